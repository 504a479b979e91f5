// rla_server.cu -- serving loop for mixed sketch-and-solve and RandSVD requests.
//
// `slots` worker threads, each with its own context (stream, memory pool, scratch), pull
// requests from one FIFO queue.  A request is admitted when its estimated device workspace
// fits the memory budget next to the work already running (a request is always admitted
// when nothing runs, so none starves).  In RLA_SERVE_BATCHED mode a worker that takes a
// RandSVD request with k <= 128 and at most 2^22 elements also takes the other pending such
// requests that fit (up to max_group) and runs them as one grouped batch (rla_batch.cu,
// eager launches); the other workers keep taking requests meanwhile, so work that arrives
// while the GPU is busy overlaps on the device.  Least-squares requests (sketch-and-solve,
// rla_ls.cu) and the other RandSVD requests run one per worker; sketches stay resident (shared by the
// workers), keyed by shape and seed, in a cache whose estimated bytes count against the
// memory budget: past its cap the least recently used sketch that no running request holds
// is destroyed.  RLA_SERVE_PLAIN is the baseline: one worker, one request at a
// time, the single-instance RandSVD path.  Latency is submit-to-completion on the host
// clock.  A request's result does not depend on what else runs: grouped kernels map every
// tile to one instance and add partial sums in a fixed order.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <tuple>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {
size_t ls_work_bytes(int64_t s, int64_t n);
int ls_sketch_solve(rla_ctx *ctx, const rla_sketch *S, int64_t m, int64_t n, const float *A, int64_t lda,
                    const float *b, float *x, void *work, int **bad_out);
}  // namespace rla

using namespace rla;

namespace {

struct Pending {
    rla_request req;
    double t_submit;
    size_t bytes;
};

struct DoneRec {
    uint64_t tag;
    double latency;
    int status;
};

size_t req_bytes(const rla_request &r) {
    if (r.kind == RLA_REQ_LS) {
        const int64_t s = std::min<int64_t>(4 * r.n, r.m);
        return ls_work_bytes(s, r.n) + (size_t)r.m * 8 * 5 + (size_t)r.m * 8 * 4;
    }
    const int64_t m = r.m, n = r.n, k = r.k;
    if (k <= 128)
        return (size_t)(4 * m * k + 4 * n * k + 16 * n * k + 32 * k * k + 4 * ((m + 2047) / 2048) * n * k) + 4096;
    return (size_t)(12 * m * k + 40 * n * k + 64 * k * k) + 4096;
}

// RandSVD requests that run in grouped batches: rank k <= 128 and at most 2^22 elements of A.
// Larger instances fill the GPU on their own, where the single-instance path (tensor-core
// products, FP64 tensor-core factorizations) is faster than the grouped kernels.  The rule
// depends on the request alone, so a request's result is the same alone and in any mix.
bool groupable(const rla_request &r) { return r.kind == RLA_REQ_SVD && r.k <= 128 && r.m * r.n <= ((int64_t)1 << 22); }

// Estimated device bytes of a resident sketch: SparseSign draws (bucket, sign, schedule
// word per entry) and their per-tile schedule, or a dense Gaussian operator.
size_t sketch_bytes(int kind, int64_t s, int64_t L) {
    if (kind == RLA_GAUSSIAN) return (size_t)(4 * s * L) + 4096;
    const int64_t nnz = std::min<int64_t>(8, s);
    return (size_t)(L * (9 * nnz + 20)) + 4096;
}

struct CacheEntry {
    rla_sketch *sk = nullptr;
    size_t bytes = 0;
    uint64_t last_use = 0;
    int refs = 0;  // requests running with this sketch
};

}  // namespace

struct rla_server {
    rla_server_config cfg{};
    std::vector<std::thread> workers;
    std::vector<rla_ctx *> ctxs;
    std::mutex mu;
    std::condition_variable cv_work, cv_idle;
    std::deque<Pending> queue;
    std::vector<DoneRec> done;
    size_t in_use = 0;
    int running = 0;
    bool stopping = false;
    std::string first_error;
    // resident sketches shared by all workers (read-only once created; creation synchronises
    // its stream), keyed by kind, dimensions and seed; cache_bytes is changed under both
    // locks (sk_mu, then mu) and read under mu by the admission check
    std::mutex sk_mu;
    std::map<std::tuple<int, int64_t, int64_t, uint64_t>, CacheEntry> sketches;
    size_t cache_bytes = 0;
    uint64_t use_clock = 0;
    int64_t evictions = 0;
    std::set<uint64_t> inject_oom;  // tags whose workspace allocation fails (under mu)
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

bool admissible(const rla_server *S) {
    if (S->queue.empty()) return false;
    return S->in_use == 0 || S->in_use + S->cache_bytes + S->queue.front().bytes <= S->cfg.memory_budget;
}

using SketchKey = std::tuple<int, int64_t, int64_t, uint64_t>;

// Sketches are created once per key for the whole server: creation allocates device memory,
// which can synchronise the device, so doing it per worker would serialise the workers.  The
// caller holds a reference until its request is finished (release_sketch).
int get_sketch(rla_server *S, rla_ctx *ctx, int kind, int64_t s, int64_t L, uint64_t seed, rla_sketch **out) {
    const SketchKey key{kind, s, L, seed};
    std::lock_guard<std::mutex> lk(S->sk_mu);
    auto &cache = S->sketches;
    auto it = cache.find(key);
    if (it != cache.end()) {
        it->second.refs++;
        it->second.last_use = ++S->use_clock;
        *out = it->second.sk;
        return RLA_OK;
    }
    const size_t need = sketch_bytes(kind, s, L);
    // Make room: destroy least recently used sketches that no running request holds (their
    // last users have synchronised their streams, so no kernel still reads them).
    while (S->cache_bytes + need > S->cfg.sketch_cache_bytes) {
        auto victim = cache.end();
        for (auto c = cache.begin(); c != cache.end(); ++c)
            if (c->second.refs == 0 && (victim == cache.end() || c->second.last_use < victim->second.last_use))
                victim = c;
        if (victim == cache.end()) break;  // every resident sketch is in use: exceed the cap for now
        rla_sketch_destroy(victim->second.sk);
        {
            std::lock_guard<std::mutex> lk2(S->mu);
            S->cache_bytes -= victim->second.bytes;
            S->evictions++;
        }
        cache.erase(victim);
    }
    rla_sketch_params p{};
    p.kind = kind;
    p.card = kind == RLA_GAUSSIAN ? RLA_RIGHT : RLA_LEFT;
    p.dtype = RLA_F32;
    p.compression_dim = s;
    p.long_dim = L;
    p.nnz = std::min<int64_t>(8, s);
    p.seed = seed;
    rla_sketch *sk = nullptr;
    RLA_TRY(rla_sketch_create(ctx, &p, &sk));
    CacheEntry e;
    e.sk = sk;
    e.bytes = need;
    e.refs = 1;
    e.last_use = ++S->use_clock;
    cache[key] = e;
    {
        std::lock_guard<std::mutex> lk2(S->mu);
        S->cache_bytes += need;
    }
    *out = sk;
    return RLA_OK;
}

void release_sketch(rla_server *S, int kind, int64_t s, int64_t L, uint64_t seed) {
    std::lock_guard<std::mutex> lk(S->sk_mu);
    auto it = S->sketches.find(SketchKey{kind, s, L, seed});
    if (it != S->sketches.end() && it->second.refs > 0) it->second.refs--;
}

int run_ls(rla_server *srv, rla_ctx *ctx, const rla_request &r) {
    const int64_t s = std::min<int64_t>(4 * r.n, r.m);
    rla_sketch *S = nullptr;
    RLA_TRY(get_sketch(srv, ctx, RLA_SPARSE_SIGN, s, r.m, r.seed, &S));
    struct Rel {
        rla_server *srv;
        int64_t s, m;
        uint64_t seed;
        ~Rel() { release_sketch(srv, RLA_SPARSE_SIGN, s, m, seed); }
    } rel{srv, s, r.m, r.seed};
    void *work = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &work, ls_work_bytes(s, r.n), ctx->stream));
    int *bad = nullptr;
    int rc = ls_sketch_solve(ctx, S, r.m, r.n, r.A, r.lda, r.b, r.x, work, &bad);
    int hbad = 0;
    if (rc == RLA_OK) {
        cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = RLA_E_CUDA;
    }
    cudaFreeAsync(work, ctx->stream);
    RLA_TRY(rc);
    return hbad ? RLA_E_NUMERIC : RLA_OK;
}

int run_svd_single(rla_server *srv, rla_ctx *ctx, const rla_request &r) {
    rla_sketch *om = nullptr;
    RLA_TRY(get_sketch(srv, ctx, RLA_GAUSSIAN, r.k, r.n, r.seed, &om));
    rla_range_params pr{0, 0, RLA_PREC_NATIVE};
    const int rc = rla_randsvd(ctx, om, RLA_F32, r.m, r.n, r.A, r.lda, &pr, RLA_F32, r.U, r.ldu, r.S, r.V, r.ldv);
    release_sketch(srv, RLA_GAUSSIAN, r.k, r.n, r.seed);
    return rc;
}

int run_svd_group(rla_ctx *ctx, const std::vector<Pending> &job) {
    std::vector<rla_svd_problem> probs;
    for (const Pending &p : job) {
        const rla_request &r = p.req;
        probs.push_back(rla_svd_problem{r.m, r.n, r.k, r.A, r.lda, r.U, r.ldu, r.S, r.V, r.ldv, r.seed});
    }
    rla_range_params pr{0, 0, RLA_PREC_NATIVE};
    rla_batch *b = nullptr;
    RLA_TRY(rla_randsvd_batch_create(ctx, (int)probs.size(), probs.data(), &pr, RLA_BATCH_EAGER, &b));
    const int rc = rla_randsvd_batch_run(ctx, b);
    rla_randsvd_batch_destroy(b);
    RLA_TRY(rc);
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

void worker_main(rla_server *S, int w) {
    cudaSetDevice(S->cfg.device);
    rla_ctx *ctx = S->ctxs[w];
    const bool batched = S->cfg.mode == RLA_SERVE_BATCHED;
    for (;;) {
        std::vector<Pending> job;
        size_t bytes = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return admissible(S) || (S->stopping && S->queue.empty()); });
            if (S->queue.empty()) break;  // stopping
            Pending f = S->queue.front();
            S->queue.pop_front();
            job.push_back(f);
            bytes += f.bytes;
            S->in_use += f.bytes;
            const bool group = batched && groupable(f.req);
            if (group) {
                for (auto it = S->queue.begin(); it != S->queue.end() && (int)job.size() < S->cfg.max_group;) {
                    if (groupable(it->req) &&
                        S->in_use + it->bytes <= S->cfg.memory_budget) {
                        job.push_back(*it);
                        bytes += it->bytes;
                        S->in_use += it->bytes;
                        it = S->queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            ++S->running;
        }
        // requests whose workspace allocation is made to fail (host-side fault injection)
        // complete with RLA_E_OOM on their own; the rest of the job runs
        std::vector<Pending> failed;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (!S->inject_oom.empty()) {
                for (auto it = job.begin(); it != job.end();) {
                    if (S->inject_oom.erase(it->req.tag)) {
                        failed.push_back(*it);
                        it = job.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
        }
        int rc = RLA_OK;
        if (!job.empty()) {
            const rla_request &r0 = job.front().req;
            if (r0.kind == RLA_REQ_LS) rc = run_ls(S, ctx, r0);
            else if (job.size() > 1 || (batched && groupable(r0))) rc = run_svd_group(ctx, job);
            else rc = run_svd_single(S, ctx, r0);
            if (rc == RLA_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = RLA_E_CUDA;
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (rc != RLA_OK && S->first_error.empty())
                S->first_error = std::string(rla_status_string(rc)) + ": " + ctx->last_error;
            if (!failed.empty() && S->first_error.empty())
                S->first_error = std::string(rla_status_string(RLA_E_OOM)) + ": injected workspace allocation failure";
            const double t = S->now();
            for (const Pending &p : job) S->done.push_back(DoneRec{p.req.tag, t - p.t_submit, rc});
            for (const Pending &p : failed) S->done.push_back(DoneRec{p.req.tag, t - p.t_submit, RLA_E_OOM});
            S->in_use -= bytes;
            --S->running;
        }
        S->cv_work.notify_all();
        S->cv_idle.notify_all();
    }
}

}  // namespace

extern "C" {

int rla_server_start(const rla_server_config *cfg, rla_server **out) {
    if (!cfg || !out) return RLA_E_ARG;
    *out = nullptr;
    if (cfg->slots <= 0 || cfg->max_group <= 0 || (cfg->mode != RLA_SERVE_BATCHED && cfg->mode != RLA_SERVE_PLAIN))
        return RLA_E_ARG;
    rla_server *S = new rla_server();
    S->cfg = *cfg;
    if (S->cfg.mode == RLA_SERVE_PLAIN) {
        S->cfg.slots = 1;
        S->cfg.max_group = 1;
    }
    if (S->cfg.memory_budget == 0) S->cfg.memory_budget = (uint64_t)150 << 30;
    if (S->cfg.sketch_cache_bytes == 0) S->cfg.sketch_cache_bytes = S->cfg.memory_budget / 8;
    for (int w = 0; w < S->cfg.slots; ++w) {
        rla_ctx *c = nullptr;
        const int rc = rla_ctx_create(cfg->device, nullptr, &c);
        if (rc != RLA_OK) {
            for (rla_ctx *x : S->ctxs) rla_ctx_destroy(x);
            delete S;
            return rc;
        }
        S->ctxs.push_back(c);
    }
    for (int w = 0; w < S->cfg.slots; ++w) S->workers.emplace_back(worker_main, S, w);
    *out = S;
    return RLA_OK;
}

int rla_server_submit(rla_server *S, const rla_request *req) {
    if (!S || !req) return RLA_E_ARG;
    const rla_request &r = *req;
    if (r.kind != RLA_REQ_LS && r.kind != RLA_REQ_SVD) return RLA_E_ARG;
    if (r.m <= 0 || r.n <= 0 || !r.A || r.lda < r.m) return RLA_E_ARG;
    if (r.kind == RLA_REQ_LS && (!r.b || !r.x || r.n > r.m || r.n > 4096)) return RLA_E_ARG;
    if (r.kind == RLA_REQ_SVD && (r.k <= 0 || r.k > std::min(r.m, r.n) || !r.U || !r.S || !r.V || r.ldu < r.m ||
                                  r.ldv < r.n))
        return RLA_E_ARG;
    Pending p{r, S->now(), req_bytes(r)};
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) return RLA_E_ARG;
        S->queue.push_back(p);
    }
    S->cv_work.notify_one();
    return RLA_OK;
}

int rla_server_poll(rla_server *S, uint64_t *tags, double *latency_s, int *status, int max, int *count) {
    if (!S || !count || max < 0) return RLA_E_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    const int n = (int)std::min<size_t>((size_t)max, S->done.size());
    for (int i = 0; i < n; ++i) {
        if (tags) tags[i] = S->done[i].tag;
        if (latency_s) latency_s[i] = S->done[i].latency;
        if (status) status[i] = S->done[i].status;
    }
    S->done.erase(S->done.begin(), S->done.begin() + n);
    *count = n;
    return RLA_OK;
}

const char *rla_server_last_error(rla_server *S) {
    if (!S) return "";
    std::lock_guard<std::mutex> lk(S->mu);
    return S->first_error.c_str();
}

int rla_server_wait_idle(rla_server *S) {
    if (!S) return RLA_E_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_idle.wait(lk, [&] { return S->queue.empty() && S->running == 0; });
    return RLA_OK;
}

int rla_server_cancel(rla_server *S, uint64_t tag) {
    if (!S) return RLA_E_ARG;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->queue.begin();
        while (it != S->queue.end() && it->req.tag != tag) ++it;
        if (it == S->queue.end()) return RLA_E_ARG;
        S->done.push_back(DoneRec{tag, S->now() - it->t_submit, RLA_E_CANCELLED});
        S->queue.erase(it);
    }
    S->cv_work.notify_all();
    S->cv_idle.notify_all();
    return RLA_OK;
}

int rla_server_inject_alloc_failure(rla_server *S, uint64_t tag) {
    if (!S) return RLA_E_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    S->inject_oom.insert(tag);
    return RLA_OK;
}

int rla_server_get_stats(rla_server *S, rla_server_stats *o) {
    if (!S || !o) return RLA_E_ARG;
    int64_t entries = 0;
    {
        std::lock_guard<std::mutex> lk(S->sk_mu);
        entries = (int64_t)S->sketches.size();
    }
    std::lock_guard<std::mutex> lk(S->mu);
    o->queued = (int64_t)S->queue.size();
    o->running = S->running;
    o->workspace_bytes = S->in_use;
    o->cache_bytes = S->cache_bytes;
    o->cache_entries = entries;
    o->evictions = S->evictions;
    return RLA_OK;
}

int rla_server_stop(rla_server *S) {
    if (!S) return RLA_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto &t : S->workers) t.join();
    for (auto &kv : S->sketches) rla_sketch_destroy(kv.second.sk);
    for (rla_ctx *c : S->ctxs) rla_ctx_destroy(c);
    delete S;
    return RLA_OK;
}

}  // extern "C"
