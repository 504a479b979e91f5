// rla_sketch.cu -- complete_compressor / update_compressor! : device draws and tables.
//
// The random draws are made on the device from a counter-based generator (Philox4x32-10)
// keyed by the sketch seed and the draw count, so a sketch is reproducible from
// (seed, number of updates).  The reference draws the same distributions on the host:
//   SparseSign  nnz distinct rows per long index, values +-T(1/sqrt(nnz))   sparse_sign.jl:155-172, :248-252
//   CountSketch one uniform bucket and one +-1 per long index               count_sketch.jl:124-127, :160-161
//   SRHT        N sign bits, s rows of 0:N-1 without replacement, unordered  srht.jl:150-151
//   FJLT        K = sprandn(.., q): Bernoulli(q) pattern, N(0,1) values     fjlt.jl:183, :217
//   Gaussian    T(1/sqrt(s)) * randn(T, ..)                                  gaussian.jl:106-107, :121-122
#include <math.h>

#include <algorithm>
#include <vector>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

// SparseSign / CountSketch: per long index j, nnz distinct buckets (Floyd's algorithm,
// then sorted ascending like StatsBase.sample!(...; ordered=true)) and nnz sign bits.
__global__ void draw_sparse_kernel(Rng rng, uint32_t stream, int64_t L, int nnz, int64_t s,
                                   int32_t *bucket, uint8_t *negative) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= L) return;
    WordStream ws{rng, stream, (uint64_t)j << 24};
    int32_t *out = bucket + j * nnz;
    int cnt = 0;
    for (int64_t t = s - nnz; t < s; ++t) {
        uint32_t r = uniform_below((uint32_t)(t + 1), ws);
        bool found = false;
        for (int q = 0; q < cnt; ++q) found |= (out[q] == (int32_t)r);
        out[cnt++] = found ? (int32_t)t : (int32_t)r;
    }
    for (int a = 1; a < cnt; ++a) {  // insertion sort (nnz is small)
        int32_t v = out[a];
        int b = a - 1;
        while (b >= 0 && out[b] > v) {
            out[b + 1] = out[b];
            --b;
        }
        out[b + 1] = v;
    }
    for (int e = 0; e < nnz; ++e) negative[j * nnz + e] = (uint8_t)(ws() & 1u);
}

// Metadata of the contiguous-vector compress kernel.  The kernel maps element
// j = 128*tile + 4*lane + t of a tile to lane `lane`, and runs one sub-round per (t, e)
// with every lane adding one value to its bucket.  Here, per tile (one warp per tile):
//  * in every sub-round, lanes whose bucket repeats an earlier lane's are marked deferred
//    (bit 30 of their main word), so the main sub-rounds touch distinct bins;
//  * deferred items are packed first-fit, in (sub-round, lane) order, into extra rounds in
//    which each lane holds at most one item and all shared-memory banks (bucket mod 32),
//    hence all buckets, differ: an extra round costs one wavefront per access;
//  * tiles with more than SS_MAX_DEFER deferred items or SS_MAX_XROUNDS extra rounds are
//    marked SLOW and resolved at run time instead (only for tiny compression dimensions).
// The packing runs on all lanes at once: lane r keeps the lane and bank masks of extra
// round r, and a ballot picks the first round that takes an item.
// Pass 0 writes the main words and counts extra rounds; pass 1 (after an exclusive scan of
// the counts) writes the extra words and the tile flags.  Both passes schedule identically.
constexpr int SCHED_WARPS = 8, SS_MAX_DEFER = 512, SS_MAX_XROUNDS = 32;
constexpr int MAX_DEFER = 64;  // CountSketch schedule: deferred entries per batch
constexpr uint32_t TILE_SLOW = 0x80000000u;

template <int PASS>
__global__ void __launch_bounds__(SCHED_WARPS * 32) sparse_sched_kernel(const int32_t *bucket, const uint8_t *negative,
                                                                         int64_t L, int nnz, uint32_t *meta,
                                                                         int32_t *nrounds, const int64_t *round_base,
                                                                         uint32_t *tile_flags, uint32_t *extra) {
    __shared__ uint32_t list[SCHED_WARPS][SS_MAX_DEFER];
    __shared__ uint8_t place[SCHED_WARPS][SS_MAX_DEFER];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t tile = (int64_t)blockIdx.x * SCHED_WARPS + w;
    const int64_t ntile = (L + 127) / 128;
    if (tile >= ntile) return;  // warp-uniform
    const unsigned lt = (1u << lane) - 1u;
    int cnt = 0;
    for (int e = 0; e < nnz; ++e)
        for (int t = 0; t < 4; ++t) {
            const int64_t j = tile * 128 + 4 * lane + t;
            const bool valid = j < L;
            const uint32_t b = valid ? (uint32_t)bucket[j * nnz + e] : 0u;
            const uint32_t neg = valid ? (uint32_t)negative[j * nnz + e] : 0u;
            const unsigned grp = __match_any_sync(FULL, valid ? b : (0x80000000u | (unsigned)lane));
            const bool defer = valid && (grp & lt) != 0u;
            if (PASS == 0 && valid) meta[(tile * nnz + e) * 128 + 4 * lane + t] = b | ((uint32_t)defer << 30) | (neg << 31);
            const unsigned bal = __ballot_sync(FULL, defer);
            if (defer) {
                const int pos = cnt + __popc(bal & lt);
                if (pos < SS_MAX_DEFER) list[w][pos] = b | ((uint32_t)t << 22) | ((uint32_t)lane << 24) | (neg << 31);
            }
            cnt += __popc(bal);
        }
    __syncwarp();
    int R = 0;
    bool slow = cnt > SS_MAX_DEFER;
    uint32_t rl = 0u, rb = 0u;  // lane r: lanes and banks taken in extra round r
    for (int k = 0; k < cnt && !slow; ++k) {  // warp-uniform trip count
        const uint32_t it = list[w][k];
        const uint32_t lbit = 1u << ((it >> 24) & 31u), bbit = 1u << (it & 31u);
        const unsigned fits = __ballot_sync(FULL, lane < R && !((rl & lbit) | (rb & bbit)));
        int r;
        if (fits) {
            r = __ffs(fits) - 1;
        } else if (R < SS_MAX_XROUNDS) {
            r = R++;
        } else {
            slow = true;
            break;
        }
        if (lane == r) {
            rl |= lbit;
            rb |= bbit;
        }
        if (lane == 0) place[w][k] = (uint8_t)r;
    }
    if (slow) R = 0;
    if (PASS == 0) {
        if (lane == 0) nrounds[tile] = slow ? 0 : R;
        return;
    }
    if (slow) {
        if (lane == 0) tile_flags[tile] = TILE_SLOW;
        return;
    }
    const int64_t base = round_base[tile];
    for (int r = 0; r < R; ++r) extra[(base + r) * 32 + lane] = 0u;
    __syncwarp();
    if (lane == 0) {
        for (int k = 0; k < cnt; ++k) {
            const uint32_t it = list[w][k];
            const uint32_t ln = (it >> 24) & 31u;
            extra[(base + place[w][k]) * 32 + ln] = (it & 0x3fffffu) | (it & (3u << 22)) | (1u << 30) | (it & 0x80000000u);
        }
        tile_flags[tile] = R == 0 ? 0u : (uint32_t)((base << 8) | (uint32_t)R);
    }
}

// base[i] = sum_{k < i} nr[k] (exclusive scan of the per-tile extra-round counts), one CTA:
// each thread sums a contiguous chunk, the chunk totals are scanned in shared memory.
__global__ void __launch_bounds__(1024) sched_scan_kernel(const int32_t *nr, int64_t n, int64_t *base) {
    __shared__ int64_t part[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int64_t per = (n + nt - 1) / nt, lo = min(n, (int64_t)t * per), hi = min(n, lo + per);
    int64_t sum = 0;
    for (int64_t i = lo; i < hi; ++i) sum += nr[i];
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        const int64_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int64_t run = part[t] - sum;
    for (int64_t i = lo; i < hi; ++i) {
        base[i] = run;
        run += nr[i];
    }
}

// CountSketch (nnz = 1, s <= 2^16): 512-element batches (4 tiles, 16 sub-rounds of 32
// lanes).  An element is deferred when its bucket already occurred earlier in the batch,
// in (sub-round, lane) order, so all non-deferred elements of a batch hit distinct bins and
// the apply kernel issues a whole batch's read-modify-writes at once.  The apply kernel's
// shared memory holds, per warp, s bins, a 64-entry list and 32 dummy slots; each element's
// word is the byte offset (element size es) of the slot it is added to -- its bin, or for a
// deferred element its list entry -- with the sign in bit 31.  Up to CS_XROUNDS extra
// rounds then add list entry r*32 + lane to the bin at byte offset xbucket[batch*64 +
// r*32 + lane] and clear the entry; the list is ordered here so that each round's buckets
// are distinct, and empty entries point at the lane's dummy slot.  flags[batch] is the
// number of extra rounds, or TILE_SLOW when the batch needs run-time resolution (its words
// then all point at bins).
constexpr int CS_SCHED_WARPS = 4, CS_BATCH = 512, CS_XROUNDS = 2;

__global__ void __launch_bounds__(CS_SCHED_WARPS * 32) cs_sched_kernel(const int32_t *bucket, const uint8_t *negative,
                                                                        int64_t L, int64_t s, uint32_t es,
                                                                        uint32_t *meta, uint32_t *flags,
                                                                        uint32_t *xbucket) {
    extern __shared__ uint32_t bm_all[];
    __shared__ uint32_t list[CS_SCHED_WARPS][MAX_DEFER];
    __shared__ uint32_t slot[CS_SCHED_WARPS][CS_XROUNDS * 32];
    __shared__ int pos_of[CS_SCHED_WARPS][MAX_DEFER];
    __shared__ int ok_s[CS_SCHED_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t batch = (int64_t)blockIdx.x * CS_SCHED_WARPS + w;
    const int64_t nb = (L + CS_BATCH - 1) / CS_BATCH;
    if (batch >= nb) return;  // warp-uniform
    const int nw = (int)((s + 31) / 32);
    uint32_t *bm = bm_all + (int64_t)w * nw;
    for (int i = lane; i < nw; i += 32) bm[i] = 0u;
    __syncwarp();
    const unsigned lt = (1u << lane) - 1u;
    int cnt = 0;
    uint32_t myword[16];
    int mylist[16];
    for (int r = 0; r < 16; ++r) {
        const int64_t j = batch * CS_BATCH + (r >> 2) * 128 + 4 * lane + (r & 3);
        const bool valid = j < L;
        const uint32_t b = valid ? (uint32_t)bucket[j] : 0u;
        const uint32_t neg = valid ? (uint32_t)negative[j] : 0u;
        const unsigned grp = __match_any_sync(FULL, valid ? b : (0x80000000u | (unsigned)lane));
        const bool leader = valid && (grp & lt) == 0u;
        const bool seen = leader && ((bm[b >> 5] >> (b & 31)) & 1u);
        const bool defer = valid && (!leader || seen);
        __syncwarp();
        if (leader && !seen) atomicOr(&bm[b >> 5], 1u << (b & 31));
        __syncwarp();
        const unsigned bal = __ballot_sync(FULL, defer);
        mylist[r] = -1;
        if (defer) {
            const int pos = cnt + __popc(bal & lt);
            if (pos < MAX_DEFER) list[w][pos] = b;
            mylist[r] = pos;
        }
        cnt += __popc(bal);
        myword[r] = (b * es) | (neg << 31);
    }
    __syncwarp();
    // order the deferred entries into rounds of 32 with distinct buckets (lane 0, greedy)
    if (lane == 0) {
        int ok = cnt <= MAX_DEFER;
        int fill[CS_XROUNDS] = {0};
        for (int k = 0; k < cnt && ok; ++k) {
            const uint32_t bk = list[w][k];
            int r = 0;
            for (; r < CS_XROUNDS; ++r) {
                if (fill[r] == 32) continue;
                bool clash = false;
                for (int q = 0; q < fill[r] && !clash; ++q) clash = slot[w][r * 32 + q] == bk;
                if (!clash) break;
            }
            if (r == CS_XROUNDS) {
                ok = 0;
                break;
            }
            slot[w][r * 32 + fill[r]] = bk;
            pos_of[w][k] = r * 32 + fill[r];
            ++fill[r];
        }
        for (int r = 0; r < CS_XROUNDS; ++r)
            for (int q = fill[r]; q < 32; ++q) slot[w][r * 32 + q] = 0xffffffffu;
        ok_s[w] = ok ? (fill[1] > 0 ? 2 : (fill[0] > 0 ? 1 : 0)) : -1;
    }
    __syncwarp();
    const int R = ok_s[w];
    for (int r = 0; r < 16; ++r) {
        const int64_t j = batch * CS_BATCH + (r >> 2) * 128 + 4 * lane + (r & 3);
        if (j >= L) continue;
        uint32_t word = myword[r];
        if (R >= 0 && mylist[r] >= 0)
            word = ((uint32_t)(s + pos_of[w][mylist[r]]) * es) | (word & 0x80000000u);
        meta[j] = word;
    }
    const uint32_t dummy = (uint32_t)(s + 64 + lane) * es;
    for (int k = lane; k < CS_XROUNDS * 32; k += 32)
        xbucket[batch * 64 + k] = (R > 0 && slot[w][k] != 0xffffffffu) ? slot[w][k] * es : dummy;
    if (lane == 0) flags[batch] = R < 0 ? TILE_SLOW : (uint32_t)R;
}

__global__ void draw_signbits_kernel(Rng rng, int64_t nwords, uint32_t *bits) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i * 4 >= nwords) return;
    P4 r = rng.at(STREAM_SRHT_SIGNS, (uint64_t)i);
    uint32_t v[4] = {r.x, r.y, r.z, r.w};
    for (int k = 0; k < 4; ++k)
        if (i * 4 + k < nwords) bits[i * 4 + k] = v[k];
}

// s distinct rows of 0:N-1 in random order: Floyd's algorithm over a bitmap, followed by
// a Fisher-Yates shuffle (Floyd's insertion order is not uniform).  Single thread; the
// bitmap lives in shared memory when it fits.
__global__ void draw_rows_kernel(Rng rng, int64_t N, int64_t s, uint32_t *gbitmap,
                                 int use_smem, int32_t *rows) {
    extern __shared__ uint32_t sbitmap[];
    uint32_t *bm = use_smem ? sbitmap : gbitmap;
    int64_t nw = (N + 31) / 32;
    for (int64_t i = threadIdx.x; i < nw; i += blockDim.x) bm[i] = 0;
    __syncthreads();
    if (threadIdx.x != 0) return;
    WordStream ws{rng, STREAM_SRHT_ROWS, 0};
    int64_t cnt = 0;
    for (int64_t t = N - s; t < N; ++t) {
        uint32_t r = uniform_below((uint32_t)(t + 1), ws);
        uint32_t bit = 1u << (r & 31);
        uint32_t pick = (bm[r >> 5] & bit) ? (uint32_t)t : r;
        bm[pick >> 5] |= 1u << (pick & 31);
        rows[cnt++] = (int32_t)pick;
    }
    for (int64_t i = s - 1; i > 0; --i) {
        uint32_t k = uniform_below((uint32_t)(i + 1), ws);
        int32_t tmp = rows[i];
        rows[i] = rows[k];
        rows[k] = tmp;
    }
}


// FJLT: rows of Kc (s x N) with a Bernoulli(q) pattern drawn by geometric gaps.
// Pass 0 counts, pass 1 fills; both passes replay the same word stream.
template <class T>
__global__ void draw_fjlt_rows_kernel(Rng rng, int64_t s, int64_t N, double q, int pass,
                                      int32_t *counts, const int32_t *ptr, int32_t *col, T *val) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= s) return;
    WordStream ws{rng, STREAM_FJLT_K, (uint64_t)i << 28};
    double lq = log1p(-q);
    int64_t pos = -1;
    int32_t c = 0;
    int32_t base = pass ? ptr[i] : 0;
    while (true) {
        double u = u01_open_d(ws(), ws());
        double g = (q >= 1.0) ? 0.0 : floor(log(u) / lq);
        if (!(g < (double)N)) break;
        pos += (int64_t)g + 1;
        if (pos >= N) break;
        double z2;
        double z = normal_pair(ws, &z2);
        if (pass) {
            col[base + c] = (int32_t)pos;
            val[base + c] = (T)z;
        }
        ++c;
    }
    if (!pass) counts[i] = c;
}

template <class T>
__global__ void draw_gaussian_kernel(Rng rng, int64_t n, T scale, T *out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (2 * i >= n) return;
    WordStream ws{rng, STREAM_GAUSS, (uint64_t)i};
    double z2;
    double z1 = normal_pair(ws, &z2);
    out[2 * i] = scale * (T)z1;
    if (2 * i + 1 < n) out[2 * i + 1] = scale * (T)z2;
}

template <class T>
static int fjlt_build(rla_ctx *ctx, rla_sketch *sk, const Rng &rng) {
    int64_t s = sk->s, N = sk->N;
    int32_t *counts = nullptr;
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&counts, sizeof(int32_t) * (s + 1), ctx->stream));
    draw_fjlt_rows_kernel<T><<<ceil_div_i(s, 128), 128, 0, ctx->stream>>>(rng, s, N, sk->sparsity, 0,
                                                                         counts, nullptr, nullptr, nullptr);
    RLA_TRY(check_launch(ctx, "draw_fjlt_rows(count)"));
    std::vector<int32_t> hc(s);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(hc.data(), counts, sizeof(int32_t) * s, cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> hp(s + 1, 0);
    for (int64_t i = 0; i < s; ++i) hp[i + 1] = hp[i] + hc[i];
    int64_t nnz = hp[s];
    if (sk->k_ptr) cudaFreeAsync(sk->k_ptr, ctx->stream);
    if (sk->k_col) cudaFreeAsync(sk->k_col, ctx->stream);
    if (sk->k_val) cudaFreeAsync(sk->k_val, ctx->stream);
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&sk->k_ptr, sizeof(int32_t) * (s + 1), ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&sk->k_col, sizeof(int32_t) * std::max<int64_t>(nnz, 1), ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&sk->k_val, sizeof(T) * std::max<int64_t>(nnz, 1), ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->k_ptr, hp.data(), sizeof(int32_t) * (s + 1), cudaMemcpyHostToDevice, ctx->stream));
    draw_fjlt_rows_kernel<T><<<ceil_div_i(s, 128), 128, 0, ctx->stream>>>(rng, s, N, sk->sparsity, 1, nullptr,
                                                                         sk->k_ptr, sk->k_col, (T *)sk->k_val);
    RLA_TRY(check_launch(ctx, "draw_fjlt_rows(fill)"));
    RLA_CUDA_TRY(ctx, cudaFreeAsync(counts, ctx->stream));
    sk->k_nnz = nnz;
    return RLA_OK;
}

// Transpose Kc (CSR s x N) into CSR of Kc' (N x s) on the host; entries of each row of
// the transpose are in ascending column order.
template <class T>
static int fjlt_transpose(rla_ctx *ctx, rla_sketch *sk) {
    int64_t s = sk->s, N = sk->N, nnz = sk->k_nnz;
    std::vector<int32_t> p(s + 1), c(std::max<int64_t>(nnz, 1));
    std::vector<T> v(std::max<int64_t>(nnz, 1));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(p.data(), sk->k_ptr, sizeof(int32_t) * (s + 1), cudaMemcpyDeviceToHost, ctx->stream));
    if (nnz) {
        RLA_CUDA_TRY(ctx, cudaMemcpyAsync(c.data(), sk->k_col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, ctx->stream));
        RLA_CUDA_TRY(ctx, cudaMemcpyAsync(v.data(), sk->k_val, sizeof(T) * nnz, cudaMemcpyDeviceToHost, ctx->stream));
    }
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> tp(N + 1, 0), tr(std::max<int64_t>(nnz, 1));
    std::vector<T> tv(std::max<int64_t>(nnz, 1));
    for (int64_t k = 0; k < nnz; ++k) tp[c[k] + 1]++;
    for (int64_t r = 0; r < N; ++r) tp[r + 1] += tp[r];
    std::vector<int32_t> fill(tp.begin(), tp.end() - 1);
    for (int64_t i = 0; i < s; ++i)
        for (int32_t k = p[i]; k < p[i + 1]; ++k) {
            int32_t d = fill[c[k]]++;
            tr[d] = (int32_t)i;
            tv[d] = v[k];
        }
    if (sk->kt_ptr) cudaFreeAsync(sk->kt_ptr, ctx->stream);
    if (sk->kt_row) cudaFreeAsync(sk->kt_row, ctx->stream);
    if (sk->kt_val) cudaFreeAsync(sk->kt_val, ctx->stream);
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&sk->kt_ptr, sizeof(int32_t) * (N + 1), ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&sk->kt_row, sizeof(int32_t) * std::max<int64_t>(nnz, 1), ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMallocAsync(&sk->kt_val, sizeof(T) * std::max<int64_t>(nnz, 1), ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->kt_ptr, tp.data(), sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice, ctx->stream));
    if (nnz) {
        RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->kt_row, tr.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, ctx->stream));
        RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->kt_val, tv.data(), sizeof(T) * nnz, cudaMemcpyHostToDevice, ctx->stream));
    }
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

// SRHT expand tables: samples grouped by their low log2(chunk) bits.
static int srht_tables(rla_ctx *ctx, rla_sketch *sk) {
    int64_t s = sk->s;
    sk->chunk = std::min<int64_t>(sk->N, 4096);
    int64_t ch = sk->chunk;
    std::vector<int32_t> rows(s);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(rows.data(), sk->rows, sizeof(int32_t) * s, cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> ptr(ch + 1, 0), list(s);
    for (int64_t k = 0; k < s; ++k) ptr[(rows[k] & (ch - 1)) + 1]++;
    for (int64_t r = 0; r < ch; ++r) ptr[r + 1] += ptr[r];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t k = 0; k < s; ++k) list[fill[rows[k] & (ch - 1)]++] = (int32_t)k;
    if (!sk->p2_ptr) RLA_CUDA_TRY(ctx, cudaMalloc(&sk->p2_ptr, sizeof(int32_t) * (4096 + 1)));
    if (!sk->p2_list) RLA_CUDA_TRY(ctx, cudaMalloc(&sk->p2_list, sizeof(int32_t) * s));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->p2_ptr, ptr.data(), sizeof(int32_t) * (ch + 1), cudaMemcpyHostToDevice, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->p2_list, list.data(), sizeof(int32_t) * s, cudaMemcpyHostToDevice, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

static int build_meta(rla_ctx *ctx, rla_sketch *sk) {
    if (sk->s > (1 << 22)) return RLA_OK;  // compression dimension beyond the packed form: strided/expand paths only
    sk->batch_mode = (sk->nnz == 1 && sk->s <= 65536) ? 1 : 0;
    if (sk->batch_mode) {
        const int64_t nb = ceil_div(sk->L, CS_BATCH);
        const size_t bm_bytes = (size_t)CS_SCHED_WARPS * ceil_div(sk->s, 32) * 4;
        if (!sk->tile_flags) RLA_CUDA_TRY(ctx, cudaMalloc(&sk->tile_flags, sizeof(uint32_t) * nb));
        if (!sk->extra) {
            RLA_CUDA_TRY(ctx, cudaMalloc(&sk->extra, sizeof(uint32_t) * 64 * nb));
            sk->extra_rounds_cap = 2 * nb;
        }
        if (bm_bytes > 48 * 1024)
            RLA_CUDA_TRY(ctx, set_smem_max(cs_sched_kernel));
        cs_sched_kernel<<<ceil_div_i(nb, CS_SCHED_WARPS), CS_SCHED_WARPS * 32, bm_bytes, ctx->stream>>>(
            sk->bucket, sk->negative, sk->L, sk->s, (uint32_t)dtype_size(sk->p.dtype), sk->meta, sk->tile_flags,
            sk->extra);
        return check_launch(ctx, "cs_sched");
    }
    const int64_t ntile = ceil_div(sk->L, 128);
    const int blocks = ceil_div_i(ntile, SCHED_WARPS);
    int32_t *nr = nullptr;
    int64_t *base = nullptr;
    RLA_CUDA_TRY(ctx, cudaMallocAsync((void **)&nr, sizeof(int32_t) * ntile, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMallocAsync((void **)&base, sizeof(int64_t) * ntile, ctx->stream));
    sparse_sched_kernel<0><<<blocks, SCHED_WARPS * 32, 0, ctx->stream>>>(sk->bucket, sk->negative, sk->L, (int)sk->nnz,
                                                                         sk->meta, nr, nullptr, nullptr, nullptr);
    RLA_TRY(check_launch(ctx, "sparse_sched(0)"));
    if (ntile * SS_MAX_XROUNDS < (int64_t(1) << 23)) {
        // the schedule never needs more than SS_MAX_XROUNDS rounds per tile: size `extra` for
        // that once and scan the counts on the device, so a redraw waits on nothing
        const int64_t cap = std::max<int64_t>(ntile * SS_MAX_XROUNDS, 1);
        if (sk->extra_rounds_cap < cap) {
            if (sk->extra) RLA_CUDA_TRY(ctx, cudaFree(sk->extra));
            sk->extra = nullptr;
            RLA_CUDA_TRY(ctx, cudaMalloc(&sk->extra, sizeof(uint32_t) * 32 * cap));
            sk->extra_rounds_cap = cap;
        }
        if (!sk->tile_flags) RLA_CUDA_TRY(ctx, cudaMalloc(&sk->tile_flags, sizeof(uint32_t) * std::max<int64_t>(ntile, 1)));
        sched_scan_kernel<<<1, 1024, 0, ctx->stream>>>(nr, ntile, base);
        RLA_TRY(check_launch(ctx, "sched_scan"));
        sparse_sched_kernel<1><<<blocks, SCHED_WARPS * 32, 0, ctx->stream>>>(
            sk->bucket, sk->negative, sk->L, (int)sk->nnz, sk->meta, nr, base, sk->tile_flags, sk->extra);
        RLA_TRY(check_launch(ctx, "sparse_sched(1)"));
        RLA_CUDA_TRY(ctx, cudaFreeAsync(nr, ctx->stream));
        RLA_CUDA_TRY(ctx, cudaFreeAsync(base, ctx->stream));
        return RLA_OK;
    }
    std::vector<int32_t> hn(ntile);
    std::vector<int64_t> hb(ntile);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(hn.data(), nr, sizeof(int32_t) * ntile, cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    int64_t tot = 0;
    for (int64_t i = 0; i < ntile; ++i) {
        hb[i] = tot;
        tot += hn[i];
    }
    // a tile flag holds the tile's first extra round in bits 8..30
    if (tot >= (int64_t(1) << 23)) return set_error(ctx, RLA_E_UNSUPPORTED, "too many deferred rounds");
    if (tot > sk->extra_rounds_cap) {
        if (sk->extra) RLA_CUDA_TRY(ctx, cudaFree(sk->extra));
        sk->extra = nullptr;
        sk->extra_rounds_cap = std::max<int64_t>(tot, 1) + tot / 4;
        RLA_CUDA_TRY(ctx, cudaMalloc(&sk->extra, sizeof(uint32_t) * 32 * sk->extra_rounds_cap));
    }
    if (!sk->tile_flags) RLA_CUDA_TRY(ctx, cudaMalloc(&sk->tile_flags, sizeof(uint32_t) * std::max<int64_t>(ntile, 1)));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(base, hb.data(), sizeof(int64_t) * ntile, cudaMemcpyHostToDevice, ctx->stream));
    sparse_sched_kernel<1><<<blocks, SCHED_WARPS * 32, 0, ctx->stream>>>(sk->bucket, sk->negative, sk->L, (int)sk->nnz,
                                                                         sk->meta, nr, base, sk->tile_flags, sk->extra);
    RLA_TRY(check_launch(ctx, "sparse_sched(1)"));
    RLA_CUDA_TRY(ctx, cudaFreeAsync(nr, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaFreeAsync(base, ctx->stream));
    return RLA_OK;
}

static Rng make_rng(const rla_sketch *sk) {
    Rng r;
    r.k0 = (uint32_t)sk->p.seed;
    r.k1 = (uint32_t)(sk->p.seed >> 32);
    r.epoch = (uint32_t)sk->draw_count;
    return r;
}

static int draw(rla_ctx *ctx, rla_sketch *sk, bool sync = true) {
    Rng rng = make_rng(sk);
    const int kind = sk->p.kind;
    if (kind == RLA_SAMPLING) return sampling_draw(ctx, sk, sync);
    if (kind == RLA_SPARSE_SIGN || kind == RLA_COUNT_SKETCH) {
        draw_sparse_kernel<<<ceil_div_i(sk->L, 128), 128, 0, ctx->stream>>>(
            rng, kind == RLA_SPARSE_SIGN ? STREAM_SPARSE : STREAM_COUNT, sk->L, (int)sk->nnz, sk->s,
            sk->bucket, sk->negative);
        RLA_TRY(check_launch(ctx, "draw_sparse"));
        RLA_TRY(build_meta(ctx, sk));
    } else if (kind == RLA_SRHT || kind == RLA_FJLT) {
        int64_t nwords = ceil_div(sk->N, 32);
        Rng r2 = rng;
        draw_signbits_kernel<<<ceil_div_i(ceil_div(nwords, 4), 256), 256, 0, ctx->stream>>>(r2, nwords, sk->signbits);
        RLA_TRY(check_launch(ctx, "draw_signbits"));
        if (kind == RLA_SRHT) {
            size_t bm_bytes = sizeof(uint32_t) * nwords;
            int use_smem = bm_bytes <= 160 * 1024;
            uint32_t *gbm = nullptr;
            if (!use_smem) {
                void *p;
                RLA_TRY(scratch_get(ctx, bm_bytes, &p));
                gbm = (uint32_t *)p;
            } else {
                RLA_CUDA_TRY(ctx, set_smem_max(draw_rows_kernel));
            }
            draw_rows_kernel<<<1, 256, use_smem ? bm_bytes : 0, ctx->stream>>>(rng, sk->N, sk->s, gbm, use_smem, sk->rows);
            RLA_TRY(check_launch(ctx, "draw_rows"));
            RLA_TRY(srht_tables(ctx, sk));
            RLA_TRY(build_srht_sign_table(ctx, sk));
        } else {
            if (sk->p.dtype == RLA_F32) {
                RLA_TRY(fjlt_build<float>(ctx, sk, rng));
                RLA_TRY(fjlt_transpose<float>(ctx, sk));
            } else {
                RLA_TRY(fjlt_build<double>(ctx, sk, rng));
                RLA_TRY(fjlt_transpose<double>(ctx, sk));
            }
        }
    } else if (kind == RLA_GAUSSIAN) {
        int64_t n = sk->n_rows * sk->n_cols;
        if (sk->p.dtype == RLA_F32)
            draw_gaussian_kernel<float><<<ceil_div_i(ceil_div(n, 2), 256), 256, 0, ctx->stream>>>(
                rng, n, (float)sk->scale, (float *)sk->dense);
        else
            draw_gaussian_kernel<double><<<ceil_div_i(ceil_div(n, 2), 256), 256, 0, ctx->stream>>>(
                rng, n, (double)sk->scale, (double *)sk->dense);
        RLA_TRY(check_launch(ctx, "draw_gaussian"));
    }
    if (sync) RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

// update_compressor! without the final synchronisation: the new draws are complete when
// the context's stream reaches this point.
int sketch_redraw_async(rla_ctx *ctx, rla_sketch *sk) {
    int rc = draw(ctx, sk, false);
    if (rc == RLA_OK) sk->draw_count++;
    return rc;
}

static void free_sketch_buffers(rla_sketch *sk) {
    void *ptrs[] = {sk->bucket, sk->negative, sk->meta, sk->rows, sk->signbits, sk->sign_tl, sk->tile_flags, sk->extra, sk->p2_ptr, sk->p2_list,
                    sk->k_ptr, sk->k_col, sk->k_val, sk->kt_ptr, sk->kt_row, sk->kt_val, sk->dense,
                    sk->sidx, sk->splan, sk->sweights, sk->s_err, sk->tp_ptr, sk->tp_idx};
    for (void *p : ptrs)
        if (p) cudaFree(p);
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_sketch_create(rla_ctx *ctx, const rla_sketch_params *pp, rla_sketch **out) {
    if (!ctx || !pp || !out) return RLA_E_ARG;
    *out = nullptr;
    const rla_sketch_params &p = *pp;
    if (p.kind == RLA_SAMPLING) return set_error(ctx, RLA_E_ARG, "Sampling recipes are made by rla_sampling_create.");
    if (p.kind < RLA_SPARSE_SIGN || p.kind > RLA_GAUSSIAN) return set_error(ctx, RLA_E_ARG, "Unknown compressor kind %d.", p.kind);
    if (p.card != RLA_LEFT && p.card != RLA_RIGHT)
        return set_error(ctx, RLA_E_ARG, "`cardinality` must be specified as `Left()` or `Right()`.");
    if (p.dtype != RLA_F32 && p.dtype != RLA_F64) return set_error(ctx, RLA_E_ARG, "Element type must be Float32 or Float64.");
    // Constructor checks, with the reference's messages.
    if (p.compression_dim <= 0) {
        if (p.kind == RLA_COUNT_SKETCH || p.kind == RLA_GAUSSIAN)
            return set_error(ctx, RLA_E_ARG, "Field 'compression_dim' must be positive.");
        return set_error(ctx, RLA_E_ARG, "Field `compression_dim` must be positive.");
    }
    if (p.kind == RLA_SPARSE_SIGN) {
        if (p.nnz > p.compression_dim)
            return set_error(ctx, RLA_E_ARG,
                             "Number of non-zero indices, %lld, must be less than or equal to compression dimension, %lld.",
                             (long long)p.nnz, (long long)p.compression_dim);
        if (p.nnz <= 0) return set_error(ctx, RLA_E_ARG, "Field `nnz` must be positive.");
    }
    if ((p.kind == RLA_SRHT || p.kind == RLA_FJLT) && p.block_size <= 0)
        return set_error(ctx, RLA_E_ARG, "Field `block_size` must be positive.");
    if (p.long_dim <= 0) return set_error(ctx, RLA_E_ARG, "The sketched dimension must be positive.");
    if (p.compression_dim >= (int64_t(1) << 30) || p.long_dim >= (int64_t(1) << 31))
        return set_error(ctx, RLA_E_UNSUPPORTED, "Dimensions beyond 2^30 (compression) / 2^31 (sketched) are not supported.");
    if (p.kind == RLA_FJLT && (p.sparsity < 0.0 || p.sparsity > 1.0))
        return set_error(ctx, RLA_E_ARG, "Field `sparsity` must be in [0, 1].");

    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    rla_sketch *sk = new rla_sketch();
    sk->p = p;
    sk->device = ctx->device;
    sk->s = p.compression_dim;
    sk->L = p.long_dim;
    sk->n_rows = p.card == RLA_LEFT ? sk->s : sk->L;
    sk->n_cols = p.card == RLA_LEFT ? sk->L : sk->s;
    const size_t es = dtype_size(p.dtype);
    int rc = RLA_OK;
    auto alloc = [&](void **ptr, size_t bytes) {
        if (rc != RLA_OK) return;
        cudaError_t e = cudaMalloc(ptr, std::max<size_t>(bytes, 16));
        if (e != cudaSuccess) rc = set_error(ctx, RLA_E_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    };
    switch (p.kind) {
        case RLA_SPARSE_SIGN:
        case RLA_COUNT_SKETCH: {
            sk->nnz = p.kind == RLA_SPARSE_SIGN ? p.nnz : 1;
            sk->scale = p.kind == RLA_SPARSE_SIGN
                            ? (p.dtype == RLA_F32 ? (double)(float)(1.0 / sqrt((double)sk->nnz)) : 1.0 / sqrt((double)sk->nnz))
                            : 1.0;
            size_t ne = (size_t)(sk->L * sk->nnz);
            alloc((void **)&sk->bucket, ne * 4);
            alloc((void **)&sk->negative, ne);
            alloc((void **)&sk->meta, (size_t)ceil_div(sk->L, 128) * 128 * sk->nnz * 4);
            break;
        }
        case RLA_SRHT:
        case RLA_FJLT: {
            sk->N = next_pow2(sk->L);
            if (p.kind == RLA_SRHT) {
                if (sk->s > sk->N) {
                    delete sk;
                    return set_error(ctx, RLA_E_ARG, "Cannot draw %lld rows without replacement from %lld.",
                                     (long long)p.compression_dim, (long long)next_pow2(p.long_dim));
                }
                double sc = sqrt((double)sk->s) / sqrt((double)sk->N);
                sk->scale = p.dtype == RLA_F32 ? (double)(float)sc : sc;
                alloc((void **)&sk->rows, (size_t)sk->s * 4);
            } else {
                sk->sparsity = p.sparsity == 0.0 ? 0.25 * log((double)sk->L) * log((double)sk->L) / (double)sk->L
                                                 : p.sparsity;
                if (sk->sparsity > 1.0) sk->sparsity = 1.0;
                double sc = 1.0 / (sqrt((double)sk->N) * sqrt(sk->sparsity) * sqrt((double)sk->s));
                sk->scale = p.dtype == RLA_F32 ? (double)(float)sc : sc;
            }
            alloc((void **)&sk->signbits, (size_t)ceil_div(sk->N, 32) * 4);
            break;
        }
        case RLA_GAUSSIAN: {
            double sc = 1.0 / sqrt((double)sk->s);
            sk->scale = p.dtype == RLA_F32 ? (double)(float)sc : sc;
            alloc(&sk->dense, (size_t)(sk->n_rows * sk->n_cols) * es);
            break;
        }
    }
    if (rc == RLA_OK) rc = draw(ctx, sk);
    if (rc != RLA_OK) {
        free_sketch_buffers(sk);
        delete sk;
        return rc;
    }
    sk->draw_count = 1;
    *out = sk;
    return RLA_OK;
}

int rla_sketch_update(rla_ctx *ctx, rla_sketch *sk) {
    if (!ctx || !sk) return RLA_E_ARG;
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    int rc = draw(ctx, sk);
    if (rc == RLA_OK) sk->draw_count++;
    return rc;
}

int rla_sketch_destroy(rla_sketch *sk) {
    if (!sk) return RLA_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(sk->device);
    cudaDeviceSynchronize();
    free_sketch_buffers(sk);
    cudaSetDevice(cur);
    delete sk;
    return RLA_OK;
}

int rla_sketch_get_info(const rla_sketch *sk, rla_sketch_info *o) {
    if (!sk || !o) return RLA_E_ARG;
    o->kind = sk->p.kind;
    o->card = sk->p.card;
    o->dtype = sk->p.dtype;
    o->n_rows = sk->n_rows;
    o->n_cols = sk->n_cols;
    o->compression_dim = sk->s;
    o->long_dim = sk->L;
    o->nnz = sk->nnz;
    o->block_size = sk->p.block_size;
    o->padded = sk->N;
    o->k_nnz = sk->k_nnz;
    o->sparsity = sk->sparsity;
    o->scale = sk->scale;
    o->draw_count = sk->draw_count;
    return RLA_OK;
}

int rla_sketch_get_draws(rla_ctx *ctx, const rla_sketch *sk, int64_t *idx, void *vals, uint8_t *signs, int64_t *kptr) {
    if (!ctx || !sk) return RLA_E_ARG;
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    const int kind = sk->p.kind;
    const size_t es = dtype_size(sk->p.dtype);
    if (kind == RLA_SAMPLING) {
        if (idx) RLA_CUDA_TRY(ctx, cudaMemcpy(idx, sk->sidx, sizeof(int64_t) * sk->s, cudaMemcpyDeviceToHost));
        return RLA_OK;
    }
    if (kind == RLA_SPARSE_SIGN || kind == RLA_COUNT_SKETCH) {
        size_t ne = (size_t)(sk->L * sk->nnz);
        std::vector<int32_t> b(ne);
        std::vector<uint8_t> ng(ne);
        RLA_CUDA_TRY(ctx, cudaMemcpy(b.data(), sk->bucket, ne * 4, cudaMemcpyDeviceToHost));
        RLA_CUDA_TRY(ctx, cudaMemcpy(ng.data(), sk->negative, ne, cudaMemcpyDeviceToHost));
        if (idx)
            for (size_t i = 0; i < ne; ++i) idx[i] = b[i];
        if (vals) {
            for (size_t i = 0; i < ne; ++i) {
                double v = ng[i] ? -sk->scale : sk->scale;
                if (es == 4) ((float *)vals)[i] = (float)v;
                else ((double *)vals)[i] = v;
            }
        }
    } else if (kind == RLA_SRHT || kind == RLA_FJLT) {
        if (signs) {
            int64_t nw = ceil_div(sk->N, 32);
            std::vector<uint32_t> w(nw);
            RLA_CUDA_TRY(ctx, cudaMemcpy(w.data(), sk->signbits, nw * 4, cudaMemcpyDeviceToHost));
            for (int64_t r = 0; r < sk->N; ++r) signs[r] = (uint8_t)((w[r >> 5] >> (r & 31)) & 1u);
        }
        if (kind == RLA_SRHT) {
            if (idx) {
                std::vector<int32_t> r(sk->s);
                RLA_CUDA_TRY(ctx, cudaMemcpy(r.data(), sk->rows, sk->s * 4, cudaMemcpyDeviceToHost));
                for (int64_t i = 0; i < sk->s; ++i) idx[i] = r[i];
            }
        } else {
            // Left: op = Kc (s x N) as CSC == CSR of Kc' ; Right: op = Kc' (N x s) as CSC == CSR of Kc
            bool left = sk->p.card == RLA_LEFT;
            int64_t ncol = left ? sk->N : sk->s;
            const int32_t *dptr = left ? sk->kt_ptr : sk->k_ptr;
            const int32_t *didx = left ? sk->kt_row : sk->k_col;
            const void *dval = left ? sk->kt_val : sk->k_val;
            std::vector<int32_t> hp(ncol + 1), hi(std::max<int64_t>(sk->k_nnz, 1));
            RLA_CUDA_TRY(ctx, cudaMemcpy(hp.data(), dptr, (ncol + 1) * 4, cudaMemcpyDeviceToHost));
            if (sk->k_nnz) RLA_CUDA_TRY(ctx, cudaMemcpy(hi.data(), didx, sk->k_nnz * 4, cudaMemcpyDeviceToHost));
            if (kptr)
                for (int64_t i = 0; i <= ncol; ++i) kptr[i] = hp[i];
            if (idx)
                for (int64_t i = 0; i < sk->k_nnz; ++i) idx[i] = hi[i];
            if (vals && sk->k_nnz) RLA_CUDA_TRY(ctx, cudaMemcpy(vals, dval, sk->k_nnz * es, cudaMemcpyDeviceToHost));
        }
    } else if (kind == RLA_GAUSSIAN) {
        if (vals) RLA_CUDA_TRY(ctx, cudaMemcpy(vals, sk->dense, sk->n_rows * sk->n_cols * es, cudaMemcpyDeviceToHost));
    }
    return RLA_OK;
}

int rla_sketch_set_draws(rla_ctx *ctx, rla_sketch *sk, const int64_t *idx, const void *vals, const uint8_t *signs,
                         const int64_t *kptr, int64_t k_nnz) {
    if (!ctx || !sk) return RLA_E_ARG;
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    const int kind = sk->p.kind;
    const size_t es = dtype_size(sk->p.dtype);
    auto val_at = [&](size_t i) -> double { return es == 4 ? (double)((const float *)vals)[i] : ((const double *)vals)[i]; };
    if (kind == RLA_SAMPLING) {
        if (!idx) return set_error(ctx, RLA_E_ARG, "Sampling draws need the indices.");
        return sampling_set_indices(ctx, sk, idx);
    }
    if (kind == RLA_SPARSE_SIGN || kind == RLA_COUNT_SKETCH) {
        if (!idx || !vals) return set_error(ctx, RLA_E_ARG, "Sparse draws need indices and values.");
        size_t ne = (size_t)(sk->L * sk->nnz);
        std::vector<int32_t> b(ne);
        std::vector<uint8_t> ng(ne);
        for (size_t i = 0; i < ne; ++i) {
            if (idx[i] < 0 || idx[i] >= sk->s)
                return set_error(ctx, RLA_E_ARG, "Row index %lld out of range 0:%lld.", (long long)idx[i], (long long)sk->s - 1);
            b[i] = (int32_t)idx[i];
            double v = val_at(i);
            if (v == sk->scale) ng[i] = 0;
            else if (v == -sk->scale) ng[i] = 1;
            else
                return set_error(ctx, RLA_E_ARG, "Nonzero values must be +-%.17g (the compressor's scale).", sk->scale);
        }
        RLA_CUDA_TRY(ctx, cudaMemcpy(sk->bucket, b.data(), ne * 4, cudaMemcpyHostToDevice));
        RLA_CUDA_TRY(ctx, cudaMemcpy(sk->negative, ng.data(), ne, cudaMemcpyHostToDevice));
        RLA_TRY(build_meta(ctx, sk));
    } else if (kind == RLA_SRHT || kind == RLA_FJLT) {
        if (!signs) return set_error(ctx, RLA_E_ARG, "SRHT/FJLT draws need signs.");
        int64_t nw = ceil_div(sk->N, 32);
        std::vector<uint32_t> w(nw, 0);
        for (int64_t r = 0; r < sk->N; ++r) w[r >> 5] |= (signs[r] ? 1u : 0u) << (r & 31);
        RLA_CUDA_TRY(ctx, cudaMemcpy(sk->signbits, w.data(), nw * 4, cudaMemcpyHostToDevice));
        if (kind == RLA_SRHT) {
            if (!idx) return set_error(ctx, RLA_E_ARG, "SRHT draws need the sampled rows.");
            std::vector<int32_t> r(sk->s);
            for (int64_t i = 0; i < sk->s; ++i) {
                if (idx[i] < 0 || idx[i] >= sk->N)
                    return set_error(ctx, RLA_E_ARG, "Sampled row %lld out of range 0:%lld.", (long long)idx[i], (long long)sk->N - 1);
                r[i] = (int32_t)idx[i];
            }
            RLA_CUDA_TRY(ctx, cudaMemcpy(sk->rows, r.data(), sk->s * 4, cudaMemcpyHostToDevice));
            RLA_TRY(srht_tables(ctx, sk));
            RLA_TRY(build_srht_sign_table(ctx, sk));
        } else {
            if (!idx || !vals || !kptr) return set_error(ctx, RLA_E_ARG, "FJLT draws need op.colptr, op.rowval and op.nzval.");
            bool left = sk->p.card == RLA_LEFT;
            // Given CSC of op: Left op = Kc (s x N) -> CSC == CSR of Kc' (N rows of s);
            // Right op = Kc' (N x s) -> CSC == CSR of Kc (s rows of N).  Build CSR of Kc.
            int64_t ncol = left ? sk->N : sk->s;
            int64_t nrow = left ? sk->s : sk->N;
            if (kptr[0] != 0 || kptr[ncol] != k_nnz) return set_error(ctx, RLA_E_ARG, "Inconsistent op.colptr.");
            for (int64_t c = 0; c < ncol; ++c)
                if (kptr[c + 1] < kptr[c]) return set_error(ctx, RLA_E_ARG, "op.colptr must be nondecreasing.");
            for (int64_t k = 0; k < k_nnz; ++k)
                if (idx[k] < 0 || idx[k] >= nrow) return set_error(ctx, RLA_E_ARG, "op.rowval out of range.");
            std::vector<int32_t> cp(sk->s + 1, 0), cc(std::max<int64_t>(k_nnz, 1));
            std::vector<char> cv(std::max<int64_t>(k_nnz, 1) * es);
            if (!left) {
                for (int64_t c = 0; c <= sk->s; ++c) cp[c] = (int32_t)kptr[c];
                for (int64_t k = 0; k < k_nnz; ++k) cc[k] = (int32_t)idx[k];
                memcpy(cv.data(), vals, k_nnz * es);
            } else {
                for (int64_t k = 0; k < k_nnz; ++k) cp[idx[k] + 1]++;
                for (int64_t i = 0; i < sk->s; ++i) cp[i + 1] += cp[i];
                std::vector<int32_t> fill(cp.begin(), cp.end() - 1);
                for (int64_t c = 0; c < ncol; ++c)
                    for (int64_t k = kptr[c]; k < kptr[c + 1]; ++k) {
                        int32_t d = fill[idx[k]]++;
                        cc[d] = (int32_t)c;
                        memcpy(cv.data() + d * es, (const char *)vals + k * es, es);
                    }
            }
            if (sk->k_ptr) cudaFree(sk->k_ptr);
            if (sk->k_col) cudaFree(sk->k_col);
            if (sk->k_val) cudaFree(sk->k_val);
            sk->k_ptr = sk->k_col = nullptr;
            sk->k_val = nullptr;
            RLA_CUDA_TRY(ctx, cudaMalloc(&sk->k_ptr, (sk->s + 1) * 4));
            RLA_CUDA_TRY(ctx, cudaMalloc(&sk->k_col, std::max<int64_t>(k_nnz, 1) * 4));
            RLA_CUDA_TRY(ctx, cudaMalloc(&sk->k_val, std::max<int64_t>(k_nnz, 1) * es));
            RLA_CUDA_TRY(ctx, cudaMemcpy(sk->k_ptr, cp.data(), (sk->s + 1) * 4, cudaMemcpyHostToDevice));
            if (k_nnz) {
                RLA_CUDA_TRY(ctx, cudaMemcpy(sk->k_col, cc.data(), k_nnz * 4, cudaMemcpyHostToDevice));
                RLA_CUDA_TRY(ctx, cudaMemcpy(sk->k_val, cv.data(), k_nnz * es, cudaMemcpyHostToDevice));
            }
            sk->k_nnz = k_nnz;
            if (sk->p.dtype == RLA_F32) RLA_TRY(fjlt_transpose<float>(ctx, sk));
            else RLA_TRY(fjlt_transpose<double>(ctx, sk));
        }
    } else if (kind == RLA_GAUSSIAN) {
        if (!vals) return set_error(ctx, RLA_E_ARG, "Gaussian draws need values.");
        RLA_CUDA_TRY(ctx, cudaMemcpy(sk->dense, vals, sk->n_rows * sk->n_cols * es, cudaMemcpyHostToDevice));
    }
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

}  // extern "C"
