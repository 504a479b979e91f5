// rla_sampling.cu -- the Sampling compressor (src/Compressors/sampling.jl) with its
// distributions Uniform, L2Norm and Agmon (src/Compressors/Distributions/*.jl).
//
// A Sampling recipe is a selection matrix P (s x L, P(i, idx(i)) = 1): S = P for Left
// cardinality, S = P' for Right.  In the compress/expand terms of rla_api.cu, compress is a
// gather y(i) = x(idx(i)) (view(A, idx, :), sampling.jl:145-157) and expand is a scatter-add
// y = beta*y, then y(idx(i)) += alpha*x(i) in i order (sampling.jl:160-218, where repeated
// indices of a with-replacement draw accumulate).
//
// Draws are made on the device from the sketch's seed and draw count (Julia's StatsBase
// streams are not reproduced; the distribution of the draw is):
//  * with replacement, ordered (wsample!(..., ordered = true, replace = true)): s sorted
//    uniform order statistics on [0, W) from prefix sums of s+1 Exp(1) draws, mapped
//    through the inclusive prefix sum of the weights (upper bound), so the indices come out
//    sorted without a sort;
//  * without replacement, ordered: Efraimidis-Spirakis keys E_j / w_j (E_j ~ Exp(1)), the s
//    smallest selected by an MSB-first radix select over the keys' bit patterns, then
//    compacted in index order;
//  * Agmon (agmon.jl): beta candidates (all indices when beta >= the dimension, else uniform
//    with or without replacement), residuals |A(c,:)x - b(c)| (Left) or |A(:,c)'(Ax - b)|
//    (Right), and the k largest by (-residual, candidate) in that order.
// The weights of L2Norm are the squared row (Left) or column (Right) norms of A in FP64.
#include <math.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

enum : uint32_t { STREAM_SAMPLE_EXP = 9, STREAM_SAMPLE_KEYS = 10, STREAM_SAMPLE_CAND = 11, STREAM_SAMPLE_FLOYD = 12 };

// ---- weights ----------------------------------------------------------------------
template <class T>
__global__ void sq_norms_rows_kernel(const T *A, int64_t lda, int64_t m, int64_t n, double *w) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    double acc = 0.0;
    for (int64_t j = 0; j < n; ++j) {
        const double v = (double)A[i + j * lda];
        acc += v * v;
    }
    w[i] = acc;
}

template <class T>
__global__ void sq_norms_cols_kernel(const T *A, int64_t lda, int64_t m, int64_t n, double *w) {
    const int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= n) return;
    double acc = 0.0;
    for (int64_t i = lane; i < m; i += 32) {
        const double v = (double)A[i + j * lda];
        acc += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if (lane == 0) w[j] = acc;
}

// ---- inclusive prefix sum (one CTA; w == nullptr means all ones) --------------------
__global__ void __launch_bounds__(1024) scan_f64_kernel(const double *w, int64_t n, double *out) {
    __shared__ double part[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int64_t per = (n + nt - 1) / nt, lo = min(n, (int64_t)t * per), hi = min(n, lo + per);
    double sum = 0.0;
    for (int64_t i = lo; i < hi; ++i) sum += w ? w[i] : 1.0;
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        const double v = t >= off ? part[t - off] : 0.0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    double run = part[t] - sum;
    for (int64_t i = lo; i < hi; ++i) {
        run += w ? w[i] : 1.0;
        out[i] = run;
    }
}

__global__ void exp_draw_kernel(Rng rng, int64_t k, double *e) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= k) return;
    const P4 r = rng.at(STREAM_SAMPLE_EXP, (uint64_t)i);
    e[i] = -log(u01_open_d(r.x, r.y));
}

// idx(i) = the first j with cdf(j) > W * P(i) / P(s): the (i+1)-th of s sorted draws.
__global__ void cdf_search_kernel(const double *P, int64_t s, const double *cdf, int64_t L, int64_t *idx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= s) return;
    const double u = cdf[L - 1] * (P[i] / P[s]);
    int64_t lo = 0, hi = L - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    idx[i] = lo;
}

// ---- selection of the k smallest 64-bit keys ----------------------------------------
// key_j = E_j / w_j as an IEEE bit pattern (positive doubles order like their bits;
// w_j = 0 gives +inf, which is never selected while positive weights remain).
__global__ void es_keys_kernel(Rng rng, int64_t L, const double *w, uint64_t *key) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= L) return;
    const P4 r = rng.at(STREAM_SAMPLE_KEYS, (uint64_t)j);
    const double e = -log(u01_open_d(r.x, r.y));
    const double wj = w ? w[j] : 1.0;
    const double k = wj > 0.0 ? e / wj : INFINITY;
    key[j] = (uint64_t)__double_as_longlong(k);
}

// Uniform sampling without replacement for small s: Floyd's algorithm (Bentley and Floyd,
// "A sample of brilliance", CACM 30(9), 1987).  For j = L-s .. L-1 take t uniform in [0, j],
// or j when t was taken already; every s-subset of [0, L) is equally likely.  One warp: lane
// 0 draws, the warp tests membership in the shared-memory list, then sorts the list
// (bitonic) so the indices come out in increasing order like the selection path's.
constexpr int FLOYD_MAX = 256;

__global__ void __launch_bounds__(32) floyd_sample_kernel(Rng rng, int64_t L, int s, int64_t *idx) {
    __shared__ uint32_t set[FLOYD_MAX];
    const int lane = threadIdx.x;
    WordStream ws{rng, STREAM_SAMPLE_FLOYD, 0};
    for (int i = 0; i < s; ++i) {
        const uint32_t j = (uint32_t)(L - s + i);
        uint32_t t = 0;
        if (lane == 0) t = uniform_below(j + 1u, ws);
        t = __shfl_sync(FULL, t, 0);
        bool hit = false;
        for (int q = lane; q < i; q += 32) hit |= set[q] == t;
        hit = __any_sync(FULL, hit);
        if (lane == 0) set[i] = hit ? j : t;
        __syncwarp();
    }
    int P = 1;
    while (P < s) P <<= 1;
    for (int q = s + lane; q < P; q += 32) set[q] = 0xffffffffu;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
        for (int h = k >> 1; h > 0; h >>= 1) {
            for (int q = lane; q < P; q += 32) {
                const int o = q ^ h;
                if (o > q) {
                    const uint32_t a = set[q], b = set[o];
                    const bool up = (q & k) == 0;
                    if ((a > b) == up) {
                        set[q] = b;
                        set[o] = a;
                    }
                }
            }
            __syncwarp();
        }
    for (int q = lane; q < s; q += 32) idx[q] = (int64_t)set[q];
}

// Radix-select state in device memory: the known high bits of the threshold key, their
// mask, and the rank of the threshold among the keys that share them.
struct SelState {
    uint64_t prefix, mask;
    int64_t rem;
};

__global__ void sel_init_kernel(SelState *st, int64_t k, unsigned *hist) {
    if (threadIdx.x == 0) {
        st->prefix = 0;
        st->mask = 0;
        st->rem = k;
    }
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
}

__global__ void radix_hist_kernel(const uint64_t *key, int64_t n, const SelState *st, int shift, unsigned *hist) {
    __shared__ unsigned h[256];
    const uint64_t prefix = st->prefix, mask = st->mask;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[j];
        if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// The digit at `shift` of the threshold: the first digit whose cumulative count reaches
// the remaining rank.  One CTA of 256 threads; the histogram is cleared for the next pass.
__global__ void radix_pick_kernel(SelState *st, unsigned *hist, int shift) {
    __shared__ int64_t inc[256];
    const int t = threadIdx.x;
    const int64_t h = hist[t];
    inc[t] = h;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {  // inclusive prefix sums of the counts
        const int64_t v = t >= off ? inc[t - off] : 0;
        __syncthreads();
        inc[t] += v;
        __syncthreads();
    }
    const int64_t rem = st->rem, before = inc[t] - h;
    // the digit whose bucket holds the rem-th key (the last one if rounding ever overshoots)
    if ((before < rem && rem <= inc[t]) || (t == 255 && rem > inc[255])) {
        st->rem = rem - before;
        st->prefix |= (uint64_t)t << shift;
        st->mask |= (uint64_t)255 << shift;
    }
    hist[t] = 0;
}

// count(key < T) by atomics on a 64-bit counter (integer sums are order-independent).
__global__ void count_below_kernel(const uint64_t *key, int64_t n, uint64_t T, unsigned long long *count) {
    __shared__ unsigned c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    unsigned mine = 0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        mine += key[j] < T;
    atomicAdd(&c, mine);
    __syncthreads();
    if (threadIdx.x == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// err = count + 1 when fewer than s keys are below +inf (positive weights), else unchanged.
__global__ void check_positive_kernel(const unsigned long long *count, int64_t s, int64_t *err) {
    if ((int64_t)*count < s) *err = (int64_t)*count + 1;
}

// err = -1 when the weights do not sum to a positive finite number.
__global__ void check_sum_kernel(const double *cdf, int64_t L, int64_t *err) {
    const double W = cdf[L - 1];
    if (!(W > 0.0) || !isfinite(W)) *err = -1;
}

// Exclusive scans of the two block-count arrays (one CTA).
__global__ void __launch_bounds__(1024) scan2_kernel(const int64_t *a, const int64_t *b, int64_t n, int64_t *oa,
                                                     int64_t *ob) {
    __shared__ int64_t pa[1024], pb[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int64_t per = (n + nt - 1) / nt, lo = min(n, (int64_t)t * per), hi = min(n, lo + per);
    int64_t sa = 0, sb = 0;
    for (int64_t i = lo; i < hi; ++i) {
        sa += a[i];
        sb += b[i];
    }
    pa[t] = sa;
    pb[t] = sb;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        const int64_t va = t >= off ? pa[t - off] : 0, vb = t >= off ? pb[t - off] : 0;
        __syncthreads();
        pa[t] += va;
        pb[t] += vb;
        __syncthreads();
    }
    int64_t ra = pa[t] - sa, rb = pb[t] - sb;
    for (int64_t i = lo; i < hi; ++i) {
        oa[i] = ra;
        ob[i] = rb;
        ra += a[i];
        rb += b[i];
    }
}

// Per 1024-element block: how many keys are below T and how many equal it.
__global__ void __launch_bounds__(1024) select_count_kernel(const uint64_t *key, int64_t n, const SelState *st,
                                                            int64_t *blk_lt, int64_t *blk_eq) {
    __shared__ int wl[32], we[32];
    const uint64_t T = st->prefix;
    const int64_t j = blockIdx.x * 1024ll + threadIdx.x;
    const uint64_t k = j < n ? key[j] : ~0ull;
    const unsigned bl = __ballot_sync(FULL, j < n && k < T), be = __ballot_sync(FULL, j < n && k == T);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        wl[w] = __popc(bl);
        we[w] = __popc(be);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t a = 0, b = 0;
        for (int i = 0; i < 32; ++i) {
            a += wl[i];
            b += we[i];
        }
        blk_lt[blockIdx.x] = a;
        blk_eq[blockIdx.x] = b;
    }
}

// The selected set is {key < T} plus the first `need` keys equal to T (index order); a
// selected j lands at lt_before(j) + min(eq_before(j), need), so the output is in index
// order.  off_lt / off_eq: exclusive prefix sums of the block counts.
__global__ void __launch_bounds__(1024) select_write_kernel(const uint64_t *key, int64_t n, const SelState *st,
                                                            const int64_t *off_lt, const int64_t *off_eq,
                                                            const int64_t *cand, int64_t *out) {
    __shared__ int wl[32], we[32];
    const uint64_t T = st->prefix;
    const int64_t need = st->rem;
    const int64_t j = blockIdx.x * 1024ll + threadIdx.x;
    const uint64_t k = j < n ? key[j] : ~0ull;
    const bool lt = j < n && k < T, eq = j < n && k == T;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned bl = __ballot_sync(FULL, lt), be = __ballot_sync(FULL, eq);
    if (lane == 0) {
        wl[w] = __popc(bl);
        we[w] = __popc(be);
    }
    __syncthreads();
    int bl_before = 0, be_before = 0;
    for (int i = 0; i < w; ++i) {
        bl_before += wl[i];
        be_before += we[i];
    }
    const unsigned below = (1u << lane) - 1u;
    const int64_t ltb = off_lt[blockIdx.x] + bl_before + __popc(bl & below);
    const int64_t eqb = off_eq[blockIdx.x] + be_before + __popc(be & below);
    if (lt || (eq && eqb < need)) out[ltb + min(eqb, need)] = cand ? cand[j] : j;
}

// ---- Agmon --------------------------------------------------------------------------
__global__ void cand_uniform_kernel(Rng rng, int64_t beta, int64_t L, int64_t *cand) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= beta) return;
    WordStream ws{rng, STREAM_SAMPLE_CAND, (uint64_t)i * 4};
    cand[i] = uniform_below((uint32_t)L, ws);
}

// res(p) = |A(c,:) x - b(c)| for Left (or |r(c)| when r is given), c = cand(p) (or p).
template <class T>
__global__ void agmon_res_left_kernel(const T *A, int64_t lda, int64_t n, const T *x, const T *b, const T *r,
                                      const int64_t *cand, int64_t nc, double *res) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= nc) return;
    const int64_t c = cand ? cand[p] : p;
    double v;
    if (r) {
        v = (double)r[c];
    } else {
        v = -(double)b[c];
        for (int64_t j = 0; j < n; ++j) v += (double)A[c + j * lda] * (double)x[j];
    }
    res[p] = fabs(v);
}

// rv = A x - b (m rows), one thread per row.
template <class T>
__global__ void agmon_rv_kernel(const T *A, int64_t lda, int64_t m, int64_t n, const T *x, const T *b, double *rv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    double v = -(double)b[i];
    for (int64_t j = 0; j < n; ++j) v += (double)A[i + j * lda] * (double)x[j];
    rv[i] = v;
}

// res(p) = |A(:, c)' rv| for Right, one warp per candidate (rv in FP64, or the given r).
template <class T>
__global__ void agmon_res_right_kernel(const T *A, int64_t lda, int64_t m, const double *rv, const T *r,
                                       const int64_t *cand, int64_t nc, double *res) {
    const int64_t p = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= nc) return;
    const int64_t c = cand ? cand[p] : p;
    double acc = 0.0;
    for (int64_t i = lane; i < m; i += 32) acc += (double)A[i + c * lda] * (r ? (double)r[i] : rv[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if (lane == 0) res[p] = fabs(acc);
}

// Larger residual first: the key is the complement of the residual's bit pattern.
__global__ void res_keys_kernel(const double *res, int64_t nc, uint64_t *key) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= nc) return;
    key[p] = ~(uint64_t)__double_as_longlong(res[p]);
}

// Sort the k selected candidates by (-residual, candidate): one CTA, odd-even merge-free
// bitonic sort of (key, candidate) pairs padded to a power of two in shared memory.
__global__ void __launch_bounds__(1024) agmon_order_kernel(const int64_t *sel, int64_t k, const double *res_of,
                                                           const int64_t *pos_of, int64_t *idx) {
    __shared__ double rs[1024];
    __shared__ int64_t cs[1024];
    int np = 1;
    while (np < k) np <<= 1;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        if (i < k) {
            rs[i] = res_of[pos_of[i]];
            cs[i] = sel[i];
        } else {
            rs[i] = -1.0;
            cs[i] = INT64_MAX;
        }
    }
    __syncthreads();
    auto before = [&](int a, int b) { return rs[a] > rs[b] || (rs[a] == rs[b] && cs[a] < cs[b]); };
    for (int size = 2; size <= np; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < np; i += blockDim.x) {
                const int jx = i ^ stride;
                if (jx > i) {
                    const bool up = (i & size) == 0;
                    if (up ? before(jx, i) : before(i, jx)) {
                        const double tr = rs[i];
                        rs[i] = rs[jx];
                        rs[jx] = tr;
                        const int64_t tc = cs[i];
                        cs[i] = cs[jx];
                        cs[jx] = tc;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < k; i += blockDim.x) idx[i] = cs[i];
}

// ---- apply ----------------------------------------------------------------------------
// compress: Y(i, v) = alpha * X(idx(i), v) + beta * Y(i, v); the fastest-varying thread
// index follows whichever of the element or vector stride of X is 1.
template <class T>
__global__ void sample_gather_kernel(const T *X, int64_t x_es, int64_t x_vs, int64_t nv, const int64_t *idx,
                                     int64_t s, T *Y, int64_t y_es, int64_t y_vs, T alpha, T beta, int beta_zero,
                                     int v_fast) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= s * nv) return;
    const int64_t i = v_fast ? t / nv : t % s, v = v_fast ? t % nv : t / s;
    T *yp = Y + i * y_es + v * y_vs;
    const T val = alpha * X[idx[i] * x_es + v * x_vs];
    *yp = beta_zero ? val : val + beta * *yp;
}

// expand, step 1: Y = beta * Y over all L x nv entries (zero when beta == 0).
template <class T>
__global__ void sample_scale_kernel(T *Y, int64_t y_es, int64_t y_vs, int64_t L, int64_t nv, T beta, int beta_zero,
                                    int v_fast) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= L * nv) return;
    const int64_t i = v_fast ? t / nv : t % L, v = v_fast ? t % nv : t / L;
    T *yp = Y + i * y_es + v * y_vs;
    *yp = beta_zero ? T(0) : beta * *yp;
}

// expand, step 2: for every distinct target u, Y(tgt(u), v) += alpha * X(p, v) for the
// positions p of u in increasing order (the reference's accumulation order).
// plan layout [tgt: s][run_ptr: s+1][run_pos: s][U]; threads u >= U exit.
template <class T>
__global__ void sample_scatter_kernel(const T *X, int64_t x_es, int64_t x_vs, int64_t nv, const int64_t *plan,
                                      int64_t s, T *Y, int64_t y_es, int64_t y_vs, T alpha, int v_fast) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= s * nv) return;
    const int64_t u = v_fast ? t / nv : t % s, v = v_fast ? t % nv : t / s;
    if (u >= plan[3 * s + 1]) return;
    const int64_t *tgt = plan, *run_ptr = plan + s, *run_pos = plan + 2 * s + 1;
    T *yp = Y + tgt[u] * y_es + v * y_vs;
    T acc = *yp;
    for (int64_t q = run_ptr[u]; q < run_ptr[u + 1]; ++q) acc += alpha * X[run_pos[q] * x_es + v * x_vs];
    *yp = acc;
}

__global__ void pos_to_cand_kernel(const int64_t *pos, int64_t k, const int64_t *cand, int64_t *sel) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < k) sel[i] = cand ? cand[pos[i]] : pos[i];
}

// ---- host side ----------------------------------------------------------------------
static Rng sampling_rng(const rla_sketch *sk) {
    Rng r;
    r.k0 = (uint32_t)sk->p.seed;
    r.k1 = (uint32_t)(sk->p.seed >> 32);
    r.epoch = (uint32_t)sk->draw_count;
    return r;
}

static int sel_check(rla_ctx *ctx, const char *what) { return check_launch(ctx, what); }

// The k smallest keys of key[0:n) (k <= n), written to out in index order (cand maps
// positions to indices when given).  Everything stays on the stream: 8 histogram/pick pairs
// over the key bytes (MSB first), block counts, their scans, the ordered write.
static int select_smallest(rla_ctx *ctx, const uint64_t *key, int64_t n, int64_t k, const int64_t *cand,
                           int64_t *out) {
    const int64_t nb = ceil_div(n, 1024);
    void *p = nullptr;
    const size_t st_bytes = 64, hist_bytes = 256 * sizeof(unsigned);
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &p, st_bytes + hist_bytes + sizeof(int64_t) * 4 * nb, ctx->stream));
    SelState *st = (SelState *)p;
    unsigned *hist = (unsigned *)((char *)p + st_bytes);
    int64_t *blk = (int64_t *)((char *)p + st_bytes + hist_bytes);
    sel_init_kernel<<<1, 256, 0, ctx->stream>>>(st, k, hist);
    const int gb = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), 4 * (int64_t)ctx->sm_count));
    for (int shift = 56; shift >= 0; shift -= 8) {
        radix_hist_kernel<<<gb, 256, 0, ctx->stream>>>(key, n, st, shift, hist);
        radix_pick_kernel<<<1, 256, 0, ctx->stream>>>(st, hist, shift);
    }
    select_count_kernel<<<(unsigned)nb, 1024, 0, ctx->stream>>>(key, n, st, blk, blk + nb);
    scan2_kernel<<<1, 1024, 0, ctx->stream>>>(blk, blk + nb, nb, blk + 2 * nb, blk + 3 * nb);
    select_write_kernel<<<(unsigned)nb, 1024, 0, ctx->stream>>>(key, n, st, blk + 2 * nb, blk + 3 * nb, cand, out);
    RLA_TRY(sel_check(ctx, "select_smallest"));
    RLA_CUDA_TRY(ctx, cudaFreeAsync(p, ctx->stream));
    return RLA_OK;
}

// Expand plan of sorted indices on the device: targets are the run heads, positions the
// identity.  One CTA; plan layout [tgt: s][ptr: s+1][pos: s][U].
__global__ void __launch_bounds__(1024) plan_sorted_kernel(const int64_t *idx, int64_t s, int64_t *plan) {
    __shared__ int64_t part[1024];
    int64_t *tgt = plan, *ptr = plan + s, *pos = plan + 2 * s + 1, *U = plan + 3 * s + 1;
    const int t = threadIdx.x, nt = blockDim.x;
    const int64_t per = (s + nt - 1) / nt, lo = min(s, (int64_t)t * per), hi = min(s, lo + per);
    int64_t c = 0;
    for (int64_t i = lo; i < hi; ++i) c += (i == 0 || idx[i] != idx[i - 1]);
    part[t] = c;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        const int64_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int64_t u = part[t] - c;
    for (int64_t i = lo; i < hi; ++i) {
        pos[i] = i;
        if (i == 0 || idx[i] != idx[i - 1]) {
            tgt[u] = idx[i];
            ptr[u] = i;
            ++u;
        }
    }
    if (t == nt - 1) {
        ptr[part[t]] = s;
        *U = part[t];
    }
}

// Expand plan from the current indices: distinct targets with their positions in order.
static int sampling_plan(rla_ctx *ctx, rla_sketch *sk) {
    const int64_t s = sk->s;
    std::vector<int64_t> h(s);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), sk->sidx, sizeof(int64_t) * s, cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int64_t> pos(s);
    std::iota(pos.begin(), pos.end(), 0);
    if (!std::is_sorted(h.begin(), h.end()))
        std::stable_sort(pos.begin(), pos.end(), [&](int64_t a, int64_t b) { return h[a] < h[b]; });
    std::vector<int64_t> tgt, ptr;
    tgt.reserve(s);
    ptr.reserve(s + 1);
    for (int64_t q = 0; q < s; ++q)
        if (q == 0 || h[pos[q]] != h[pos[q - 1]]) {
            tgt.push_back(h[pos[q]]);
            ptr.push_back(q);
        }
    ptr.push_back(s);
    std::vector<int64_t> plan(3 * s + 2, 0);  // [tgt: s][ptr: s+1][pos: s][U]
    std::copy(tgt.begin(), tgt.end(), plan.begin());
    std::copy(ptr.begin(), ptr.end(), plan.begin() + s);
    std::copy(pos.begin(), pos.end(), plan.begin() + 2 * s + 1);
    plan[3 * s + 1] = (int64_t)tgt.size();
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->splan, plan.data(), sizeof(int64_t) * plan.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

// sample_distribution! for Uniform / L2Norm: `w` holds the weights (nullptr: uniform).
// Failed preconditions are flagged in sk->s_err (read by sampling_finish).
static int sample_weighted(rla_ctx *ctx, rla_sketch *sk, const double *w) {
    const int64_t s = sk->s, L = sk->L;
    Rng rng = sampling_rng(sk);
    if (sk->s_replace) {
        void *p = nullptr;
        RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &p, sizeof(double) * (L + 2 * (s + 1)), ctx->stream));
        double *cdf = (double *)p, *e = cdf + L, *P = e + (s + 1);
        scan_f64_kernel<<<1, 1024, 0, ctx->stream>>>(w, L, cdf);
        exp_draw_kernel<<<ceil_div_i(s + 1, 256), 256, 0, ctx->stream>>>(rng, s + 1, e);
        scan_f64_kernel<<<1, 1024, 0, ctx->stream>>>(e, s + 1, P);
        check_sum_kernel<<<1, 1, 0, ctx->stream>>>(cdf, L, sk->s_err);
        cdf_search_kernel<<<ceil_div_i(s, 256), 256, 0, ctx->stream>>>(P, s, cdf, L, sk->sidx);
        RLA_TRY(check_launch(ctx, "sample_with_replacement"));
        RLA_CUDA_TRY(ctx, cudaFreeAsync(p, ctx->stream));
        return RLA_OK;
    }
    if (s > L)
        return set_error(ctx, RLA_E_ARG, "Cannot draw %lld samples from %lld samples without replacement.",
                         (long long)s, (long long)L);
    if (!w && s <= FLOYD_MAX) {  // uniform, few samples: one warp instead of a selection over L keys
        floyd_sample_kernel<<<1, 32, 0, ctx->stream>>>(rng, L, (int)s, sk->sidx);
        return check_launch(ctx, "floyd_sample");
    }
    void *p = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &p, sizeof(uint64_t) * L + 64, ctx->stream));
    uint64_t *key = (uint64_t *)p;
    unsigned long long *cnt = (unsigned long long *)(key + L);
    es_keys_kernel<<<ceil_div_i(L, 256), 256, 0, ctx->stream>>>(rng, L, w, key);
    RLA_TRY(check_launch(ctx, "es_keys"));
    if (w) {
        // at least s positive weights (keys below +inf)
        RLA_CUDA_TRY(ctx, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), ctx->stream));
        count_below_kernel<<<(int)std::min<int64_t>(ceil_div(L, 256), 4 * (int64_t)ctx->sm_count), 256, 0,
                             ctx->stream>>>(key, L, 0x7ff0000000000000ull, cnt);
        check_positive_kernel<<<1, 1, 0, ctx->stream>>>(cnt, s, sk->s_err);
    }
    int rc = select_smallest(ctx, key, L, s, nullptr, sk->sidx);
    cudaFreeAsync(p, ctx->stream);
    return rc;
}

// Read the precondition flags of the last draw (synchronises the stream).
static int sampling_finish(rla_ctx *ctx, rla_sketch *sk) {
    int64_t err = 0;
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&err, sk->s_err, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (err == 0) return RLA_OK;
    RLA_CUDA_TRY(ctx, cudaMemsetAsync(sk->s_err, 0, sizeof(int64_t), ctx->stream));
    if (err < 0) return set_error(ctx, RLA_E_ARG, "The sampling weights must have a positive finite sum.");
    return set_error(ctx, RLA_E_ARG, "Cannot draw %lld samples without replacement from %lld indices of positive weight.",
                     (long long)sk->s, (long long)(err - 1));
}

template <class T>
static int sample_agmon_t(rla_ctx *ctx, rla_sketch *sk, int64_t a_rows, int64_t a_cols, const T *A, int64_t lda,
                          const T *x, const T *b, const T *r) {
    const int64_t k = sk->s, L = sk->L, beta = sk->s_beta;
    Rng rng = sampling_rng(sk);
    if (beta == 1) {  // agmon.jl: indices[1] = rand(state_space)
        cand_uniform_kernel<<<1, 32, 0, ctx->stream>>>(rng, 1, L, sk->sidx);
        return check_launch(ctx, "agmon_single");
    }
    const bool all = beta >= L;
    const int64_t nc = all ? L : beta;
    void *p = nullptr;
    // cand [nc] | res [nc] | rv [a_rows] | key [max(nc, L)] | pos [k] | sel [k]
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &p, sizeof(int64_t) * nc + sizeof(double) * (nc + a_rows) +
                                                 sizeof(uint64_t) * std::max(nc, L) + 2 * sizeof(int64_t) * k,
                                   ctx->stream));
    int64_t *cand = (int64_t *)p;
    double *res = (double *)(cand + nc);
    double *rv = res + nc;
    uint64_t *key = (uint64_t *)(rv + a_rows);
    int64_t *pos = (int64_t *)(key + std::max(nc, L));
    int64_t *sel = pos + k;
    int rc = RLA_OK;
    if (!all) {
        if (sk->s_replace) {
            cand_uniform_kernel<<<ceil_div_i(nc, 256), 256, 0, ctx->stream>>>(rng, nc, L, cand);
            rc = check_launch(ctx, "agmon_candidates");
        } else {
            es_keys_kernel<<<ceil_div_i(L, 256), 256, 0, ctx->stream>>>(rng, L, nullptr, key);
            rc = select_smallest(ctx, key, L, nc, nullptr, cand);
        }
    }
    const int64_t *cp = all ? nullptr : cand;
    if (rc == RLA_OK) {
        if (sk->p.card == RLA_LEFT) {
            agmon_res_left_kernel<T><<<ceil_div_i(nc, 256), 256, 0, ctx->stream>>>(A, lda, a_cols, x, b, r, cp, nc, res);
        } else {
            if (!r) agmon_rv_kernel<T><<<ceil_div_i(a_rows, 256), 256, 0, ctx->stream>>>(A, lda, a_rows, a_cols, x, b, rv);
            agmon_res_right_kernel<T><<<ceil_div_i(nc * 32, 256), 256, 0, ctx->stream>>>(A, lda, a_rows, rv, r, cp, nc,
                                                                                         res);
        }
        res_keys_kernel<<<ceil_div_i(nc, 256), 256, 0, ctx->stream>>>(res, nc, key);
        rc = check_launch(ctx, "agmon_residuals");
    }
    // positions of the k largest residuals (ties: earlier position), then the candidates
    // they name, ordered by (-residual, candidate)
    if (rc == RLA_OK) rc = select_smallest(ctx, key, nc, k, nullptr, pos);
    if (rc == RLA_OK) {
        pos_to_cand_kernel<<<ceil_div_i(k, 256), 256, 0, ctx->stream>>>(pos, k, cp, sel);
        agmon_order_kernel<<<1, 1024, 0, ctx->stream>>>(sel, k, res, pos, sk->sidx);
        rc = check_launch(ctx, "agmon_order");
    }
    cudaFreeAsync(p, ctx->stream);
    return rc;
}


// Draw for the current distribution.  Uniform needs no data; L2Norm uses the weights of the
// last rla_sampling_update (or those passed in); Agmon needs x, A, b every time.
int sampling_draw(rla_ctx *ctx, rla_sketch *sk, bool sync) {
    int rc = RLA_OK;
    if (sk->s_dist == RLA_DIST_UNIFORM) rc = sample_weighted(ctx, sk, nullptr);
    else if (sk->s_dist == RLA_DIST_L2NORM) {
        if (!sk->s_has_weights)
            return set_error(ctx, RLA_E_ARG, "`L2Norm` sampling needs A: call rla_sampling_update first.");
        rc = sample_weighted(ctx, sk, sk->sweights);
    } else
        return set_error(ctx, RLA_E_ARG, "`Agmon` sampling needs x, A and b: use rla_sampling_update.");
    if (rc == RLA_OK) {
        plan_sorted_kernel<<<1, 1024, 0, ctx->stream>>>(sk->sidx, sk->s, sk->splan);
        rc = check_launch(ctx, "plan_sorted");
    }
    if (rc == RLA_OK && sync) rc = sampling_finish(ctx, sk);
    return rc;
}

template <class T>
static int sampling_update_t(rla_ctx *ctx, rla_sketch *sk, int64_t a_rows, int64_t a_cols, const T *A, int64_t lda,
                             const T *x, const T *b, const T *r) {
    if (sk->s_dist == RLA_DIST_L2NORM) {
        cudaEvent_t e0 = timing_begin(ctx);
        if (sk->p.card == RLA_LEFT)
            sq_norms_rows_kernel<T><<<ceil_div_i(a_rows, 256), 256, 0, ctx->stream>>>(A, lda, a_rows, a_cols, sk->sweights);
        else
            sq_norms_cols_kernel<T><<<ceil_div_i(a_cols * 32, 256), 256, 0, ctx->stream>>>(A, lda, a_rows, a_cols,
                                                                                         sk->sweights);
        timing_end(ctx, 3, e0);
        RLA_TRY(check_launch(ctx, "l2norm_weights"));
        sk->s_has_weights = true;
        RLA_TRY(sample_weighted(ctx, sk, sk->sweights));
    } else if (sk->s_dist == RLA_DIST_UNIFORM) {
        RLA_TRY(sample_weighted(ctx, sk, nullptr));
    } else {
        // Agmon's indices come in residual order: the plan is built on the host
        RLA_TRY(sample_agmon_t<T>(ctx, sk, a_rows, a_cols, A, lda, x, b, r));
        return sampling_plan(ctx, sk);
    }
    plan_sorted_kernel<<<1, 1024, 0, ctx->stream>>>(sk->sidx, sk->s, sk->splan);
    return check_launch(ctx, "plan_sorted");
}

int sampling_update(rla_ctx *ctx, rla_sketch *sk, int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                    const void *x, const void *b, const void *r) {
    if (sk->p.dtype == RLA_F32)
        return sampling_update_t<float>(ctx, sk, a_rows, a_cols, (const float *)A, lda, (const float *)x,
                                        (const float *)b, (const float *)r);
    return sampling_update_t<double>(ctx, sk, a_rows, a_cols, (const double *)A, lda, (const double *)x,
                                     (const double *)b, (const double *)r);
}

template <class T>
int sampling_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                      int64_t y_es, int64_t y_vs, double alpha, double beta) {
    const int64_t tot = sk->s * nv;
    if (tot == 0) return RLA_OK;
    sample_gather_kernel<T><<<ceil_div_i(tot, 256), 256, 0, ctx->stream>>>(
        X, x_es, x_vs, nv, sk->sidx, sk->s, Y, y_es, y_vs, (T)alpha, (T)beta, beta == 0.0, x_es != 1 ? 1 : 0);
    return check_launch(ctx, "sample_gather");
}

template <class T>
int sampling_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                    int64_t y_es, int64_t y_vs, double alpha, double beta) {
    const int v_fast = y_es != 1 ? 1 : 0;
    if (beta != 1.0 && sk->L * nv > 0) {
        sample_scale_kernel<T><<<ceil_div_i(sk->L * nv, 256), 256, 0, ctx->stream>>>(Y, y_es, y_vs, sk->L, nv, (T)beta,
                                                                                    beta == 0.0, v_fast);
        RLA_TRY(check_launch(ctx, "sample_scale"));
    }
    if (sk->s * nv == 0) return RLA_OK;
    sample_scatter_kernel<T><<<ceil_div_i(sk->s * nv, 256), 256, 0, ctx->stream>>>(X, x_es, x_vs, nv, sk->splan, sk->s,
                                                                                    Y, y_es, y_vs, (T)alpha, v_fast);
    return check_launch(ctx, "sample_scatter");
}

template int sampling_compress<float>(rla_ctx *, const rla_sketch *, const float *, int64_t, int64_t, int64_t, float *,
                                      int64_t, int64_t, double, double);
template int sampling_compress<double>(rla_ctx *, const rla_sketch *, const double *, int64_t, int64_t, int64_t,
                                       double *, int64_t, int64_t, double, double);
template int sampling_expand<float>(rla_ctx *, const rla_sketch *, const float *, int64_t, int64_t, int64_t, float *,
                                    int64_t, int64_t, double, double);
template int sampling_expand<double>(rla_ctx *, const rla_sketch *, const double *, int64_t, int64_t, int64_t,
                                     double *, int64_t, int64_t, double, double);

// Load externally supplied indices (parity mode) and rebuild the expand plan.
int sampling_set_indices(rla_ctx *ctx, rla_sketch *sk, const int64_t *idx) {
    for (int64_t i = 0; i < sk->s; ++i)
        if (idx[i] < 0 || idx[i] >= sk->L)
            return set_error(ctx, RLA_E_ARG, "Index %lld out of range 0:%lld.", (long long)idx[i], (long long)sk->L - 1);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(sk->sidx, idx, sizeof(int64_t) * sk->s, cudaMemcpyHostToDevice, ctx->stream));
    return sampling_plan(ctx, sk);
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_sampling_create(rla_ctx *ctx, int card, int dtype, int64_t compression_dim, int64_t long_dim,
                        int distribution, int replace, int64_t beta, uint64_t seed, rla_sketch **out) {
    if (!ctx || !out) return RLA_E_ARG;
    *out = nullptr;
    // Sampling / distribution constructor checks (sampling.jl:50-61, agmon.jl Agmon)
    if (compression_dim <= 0) return set_error(ctx, RLA_E_ARG, "Field `compression_dim` must be positive.");
    if (card != RLA_LEFT && card != RLA_RIGHT)
        return set_error(ctx, RLA_E_ARG,
                         "`cardinality` must be specified as `Left()` or `Right()`.`Undef()` is not allowed in "
                         "`Sampling` structure.");
    if (dtype != RLA_F32 && dtype != RLA_F64) return set_error(ctx, RLA_E_ARG, "Element type must be Float32 or Float64.");
    if (distribution < RLA_DIST_UNIFORM || distribution > RLA_DIST_AGMON)
        return set_error(ctx, RLA_E_ARG, "Unknown distribution %d.", distribution);
    if (distribution == RLA_DIST_AGMON) {
        if (beta < 1) return set_error(ctx, RLA_E_ARG, "`Agmon` beta must be >= 1, got beta=%lld", (long long)beta);
        if (beta > long_dim)
            return set_error(ctx, RLA_E_ARG, "`Agmon` beta must be <= number of %s (%lld), got beta=%lld",
                             card == RLA_LEFT ? "rows" : "columns", (long long)long_dim, (long long)beta);
        if (compression_dim > beta)
            return set_error(ctx, RLA_E_ARG, "`Agmon` cannot output %lld indices when beta=%lld.",
                             (long long)compression_dim, (long long)beta);
        if (compression_dim > 1024)
            return set_error(ctx, RLA_E_UNSUPPORTED, "`Agmon` sampling takes compression_dim <= 1024.");
    }
    if (long_dim <= 0) return set_error(ctx, RLA_E_ARG, "The sketched dimension must be positive.");
    if (long_dim >= (int64_t(1) << 31) || compression_dim >= (int64_t(1) << 30))
        return set_error(ctx, RLA_E_UNSUPPORTED, "Dimensions beyond 2^30 (compression) / 2^31 (sampled) are not supported.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    rla_sketch *sk = new rla_sketch();
    sk->p.kind = RLA_SAMPLING;
    sk->p.card = card;
    sk->p.dtype = dtype;
    sk->p.compression_dim = compression_dim;
    sk->p.long_dim = long_dim;
    sk->p.seed = seed;
    sk->device = ctx->device;
    sk->s = compression_dim;
    sk->L = long_dim;
    sk->n_rows = card == RLA_LEFT ? sk->s : sk->L;
    sk->n_cols = card == RLA_LEFT ? sk->L : sk->s;
    sk->s_dist = distribution;
    sk->s_replace = replace != 0;
    sk->s_beta = beta;
    sk->scale = 1.0;
    cudaError_t e = cudaMalloc((void **)&sk->sidx, sizeof(int64_t) * sk->s);
    if (e == cudaSuccess) e = cudaMalloc((void **)&sk->splan, sizeof(int64_t) * (3 * sk->s + 2));
    if (e == cudaSuccess) e = cudaMalloc((void **)&sk->s_err, sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(sk->s_err, 0, sizeof(int64_t), ctx->stream);
    if (e == cudaSuccess && distribution == RLA_DIST_L2NORM) e = cudaMalloc((void **)&sk->sweights, sizeof(double) * sk->L);
    if (e == cudaSuccess) e = cudaMemsetAsync(sk->sidx, 0, sizeof(int64_t) * sk->s, ctx->stream);
    int rc = e == cudaSuccess ? RLA_OK : set_error(ctx, RLA_E_OOM, "%s", cudaGetErrorString(e));
    // Uniform draws at once; L2Norm and Agmon draw in rla_sampling_update (they need A)
    if (rc == RLA_OK) rc = distribution == RLA_DIST_UNIFORM ? sampling_draw(ctx, sk, true) : sampling_plan(ctx, sk);
    if (rc == RLA_OK) RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (rc != RLA_OK) {
        rla_sketch_destroy(sk);
        return rc;
    }
    sk->draw_count = 1;
    *out = sk;
    return RLA_OK;
}

int rla_sampling_update(rla_ctx *ctx, rla_sketch *sk, int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                        const void *x, int64_t x_len, const void *b, int64_t b_len, const void *r) {
    if (!ctx) return RLA_E_ARG;
    if (!sk || sk->p.kind != RLA_SAMPLING) return set_error(ctx, RLA_E_ARG, "Not a Sampling recipe.");
    const int64_t dim = sk->p.card == RLA_LEFT ? a_rows : a_cols;
    if (dim != sk->L)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld %s while the recipe samples %lld.", (long long)dim,
                         sk->p.card == RLA_LEFT ? "rows" : "columns", (long long)sk->L);
    if (sk->s_dist != RLA_DIST_UNIFORM && (!A || lda < std::max<int64_t>(1, a_rows)))
        return set_error(ctx, RLA_E_ARG, "A (device, leading dimension >= rows) is required.");
    if (sk->s_dist == RLA_DIST_AGMON) {
        // agmon.jl update_distribution! / complete_distribution checks
        if (b_len != a_rows)
            return set_error(ctx, RLA_E_DIM, "Vector b has length %lld, expected %lld to match rows of A",
                             (long long)b_len, (long long)a_rows);
        if (x_len != a_cols)
            return set_error(ctx, RLA_E_DIM, "Vector x has length %lld, expected %lld to match columns of A",
                             (long long)x_len, (long long)a_cols);
        if (!r && (!x || !b)) return set_error(ctx, RLA_E_ARG, "`Agmon` needs x and b (or the residual r).");
    }
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    const uint64_t saved = sk->draw_count;
    int rc = sampling_update(ctx, sk, a_rows, a_cols, A, lda, x, b, r);
    if (rc == RLA_OK) rc = sampling_finish(ctx, sk);
    if (rc == RLA_OK) sk->draw_count = saved + 1;
    return rc;
}

}  // extern "C"
