// rla_ls.cu -- least squares on the device: one-shot sketch-and-solve, and the Iterative
// Hessian Sketch solver (src/Solvers/ihs.jl).
//
// x = argmin || S (A x - b) || for a Left compressor S (s x m, s >= n), A (m x n) and b (m),
// Float32 data: SA = S*A and Sb = S*b with the library's sketch kernels, then the sketched
// normal equations through the FP64 Cholesky factor of the equilibrated Gram matrix,
// D (SA)'(SA) D = R'R, x = D R^-1 R^-T D (SA)' Sb.  This is the solve of the serving
// workload's least-squares requests (a SparseSign sketch with s = 4n); the reference's
// solvers reach the same sketch through mul! (src/Solvers/ihs.jl:231-236).
#include <math.h>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

// d = diag(G)^-1/2
__global__ void ls_diag_kernel(const double *G, int64_t l, double *d) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= l) return;
    const double g = G[i + i * l];
    d[i] = g > 0.0 ? rsqrt(g) : 1.0;
}

// G <- D G D, one CTA per column
__global__ void ls_scale_kernel(double *G, int64_t l, const double *d) {
    const int64_t j = blockIdx.x;
    for (int64_t i = threadIdx.x; i < l; i += blockDim.x) G[i + j * l] *= d[i] * d[j];
}

// c(i) = sum_r X(r, i) y(r) in FP64, one warp per output (X rows x n, ld ldx; Float32).
__global__ void ls_gemv_t_kernel(const float *X, int64_t rows, int64_t n, int64_t ldx, const float *y, double *c) {
    const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const float *xi = X + i * ldx;
    double acc = 0.0;
    for (int64_t r = lane; r < rows; r += 32) acc += (double)xi[r] * (double)y[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if (lane == 0) c[i] = acc;
}

// With R upper (l x l): y = R^-T (d .* c), z = R^-1 y, x = d .* z.  Blocked by 32: warp 0
// solves a 32 x 32 diagonal triangle with shuffles, its lane holding the block's column
// (forward) or row (backward) of R in registers with the pivot reciprocal, so the serial
// steps wait on no memory; then all threads apply the block to the rest of the vector.  The
// R entries of a thread's first TS_PF update columns are loaded at the top of the block
// step, together with warp 0's diagonal block, so one memory latency is paid per block.
// Two barriers per block.  One CTA; the vector in shared memory.
constexpr int TS_THREADS = 256, TS_PF = 2;

template <class TX>
__global__ void __launch_bounds__(TS_THREADS) ls_trisolve_kernel(const double *R, int64_t l, const double *d,
                                                                const double *c, TX *x) {
    extern __shared__ double v[];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t i = tid; i < l; i += nt) v[i] = d[i] * c[i];
    __syncthreads();
    // forward: R' y = v, R' lower; block rows [b, b+32)
    for (int64_t b = 0; b < l; b += 32) {
        const int nb = (int)min((int64_t)32, l - b);
        double pf[TS_PF][32];
#pragma unroll
        for (int k = 0; k < TS_PF; ++k) {
            const int64_t j = b + nb + tid + (int64_t)k * nt;
#pragma unroll
            for (int t = 0; t < 32; ++t) pf[k][t] = (j < l && t < nb) ? R[(b + t) + j * l] : 0.0;
        }
        if (warp == 0) {
            double col[32];  // col[t] = R(b+t, b+lane) = R'(b+lane, b+t)
#pragma unroll
            for (int t = 0; t < 32; ++t) col[t] = (t < nb && lane < nb) ? R[(b + t) + (b + lane) * l] : 1.0;
            const double rinv = 1.0 / (lane < nb ? R[(b + lane) + (b + lane) * l] : 1.0);
            double yv = lane < nb ? v[b + lane] : 0.0;
#pragma unroll
            for (int t = 0; t < 32; ++t) {
                if (t < nb) {
                    if (lane == t) yv *= rinv;
                    const double yt = __shfl_sync(FULL, yv, t);
                    if (lane > t) yv -= yt * col[t];
                }
            }
            if (lane < nb) v[b + lane] = yv;
        }
        __syncthreads();
        // v(j) -= sum_{t in block} R(b+t, j) y(b+t) for j >= b+nb
#pragma unroll
        for (int k = 0; k < TS_PF; ++k) {
            const int64_t j = b + nb + tid + (int64_t)k * nt;
            if (j < l) {
                double acc = 0.0;
#pragma unroll
                for (int t = 0; t < 32; ++t) acc += pf[k][t] * v[b + min(t, nb - 1)];
                v[j] -= acc;
            }
        }
        for (int64_t j = b + nb + tid + (int64_t)TS_PF * nt; j < l; j += nt) {
            const double *rj = R + b + j * l;
            double acc = 0.0;
            for (int t = 0; t < nb; ++t) acc += rj[t] * v[b + t];
            v[j] -= acc;
        }
        __syncthreads();
    }
    // backward: R z = y; block rows [b, b+nb) from the bottom
    for (int64_t e = l; e > 0; e -= 32) {
        const int nb = (int)min((int64_t)32, e);
        const int64_t b = e - nb;
        double pf[TS_PF][32];
#pragma unroll
        for (int k = 0; k < TS_PF; ++k) {
            const int64_t j = tid + (int64_t)k * nt;
#pragma unroll
            for (int t = 0; t < 32; ++t) pf[k][t] = (j < b && t < nb) ? R[j + (b + t) * l] : 0.0;
        }
        if (warp == 0) {
            double row[32];  // row[t] = R(b+lane, b+t)
#pragma unroll
            for (int t = 0; t < 32; ++t) row[t] = (t < nb && lane < nb) ? R[(b + lane) + (b + t) * l] : 1.0;
            const double rinv = 1.0 / (lane < nb ? R[(b + lane) + (b + lane) * l] : 1.0);
            double zv = lane < nb ? v[b + lane] : 0.0;
#pragma unroll
            for (int t = 31; t >= 0; --t) {
                if (t < nb) {
                    if (lane == t) zv *= rinv;
                    const double zt = __shfl_sync(FULL, zv, t);
                    if (lane < t) zv -= zt * row[t];
                }
            }
            if (lane < nb) v[b + lane] = zv;
        }
        __syncthreads();
        // v(j) -= sum_{t in block} R(j, b+t) z(b+t) for j < b
#pragma unroll
        for (int k = 0; k < TS_PF; ++k) {
            const int64_t j = tid + (int64_t)k * nt;
            if (j < b) {
                double acc = 0.0;
#pragma unroll
                for (int t = 0; t < 32; ++t) acc += pf[k][t] * v[b + min(t, nb - 1)];
                v[j] -= acc;
            }
        }
        for (int64_t j = tid + (int64_t)TS_PF * nt; j < b; j += nt) {
            double acc = 0.0;
            for (int t = 0; t < nb; ++t) acc += R[j + (b + t) * l] * v[b + t];
            v[j] -= acc;
        }
        __syncthreads();
    }
    for (int64_t i = tid; i < l; i += nt) x[i] = (TX)(d[i] * v[i]);
}

// D G D with d = diag(G)^-1/2 (so the Cholesky factor is of an equilibrated matrix).
int ls_equilibrate(rla_ctx *ctx, double *G, int64_t l, double *d) {
    ls_diag_kernel<<<ceil_div_i(l, 256), 256, 0, ctx->stream>>>(G, l, d);
    ls_scale_kernel<<<(unsigned)l, 256, 0, ctx->stream>>>(G, l, d);
    return check_launch(ctx, "ls_equilibrate");
}

// x = d .* R^-1 R^-T (d .* c) for the factor R of the equilibrated matrix.
template <class TX>
int ls_chol_solve(rla_ctx *ctx, const double *R, int64_t l, const double *d, const double *c, TX *x) {
    const size_t smem = sizeof(double) * (size_t)l;
    if (smem > 48 * 1024) RLA_CUDA_TRY(ctx, set_smem_max(ls_trisolve_kernel<TX>));
    ls_trisolve_kernel<TX><<<1, TS_THREADS, smem, ctx->stream>>>(R, l, d, c, x);
    return check_launch(ctx, "ls_trisolve");
}
template int ls_chol_solve<float>(rla_ctx *, const double *, int64_t, const double *, const double *, float *);
template int ls_chol_solve<double>(rla_ctx *, const double *, int64_t, const double *, const double *, double *);

size_t ls_work_bytes(int64_t s, int64_t n) {
    auto r = [](size_t b) { return (b + 255) & ~size_t(255); };
    return r(sizeof(float) * s * n) + r(sizeof(float) * s) + r(sizeof(double) * n * n) + r(sizeof(double) * 3 * n) +
           r(sizeof(int));
}

// Asynchronous on ctx->stream; `work` holds ls_work_bytes(s, n) bytes; *bad (device int)
// reports a Cholesky breakdown after the stream completes.
int ls_sketch_solve(rla_ctx *ctx, const rla_sketch *S, int64_t m, int64_t n, const float *A, int64_t lda,
                    const float *b, float *x, void *work, int **bad_out) {
    const int64_t s = S->s;
    auto r = [](size_t bb) { return (bb + 255) & ~size_t(255); };
    char *w = (char *)work;
    float *SA = (float *)w;
    w += r(sizeof(float) * s * n);
    float *Sb = (float *)w;
    w += r(sizeof(float) * s);
    double *G = (double *)w;
    w += r(sizeof(double) * n * n);
    double *c = (double *)w;
    double *tmp = c + n;
    w += r(sizeof(double) * 3 * n);
    int *bad = (int *)w;
    RLA_TRY(sketch_mul_impl(ctx, S, RLA_SIDE_LEFT, 0, s, n, SA, s, 0, m, n, A, lda, 0, 1.0, 0.0));
    RLA_TRY(sketch_mul_impl(ctx, S, RLA_SIDE_LEFT, 0, s, 1, Sb, s, 0, m, 1, b, m, 0, 1.0, 0.0));
    RLA_TRY(gram_fp64<float>(ctx, SA, s, n, s, G));
    ls_gemv_t_kernel<<<ceil_div_i(n * 32, 256), 256, 0, ctx->stream>>>(SA, s, n, s, Sb, c);
    RLA_TRY(check_launch(ctx, "ls_gemv_t"));
    ls_diag_kernel<<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(G, n, tmp);
    ls_scale_kernel<<<(unsigned)n, 256, 0, ctx->stream>>>(G, n, tmp);
    RLA_TRY(check_launch(ctx, "ls_equilibrate"));
    RLA_TRY(cholesky_upper(ctx, G, n, 0.0, bad));
    const size_t smem = sizeof(double) * (size_t)n;
    if (smem > 48 * 1024)
        RLA_CUDA_TRY(ctx, set_smem_max(ls_trisolve_kernel<float>));
    ls_trisolve_kernel<float><<<1, TS_THREADS, smem, ctx->stream>>>(G, n, tmp, c, x);
    RLA_TRY(check_launch(ctx, "ls_trisolve"));
    *bad_out = bad;
    return RLA_OK;
}


// ---- Iterative Hessian Sketch (src/Solvers/ihs.jl:214-254) ---------------------------
//
// Iteration i of rsolve! reads A four times in the reference: A'r (:223), the error
// b - Ax (full_residual.jl), S*A (:236) and r -= A*u (:249).  Here the residual update of
// iteration i-1, the error and the gradient of iteration i share one pass over A
// (ihs_pass_kernel), and the sketch apply is the second:
//   r <- r - A u          (the reference updates r by A*u also when alpha != 1)
//   e  = ||b - A x||      (x already advanced by alpha*u)
//   g  = A' r
// The sub-problem solve R'R u = g uses the FP64 Cholesky factor of the equilibrated
// sketched Gram matrix (the same R'R as the reference's qr!(S*A).R, so u is the same).

// CTA = WARPS warps; a tile is 32 consecutive rows; warp w keeps columns
// [w*CPW, (w+1)*CPW) of the tile in registers (lane = row), the next tile prefetched.
// The row dots with u and x reduce over the warps in shared memory; A'r accumulates per
// lane in registers over the CTA's tiles and is reduced over lanes once at the end.
// Partial results per CTA: g_part[blk*n + c] (FP64) and e_part[blk] (FP64 sum of squares).
template <class T, int WARPS, int CPW>
__global__ void __launch_bounds__(WARPS * 32, 1)
    ihs_pass_kernel(const T *__restrict__ A, int64_t lda, int64_t m, int n, T *__restrict__ r,
                    const T *__restrict__ u, const T *__restrict__ x, const T *__restrict__ b, double *g_part,
                    double *e_part) {
    __shared__ T su[WARPS * CPW], sx[WARPS * CPW];
    __shared__ T red_u[WARPS][33], red_x[WARPS][33];
    __shared__ T rn[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c = threadIdx.x; c < WARPS * CPW; c += WARPS * 32) {
        su[c] = c < n ? u[c] : T(0);
        sx[c] = c < n ? x[c] : T(0);
    }
    __syncthreads();
    const int c0 = w * CPW;
    const int64_t ntiles = (m + 31) / 32;
    T a[CPW], an[CPW], gacc[CPW];
#pragma unroll
    for (int k = 0; k < CPW; ++k) gacc[k] = T(0);
    auto load = [&](int64_t t, T *dst) {
        const int64_t row = t * 32 + lane;
        const bool rok = row < m;
        const T *ap = A + row + (int64_t)c0 * lda;
#pragma unroll
        for (int k = 0; k < CPW; ++k) dst[k] = (rok && c0 + k < n) ? __ldcs(ap + (int64_t)k * lda) : T(0);
    };
    // warp 0 also keeps the tile's r and b entries, prefetched one tile ahead like A
    auto load_rb = [&](int64_t t, T &rv, T &bv) {
        const int64_t row = t * 32 + lane;
        rv = row < m ? r[row] : T(0);
        bv = row < m ? b[row] : T(0);
    };
    double e2 = 0.0;
    T r_cur = T(0), b_cur = T(0), r_nx = T(0), b_nx = T(0);
    int64_t tile = blockIdx.x;
    if (tile < ntiles) {
        load(tile, a);
        if (w == 0) load_rb(tile, r_cur, b_cur);
    }
    for (; tile < ntiles; tile += gridDim.x) {
        const int64_t nxt = tile + gridDim.x;
        if (nxt < ntiles) {
            load(nxt, an);
            if (w == 0) load_rb(nxt, r_nx, b_nx);
        }
        T pu = T(0), px = T(0);
#pragma unroll
        for (int k = 0; k < CPW; ++k) {
            pu += a[k] * su[c0 + k];
            px += a[k] * sx[c0 + k];
        }
        red_u[w][lane] = pu;
        red_x[w][lane] = px;
        __syncthreads();
        if (w == 0) {
            const int64_t row = tile * 32 + lane;
            T au = T(0), ax = T(0);
#pragma unroll
            for (int ww = 0; ww < WARPS; ++ww) {
                au += red_u[ww][lane];
                ax += red_x[ww][lane];
            }
            T rv = T(0);
            if (row < m) {
                rv = r_cur - au;
                r[row] = rv;
                const double e = (double)b_cur - (double)ax;
                e2 += e * e;
            }
            rn[lane] = rv;
            r_cur = r_nx;
            b_cur = b_nx;
        }
        __syncthreads();
        const T rv = rn[lane];
#pragma unroll
        for (int k = 0; k < CPW; ++k) {
            gacc[k] += a[k] * rv;
            a[k] = an[k];
        }
    }
#pragma unroll
    for (int k = 0; k < CPW; ++k) {
        double v = (double)gacc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        if (lane == 0 && c0 + k < n) g_part[(int64_t)blockIdx.x * n + c0 + k] = v;
    }
    if (w == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(FULL, e2, o);
        if (lane == 0) e_part[blockIdx.x] = e2;
    }
}

// Any n: r <- r - A u and the error partials, one thread per row (FP64 accumulation).
template <class T>
__global__ void __launch_bounds__(256) ihs_rows_kernel(const T *A, int64_t lda, int64_t m, int64_t n, T *r, const T *u,
                                                       const T *x, const T *b, double *e_part) {
    __shared__ double red[8];
    const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double e = 0.0;
    if (row < m) {
        double au = 0.0, ax = 0.0;
        for (int64_t c = 0; c < n; ++c) {
            const double v = (double)A[row + c * lda];
            au += v * (double)u[c];
            ax += v * (double)x[c];
        }
        r[row] = (T)((double)r[row] - au);
        e = (double)b[row] - ax;
        e *= e;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(FULL, e, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
        e_part[blockIdx.x] = t;
    }
}

// Any n: g_part[c] = sum_rows A(row, c) r(row), one warp per column (FP64 accumulation).
template <class T>
__global__ void ihs_cols_kernel(const T *A, int64_t lda, int64_t m, int64_t n, const T *r, double *g_part) {
    const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= n) return;
    const T *ac = A + c * lda;
    double acc = 0.0;
    for (int64_t i = lane; i < m; i += 32) acc += (double)ac[i] * (double)r[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if (lane == 0) g_part[c] = acc;
}

// g(c) = sum over the partials (CTA order), in T and FP64.
template <class T>
__global__ void ihs_reduce_kernel(const double *g_part, int nblk, int64_t n, T *g, double *gd) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n) return;
    double v = 0.0;
    for (int k = 0; k < nblk; ++k) v += g_part[(int64_t)k * n + c];
    g[c] = (T)v;
    gd[c] = v;
}

// stat[0] = ||b - A x|| (FullResidual), stat[1] = ||A' r|| (LSGradient), stat[2] = the
// Cholesky breakdown flag of the last step.  One CTA.
__global__ void __launch_bounds__(1024) ihs_norms_kernel(const double *e_part, int ne, const double *gd, int64_t n,
                                                         const int *bad, double *stat) {
    __shared__ double re[32], rg[32];
    double e = 0.0, gg = 0.0;
    for (int i = threadIdx.x; i < ne; i += blockDim.x) e += e_part[i];
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) gg += gd[i] * gd[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(FULL, e, o);
        gg += __shfl_xor_sync(FULL, gg, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        re[w] = e;
        rg[w] = gg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double te = 0.0, tg = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            te += re[i];
            tg += rg[i];
        }
        stat[0] = sqrt(te);
        stat[1] = sqrt(tg);
        stat[2] = bad ? (double)*bad : 0.0;
    }
}

template <class T>
__global__ void ihs_axpy_kernel(int64_t n, double alpha, const T *u, T *x) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) x[i] = (T)((double)x[i] + alpha * (double)u[i]);
}

}  // namespace rla

// Solver state: the compressor (not owned), the step size and the device workspaces.
struct rla_ihs {
    rla_sketch *S = nullptr;
    int dtype = RLA_F32;
    int64_t m = 0, n = 0, s = 0;
    double alpha = 1.0;
    int device = 0;
    int nblk = 0;       // partial rows of the fused pass (0: the any-n kernels)
    int warps = 0, cpw = 0;
    void *SA = nullptr;  // compressed_mat, s x n in the element type
    void *u = nullptr;   // the sub-problem solution of the last step, n
    double *G = nullptr, *d = nullptr, *gd = nullptr, *g_part = nullptr, *e_part = nullptr, *stat = nullptr;
    int *bad = nullptr;
    int ne = 0;
    double *hstat = nullptr;  // pinned host copy of stat
    // update_compressor! runs on a private stream, after the last S*A that read the draws
    // (ev_apply) and before the next one (ev_draw), so it overlaps the previous iteration's
    // tail and the host never waits for it.
    rla_ctx *side = nullptr;
    cudaEvent_t ev_apply = nullptr, ev_draw = nullptr;
};

namespace rla {

template <class T, int WARPS>
static int ihs_pass_fused(rla_ctx *ctx, rla_ihs *h, const T *A, int64_t lda, T *r, const T *u, const T *x,
                          const T *b) {
    auto go = [&](auto kern) {
        cudaEvent_t e0 = timing_begin(ctx);
        kern<<<h->nblk, WARPS * 32, 0, ctx->stream>>>(A, lda, h->m, (int)h->n, r, u, x, b, h->g_part, h->e_part);
        timing_end(ctx, 1, e0);
    };
    switch (h->cpw) {
    case 1: go(ihs_pass_kernel<T, WARPS, 1>); break;
    case 2: go(ihs_pass_kernel<T, WARPS, 2>); break;
    case 4: go(ihs_pass_kernel<T, WARPS, 4>); break;
    case 8: go(ihs_pass_kernel<T, WARPS, 8>); break;
    case 16: go(ihs_pass_kernel<T, WARPS, 16>); break;
    default: go(ihs_pass_kernel<T, WARPS, 32>); break;
    }
    return check_launch(ctx, "ihs_pass");
}

// r <- r - A u, e = ||b - A x||, g = A' r (+ FP64 copy), norms into h->stat.
template <class T>
static int ihs_pass(rla_ctx *ctx, rla_ihs *h, const T *A, int64_t lda, T *r, const T *u, const T *x, const T *b,
                    T *g) {
    const int64_t m = h->m, n = h->n;
    int nparts = 1;
    if (h->nblk > 0) {
        if constexpr (sizeof(T) == 4) RLA_TRY((ihs_pass_fused<T, 16>(ctx, h, A, lda, r, u, x, b)));
        else RLA_TRY((ihs_pass_fused<T, 8>(ctx, h, A, lda, r, u, x, b)));
        nparts = h->nblk;
        h->ne = h->nblk;
    } else {
        const int rb = ceil_div_i(m, 256);
        ihs_rows_kernel<T><<<rb, 256, 0, ctx->stream>>>(A, lda, m, n, r, u, x, b, h->e_part);
        RLA_TRY(check_launch(ctx, "ihs_rows"));
        ihs_cols_kernel<T><<<ceil_div_i(n * 32, 256), 256, 0, ctx->stream>>>(A, lda, m, n, r, h->g_part);
        RLA_TRY(check_launch(ctx, "ihs_cols"));
        h->ne = rb;
    }
    ihs_reduce_kernel<T><<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(h->g_part, nparts, n, g, h->gd);
    ihs_norms_kernel<<<1, 1024, 0, ctx->stream>>>(h->e_part, h->ne, h->gd, n, h->bad, h->stat);
    return check_launch(ctx, "ihs_reduce");
}

template <class T>
static int ihs_start_t(rla_ctx *ctx, rla_ihs *h, const T *A, int64_t lda, const T *b, const T *x, T *r, T *g) {
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(r, b, sizeof(T) * h->m, cudaMemcpyDeviceToDevice, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemsetAsync(h->bad, 0, sizeof(int), ctx->stream));
    // the first redraw waits for whatever the caller queued before the solve
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_apply, ctx->stream));
    return ihs_pass<T>(ctx, h, A, lda, r, x, x, b, g);
}

template <class T>
static int ihs_step_t(rla_ctx *ctx, rla_ihs *h, const T *A, int64_t lda, const T *b, T *x, T *r, T *g) {
    const int64_t n = h->n, s = h->s;
    // update_compressor! (ihs.jl:231) and mat_view = S*A (:236)
    RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(h->side->stream, h->ev_apply, 0));
    if (int rc = sketch_redraw_async(h->side, h->S)) return set_error(ctx, rc, "%s", h->side->last_error.c_str());
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_draw, h->side->stream));
    RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, h->ev_draw, 0));
    T *SA = (T *)h->SA;
    cudaEvent_t e0 = timing_begin(ctx);
    RLA_TRY(sketch_mul_impl(ctx, h->S, RLA_SIDE_LEFT, 0, s, n, SA, s, 0, h->m, n, A, lda, 0, 1.0, 0.0));
    timing_end(ctx, 2, e0);
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_apply, ctx->stream));
    // R'R = (SA)'(SA) (ihs.jl:239), equilibrated: D G D = R'R
    RLA_TRY(gram_fp64<T>(ctx, SA, s, n, s, h->G));
    ls_diag_kernel<<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(h->G, n, h->d);
    ls_scale_kernel<<<(unsigned)n, 256, 0, ctx->stream>>>(h->G, n, h->d);
    RLA_TRY(check_launch(ctx, "ihs_equilibrate"));
    RLA_TRY(cholesky_upper(ctx, h->G, n, 0.0, h->bad));
    // u = R \ (R' \ g) (ihs.jl:241-243), x += alpha*u (:246)
    const size_t smem = sizeof(double) * (size_t)n;
    if (smem > 48 * 1024) RLA_CUDA_TRY(ctx, set_smem_max(ls_trisolve_kernel<T>));
    T *u = (T *)h->u;
    ls_trisolve_kernel<T><<<1, TS_THREADS, smem, ctx->stream>>>(h->G, n, h->d, h->gd, u);
    ihs_axpy_kernel<T><<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(n, h->alpha, u, x);
    RLA_TRY(check_launch(ctx, "ihs_solve"));
    // r -= A*u (:249) with the next iteration's error and gradient
    return ihs_pass<T>(ctx, h, A, lda, r, u, x, b, g);
}

static void ihs_free(rla_ihs *h) {
    void *p[] = {h->SA, h->u, h->G, h->d, h->gd, h->g_part, h->e_part, h->stat, h->bad};
    for (void *q : p)
        if (q) cudaFree(q);
    if (h->hstat) cudaFreeHost(h->hstat);
    if (h->ev_apply) cudaEventDestroy(h->ev_apply);
    if (h->ev_draw) cudaEventDestroy(h->ev_draw);
    if (h->side) rla_ctx_destroy(h->side);
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_sketch_solve(rla_ctx *ctx, const rla_sketch *sk, int64_t m, int64_t n, const float *A, int64_t lda,
                     const float *b, float *x) {
    if (!ctx) return RLA_E_ARG;
    if (!sk || !A || !b || !x) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (sk->p.dtype != RLA_F32) return set_error(ctx, RLA_E_ARG, "Sketch-and-solve takes a Float32 compressor.");
    if (sk->n_cols != m || sk->n_rows != sk->s)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)m,
                         (long long)sk->n_cols);
    if (n <= 0 || sk->s < n || lda < m) return set_error(ctx, RLA_E_ARG, "Need 0 < n <= compression dimension.");
    if (n > 4096) return set_error(ctx, RLA_E_UNSUPPORTED, "sketch-and-solve takes n <= 4096");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    void *work = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &work, ls_work_bytes(sk->s, n), ctx->stream));
    int *bad = nullptr;
    int rc = ls_sketch_solve(ctx, sk, m, n, A, lda, b, x, work, &bad);
    int hbad = 0;
    if (rc == RLA_OK) {
        cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = set_error(ctx, RLA_E_CUDA, "%s", cudaGetErrorString(e));
    }
    cudaFreeAsync(work, ctx->stream);
    RLA_TRY(rc);
    if (hbad) return set_error(ctx, RLA_E_NUMERIC, "Sketched Gram matrix is not positive definite.");
    return RLA_OK;
}

int rla_ihs_create(rla_ctx *ctx, rla_sketch *compressor, int dtype, int64_t m, int64_t n, double alpha,
                   rla_ihs **out) {
    if (!ctx) return RLA_E_ARG;
    if (!compressor || !out) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    *out = nullptr;
    if (dtype != RLA_F32 && dtype != RLA_F64) return set_error(ctx, RLA_E_ARG, "dtype must be Float32 or Float64.");
    if (compressor->p.dtype != dtype)
        return set_error(ctx, RLA_E_ARG, "The compressor's element type differs from the matrix's.");
    if (compressor->p.card != RLA_LEFT)
        return set_error(ctx, RLA_E_ARG, "IHS compresses from the `Left`; the compressor has cardinality `Right`.");
    const int64_t s = compressor->n_rows;
    // complete_solver's checks, in the reference's order and wording (ihs.jl:160-190)
    if (n > s)
        return set_error(ctx, RLA_E_ARG,
                         "Compression dimension not larger than column dimension this will lead to singular QR "
                         "decompositions, which cannot be inverted.");
    if (m < s) return set_error(ctx, RLA_E_ARG, "Compression dimension larger row dimension.");
    if (n >= m) return set_error(ctx, RLA_E_ARG, "Matrix must have more rows than columns.");
    if (compressor->n_cols != m)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)m,
                         (long long)compressor->n_cols);
    if (n < 1) return set_error(ctx, RLA_E_ARG, "Matrix must have at least one column.");
    if (n > 4096) return set_error(ctx, RLA_E_UNSUPPORTED, "IHS takes n <= 4096 columns.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    rla_ihs *h = new rla_ihs;
    h->S = compressor;
    h->dtype = dtype;
    h->m = m;
    h->n = n;
    h->s = s;
    h->alpha = alpha;
    h->device = ctx->device;
    const int es = dtype == RLA_F32 ? 4 : 8;
    h->warps = dtype == RLA_F32 ? 16 : 8;
    h->cpw = 1;
    while (h->cpw < 32 && (int64_t)h->warps * h->cpw < n) h->cpw *= 2;
    h->nblk = (int64_t)h->warps * h->cpw >= n ? ctx->sm_count : 0;
    const int64_t parts = h->nblk > 0 ? (int64_t)h->nblk * n : n;
    const int64_t eparts = std::max<int64_t>(h->nblk, ceil_div(m, 256));
    cudaError_t e = cudaSuccess;
    auto grab = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    };
    grab(&h->SA, (size_t)es * s * n);
    grab(&h->u, (size_t)es * n);
    grab((void **)&h->G, sizeof(double) * n * n);
    grab((void **)&h->d, sizeof(double) * n);
    grab((void **)&h->gd, sizeof(double) * n);
    grab((void **)&h->g_part, sizeof(double) * parts);
    grab((void **)&h->e_part, sizeof(double) * eparts);
    grab((void **)&h->stat, sizeof(double) * 4);
    grab((void **)&h->bad, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hstat, sizeof(double) * 4);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_apply, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_draw, cudaEventDisableTiming);
    if (e == cudaSuccess && rla_ctx_create(ctx->device, nullptr, &h->side) != RLA_OK) e = cudaErrorUnknown;
    if (e == cudaSuccess) e = cudaMemsetAsync(h->bad, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->u, 0, (size_t)es * n, ctx->stream);
    if (e != cudaSuccess) {
        ihs_free(h);
        delete h;
        return set_error(ctx, e == cudaErrorMemoryAllocation ? RLA_E_OOM : RLA_E_CUDA, "%s", cudaGetErrorString(e));
    }
    *out = h;
    return RLA_OK;
}

static int ihs_check(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, const void *x, const void *r,
                     const void *g) {
    if (!ctx) return RLA_E_ARG;
    if (!h || !A || !b || !x || !r || !g) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (lda < h->m) return set_error(ctx, RLA_E_ARG, "lda must be at least m.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    return RLA_OK;
}

int rla_ihs_start(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, const void *x, void *r,
                  void *g) {
    RLA_TRY(ihs_check(ctx, h, A, lda, b, x, r, g));
    if (h->dtype == RLA_F32)
        return ihs_start_t<float>(ctx, h, (const float *)A, lda, (const float *)b, (const float *)x, (float *)r,
                                  (float *)g);
    return ihs_start_t<double>(ctx, h, (const double *)A, lda, (const double *)b, (const double *)x, (double *)r,
                               (double *)g);
}

int rla_ihs_step(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, void *x, void *r, void *g) {
    RLA_TRY(ihs_check(ctx, h, A, lda, b, x, r, g));
    if (h->dtype == RLA_F32)
        return ihs_step_t<float>(ctx, h, (const float *)A, lda, (const float *)b, (float *)x, (float *)r, (float *)g);
    return ihs_step_t<double>(ctx, h, (const double *)A, lda, (const double *)b, (double *)x, (double *)r,
                              (double *)g);
}

int rla_ihs_errors(rla_ctx *ctx, rla_ihs *h, double *full_residual, double *ls_gradient) {
    if (!ctx) return RLA_E_ARG;
    if (!h) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(h->hstat, h->stat, sizeof(double) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h->hstat[2] != 0.0) return set_error(ctx, RLA_E_NUMERIC, "Sketched Gram matrix is not positive definite.");
    if (full_residual) *full_residual = h->hstat[0];
    if (ls_gradient) *ls_gradient = h->hstat[1];
    return RLA_OK;
}

int rla_ihs_solve(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, void *x, void *r, void *g,
                  int64_t max_it, int64_t collection_rate, double threshold, int error_kind, double *hist,
                  int64_t hist_len, int64_t *iterations, int *converged) {
    RLA_TRY(ihs_check(ctx, h, A, lda, b, x, r, g));
    // BasicLogger (src/Solvers/Loggers/basic_logger.jl:15-33) argument checks
    if (max_it < 0) return set_error(ctx, RLA_E_ARG, "Field `max_it` must be positive or 0.");
    if (collection_rate < 1) return set_error(ctx, RLA_E_ARG, "Field `colection_rate` must be positive.");
    if (collection_rate > max_it && max_it > 0)
        return set_error(ctx, RLA_E_ARG, "Field `colection_rate` must be smaller than `max_it`.");
    if (error_kind != RLA_IHS_FULL_RESIDUAL && error_kind != RLA_IHS_LS_GRADIENT)
        return set_error(ctx, RLA_E_ARG, "error_kind must be RLA_IHS_FULL_RESIDUAL or RLA_IHS_LS_GRADIENT.");
    const int64_t need = (max_it + collection_rate - 1) / collection_rate + 1;
    if (hist && hist_len < need) return set_error(ctx, RLA_E_ARG, "hist needs %lld entries.", (long long)need);
    if (hist)
        for (int64_t i = 0; i < need; ++i) hist[i] = 0.0;
    // rsolve! (ihs.jl:214-254) with update_logger! (basic_logger.jl:84-101)
    int64_t rec = 0, it = 0;
    bool conv = false;
    RLA_TRY(rla_ihs_start(ctx, h, A, lda, b, x, r, g));
    for (int64_t i = 1; i <= max_it; ++i) {
        double ef = 0.0, eg = 0.0;
        RLA_TRY(rla_ihs_errors(ctx, h, &ef, &eg));
        const double err = error_kind == RLA_IHS_FULL_RESIDUAL ? ef : eg;
        it = i;
        conv = i < max_it ? err < threshold : true;
        if (conv) {
            if (hist) hist[rec] = err;
        } else if (i % collection_rate == 0) {
            if (hist) hist[rec] = err;
            ++rec;
        }
        if (conv) break;
        RLA_TRY(rla_ihs_step(ctx, h, A, lda, b, x, r, g));
    }
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
    return RLA_OK;
}

int rla_ihs_workspace(const rla_ihs *h, void **compressed_mat, void **update, double **R_equilibrated,
                      double **d) {
    if (!h) return RLA_E_ARG;
    if (compressed_mat) *compressed_mat = h->SA;
    if (update) *update = h->u;
    if (R_equilibrated) *R_equilibrated = h->G;
    if (d) *d = h->d;
    return RLA_OK;
}

int rla_ihs_destroy(rla_ihs *h) {
    if (!h) return RLA_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    ihs_free(h);
    cudaSetDevice(cur);
    delete h;
    return RLA_OK;
}

}  // extern "C"
