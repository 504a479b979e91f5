// rla_proj.cu -- the row- and column-action projection solvers on the device:
// Kaczmarz (src/Solvers/kaczmarz.jl) and ColumnProjection (src/Solvers/col_projection.jl).
//
// Kaczmarz, one iteration (kaczmarz.jl:262-368): update_compressor! (Left S, s x m),
// mat_view = S*A (s x n), vec_view = S*b, then the minimum-norm correction of the sketched
// rows, u = (SA)' (SA (SA)')^-1 (Sb - SA x) (the LQ sub-solver, lq.jl; for s = 1 the
// scalar kaczmarz_update!), x += alpha*u.  S*A is formed transposed, Y = (SA)' (n x s),
// so that SA (SA)' is the FP64 Gram matrix of Y's columns.
//
// ColumnProjection, one iteration (col_projection.jl:276-372): update_compressor! (Right S,
// n x s), mat_view = A*S (m x s), the least-squares correction u = argmin ||AS u - r|| (the
// QR sub-solver, qr.jl; for s = 1 colproj_update!), x += alpha*S*u, r -= alpha*AS*u.
//
// Both sub-problems are solved through the FP64 Cholesky factor of the equilibrated s x s
// Gram matrix (the reference's LQ / QR factors give the same solution when the sketched
// block has full rank).  The redraw runs on a private stream ordered by events, as in IHS.
#include <math.h>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

// out(j) = sum_r X(r, j) v(r) (X rows x cols, ld ldx), one warp per column, FP64.
template <class T>
__global__ void proj_gemv_t_kernel(const T *X, int64_t rows, int64_t cols, int64_t ldx, const T *v, double *out) {
    const int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= cols) return;
    const T *xj = X + j * ldx;
    double acc = 0.0;
    for (int64_t r = lane; r < rows; r += 32) acc += (double)xj[r] * (double)v[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if (lane == 0) out[j] = acc;
}

// target(i) += coef * sum_j X(i, j) w(j) (X rows x cols, ld ldx), one thread per row.
template <class T>
__global__ void proj_gemv_n_kernel(const T *X, int64_t rows, int64_t cols, int64_t ldx, const double *w, double coef,
                                   T *target) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= rows) return;
    double acc = 0.0;
    for (int64_t j = 0; j < cols; ++j) acc += (double)X[i + j * ldx] * w[j];
    target[i] = (T)((double)target[i] + coef * acc);
}

// c(j) = sb(j) - c(j) (the sketched residual Sb - SA x).
template <class T>
__global__ void proj_sub_kernel(const T *sb, int64_t s, double *c) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < s) c[j] = (double)sb[j] - c[j];
}

// part(blk) = sum over the block's rows of (b - A x)^2, one thread per row.
template <class T>
__global__ void __launch_bounds__(256) proj_resid_kernel(const T *A, int64_t lda, int64_t m, int64_t n, const T *x,
                                                         const T *b, double *part) {
    __shared__ double red[8];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < m) {
        double v = (double)b[i];
        for (int64_t j = 0; j < n; ++j) v -= (double)A[i + j * lda] * (double)x[j];
        e = v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(FULL, e, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        part[blockIdx.x] = t;
    }
}

// out(0) = sqrt(sum of v(0:n)) (sq = 0) or sqrt(sum of v^2) (sq = 1); one CTA, fixed order.
__global__ void __launch_bounds__(1024) proj_norm_kernel(const double *v, int64_t n, int sq, double *out) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += sq ? v[i] * v[i] : v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        out[0] = sqrt(t);
    }
}

template <class T>
__global__ void proj_cast_kernel(const double *y, int64_t s, T *out) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < s) out[j] = (T)y[j];
}

// r = b - A x (the start of ColumnProjection's rsolve!, col_projection.jl:328-329).
template <class T>
__global__ void proj_r0_kernel(const T *A, int64_t lda, int64_t m, int64_t n, const T *x, const T *b, T *r) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    double v = (double)b[i];
    for (int64_t j = 0; j < n; ++j) v -= (double)A[i + j * lda] * (double)x[j];
    r[i] = (T)v;
}

// kaczmarz_update!'s guard (kaczmarz.jl: `if !iszero(mat_view)`): skip[0] = 1 when the
// sketched rows are all zero (their Gram matrix has a zero diagonal).
__global__ void proj_zero_check_kernel(const double *G, int64_t s, int *skip) {
    double t = 0.0;
    for (int64_t j = 0; j < s; ++j) t += G[j + j * s];
    *skip = t == 0.0;
}

// y(j) = 0 when skip is set (no update).
__global__ void proj_mask_kernel(const int *skip, int64_t s, double *y) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < s && *skip) y[j] = 0.0;
}

}  // namespace rla

struct rla_proj {
    rla_sketch *S = nullptr;
    int kind = RLA_PROJ_KACZMARZ;
    int dtype = RLA_F32;
    int64_t m = 0, n = 0, s = 0;
    double alpha = 1.0;
    int device = 0;
    void *Y = nullptr;     // Kaczmarz: (SA)' (n x s); ColumnProjection: AS (m x s)
    void *Sb = nullptr;    // Kaczmarz: S*b (s)
    void *uT = nullptr;    // ColumnProjection: u in the element type (s)
    double *G = nullptr, *d = nullptr, *c = nullptr, *y = nullptr, *part = nullptr, *vec = nullptr, *stat = nullptr;
    int *bad = nullptr, *skip = nullptr;
    double *hstat = nullptr;
    bool sketched = false;  // a sketched system exists (CompressedResidual)
    rla_ctx *side = nullptr;
    cudaEvent_t ev_apply = nullptr, ev_draw = nullptr;
};

namespace rla {

static void proj_free(rla_proj *h) {
    void *p[] = {h->Y, h->Sb, h->uT, h->G, h->d, h->c, h->y, h->part, h->vec, h->stat, h->bad, h->skip};
    for (void *q : p)
        if (q) cudaFree(q);
    if (h->hstat) cudaFreeHost(h->hstat);
    if (h->ev_apply) cudaEventDestroy(h->ev_apply);
    if (h->ev_draw) cudaEventDestroy(h->ev_draw);
    if (h->side) rla_ctx_destroy(h->side);
}

// update_compressor! on the private stream, ordered after the last use of the draws.
static int proj_redraw(rla_ctx *ctx, rla_proj *h) {
    RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(h->side->stream, h->ev_apply, 0));
    if (int rc = sketch_redraw_async(h->side, h->S)) return set_error(ctx, rc, "%s", h->side->last_error.c_str());
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_draw, h->side->stream));
    RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, h->ev_draw, 0));
    return RLA_OK;
}

// Solve G y = c through the equilibrated FP64 Cholesky factor (G s x s in h->G).
static int proj_gram_solve(rla_ctx *ctx, rla_proj *h) {
    const int64_t s = h->s;
    RLA_TRY(ls_equilibrate(ctx, h->G, s, h->d));
    RLA_TRY(cholesky_upper(ctx, h->G, s, 0.0, h->bad));
    return ls_chol_solve<double>(ctx, h->G, s, h->d, h->c, h->y);
}

template <class T>
static int kaczmarz_step_t(rla_ctx *ctx, rla_proj *h, const T *A, int64_t lda, const T *b, T *x) {
    const int64_t n = h->n, s = h->s, m = h->m;
    RLA_TRY(proj_redraw(ctx, h));
    T *Y = (T *)h->Y, *Sb = (T *)h->Sb;
    // (SA)' = A' S' (n x s) and S*b
    RLA_TRY(sketch_mul_impl(ctx, h->S, RLA_SIDE_LEFT, 0, s, n, Y, n, 1, m, n, A, lda, 0, 1.0, 0.0));
    RLA_TRY(sketch_mul_impl(ctx, h->S, RLA_SIDE_LEFT, 0, s, 1, Sb, s, 0, m, 1, b, m, 0, 1.0, 0.0));
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_apply, ctx->stream));
    // c = Sb - SA x, G = SA (SA)'
    proj_gemv_t_kernel<T><<<ceil_div_i(s * 32, 256), 256, 0, ctx->stream>>>(Y, n, s, n, x, h->c);
    proj_sub_kernel<T><<<ceil_div_i(s, 256), 256, 0, ctx->stream>>>(Sb, s, h->c);
    RLA_TRY(check_launch(ctx, "kaczmarz_residual"));
    RLA_TRY(gram_fp64<T>(ctx, Y, n, s, n, h->G));
    proj_zero_check_kernel<<<1, 1, 0, ctx->stream>>>(h->G, s, h->skip);
    RLA_TRY(proj_gram_solve(ctx, h));
    proj_mask_kernel<<<ceil_div_i(s, 256), 256, 0, ctx->stream>>>(h->skip, s, h->y);
    // x += alpha * (SA)' y
    proj_gemv_n_kernel<T><<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(Y, n, s, n, h->y, h->alpha, x);
    h->sketched = true;
    return check_launch(ctx, "kaczmarz_update");
}

template <class T>
static int colproj_step_t(rla_ctx *ctx, rla_proj *h, const T *A, int64_t lda, T *x, T *r) {
    const int64_t n = h->n, s = h->s, m = h->m;
    RLA_TRY(proj_redraw(ctx, h));
    T *Y = (T *)h->Y;
    // AS (m x s)
    RLA_TRY(sketch_mul_impl(ctx, h->S, RLA_SIDE_RIGHT, 0, m, s, Y, m, 0, m, n, A, lda, 0, 1.0, 0.0));
    // u = (AS'AS)^-1 AS' r
    proj_gemv_t_kernel<T><<<ceil_div_i(s * 32, 256), 256, 0, ctx->stream>>>(Y, m, s, m, r, h->c);
    RLA_TRY(check_launch(ctx, "colproj_rhs"));
    RLA_TRY(gram_fp64<T>(ctx, Y, m, s, m, h->G));
    RLA_TRY(proj_gram_solve(ctx, h));
    // x += alpha * S u (S: n x s), r -= alpha * AS u
    T *uT = (T *)h->uT;
    proj_cast_kernel<T><<<ceil_div_i(s, 256), 256, 0, ctx->stream>>>(h->y, s, uT);
    RLA_TRY(check_launch(ctx, "colproj_cast"));
    RLA_TRY(sketch_mul_impl(ctx, h->S, RLA_SIDE_LEFT, 0, n, 1, x, n, 0, s, 1, uT, s, 0, h->alpha, 1.0));
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_apply, ctx->stream));
    proj_gemv_n_kernel<T><<<ceil_div_i(m, 256), 256, 0, ctx->stream>>>(Y, m, s, m, h->y, -h->alpha, r);
    h->sketched = true;
    return check_launch(ctx, "colproj_update");
}

}  // namespace rla

namespace rla {

template <class T>
static int proj_error_t(rla_ctx *ctx, rla_proj *h, int kind, const T *A, int64_t lda, const T *b, const T *x,
                        const T *r) {
    const int64_t m = h->m, n = h->n, s = h->s;
    if (kind == RLA_ERR_FULL_RESIDUAL) {
        const int nb = ceil_div_i(m, 256);
        proj_resid_kernel<T><<<nb, 256, 0, ctx->stream>>>(A, lda, m, n, x, b, h->part);
        proj_norm_kernel<<<1, 1024, 0, ctx->stream>>>(h->part, nb, 0, h->stat);
    } else if (kind == RLA_ERR_LS_GRADIENT) {
        proj_gemv_t_kernel<T><<<ceil_div_i(n * 32, 256), 256, 0, ctx->stream>>>(A, m, n, lda, r, h->vec);
        proj_norm_kernel<<<1, 1024, 0, ctx->stream>>>(h->vec, n, 1, h->stat);
    } else {
        // ||Sb - SA x|| of the last sketched system (zero before the first step)
        if (!h->sketched) {
            RLA_CUDA_TRY(ctx, cudaMemsetAsync(h->stat, 0, sizeof(double), ctx->stream));
        } else {
            proj_gemv_t_kernel<T><<<ceil_div_i(s * 32, 256), 256, 0, ctx->stream>>>((const T *)h->Y, n, s, n, x, h->vec);
            proj_sub_kernel<T><<<ceil_div_i(s, 256), 256, 0, ctx->stream>>>((const T *)h->Sb, s, h->vec);
            proj_norm_kernel<<<1, 1024, 0, ctx->stream>>>(h->vec, s, 1, h->stat);
        }
    }
    RLA_TRY(check_launch(ctx, "proj_error"));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(h->hstat, h->stat, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    int hbad = 0;
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&hbad, h->bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (hbad) {
        int skip = 0;
        cudaMemcpy(&skip, h->skip, sizeof(int), cudaMemcpyDeviceToHost);
        if (!skip) return set_error(ctx, RLA_E_NUMERIC, "The sketched block is rank deficient (singular sub-problem).");
    }
    return RLA_OK;
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_proj_create(rla_ctx *ctx, rla_sketch *compressor, int kind, int dtype, int64_t m, int64_t n, double alpha,
                    rla_proj **out) {
    if (!ctx) return RLA_E_ARG;
    if (!compressor || !out) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    *out = nullptr;
    if (kind != RLA_PROJ_KACZMARZ && kind != RLA_PROJ_COLUMN) return set_error(ctx, RLA_E_ARG, "Unknown solver kind %d.", kind);
    if (dtype != RLA_F32 && dtype != RLA_F64) return set_error(ctx, RLA_E_ARG, "dtype must be Float32 or Float64.");
    if (compressor->p.dtype != dtype)
        return set_error(ctx, RLA_E_ARG, "The compressor's element type differs from the matrix's.");
    if (m < 1 || n < 1) return set_error(ctx, RLA_E_ARG, "A must have at least one row and one column.");
    int64_t s;
    if (kind == RLA_PROJ_KACZMARZ) {
        // mul!(mat_view, S, A) needs a Left S with n_cols == size(A, 1)
        if (compressor->n_cols != m)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)m,
                             (long long)compressor->n_cols);
        s = compressor->n_rows;
    } else {
        // mul!(mat_view, A, S) needs n_rows == size(A, 2)
        if (compressor->n_rows != n)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while S has %lld rows.", (long long)n,
                             (long long)compressor->n_rows);
        s = compressor->n_cols;
    }
    if (s > 4096) return set_error(ctx, RLA_E_UNSUPPORTED, "block size above 4096 is not supported.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    rla_proj *h = new rla_proj;
    h->S = compressor;
    h->kind = kind;
    h->dtype = dtype;
    h->m = m;
    h->n = n;
    h->s = s;
    h->alpha = alpha;
    h->device = ctx->device;
    const size_t es = dtype == RLA_F32 ? 4 : 8;
    cudaError_t e = cudaSuccess;
    auto grab = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    };
    grab(&h->Y, es * (size_t)s * (kind == RLA_PROJ_KACZMARZ ? n : m));
    grab(&h->Sb, es * (size_t)s);
    grab(&h->uT, es * (size_t)s);
    grab((void **)&h->G, sizeof(double) * s * s);
    grab((void **)&h->d, sizeof(double) * s);
    grab((void **)&h->c, sizeof(double) * s);
    grab((void **)&h->y, sizeof(double) * s);
    grab((void **)&h->part, sizeof(double) * ceil_div(m, 256));
    grab((void **)&h->vec, sizeof(double) * std::max(n, s));
    grab((void **)&h->stat, sizeof(double) * 2);
    grab((void **)&h->bad, sizeof(int));
    grab((void **)&h->skip, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hstat, sizeof(double) * 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->bad, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->skip, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_apply, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_draw, cudaEventDisableTiming);
    if (e == cudaSuccess && rla_ctx_create(ctx->device, nullptr, &h->side) != RLA_OK) e = cudaErrorUnknown;
    if (e != cudaSuccess) {
        proj_free(h);
        delete h;
        return set_error(ctx, e == cudaErrorMemoryAllocation ? RLA_E_OOM : RLA_E_CUDA, "%s", cudaGetErrorString(e));
    }
    *out = h;
    return RLA_OK;
}

static int proj_check(rla_ctx *ctx, rla_proj *h, const void *A, int64_t lda) {
    if (!ctx) return RLA_E_ARG;
    if (!h || !A) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (lda < h->m) return set_error(ctx, RLA_E_ARG, "lda must be at least m.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    return RLA_OK;
}

int rla_proj_start(rla_ctx *ctx, rla_proj *h, const void *A, int64_t lda, const void *b, const void *x, void *r) {
    RLA_TRY(proj_check(ctx, h, A, lda));
    // the first redraw waits for whatever the caller queued before the solve
    RLA_CUDA_TRY(ctx, cudaEventRecord(h->ev_apply, ctx->stream));
    h->sketched = false;
    if (h->kind == RLA_PROJ_KACZMARZ) return RLA_OK;
    if (!b || !x || !r) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (h->dtype == RLA_F32)
        proj_r0_kernel<float><<<ceil_div_i(h->m, 256), 256, 0, ctx->stream>>>((const float *)A, lda, h->m, h->n,
                                                                              (const float *)x, (const float *)b,
                                                                              (float *)r);
    else
        proj_r0_kernel<double><<<ceil_div_i(h->m, 256), 256, 0, ctx->stream>>>((const double *)A, lda, h->m, h->n,
                                                                               (const double *)x, (const double *)b,
                                                                               (double *)r);
    return check_launch(ctx, "proj_start");
}

int rla_proj_step(rla_ctx *ctx, rla_proj *h, const void *A, int64_t lda, const void *b, void *x, void *r) {
    RLA_TRY(proj_check(ctx, h, A, lda));
    if (!x) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (h->kind == RLA_PROJ_KACZMARZ) {
        if (!b) return set_error(ctx, RLA_E_ARG, "NULL argument.");
        if (h->dtype == RLA_F32)
            return kaczmarz_step_t<float>(ctx, h, (const float *)A, lda, (const float *)b, (float *)x);
        return kaczmarz_step_t<double>(ctx, h, (const double *)A, lda, (const double *)b, (double *)x);
    }
    if (!r) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (h->dtype == RLA_F32) return colproj_step_t<float>(ctx, h, (const float *)A, lda, (float *)x, (float *)r);
    return colproj_step_t<double>(ctx, h, (const double *)A, lda, (double *)x, (double *)r);
}

int rla_proj_error(rla_ctx *ctx, rla_proj *h, int kind, const void *A, int64_t lda, const void *b, const void *x,
                   const void *r, double *value) {
    RLA_TRY(proj_check(ctx, h, A, lda));
    if (!value) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (kind == RLA_ERR_FULL_RESIDUAL && (!b || !x)) return set_error(ctx, RLA_E_ARG, "FullResidual needs b and x.");
    if (kind == RLA_ERR_LS_GRADIENT && !r) return set_error(ctx, RLA_E_ARG, "LSGradient needs the residual vector.");
    if (kind == RLA_ERR_COMPRESSED_RESIDUAL && (!x || h->kind != RLA_PROJ_KACZMARZ))
        return set_error(ctx, RLA_E_ARG, "CompressedResidual needs the sketched rows of a Kaczmarz solver.");
    if (kind < RLA_ERR_FULL_RESIDUAL || kind > RLA_ERR_COMPRESSED_RESIDUAL)
        return set_error(ctx, RLA_E_ARG, "Unknown error method %d.", kind);
    int rc = h->dtype == RLA_F32
                 ? proj_error_t<float>(ctx, h, kind, (const float *)A, lda, (const float *)b, (const float *)x,
                                       (const float *)r)
                 : proj_error_t<double>(ctx, h, kind, (const double *)A, lda, (const double *)b, (const double *)x,
                                        (const double *)r);
    RLA_TRY(rc);
    *value = h->hstat[0];
    return RLA_OK;
}

int rla_proj_workspace(const rla_proj *h, void **compressed_mat, void **compressed_vec) {
    if (!h) return RLA_E_ARG;
    if (compressed_mat) *compressed_mat = h->Y;
    if (compressed_vec) *compressed_vec = h->Sb;
    return RLA_OK;
}

int rla_proj_destroy(rla_proj *h) {
    if (!h) return RLA_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    proj_free(h);
    cudaSetDevice(cur);
    delete h;
    return RLA_OK;
}

}  // extern "C"
