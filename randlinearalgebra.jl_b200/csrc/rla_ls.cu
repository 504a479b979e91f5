// rla_ls.cu -- sketch-and-solve least squares on the device.
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
// solves a 32 x 32 diagonal triangle with shuffles (the block's entries in registers), then
// all threads apply the block to the rest of the vector; two barriers per block.  One CTA;
// the vector in shared memory.
__global__ void __launch_bounds__(1024) ls_trisolve_kernel(const double *R, int64_t l, const double *d,
                                                          const double *c, float *x) {
    extern __shared__ double v[];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t i = tid; i < l; i += nt) v[i] = d[i] * c[i];
    __syncthreads();
    // forward: R' y = v, R' lower; block rows [b, b+32)
    for (int64_t b = 0; b < l; b += 32) {
        const int nb = (int)min((int64_t)32, l - b);
        if (warp == 0) {
            double yv = lane < nb ? v[b + lane] : 0.0;
            for (int t = 0; t < nb; ++t) {
                const double yt = __shfl_sync(FULL, yv, t) / R[(b + t) + (b + t) * l];
                if (lane == t) yv = yt;
                if (lane > t && lane < nb) yv -= yt * R[(b + t) + (b + lane) * l];
            }
            if (lane < nb) v[b + lane] = yv;
        }
        __syncthreads();
        // v(j) -= sum_{t in block} R(b+t, j) y(b+t) for j >= b+nb
        for (int64_t j = b + nb + tid; j < l; j += nt) {
            double acc = 0.0;
            for (int t = 0; t < nb; ++t) acc += R[(b + t) + j * l] * v[b + t];
            v[j] -= acc;
        }
        __syncthreads();
    }
    // backward: R z = y; block rows [b, b+nb) from the bottom
    for (int64_t e = l; e > 0; e -= 32) {
        const int nb = (int)min((int64_t)32, e);
        const int64_t b = e - nb;
        if (warp == 0) {
            double zv = lane < nb ? v[b + lane] : 0.0;
            for (int t = nb - 1; t >= 0; --t) {
                const double zt = __shfl_sync(FULL, zv, t) / R[(b + t) + (b + t) * l];
                if (lane == t) zv = zt;
                if (lane < t) zv -= zt * R[(b + lane) + (b + t) * l];
            }
            if (lane < nb) v[b + lane] = zv;
        }
        __syncthreads();
        // v(j) -= sum_{t in block} R(j, b+t) z(b+t) for j < b
        for (int64_t j = tid; j < b; j += nt) {
            double acc = 0.0;
            for (int t = 0; t < nb; ++t) acc += R[j + (b + t) * l] * v[b + t];
            v[j] -= acc;
        }
        __syncthreads();
    }
    for (int64_t i = tid; i < l; i += nt) x[i] = (float)(d[i] * v[i]);
}

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
        RLA_CUDA_TRY(ctx, set_smem_max(ls_trisolve_kernel));
    ls_trisolve_kernel<<<1, 1024, smem, ctx->stream>>>(G, n, tmp, c, x);
    RLA_TRY(check_launch(ctx, "ls_trisolve"));
    *bad_out = bad;
    return RLA_OK;
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

}  // extern "C"
