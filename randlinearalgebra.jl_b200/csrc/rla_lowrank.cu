// rla_lowrank.cu -- mul! for completed range approximators.
//
// RandSVD (randsvd.jl:198-293): C = alpha*U*diag(S)*V'*A + beta*C from the left (V'A is
// formed first, then U*(.)), and C = alpha*A*U*diag(S)*V' + beta*C from the right (A*U
// first); the adjoint swaps U and V.  RangeFinder (rangefinder.jl:151-191) is the same
// with S = NULL and V = NULL: C = alpha*range*A + beta*C.  The reference walks A in
// blocks of `block_size` columns/rows to bound its buffer; that changes no value and is
// not reproduced.  Intermediate products accumulate in FP64.
#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

__global__ void scale_rows_kernel(double *M, int64_t rows, int64_t cols, const double *s) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx < rows * cols) M[idx] *= s[idx % rows];
}

__global__ void scale_cols_kernel(double *M, int64_t rows, int64_t cols, const double *s) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx < rows * cols) M[idx] *= s[idx / rows];
}

// C = alpha*X*Y + beta*C where C may be stored transposed (trans_c).
template <class TX, class TY, class TC>
static int gemm_tc(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const TX *X, int64_t ldx, int tx, const TY *Y,
                   int64_t ldy, int ty, TC *C, int64_t ldc, int trans_c, double alpha, double beta) {
    if (!trans_c) return gemm<TX, TY, TC, double>(ctx, M, N, K, X, ldx, tx, Y, ldy, ty, C, ldc, alpha, beta);
    return gemm<TY, TX, TC, double>(ctx, N, M, K, Y, ldy, !ty, X, ldx, !tx, C, ldc, alpha, beta);
}

template <class F, class T>
static int lowrank_t(rla_ctx *ctx, int side, int trans_r, int64_t m, int64_t n, int64_t k, const F *U, int64_t ldu,
                     const double *S, const F *V, int64_t ldv, int64_t c_rows, int64_t c_cols, T *C, int64_t ldc,
                     int trans_c, int64_t a_rows, int64_t a_cols, const T *A, int64_t lda, int trans_a, double alpha,
                     double beta) {
    // R = U diag(S) V' (m x n); with V == NULL, R = U (m x k, n == k).
    const F *P = trans_r ? V : U;  // left factor of op(R)
    const F *Qf = trans_r ? U : V; // right factor (op(R) = P diag(S) Qf')
    const int64_t ldp = trans_r ? ldv : ldu, ldq = trans_r ? ldu : ldv;
    if (V == nullptr) {
        // op(R) = U or U'
        if (side == RLA_SIDE_LEFT)
            return gemm_tc<F, T, T>(ctx, c_rows, c_cols, a_rows, U, ldu, trans_r, A, lda, trans_a, C, ldc, trans_c,
                                    alpha, beta);
        return gemm_tc<T, F, T>(ctx, c_rows, c_cols, a_cols, A, lda, trans_a, U, ldu, trans_r, C, ldc, trans_c, alpha,
                                beta);
    }
    double *tmp = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&tmp, sizeof(double) * std::max<int64_t>(1, k * std::max(c_rows, c_cols)),
                                      ctx->stream));
    int rc;
    if (side == RLA_SIDE_LEFT) {
        // tmp (k x a_cols) = Qf' A ; rows scaled by S ; C = alpha * P tmp + beta C
        rc = gemm<F, T, double, double>(ctx, k, a_cols, a_rows, Qf, ldq, 1, A, lda, trans_a, tmp, k, 1.0, 0.0);
        if (rc == RLA_OK && S) {
            scale_rows_kernel<<<ceil_div_i(k * a_cols, 256), 256, 0, ctx->stream>>>(tmp, k, a_cols, S);
            rc = check_launch(ctx, "scale_rows");
        }
        if (rc == RLA_OK)
            rc = gemm_tc<F, double, T>(ctx, c_rows, c_cols, k, P, ldp, 0, tmp, k, 0, C, ldc, trans_c, alpha, beta);
    } else {
        // tmp (a_rows x k) = A P ; columns scaled by S ; C = alpha * tmp Qf' + beta C
        rc = gemm<T, F, double, double>(ctx, a_rows, k, a_cols, A, lda, trans_a, P, ldp, 0, tmp, a_rows, 1.0, 0.0);
        if (rc == RLA_OK && S) {
            scale_cols_kernel<<<ceil_div_i(a_rows * k, 256), 256, 0, ctx->stream>>>(tmp, a_rows, k, S);
            rc = check_launch(ctx, "scale_cols");
        }
        if (rc == RLA_OK)
            rc = gemm_tc<double, F, T>(ctx, c_rows, c_cols, k, tmp, a_rows, 0, Qf, ldq, 1, C, ldc, trans_c, alpha, beta);
    }
    cudaFreeAsync(tmp, ctx->stream);
    return rc;
}

}  // namespace rla

using namespace rla;

extern "C" int rla_lowrank_mul(rla_ctx *ctx, int factor_dtype, int dtype, int side, int trans_r, int64_t m, int64_t n,
                               int64_t k, const void *U, int64_t ldu, const double *S, const void *V, int64_t ldv,
                               int64_t c_rows, int64_t c_cols, void *C, int64_t ldc, int trans_c, int64_t a_rows,
                               int64_t a_cols, const void *A, int64_t lda, int trans_a, double alpha, double beta) {
    if (!ctx) return RLA_E_ARG;
    if (!U || !C || !A) return set_error(ctx, RLA_E_ARG, "NULL matrix pointer.");
    if ((V == nullptr) != (S == nullptr)) return set_error(ctx, RLA_E_ARG, "S and V are given together.");
    const int64_t r_rows = trans_r ? n : m, r_cols = trans_r ? m : n;
    // left_mul_dimcheck / right_mul_dimcheck (src/helpers/mul_dim_checks.jl:41-133)
    if (side == RLA_SIDE_LEFT) {
        if (a_rows != r_cols)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)a_rows, (long long)r_cols);
        if (a_cols != c_cols)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while C has %lld columns.", (long long)a_cols, (long long)c_cols);
        if (c_rows != r_rows)
            return set_error(ctx, RLA_E_DIM, "Matrix C has %lld rows while S has %lld rows.", (long long)c_rows, (long long)r_rows);
    } else {
        if (a_cols != r_rows)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while S has %lld rows.", (long long)a_cols, (long long)r_rows);
        if (c_cols != r_cols)
            return set_error(ctx, RLA_E_DIM, "Matrix C has %lld columns while S has %lld columns.", (long long)c_cols, (long long)r_cols);
        if (c_rows != a_rows)
            return set_error(ctx, RLA_E_DIM, "Matrix C has %lld rows while A has %lld rows.", (long long)c_rows, (long long)a_rows);
    }
    if (c_rows == 0 || c_cols == 0) return RLA_OK;
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    int rc;
#define RLA_LR(F, T)                                                                                              \
    rc = lowrank_t<F, T>(ctx, side, trans_r, m, n, k, (const F *)U, ldu, S, (const F *)V, ldv, c_rows, c_cols,    \
                         (T *)C, ldc, trans_c, a_rows, a_cols, (const T *)A, lda, trans_a, alpha, beta)
    if (factor_dtype == RLA_F64 && dtype == RLA_F64) RLA_LR(double, double);
    else if (factor_dtype == RLA_F64 && dtype == RLA_F32) RLA_LR(double, float);
    else if (factor_dtype == RLA_F32 && dtype == RLA_F32) RLA_LR(float, float);
    else RLA_LR(float, double);
#undef RLA_LR
    RLA_TRY(rc);
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}
