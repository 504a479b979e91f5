// rla_gemm.cu -- GEMM entry for the native-precision path.
//
// C(M x N) = alpha * op(A)(M x K) * op(B)(K x N) + beta * C, all column-major.
// Operand types may differ (FP32 data with an FP64 Gram accumulator, FP64 factors
// applied to FP32 data).  FP64 accumulation goes to the FP64 tensor-core kernel
// (rla_dgemm.cu); the CUDA-core kernel below serves FP32 accumulation.
#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

template <class TA, class TB, class TC, class TAcc, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
gemm_simt_kernel(int64_t M, int64_t N, int64_t K, const TA *__restrict__ A, int64_t lda, int ta,
                 const TB *__restrict__ B, int64_t ldb, int tb, TC *__restrict__ C, int64_t ldc, TAcc alpha,
                 TAcc beta, int beta_zero, int b_upper) {
    constexpr int NT = (BM / TM) * (BN / TN);
    __shared__ TAcc As[BK][BM + 1];
    __shared__ TAcc Bs[BK][BN + 1];
    const int tid = threadIdx.x;
    const int tx = tid % (BN / TN), ty = tid / (BN / TN);
    const int64_t m0 = (int64_t)blockIdx.x * BM, n0 = (int64_t)blockIdx.y * BN;
    TAcc acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = TAcc(0);
    // an upper-triangular op(B) has no rows below the diagonal of this column block
    const int64_t kend = b_upper ? min(K, n0 + BN) : K;
    for (int64_t k0 = 0; k0 < kend; k0 += BK) {
        // A tile: BM x BK ; thread order follows the contiguous dimension of A
        for (int idx = tid; idx < BM * BK; idx += NT) {
            int i, k;
            if (!ta) { i = idx % BM; k = idx / BM; }
            else { k = idx % BK; i = idx / BK; }
            const int64_t gi = m0 + i, gk = k0 + k;
            TAcc v = TAcc(0);
            if (gi < M && gk < K) v = (TAcc)(ta ? A[gk + gi * lda] : A[gi + gk * lda]);
            As[k][i] = v;
        }
        for (int idx = tid; idx < BN * BK; idx += NT) {
            int j, k;
            if (!tb) { k = idx % BK; j = idx / BK; }
            else { j = idx % BN; k = idx / BN; }
            const int64_t gj = n0 + j, gk = k0 + k;
            TAcc v = TAcc(0);
            if (gj < N && gk < K) v = (TAcc)(tb ? B[gj + gk * ldb] : B[gk + gj * ldb]);
            Bs[k][j] = v;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            TAcc a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[k][ty * TM + i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[k][tx * TN + j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
        const int64_t gj = n0 + tx * TN + j;
        if (gj >= N) continue;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int64_t gi = m0 + ty * TM + i;
            if (gi >= M) continue;
            TC *cp = C + gi + gj * ldc;
            TAcc r = alpha * acc[i][j];
            if (!beta_zero) r += beta * (TAcc)*cp;
            *cp = (TC)r;
        }
    }
}

template <class TA, class TB, class TC, class TAcc>
int gemm(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const TA *A, int64_t lda, int ta, const TB *B, int64_t ldb,
         int tb, TC *C, int64_t ldc, double alpha, double beta, int b_upper) {
    if (M <= 0 || N <= 0) return RLA_OK;
    // FP64 accumulation runs on the FP64 tensor cores
    if constexpr (std::is_same<TAcc, double>::value)
        return dgemm<TA, TB, TC>(ctx, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, alpha, beta, b_upper, 0);
    constexpr int BM = 64, BN = 64, BK = 16, TM = 4, TN = 4;
    const int64_t gx = ceil_div(M, BM), gy = ceil_div(N, BN);
    if (gy > 65535) return set_error(ctx, RLA_E_UNSUPPORTED, "GEMM grid too large (N=%lld)", (long long)N);
    dim3 grid((unsigned)gx, (unsigned)gy);
    gemm_simt_kernel<TA, TB, TC, TAcc, BM, BN, BK, TM, TN><<<grid, (BM / TM) * (BN / TN), 0, ctx->stream>>>(
        M, N, K, A, lda, ta, B, ldb, tb, C, ldc, (TAcc)alpha, (TAcc)beta, beta == 0.0, b_upper);
    return check_launch(ctx, "gemm_simt");
}

#define RLA_GEMM_INST(TA, TB, TC, TAcc)                                                                  \
    template int gemm<TA, TB, TC, TAcc>(rla_ctx *, int64_t, int64_t, int64_t, const TA *, int64_t, int, \
                                        const TB *, int64_t, int, TC *, int64_t, double, double, int);
RLA_GEMM_INST(float, float, float, float)
#define RLA_GEMM_INST_D(TA, TB) RLA_GEMM_INST(TA, TB, float, double) RLA_GEMM_INST(TA, TB, double, double)
RLA_GEMM_INST_D(float, float)
RLA_GEMM_INST_D(float, double)
RLA_GEMM_INST_D(double, float)
RLA_GEMM_INST_D(double, double)

}  // namespace rla
