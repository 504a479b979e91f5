// rla_tc.cuh -- split-BF16 tensor-core GEMM (rla_tc.cu).
#pragma once

#include <cuda_bf16.h>

#include "rla_internal.cuh"

namespace rla {

using bf16 = __nv_bfloat16;

// hi = bf16(X), lo = bf16(X - hi) for X (rows x cols, ld ldx, FP32); outputs column-major
// with ld ldo (a multiple of 8, >= rows) and 16-byte aligned.
int split_bf16(rla_ctx *ctx, const float *X, int64_t rows, int64_t cols, int64_t ldx, bf16 *hi, bf16 *lo, int64_t ldo);

// NT BF16 terms of X (rows x cols, ld ldx, FP32): t0 = bf16(x), t1 = bf16(x - t0), ...;
// out[q] column-major with ld ldo (a multiple of 8, 16-byte aligned), holding X or, with
// `transpose`, X' (cols x rows).
template <int NT>
int split_terms_launch(rla_ctx *ctx, const float *X, int64_t rows, int64_t cols, int64_t ldx, int transpose,
                       bf16 *const *out, int64_t ldo);

// C (M x N, ld ldc) = alpha * op(A) * B + beta * C from the NT split terms of A (a_kmajor ?
// K x M : M x K) and of B (K x N), the term pairs of order below NT on the tensor cores.
template <int NT, class TC>
int tc_gemm_split(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *const *A, int64_t lda, int a_kmajor,
                  const bf16 *const *B, int64_t ldb, TC *C, int64_t ldc, double alpha, double beta, int splits);

// Widest tile of B columns for NT split terms (shared memory of 4 pipeline stages).
constexpr int tc_max_bn(int NT) { return NT == 2 ? 288 : 160; }

// Launch shape of one tensor-core GEMM (columns of B handled tc_max_bn(NT) at a time).
struct TcPlan {
    int BN = 0, nch = 1, stages = 2, mt = 0, nkb = 0, kbps = 0, splits = 1;
    uint32_t tmem_cols = 32;
    size_t smem = 0;
};
TcPlan tc_plan(const rla_ctx *ctx, int64_t M, int64_t N, int64_t K, int splits, int NT = 2);

// C (M x N, ld ldc) = alpha * op(A) * B + beta * C with three BF16 tensor-core products
// (hi*hi + hi*lo + lo*hi) accumulated in FP32.  A: a_kmajor ? (K x M, op = transpose) :
// (M x K); B: K x N.  All split operands column-major with ld a multiple of 8 and 16-byte
// aligned.  splits <= 0 picks the split-K count.  Asynchronous on ctx->stream.
template <class TC>
int tc_gemm_bf16x3(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *Ahi, const bf16 *Alo, int64_t lda,
                   int a_kmajor, const bf16 *Bhi, const bf16 *Blo, int64_t ldb, TC *C, int64_t ldc, double alpha,
                   double beta, int splits);

// C (M x N, ld ldc) = alpha * op(A) * op(B) + beta * C for Float32 column-major A, B with an
// FP32-accurate product on the tensor cores (three BF16 terms per operand, six MMAs per
// k-step, FP64 accumulation across k-chunks).  Asynchronous.
template <class TC>
int gemm_f32_tc(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const float *A, int64_t lda, int ta, const float *B,
                int64_t ldb, int tb, TC *C, int64_t ldc, double alpha, double beta);

// C = alpha * op(A) * B + beta * C from three BF16 terms per operand (K-major B), FP64
// accumulation across chunks of four k-blocks.  Asynchronous.
template <class TC>
int tc_gemm_f64acc(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *const *A, int64_t lda, int a_kmajor,
                   const bf16 *const *B, int64_t ldb, TC *C, int64_t ldc, double alpha, double beta);

// Device status word of the tensor-core kernels (non-zero after a timed-out wait).
int tc_status_get(rla_ctx *ctx, int **out);
// Synchronises the stream and turns a set status word into RLA_E_TIMEOUT (clearing it).
int tc_status_check(rla_ctx *ctx);

}  // namespace rla
