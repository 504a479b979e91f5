// rla_tc.cuh -- split-BF16 tensor-core GEMM (rla_tc.cu).
#pragma once

#include <cuda_bf16.h>

#include <vector>

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
    int main_cols = 0, rem_cols = 0;  // NT = 2: column split of the tile (see TcParams)
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

// Grouped products for many instances in one launch (split BF16, two terms): item q is
// op(A_q) (M x K) * B_q (K x N, N <= 64, K-major), FP64 accumulation across k-chunks, written
// to out (and out2 when set) as Float32 or Float64 with leading dimension ldo.  The tensor
// maps and tile table are built once (tc_group_build) for fixed buffers and reused by every
// launch (tc_group_run), which allocates nothing and can be captured in a graph.
struct TcGroupSpec {
    const bf16 *a[2];
    int64_t lda;
    int a_kmajor;
    const bf16 *b[2];
    int64_t ldb;
    int64_t M, N, K;
    void *out, *out2;
    int64_t ldo;
    int out_f64;
};
// The item tables live in the building context's memory pool and are released in the order
// of its stream (a synchronous free would wait for every stream on the device).
struct TcGroup {
    void *items = nullptr;
    int *tstart = nullptr;
    int count = 0, tiles = 0, stages = 2;
    size_t smem = 0;
    int *status = nullptr;
    cudaStream_t stream = nullptr;  // stream the tables are allocated and released on
};
int tc_group_build(rla_ctx *ctx, const std::vector<TcGroupSpec> &specs, TcGroup *g);
int tc_group_run(rla_ctx *ctx, const TcGroup &g, cudaStream_t st);
void tc_group_free(TcGroup *g);

// Grouped FP32 -> (hi, lo) BF16 splits of many matrices in one launch.
struct SplitSpec {
    const float *X;
    int64_t rows, cols, ldx;
    bf16 *hi, *lo;
    int64_t ldo;
};
struct SplitGroup {
    void *items = nullptr;
    int *bstart = nullptr;
    int count = 0, blocks = 0;
    cudaStream_t stream = nullptr;  // stream the tables are allocated and released on
};
int split_group_build(rla_ctx *ctx, const std::vector<SplitSpec> &specs, SplitGroup *g);
int split_group_run(rla_ctx *ctx, const SplitGroup &g, cudaStream_t st);
void split_group_free(SplitGroup *g);

// Device status word of the tensor-core kernels (non-zero after a timed-out wait).
int tc_status_get(rla_ctx *ctx, int **out);
// Synchronises the stream and turns a set status word into RLA_E_TIMEOUT (clearing it).
int tc_status_check(rla_ctx *ctx);

}  // namespace rla
