// rla_kernels.cuh -- internal launcher declarations shared by the translation units.
#pragma once

#include "rla_internal.cuh"

namespace rla {

// mul! without the final stream synchronisation (rla_api.cu).
int sketch_mul_impl(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s, int64_t c_rows, int64_t c_cols,
                    void *C, int64_t ldc, int trans_c, int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                    int trans_a, double alpha, double beta);

// update_compressor! ordered on ctx's stream, without waiting for it (rla_sketch.cu).
int sketch_redraw_async(rla_ctx *ctx, rla_sketch *sk);

// Sampling (rla_sampling.cu): draw for the current distribution, gather / scatter-add
// applies, parity-mode indices.
// `sync`: read the draw's precondition flags (and wait); without it they stay on the device
// for the next synchronous call to report.
int sampling_draw(rla_ctx *ctx, rla_sketch *sk, bool sync);
int sampling_set_indices(rla_ctx *ctx, rla_sketch *sk, const int64_t *idx);
template <class T>
int sampling_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                      int64_t y_es, int64_t y_vs, double alpha, double beta);
template <class T>
int sampling_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                    int64_t y_es, int64_t y_vs, double alpha, double beta);

// SparseSign / CountSketch (rla_sparse.cu).  Vectors of the input X: element (k, v) at
// X[k*x_es + v*x_vs]; the output likewise.  Compress maps length-L vectors to length s,
// expand maps length-s vectors to length L.
template <class T>
int sparse_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                    int64_t y_es, int64_t y_vs, double alpha, double beta);
template <class T>
int sparse_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                  int64_t y_es, int64_t y_vs, double alpha, double beta);

// SRHT / FJLT (rla_wht.cu)
// Builds sk->sign_tl (per-thread sign masks of the fused compress kernel) from sk->signbits.
int build_srht_sign_table(rla_ctx *ctx, rla_sketch *sk);
template <class T>
int srht_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                  int64_t y_es, int64_t y_vs, double alpha, double beta);
template <class T>
int srht_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                int64_t y_es, int64_t y_vs, double alpha, double beta);
template <class T>
int fjlt_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                  int64_t y_es, int64_t y_vs, double alpha, double beta);
template <class T>
int fjlt_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                int64_t y_es, int64_t y_vs, double alpha, double beta);

// CUDA-core GEMM (rla_gemm.cu): C = alpha*op(A)*op(B) + beta*C, column-major.  b_upper:
// op(B) is upper triangular (its entries below the diagonal are not read).
template <class TA, class TB, class TC, class TAcc>
int gemm(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const TA *A, int64_t lda, int ta, const TB *B, int64_t ldb,
         int tb, TC *C, int64_t ldc, double alpha, double beta, int b_upper = 0);

// FP64-accumulating GEMM on the FP64 tensor cores (rla_dgemm.cu): C = alpha*op(A)*op(B) +
// beta*C, column-major, Float32 or Float64 operands.  b_upper as for gemm; sym: the product
// is symmetric (M == N), only its upper tiles are computed and mirrored.
template <class TA, class TB, class TC>
int dgemm(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const TA *A, int64_t lda, int ta, const TB *B, int64_t ldb,
          int tb, TC *C, int64_t ldc, double alpha, double beta, int b_upper = 0, int sym = 0);

// G (l x l, ld l, FP64) = Y'Y for Y (rows x l, ld ldy), split over row chunks (rla_range.cu).
template <class T>
int gram_fp64(rla_ctx *ctx, const T *Y, int64_t rows, int64_t l, int64_t ldy, double *G);

// Least-squares pieces (rla_ls.cu): equilibration D G D (d = diag(G)^-1/2) and the
// solve x = d .* R^-1 R^-T (d .* c) with the Cholesky factor R of the equilibrated G.
int ls_equilibrate(rla_ctx *ctx, double *G, int64_t l, double *d);
template <class TX>
int ls_chol_solve(rla_ctx *ctx, const double *R, int64_t l, const double *d, const double *c, TX *x);

// Small dense FP64 kernels (rla_linalg.cu)
// In place: G (l x l, ld l) -> upper Cholesky factor R (lower part zeroed).  `shift` is
// added to the diagonal first.  *breakdown (device int) is set to 1 when a pivot is not
// positive.
int cholesky_upper(rla_ctx *ctx, double *G, int64_t l, double shift, int *breakdown);
// Explicit Q (in place, m x l, ld ldy) of LAPACK-style Householder QR (dgeqr2 + dorg2r);
// tau holds l doubles of workspace.
template <class T>
int householder_q(rla_ctx *ctx, T *Y, int64_t m, int64_t l, int64_t ldy, double *tau);
// Rinv = R^{-1} for upper-triangular R (l x l, ld l).
int tri_inv_upper(rla_ctx *ctx, const double *R, int64_t l, double *Rinv);
// Cholesky factor (into G: R upper, zero below) and Rinv = R^-1 together, blocked by 16 on the
// FP64 tensor cores (l <= 384, see chol_inv_supported); *breakdown as cholesky_upper.  work
// holds chol_inv_work_doubles(l) doubles.
bool chol_inv_supported(const rla_ctx *ctx, int64_t l);
size_t chol_inv_work_doubles(int64_t l);
int chol_inv(rla_ctx *ctx, double *G, int64_t l, double shift, int *breakdown, double *Rinv, double *work);
// One-sided Jacobi on X (l x l, ld l) with accumulated rotations J (initialised to I):
// on return the columns of X are orthogonal, sigma[i] = ||X(:, i)||, columns sorted by
// descending sigma, X(:, i) normalised, J permuted alongside.  `work` holds at least
// 2*l*l + 2*l doubles.
// Sweeps stop once no pair's relative off-diagonal |x_i'x_j| / (||x_i|| ||x_j||) exceeds tol.
int jacobi_svd(rla_ctx *ctx, double *X, double *J, double *sigma, int64_t l, double *work, double tol = 1e-15);

}  // namespace rla
