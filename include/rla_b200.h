/*
 * rla_b200.h -- C ABI of the B200 (sm_100a) sketch / randomized-rangefinder library.
 *
 * This is the drop-in boundary for RandLinearAlgebra.jl v0.2.4.  The reference's own
 * extension mechanism is Julia multiple dispatch: a package adds new `Compressor` /
 * `CompressorRecipe` and `RangeApproximator` / `RangeApproximatorRecipe` subtypes and
 * methods for `complete_compressor`, `update_compressor!`, `mul!`, `*` and
 * `complete_approximator` / `rapproximate!`.  Each entry point below is what such a
 * method reaches through `ccall`; the citations name the reference method it replaces
 * (paths relative to the RandLinearAlgebra.jl source tree).
 *
 * Conventions
 *  - Every function returns an int status (RLA_OK = 0).  After a failure,
 *    rla_ctx_last_error() holds a message; for dimension and argument errors it is the
 *    same text the reference throws (src/helpers/mul_dim_checks.jl:49-60, constructors).
 *  - All matrix arguments are DEVICE pointers owned by the caller.  Matrices are
 *    column-major with an explicit leading dimension (Julia layout).  A `trans_*` flag of
 *    1 says the logical operand is the transpose of the stored column-major matrix (the
 *    layout of Julia's `transpose(X)` / `X'` wrapper of a real matrix), so the reference's
 *    adjoint routes (src/Compressors.jl:363-410) need no copies on the caller's side.
 *  - Sketch state (random draws and the derived device tables) is owned by the opaque
 *    rla_sketch and freed by rla_sketch_destroy.
 *  - Work is issued on the context's stream.  rla_sketch_mul, rla_rangefinder and
 *    rla_randsvd return after the result is complete (Julia `mul!` semantics).
 *  - beta == 0 means C is not read (BLAS convention), so C may hold garbage or NaN.
 *  - Real Float32 (RLA_F32) and Float64 (RLA_F64) element types.
 */
#ifndef RLA_B200_H
#define RLA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define RLA_OK 0
#define RLA_E_DIM 1          /* Julia DimensionMismatch */
#define RLA_E_ARG 2          /* Julia ArgumentError */
#define RLA_E_DOMAIN 3       /* Julia DomainError */
#define RLA_E_OOM 4          /* device allocation failed */
#define RLA_E_CUDA 5         /* CUDA runtime error */
#define RLA_E_TIMEOUT 6      /* a bounded device-side wait ran out */
#define RLA_E_NUMERIC 7      /* Cholesky breakdown not repaired by the shifted fallback */
#define RLA_E_UNSUPPORTED 8  /* combination not provided by this build */
#define RLA_E_CANCELLED 9    /* serving: the request was cancelled before it started */

/* ---- enumerations ---------------------------------------------------------------- */
#define RLA_F32 0
#define RLA_F64 1

#define RLA_LEFT 0           /* Left() cardinality (src/Compressors.jl:31) */
#define RLA_RIGHT 1          /* Right() cardinality (src/Compressors.jl:38) */

#define RLA_SPARSE_SIGN 0    /* src/Compressors/sparse_sign.jl */
#define RLA_COUNT_SKETCH 1   /* src/Compressors/count_sketch.jl */
#define RLA_SRHT 2           /* src/Compressors/srht.jl */
#define RLA_FJLT 3           /* src/Compressors/fjlt.jl */
#define RLA_GAUSSIAN 4       /* src/Compressors/gaussian.jl */
#define RLA_SAMPLING 5       /* src/Compressors/sampling.jl (made by rla_sampling_create) */

#define RLA_DIST_UNIFORM 0   /* src/Compressors/Distributions/uniform.jl */
#define RLA_DIST_L2NORM 1    /* src/Compressors/Distributions/strohmer_vershynin.jl */
#define RLA_DIST_AGMON 2     /* src/Compressors/Distributions/agmon.jl */

#define RLA_SIDE_LEFT 0      /* C = alpha*op(S)*A + beta*C */
#define RLA_SIDE_RIGHT 1     /* C = alpha*A*op(S) + beta*C */

#define RLA_PREC_NATIVE 0    /* GEMMs in the element type on CUDA cores */
#define RLA_PREC_SPLIT_BF16 1 /* GEMMs as split-BF16 (hi+lo) tcgen05 products, FP32 accumulate */

typedef struct rla_ctx rla_ctx;
typedef struct rla_sketch rla_sketch;

/* ---- library / context ----------------------------------------------------------- */
int rla_version(void);
const char *rla_status_string(int status);

/* Create a context on `device`.  `stream` is a cudaStream_t to borrow, or NULL for a
 * stream owned by the context. */
int rla_ctx_create(int device, void *stream, rla_ctx **out);
int rla_ctx_destroy(rla_ctx *ctx);
const char *rla_ctx_last_error(const rla_ctx *ctx);
int rla_ctx_synchronize(rla_ctx *ctx);
/* Issue the context's work on `stream` from now on (a cudaStream_t; NULL selects the
 * legacy default stream).  A stream the context created itself is released. */
int rla_ctx_set_stream(rla_ctx *ctx, void *stream);
/* Scratch high-water mark (bytes) the context holds for partial sums and transposes. */
int rla_ctx_scratch_bytes(const rla_ctx *ctx, int64_t *bytes);

/* ---- compressors ----------------------------------------------------------------- */
typedef struct rla_sketch_params {
    int kind;                /* RLA_SPARSE_SIGN ... RLA_GAUSSIAN */
    int card;                /* RLA_LEFT / RLA_RIGHT */
    int dtype;               /* RLA_F32 / RLA_F64: the compressor's `type` field */
    int64_t compression_dim; /* s */
    int64_t long_dim;        /* size(A,1) for Left, size(A,2) for Right */
    int64_t nnz;             /* SparseSign nonzeros per long index */
    int64_t block_size;      /* SRHT/FJLT padding block (kept for parity; kernels fuse it away) */
    double sparsity;         /* FJLT; 0 selects 0.25*log(L)^2/L (fjlt.jl:181) */
    uint64_t seed;
} rla_sketch_params;

typedef struct rla_sketch_info {
    int kind, card, dtype;
    int64_t n_rows, n_cols;  /* size(S) (src/Compressors.jl:310-316) */
    int64_t compression_dim, long_dim, nnz, block_size;
    int64_t padded;          /* SRHT/FJLT padded size N */
    int64_t k_nnz;           /* FJLT: stored nonzeros of K */
    double sparsity;         /* FJLT */
    double scale;            /* SRHT/FJLT `scale`, SparseSign 1/sqrt(nnz), Gaussian 1/sqrt(s) */
    uint64_t draw_count;     /* number of draws made (1 after create, +1 per update) */
} rla_sketch_info;

/* complete_compressor(::SparseSign|CountSketch|SRHT|FJLT|Gaussian, A)
 * (sparse_sign.jl:297-305, count_sketch.jl:149-156, srht.jl:193-201, fjlt.jl:228-240,
 * gaussian.jl:126-133; constructor checks sparse_sign.jl:71-87, count_sketch.jl:65-80,
 * srht.jl:67-77, fjlt.jl (FJLT inner constructor), gaussian.jl:54-60).
 * Draws are made on the device from `seed`. */
int rla_sketch_create(rla_ctx *ctx, const rla_sketch_params *params, rla_sketch **out);

/* update_compressor!(S) (sparse_sign.jl:307-336, count_sketch.jl:158-163,
 * srht.jl:205-217, fjlt.jl:242-254, gaussian.jl:136-141): fresh draws in place. */
int rla_sketch_update(rla_ctx *ctx, rla_sketch *sk);
int rla_sketch_destroy(rla_sketch *sk);
int rla_sketch_get_info(const rla_sketch *sk, rla_sketch_info *out);

/* Parity mode: copy the draws to HOST buffers in the layout of the reference's recipe
 * fields (0-based indices; a caller filling a Julia struct adds 1):
 *   SparseSign   idx = op.rowval (Left) / op.parent.rowval (Right)  [long_dim*nnz]
 *                vals = nzval [long_dim*nnz]
 *   CountSketch  idx = mat.rowval [long_dim], vals = mat.nzval [long_dim]
 *   SRHT         idx = op [compression_dim], signs = signs [padded] (1 = +1)
 *   FJLT         kptr = op.colptr, idx = op.rowval, vals = op.nzval, signs [padded]
 *   Gaussian     vals = op, column-major n_rows x n_cols
 *   Sampling     idx = idx [compression_dim]
 * Pointers a kind does not use may be NULL. */
int rla_sketch_get_draws(rla_ctx *ctx, const rla_sketch *sk, int64_t *idx, void *vals,
                         uint8_t *signs, int64_t *kptr);
/* Load externally supplied draws (same layouts) and rebuild the derived device tables.
 * For FJLT `k_nnz` is the number of stored entries of op; otherwise it is ignored. */
int rla_sketch_set_draws(rla_ctx *ctx, rla_sketch *sk, const int64_t *idx, const void *vals,
                         const uint8_t *signs, const int64_t *kptr, int64_t k_nnz);

/* complete_compressor(::Sampling, A) (src/Compressors/sampling.jl:98-121; constructor checks
 * :50-61; Agmon's beta checks src/Compressors/Distributions/agmon.jl).  The recipe is an
 * rla_sketch of kind RLA_SAMPLING: a selection of compression_dim indices of the long_dim
 * rows (Left) or columns (Right); every rla_sketch_* call accepts it, and mul! gathers
 * (compress) or scatter-adds (expand, repeated indices accumulate in order).  `replace`
 * selects sampling with replacement; `beta` is Agmon's candidate count (compression_dim <=
 * beta <= long_dim; compression_dim <= 1024).  Uniform draws at once; L2Norm and Agmon draw in
 * rla_sampling_update. */
int rla_sampling_create(rla_ctx *ctx, int card, int dtype, int64_t compression_dim, int64_t long_dim,
                        int distribution, int replace, int64_t beta, uint64_t seed, rla_sketch **out);
/* update_compressor!(S, x, A, b) for Sampling (sampling.jl:123-128): update_distribution!
 * (L2Norm: squared row/column norms of A, strohmer_vershynin.jl; Agmon: x, A, b, agmon.jl)
 * then sample_distribution!.  A (a_rows x a_cols, ld lda), x (x_len) and b (b_len) are device
 * buffers of the recipe's element type; r (optional) is Agmon's precomputed residual.
 * rla_sketch_update redraws Uniform and L2Norm (with the last weights) without data. */
int rla_sampling_update(rla_ctx *ctx, rla_sketch *sk, int64_t a_rows, int64_t a_cols, const void *A,
                        int64_t lda, const void *x, int64_t x_len, const void *b, int64_t b_len,
                        const void *r);

/* mul!(C, S, A, alpha, beta) / mul!(C, A, S, alpha, beta) and the adjoint forms
 * (src/Compressors.jl:331-384, sparse_sign.jl:339-361, count_sketch.jl:166-213,
 * srht.jl:220-504, fjlt.jl:257-535, gaussian.jl:145-170).
 *   side == RLA_SIDE_LEFT :  C = alpha*op(S)*A + beta*C
 *   side == RLA_SIDE_RIGHT:  C = alpha*A*op(S) + beta*C
 *   op(S) = S when trans_s == 0, S' when trans_s == 1 (CompressorAdjoint).
 * A is the logical (a_rows x a_cols) operand, C the logical (c_rows x c_cols) result;
 * see the trans_* convention above.  Dimension errors carry the reference's messages
 * (left_mul_dimcheck / right_mul_dimcheck). */
int rla_sketch_mul(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s,
                   int64_t c_rows, int64_t c_cols, void *C, int64_t ldc, int trans_c,
                   int64_t a_rows, int64_t a_cols, const void *A, int64_t lda, int trans_a,
                   double alpha, double beta);

/* As rla_sketch_mul, but returns once the work is queued on the context's stream; the
 * result is valid after rla_ctx_synchronize (or later stream-ordered work).  No
 * reference counterpart: it lets a caller overlap several applies. */
int rla_sketch_mul_async(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s,
                         int64_t c_rows, int64_t c_cols, void *C, int64_t ldc, int trans_c,
                         int64_t a_rows, int64_t a_cols, const void *A, int64_t lda, int trans_a,
                         double alpha, double beta);

/* mul!(C, S, transpose(B), alpha, beta) for a Left SparseSign or CountSketch recipe S and
 * a sparse B (sparse_sign.jl:364-442, count_sketch.jl:215-262): C (c_rows x c_cols,
 * column-major, ld ldc) = alpha*S*A + beta*C with A = transpose(B) (a_rows x a_cols), B an
 * a_cols x a_rows SparseMatrixCSC.  A is passed by rows, which is B's compressed-column
 * storage: a_rowptr[a_rows+1] = B.colptr - 1, a_colidx[a_nnz] = B.rowval - 1 (distinct
 * within a row), a_vals[a_nnz] = B.nzval in S's element type; all device pointers.  Each
 * C(i, c) is summed over the long indices j in increasing order, as the reference's loops
 * do; no atomics.  The first call after a draw builds a per-recipe plan (a stable sort of
 * the draws by row of S).  Synchronous.  Other recipes or cardinalities: RLA_E_ARG. */
int rla_sketch_mul_sparse_t(rla_ctx *ctx, rla_sketch *sk, int64_t c_rows, int64_t c_cols,
                            void *C, int64_t ldc, int64_t a_rows, int64_t a_cols, int64_t a_nnz,
                            const int64_t *a_rowptr, const int64_t *a_colidx, const void *a_vals,
                            double alpha, double beta);

/* ---- range approximators --------------------------------------------------------- */
typedef struct rla_range_params {
    int64_t power_its;       /* q (randsvd.jl:339, rangefinder.jl) */
    int orthogonalize;       /* rand_ortho_it (1) or rand_power_it (0) (power_its.jl) */
    int precision;           /* RLA_PREC_NATIVE or RLA_PREC_SPLIT_BF16 */
} rla_range_params;

/* rapproximate!(::RangeFinderRecipe, A) (rangefinder.jl:134-143 with
 * power_its.jl:15-80): Q (m x l, element type of A) spans range(A*Omega) after the
 * power iterations.  `omega` is a Right-cardinality compressor with long_dim == n.
 * Orthogonalisation is CholeskyQR2 with an FP64 Gram matrix (shifted CholeskyQR3 on
 * breakdown); Q's columns follow the R-diagonal-positive sign convention. */
int rla_rangefinder(rla_ctx *ctx, const rla_sketch *omega, int dtype, int64_t m, int64_t n,
                    const void *A, int64_t lda, const rla_range_params *params,
                    void *Q, int64_t ldq);

/* rapproximate!(::RandSVDRecipe, A) (randsvd.jl:174-189): Q as above, B = Q'A, the SVD
 * of B in FP64, U = Q*W.  U (m x l) and V (n x l) are written in `out_dtype`
 * (RLA_F64 matches the reference, which promotes the factors to Float64); S (l values,
 * descending) is always Float64. */
int rla_randsvd(rla_ctx *ctx, const rla_sketch *omega, int dtype, int64_t m, int64_t n,
                const void *A, int64_t lda, const rla_range_params *params, int out_dtype,
                void *U, int64_t ldu, double *S, void *V, int64_t ldv);

/* mul! for completed approximators: RandSVD (randsvd.jl:198-293) with R = U*diag(S)*V'
 * (U m x k, V n x k, S k values in FP64), and RangeFinder (rangefinder.jl:151-191) with
 * S = V = NULL and R = U (m x k, n == k).  trans_r selects R' (ApproximatorAdjoint,
 * src/Approximators.jl:363-384).  Factors are `factor_dtype`, A and C are `dtype`;
 * A, C, side and trans flags as in rla_sketch_mul.  Device pointers; synchronous. */
int rla_lowrank_mul(rla_ctx *ctx, int factor_dtype, int dtype, int side, int trans_r,
                    int64_t m, int64_t n, int64_t k, const void *U, int64_t ldu, const double *S,
                    const void *V, int64_t ldv,
                    int64_t c_rows, int64_t c_cols, void *C, int64_t ldc, int trans_c,
                    int64_t a_rows, int64_t a_cols, const void *A, int64_t lda, int trans_a,
                    double alpha, double beta);

/* ---- batched RandSVD (grouped launches, CUDA graph) -------------------------------- */
/* Many rapproximate!(RandSVD) calls at once (randsvd.jl:174-189 per instance, with the
 * reference's defaults: Gaussian Right compressor with compression_dim = k, p = 0, the
 * given power_its / orthogonalize).  Instance i: A (m x n, Float32, column-major, device)
 * -> U (m x k, Float32), S (k, Float64, descending), V (n x k, Float32); k <= min(m, n, 128).
 * Omega is drawn exactly as rla_sketch_create(RLA_GAUSSIAN, RLA_RIGHT, RLA_F32, k, n, seed)
 * draws it.  Products with A accumulate in FP32, Gram/Cholesky/SVD in FP64.  No single
 * reference function: the reference runs the instances one after another. */
typedef struct rla_svd_problem {
    int64_t m, n, k;
    const float *A;
    int64_t lda;
    float *U;
    int64_t ldu;
    double *S;
    float *V;
    int64_t ldv;
    uint64_t seed;
} rla_svd_problem;

typedef struct rla_batch rla_batch;
#define RLA_BATCH_AUTOTUNE 1 /* time candidate tile shapes on the problem set at creation */
#define RLA_BATCH_EAGER 2    /* launch directly on the context's stream, no CUDA graph */

/* Plan a batch: workspaces, per-rank-class grouped launch tables, tuned tile shapes.  The
 * problem list (pointers included) is fixed for the plan's lifetime.  Its device memory
 * comes from the context's pool, so the context must outlive the batch. */
int rla_randsvd_batch_create(rla_ctx *ctx, int count, const rla_svd_problem *problems,
                             const rla_range_params *params, int flags, rla_batch **out);
/* Run the batch on the context's stream: the first run captures the grouped launch
 * sequence as a CUDA graph, later runs replay it.  Returns when every instance is done
 * (instances whose Cholesky broke down are recomputed by the single-instance path). */
int rla_randsvd_batch_run(rla_ctx *ctx, rla_batch *batch);
/* Tile shapes in use for rank class c (0: k <= 16, 1: <= 32, 2: <= 64, 3: <= 128): rows
 * per CTA of A*Omega (64, 128 or 256), columns of A per CTA of A'Q (64, 128 or 256) and its
 * row chunk. */
int rla_randsvd_batch_tiles(const rla_batch *batch, int c, int *rows_a_omega, int *cols_at_q,
                            int64_t *chunk_at_q);
int rla_randsvd_batch_destroy(rla_batch *batch);
/* create (no tuning) + run + destroy */
int rla_randsvd_grouped(rla_ctx *ctx, int count, const rla_svd_problem *problems,
                        const rla_range_params *params);

/* ---- sketch-and-solve least squares -------------------------------------------------- */
/* x = argmin ||S(Ax - b)|| for a Left Float32 compressor S (s x m, s >= n), A (m x n),
 * b (m), x (n): SA and Sb by the sketch kernels, then the sketched normal equations through
 * the FP64 Cholesky factor of the equilibrated Gram matrix of SA.  The least-squares request
 * of the serving loop; the reference's solvers reach the same sketch through mul!
 * (src/Solvers/ihs.jl:231-236).  Device pointers; synchronous; RLA_E_NUMERIC when the
 * sketched Gram matrix is not positive definite. */
int rla_sketch_solve(rla_ctx *ctx, const rla_sketch *sk, int64_t m, int64_t n, const float *A,
                     int64_t lda, const float *b, float *x);

/* ---- Iterative Hessian Sketch solver ------------------------------------------------------
 * IHS (src/Solvers/ihs.jl:40-254) for min ||Ax - b|| with A (m x n, m > n), a Left compressor S
 * (s x m, n <= s <= m) of the same element type, step size alpha.  All vectors are device
 * buffers the caller owns: b (m), x (n, the solution_vec, updated in place), r (m, the
 * residual_vec), g (n, the gradient_vec).
 *   rla_ihs_create  complete_solver (ihs.jl:127-206): its ArgumentError checks, same wording
 *                   and order; workspaces (compressed_mat s x n, Gram, partial sums).
 *   rla_ihs_start   the start of rsolve! (ihs.jl:214-223): r = b - A x, then iteration 1's
 *                   gradient g = A'r and error values.
 *   rla_ihs_step    the rest of an iteration (ihs.jl:231-249): update_compressor!, S*A, the
 *                   R'R of S*A (FP64 Cholesky of the equilibrated Gram matrix; the same R'R as
 *                   qr!(S*A).R), u = R \ (R' \ g), x += alpha*u, r -= A*u (by A*u also when
 *                   alpha != 1, as the reference does), then the next iteration's g and errors.
 *   rla_ihs_errors  the error values of the current iteration (synchronises): FullResidual
 *                   ||b - Ax|| (full_residual.jl) and LSGradient ||A'r|| (ls_gradient.jl);
 *                   RLA_E_NUMERIC if the last step's sketched Gram matrix was not positive
 *                   definite.
 *   rla_ihs_solve   rsolve! with BasicLogger(max_it, collection_rate, threshold) and
 *                   threshold_stop (src/Solvers/Loggers/basic_logger.jl:84-130): hist gets
 *                   ceil(max_it/collection_rate)+1 entries; *iterations = the last logged
 *                   iteration, *converged = the logger's converged flag.
 * Asynchronous on the context's stream except rla_ihs_errors and rla_ihs_solve. */
typedef struct rla_ihs rla_ihs;
#define RLA_IHS_FULL_RESIDUAL 0
#define RLA_IHS_LS_GRADIENT 1
int rla_ihs_create(rla_ctx *ctx, rla_sketch *compressor, int dtype, int64_t m, int64_t n, double alpha,
                   rla_ihs **out);
int rla_ihs_start(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, const void *x,
                  void *r, void *g);
int rla_ihs_step(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, void *x, void *r,
                 void *g);
int rla_ihs_errors(rla_ctx *ctx, rla_ihs *h, double *full_residual, double *ls_gradient);
int rla_ihs_solve(rla_ctx *ctx, rla_ihs *h, const void *A, int64_t lda, const void *b, void *x, void *r,
                  void *g, int64_t max_it, int64_t collection_rate, double threshold, int error_kind,
                  double *hist, int64_t hist_len, int64_t *iterations, int *converged);
/* ---- Kaczmarz and ColumnProjection ---------------------------------------------------------
 * Kaczmarz (src/Solvers/kaczmarz.jl:63-368; Left compressor S, s x m) and ColumnProjection
 * (src/Solvers/col_projection.jl:63-372; Right compressor S, n x s) on A (m x n, ld lda).
 * One step is one iteration after the logger check: update_compressor!, the sketched block
 * (S*A and S*b, or A*S), the sub-problem -- Kaczmarz: the minimum-norm correction of the
 * sketched rows (LQSolver, lq.jl; the scalar kaczmarz_update! for s = 1; no update when the
 * sketched rows are zero); ColumnProjection: the least-squares correction over the sketched
 * columns (QRSolver, qr.jl) -- through the FP64 Cholesky factor of the equilibrated s x s
 * Gram matrix, then x += alpha*u (and r -= alpha*A*S*u).  b, x, r are device vectors of the
 * element type the caller owns; ColumnProjection keeps the residual r = b - Ax
 * (rla_proj_start sets it).  rla_proj_error computes an error method's value for the current
 * iterate (synchronises): RLA_ERR_FULL_RESIDUAL ||b - Ax|| (full_residual.jl),
 * RLA_ERR_LS_GRADIENT ||A'r|| (ls_gradient.jl), RLA_ERR_COMPRESSED_RESIDUAL ||Sb - SAx|| of
 * the last sketched rows (compressed_residual.jl; 0 before the first step); RLA_E_NUMERIC
 * when the last sub-problem was singular.  Block sizes s <= 4096. */
typedef struct rla_proj rla_proj;
#define RLA_PROJ_KACZMARZ 0
#define RLA_PROJ_COLUMN 1
#define RLA_ERR_FULL_RESIDUAL 0
#define RLA_ERR_LS_GRADIENT 1
#define RLA_ERR_COMPRESSED_RESIDUAL 2
int rla_proj_create(rla_ctx *ctx, rla_sketch *compressor, int kind, int dtype, int64_t m, int64_t n,
                    double alpha, rla_proj **out);
int rla_proj_start(rla_ctx *ctx, rla_proj *h, const void *A, int64_t lda, const void *b, const void *x,
                   void *r);
int rla_proj_step(rla_ctx *ctx, rla_proj *h, const void *A, int64_t lda, const void *b, void *x,
                  void *r);
int rla_proj_error(rla_ctx *ctx, rla_proj *h, int kind, const void *A, int64_t lda, const void *b,
                   const void *x, const void *r, double *value);
/* The last sketched block (owned by the solver): Kaczmarz (S*A)' (n x s, ld n) and S*b (s);
 * ColumnProjection A*S (m x s, ld m). */
int rla_proj_workspace(const rla_proj *h, void **compressed_mat, void **compressed_vec);
int rla_proj_destroy(rla_proj *h);

/* Device workspaces of the solver (owned by it): compressed_mat (s x n, ld s, the element
 * type; the last S*A), update (n; the last u), R_equilibrated (n x n FP64, upper triangle; the
 * Cholesky factor of D (SA)'(SA) D) and d (n FP64; D = diag(d)), so R = R_equilibrated D^-1. */
int rla_ihs_workspace(const rla_ihs *h, void **compressed_mat, void **update, double **R_equilibrated,
                      double **d);
int rla_ihs_destroy(rla_ihs *h);

/* ---- serving loop ------------------------------------------------------------------------ */
/* No reference counterpart (the reference is a library of one-call functions).  Mixed
 * requests -- sketch-and-solve least squares (SparseSign Left, s = min(4n, m), nnz = 8) and
 * RandSVD (Gaussian, compression_dim = k, p = 0, q = 0) -- on Float32 device buffers the
 * caller owns and keeps alive until the request is polled as done. */
#define RLA_REQ_LS 0
#define RLA_REQ_SVD 1
typedef struct rla_request {
    int kind;                 /* RLA_REQ_LS or RLA_REQ_SVD */
    int64_t m, n, k;          /* A is m x n; k: RandSVD rank (ignored for LS) */
    const float *A;
    int64_t lda;
    const float *b;           /* LS: right-hand side (m) */
    float *x;                 /* LS: solution (n) */
    float *U;                 /* RandSVD: U (m x k), S (k, Float64), V (n x k) */
    int64_t ldu;
    double *S;
    float *V;
    int64_t ldv;
    uint64_t seed;            /* sketch seed (sketches are kept resident per shape and seed) */
    uint64_t tag;             /* returned by rla_server_poll */
} rla_request;

#define RLA_SERVE_BATCHED 0   /* continuous batching: slots work at once, RandSVD grouped */
#define RLA_SERVE_PLAIN 1     /* baseline: one request at a time, single-instance path */
typedef struct rla_server_config {
    int device;
    int slots;                /* concurrent workers (each with its own stream) */
    int max_group;            /* RandSVD requests (k <= 128, m*n <= 2^22) run as one grouped batch */
    int mode;                 /* RLA_SERVE_BATCHED or RLA_SERVE_PLAIN */
    uint64_t memory_budget;   /* bytes of workspace admitted at once (0: 150 GB) */
    uint64_t sketch_cache_bytes; /* cap on resident sketches (0: memory_budget / 8); counted
                                    in the budget, least recently used evicted first */
} rla_server_config;

typedef struct rla_server rla_server;
int rla_server_start(const rla_server_config *cfg, rla_server **out);
/* Queue a request (returns at once). */
int rla_server_submit(rla_server *srv, const rla_request *req);
/* Up to `max` completed requests: tags, submit-to-done latency (s) and status. */
int rla_server_poll(rla_server *srv, uint64_t *tags, double *latency_s, int *status, int max, int *count);
/* Message of the first failed request ("" when none failed); valid until the next call. */
const char *rla_server_last_error(rla_server *srv);
/* Block until the queue is empty and nothing runs. */
int rla_server_wait_idle(rla_server *srv);
/* Remove a request that is still queued; rla_server_poll then reports it with status
 * RLA_E_CANCELLED.  RLA_E_ARG when no queued request has that tag (it already started). */
int rla_server_cancel(rla_server *srv, uint64_t tag);
/* Fault injection on the host (failure-detection tests): when the request with this tag is
 * taken by a worker, its workspace allocation fails as if the device were out of memory;
 * that request alone completes with RLA_E_OOM and nothing of it reaches the GPU. */
int rla_server_inject_alloc_failure(rla_server *srv, uint64_t tag);
typedef struct rla_server_stats {
    int64_t queued, running;     /* requests waiting / being worked on */
    uint64_t workspace_bytes;    /* estimated workspace of the running requests */
    uint64_t cache_bytes;        /* resident sketches (estimated device bytes) */
    int64_t cache_entries, evictions;
} rla_server_stats;
int rla_server_get_stats(rla_server *srv, rla_server_stats *out);
/* Finish queued work and shut the workers down. */
int rla_server_stop(rla_server *srv);

/* ---- kernel timing (tracing aid, no reference counterpart) ------------------------- */
/* While enabled, the context records CUDA events around each launch of a timed kernel
 * class on its stream (class 0: the tensor-core GEMM kernel; 1: the IHS fused pass over A;
 * 2: the IHS compressor apply S*A; 3: the L2Norm weights pass of rla_sampling_update).
 * rla_ctx_kernel_time
 * synchronises the stream, returns the summed device time (ms) and launch count of the
 * class since the last call, and clears the record. */
int rla_ctx_set_timing(rla_ctx *ctx, int enable);
int rla_ctx_kernel_time(rla_ctx *ctx, int kernel_class, double *ms_total, int64_t *launches);

/* ---- bounded device-side waits (failure detection, no reference counterpart) ---------- */
/* Limit, in seconds (0 to 60, default 2), of one pipeline wait of the tensor-core GEMM
 * kernel on an mbarrier.  A wait that runs out makes every CTA of the launch stop issuing
 * work, wait (for at most 2 s more) for the copies and MMAs it already issued, release its
 * tensor memory and exit; the call then returns RLA_E_TIMEOUT and the context stays usable.
 * A limit of 0 makes any wait that is not already satisfied run out (used by the tests). */
int rla_ctx_set_wait_limit(rla_ctx *ctx, double seconds);

/* ---- split-BF16 tensor-core GEMM ------------------------------------------------ */
/* No counterpart in the reference (its products go to BLAS gemm): the product kernel used
 * by RLA_PREC_SPLIT_BF16, exposed for callers and tests.  C = alpha*op(A)*B + beta*C with
 * FP32 column-major A (op(A) = A, m x k, when trans_a = 0; A', A stored k x m, when
 * trans_a = 1), B (k x n) and C (m x n).  Each operand is split into hi = bf16(x) and
 * lo = bf16(x - hi); the 5th-generation tensor cores form hi*hi + hi*lo + lo*hi with FP32
 * accumulation (about 2^-16 relative error per product).  Device pointers; allocates the
 * split copies on the context's stream; synchronous.  RLA_E_TIMEOUT when a bounded
 * pipeline wait on the device ran out. */
int rla_gemm_bf16x3(rla_ctx *ctx, int trans_a, int64_t m, int64_t n, int64_t k,
                    const float *A, int64_t lda, const float *B, int64_t ldb,
                    float *C, int64_t ldc, double alpha, double beta);

/* ---- allocation-free SRHT apply -------------------------------------------------- */
/* No counterpart in the reference.  C = alpha*S*A + beta*C for a Left-cardinality SRHT
 * recipe S (s x m), column-major A (m x n) and C (s x n), on the context's stream, without
 * allocating device memory: for callers that cannot call cudaMalloc -- code that owns a
 * fixed device-memory budget and hands every byte out itself, code whose device memory
 * belongs to another runtime's pool, code on paths that must not touch the allocator.
 * The kernel's partial sums live in library-owned fixed device arrays of
 * RLA_NOALLOC_SCRATCH_BYTES bytes plus RLA_NOALLOC_MAX_COLS counters, held by every GPU
 * that loads the library until the process exits.  n above RLA_NOALLOC_MAX_COLS, or a
 * compression dimension whose partial sums cannot fit, is rejected with RLA_E_ARG.
 * The first call on a device looks up the arrays' device addresses; make that first call
 * before any stream capture.  All calls share the arrays, which keep the last call's
 * contents: calls whose GPU work overlaps (other streams or threads without ordering)
 * race.  The call runs on the context's device and leaves the calling thread's current
 * device as it found it.  Negative dimensions are rejected with RLA_E_ARG.  Returns once
 * the work is queued; synchronize the stream before reading C. */
#define RLA_NOALLOC_SCRATCH_BYTES (8u << 20)
#define RLA_NOALLOC_MAX_COLS 65536
int rla_srht_mul_noalloc(rla_ctx *ctx, const rla_sketch *sk,
                         int64_t c_rows, int64_t c_cols, void *C, int64_t ldc,
                         int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                         double alpha, double beta);

#ifdef __cplusplus
}
#endif
#endif /* RLA_B200_H */
