/*
 * rla_oracle.c -- CPU restatement of RandLinearAlgebra.jl's sketch-application path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline leg of bench.py load it, and only as the
 * checker (or as the timed CPU baseline).  The B200 product path never links it.
 *
 * Each routine restates, loop for loop, the Julia code it cites (paths are relative to
 * the RandLinearAlgebra.jl v0.2.4 source tree).  Matrices are strided views: element
 * (i, j) of a view lives at p[i*rs + j*cs], so Julia's column-major arrays are rs = 1,
 * cs = ld, and Julia's `transpose(X)` wrappers are the same buffer with rs/cs swapped.
 * That lets the adjoint routes of src/Compressors.jl:363-410 be restated literally as
 * calls on transposed views.  Indices are 0-based here (Julia's are 1-based).
 *
 * The sparse kernels restate the Julia 1.12 stdlib SparseArrays methods that the
 * reference reaches through `mul!(C, S.op, A, alpha, beta)`:
 *   _spmatmul!            C = a*S*A + b*C      (CSC x dense)
 *   _At_or_Ac_mul_B!      C = a*S'*A + b*C     (adjoint CSC x dense)
 *   _spmul!               C = a*X*S + b*C      (dense x CSC)
 *   _A_mul_Bt_or_Bc!      C = a*X*S' + b*C     (dense x adjoint CSC)
 * SparseArrays is not vendored with the reference; its loop order only affects the
 * last bits of rounding, and parity is checked against tolerance for floating point.
 *
 * Parity pinning: tests/test_oracle_pins.py checks every routine here against the
 * reference's own test formulas (explicit Sylvester Hadamard products, dense
 * re-materialised sparse operators) on the fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_E_DIM 1
#define ORC_E_ARG 2
#define ORC_E_OOM 3

static int is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

/* ---------------------------------------------------------------------------------
 * Template over the element type.  ORC_T is the storage/compute type, ORC_S the
 * symbol suffix (f = Float32, d = Float64).
 * ------------------------------------------------------------------------------- */
#define ORC_DEFINE(ORC_T, ORC_S)                                                          \
                                                                                           \
/* fwht!(x, signs; scaling) -- src/Compressors/helpers/fwht.jl:21-70.                      \
 * x is a strided vector (stride inc).  signs[i] != 0 means +1.  Returns ORC_E_DIM         \
 * for the two DimensionMismatch cases of fwht.jl:25-32.  Length 1 is treated as the       \
 * identity times the signed scale (the reference reads past the end there).  */           \
int orc_fwht_signed_##ORC_S(ORC_T *x, int64_t ln, int64_t inc, const uint8_t *signs,      \
                            int64_t ls, double scaling) {                                  \
    if (ls != ln) return ORC_E_DIM;                                                        \
    if (!is_pow2(ln)) return ORC_E_DIM;                                                    \
    if (ln == 1) { x[0] = (ORC_T)(x[0] * (signs[0] ? scaling : -scaling)); return 0; }     \
    int64_t h = 1, step = 2;                                                               \
    /* first pass: scale and flip signs (fwht.jl:41-48) */                                 \
    for (int64_t i = 0; i < ln; i += step) {                                               \
        double z = (double)x[i * inc] * (signs[i] ? scaling : -scaling);                   \
        double y = (double)x[(i + h) * inc] * (signs[i + h] ? scaling : -scaling);         \
        x[i * inc] = (ORC_T)(z + y);                                                       \
        x[(i + h) * inc] = (ORC_T)(z - y);                                                 \
    }                                                                                      \
    /* remaining log2(ln) - 1 butterfly passes (fwht.jl:50-66) */                          \
    while (2 * h < ln) {                                                                   \
        h <<= 1;                                                                           \
        step = h << 1;                                                                     \
        for (int64_t i = 0; i < ln; i += step) {                                           \
            for (int64_t j = i; j < i + h; ++j) {                                          \
                ORC_T z = x[j * inc];                                                      \
                ORC_T y = x[(j + h) * inc];                                                \
                x[j * inc] = z + y;                                                        \
                x[(j + h) * inc] = z - y;                                                  \
            }                                                                              \
        }                                                                                  \
    }                                                                                      \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* fwht!(x; scaling) -- src/Compressors/helpers/fwht.jl:73-118. */                         \
int orc_fwht_##ORC_S(ORC_T *x, int64_t ln, int64_t inc, double scaling) {                  \
    if (!is_pow2(ln)) return ORC_E_DIM;                                                    \
    if (ln == 1) { x[0] = (ORC_T)(x[0] * scaling); return 0; }                             \
    int64_t h = 1, step = 2;                                                               \
    for (int64_t i = 0; i < ln; i += step) {                                               \
        double z = (double)x[i * inc] * scaling;                                           \
        double y = (double)x[(i + h) * inc] * scaling;                                     \
        x[i * inc] = (ORC_T)(z + y);                                                       \
        x[(i + h) * inc] = (ORC_T)(z - y);                                                 \
    }                                                                                      \
    while (2 * h < ln) {                                                                   \
        h <<= 1;                                                                           \
        step = h << 1;                                                                     \
        for (int64_t i = 0; i < ln; i += step) {                                           \
            for (int64_t j = i; j < i + h; ++j) {                                          \
                ORC_T z = x[j * inc];                                                      \
                ORC_T y = x[(j + h) * inc];                                                \
                x[j * inc] = z + y;                                                        \
                x[(j + h) * inc] = z - y;                                                  \
            }                                                                              \
        }                                                                                  \
    }                                                                                      \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* rmul!/fill! prologue shared by the SparseArrays methods (beta == 0 fills zeros). */     \
static void orc_scale_##ORC_S(ORC_T *C, int64_t cr, int64_t cc, int64_t crs, int64_t ccs, \
                              double beta) {                                               \
    if (beta == 1.0) return;                                                               \
    for (int64_t j = 0; j < cc; ++j)                                                       \
        for (int64_t i = 0; i < cr; ++i)                                                   \
            C[i * crs + j * ccs] = beta == 0.0 ? (ORC_T)0 : (ORC_T)(C[i * crs + j * ccs] * beta); \
}                                                                                          \
                                                                                           \
/* C = alpha*S*A + beta*C with S an (sr x sc) CSC matrix (SparseArrays _spmatmul!). */     \
void orc_csc_mul_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, int64_t sr, int64_t sc,      \
                         const int64_t *colptr, const int64_t *rowval, const ORC_T *nzval, \
                         const ORC_T *A, int64_t ars, int64_t acs, int64_t n,              \
                         double alpha, double beta) {                                      \
    orc_scale_##ORC_S(C, sr, n, crs, ccs, beta);                                           \
    for (int64_t k = 0; k < n; ++k)                                                        \
        for (int64_t col = 0; col < sc; ++col) {                                           \
            ORC_T axj = (ORC_T)(A[col * ars + k * acs] * alpha);                           \
            for (int64_t j = colptr[col]; j < colptr[col + 1]; ++j)                        \
                C[rowval[j] * crs + k * ccs] += nzval[j] * axj;                            \
        }                                                                                  \
}                                                                                          \
                                                                                           \
/* C = alpha*S'*A + beta*C, S (sr x sc) CSC, C is (sc x n) (SparseArrays                   \
 * _At_or_Ac_mul_B!). */                                                                   \
void orc_csc_adj_mul_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, int64_t sr, int64_t sc,  \
                             const int64_t *colptr, const int64_t *rowval,                 \
                             const ORC_T *nzval, const ORC_T *A, int64_t ars, int64_t acs, \
                             int64_t n, double alpha, double beta) {                       \
    (void)sr;                                                                              \
    orc_scale_##ORC_S(C, sc, n, crs, ccs, beta);                                           \
    for (int64_t k = 0; k < n; ++k)                                                        \
        for (int64_t col = 0; col < sc; ++col) {                                           \
            ORC_T tmp = 0;                                                                 \
            for (int64_t j = colptr[col]; j < colptr[col + 1]; ++j)                        \
                tmp += nzval[j] * A[rowval[j] * ars + k * acs];                            \
            C[col * crs + k * ccs] += (ORC_T)(tmp * alpha);                                \
        }                                                                                  \
}                                                                                          \
                                                                                           \
/* C = alpha*X*S + beta*C, X (mx x sr) dense, S (sr x sc) CSC (SparseArrays _spmul!). */   \
void orc_dense_mul_csc_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *X,        \
                               int64_t xrs, int64_t xcs, int64_t mx, int64_t sr,           \
                               int64_t sc, const int64_t *colptr, const int64_t *rowval,   \
                               const ORC_T *nzval, double alpha, double beta) {            \
    (void)sr;                                                                              \
    orc_scale_##ORC_S(C, mx, sc, crs, ccs, beta);                                          \
    for (int64_t r = 0; r < mx; ++r)                                                       \
        for (int64_t col = 0; col < sc; ++col)                                             \
            for (int64_t k = colptr[col]; k < colptr[col + 1]; ++k)                        \
                C[r * crs + col * ccs] += (ORC_T)(alpha * X[r * xrs + rowval[k] * xcs]) * nzval[k]; \
}                                                                                          \
                                                                                           \
/* C = alpha*X*S' + beta*C, X (mx x sc) dense, S (sr x sc) CSC, C (mx x sr)                \
 * (SparseArrays _A_mul_Bt_or_Bc!). */                                                     \
void orc_dense_mul_csc_adj_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *X,    \
                                   int64_t xrs, int64_t xcs, int64_t mx, int64_t sr,       \
                                   int64_t sc, const int64_t *colptr,                      \
                                   const int64_t *rowval, const ORC_T *nzval,              \
                                   double alpha, double beta) {                            \
    orc_scale_##ORC_S(C, mx, sr, crs, ccs, beta);                                          \
    for (int64_t col = 0; col < sc; ++col)                                                 \
        for (int64_t k = colptr[col]; k < colptr[col + 1]; ++k)                            \
            for (int64_t r = 0; r < mx; ++r)                                               \
                C[r * crs + rowval[k] * ccs] += (ORC_T)(alpha * X[r * xrs + col * xcs]) * nzval[k]; \
}                                                                                          \
                                                                                           \
/* mul!(C, S::SRHTRecipe{Left}, A, alpha, beta) -- src/Compressors/srht.jl:220-286.        \
 * S is (s x m), N = padded size, op = sampled rows (0-based), A (m x n), C (s x n). */    \
int orc_srht_left_SA_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,          \
                             int64_t ars, int64_t acs, int64_t m, int64_t n, int64_t s,    \
                             int64_t N, const int64_t *op, const uint8_t *signs,           \
                             double scale, int64_t bsize, double alpha, double beta) {     \
    ORC_T *pad = (ORC_T *)malloc(sizeof(ORC_T) * N * bsize);                               \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t c0 = 0; c0 < n; c0 += bsize) {                                            \
        int64_t bw = n - c0 < bsize ? n - c0 : bsize;                                      \
        memset(pad, 0, sizeof(ORC_T) * N * bsize);                                         \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t r = 0; r < m; ++r) pad[r + i * N] = A[r * ars + (c0 + i) * acs];  \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_signed_##ORC_S(pad + i * N, N, 1, signs, N, scale); \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t k = 0; k < s; ++k) {                                              \
                ORC_T *c = &C[k * crs + (c0 + i) * ccs];                                   \
                *c = (ORC_T)(beta * *c + alpha * pad[op[k] + i * N]);                      \
            }                                                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, A, S::SRHTRecipe{Left}, alpha, beta) -- src/Compressors/srht.jl:289-363.        \
 * A (ar x s), C (ar x m).  Signs are applied after the transform (srht.jl:327-329). */    \
int orc_srht_left_AS_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,          \
                             int64_t ars, int64_t acs, int64_t ar, int64_t m, int64_t s,   \
                             int64_t N, const int64_t *op, const uint8_t *signs,           \
                             double scale, int64_t bsize, double alpha, double beta) {     \
    ORC_T *pad = (ORC_T *)malloc(sizeof(ORC_T) * N * bsize);                               \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t r0 = 0; r0 < ar; r0 += bsize) {                                           \
        int64_t bw = ar - r0 < bsize ? ar - r0 : bsize;                                    \
        memset(pad, 0, sizeof(ORC_T) * N * bsize);                                         \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t k = 0; k < s; ++k)                                                \
                pad[op[k] + i * N] = (ORC_T)(alpha * A[(r0 + i) * ars + k * acs]);         \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_##ORC_S(pad + i * N, N, 1, scale);       \
        for (int64_t i = 0; i < bsize; ++i)                                                \
            for (int64_t r = 0; r < N; ++r)                                                \
                if (!signs[r]) pad[r + i * N] = -pad[r + i * N];                           \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t j = 0; j < m; ++j) {                                              \
                ORC_T *c = &C[(r0 + i) * crs + j * ccs];                                   \
                *c = (ORC_T)(pad[j + i * N] + beta * *c);                                  \
            }                                                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, A, S::SRHTRecipe{Right}, alpha, beta) -- src/Compressors/srht.jl:366-429.       \
 * S is (n x s); A (ar x n), C (ar x s).  Padding is (bsize x N), rows transformed. */     \
int orc_srht_right_AS_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,         \
                              int64_t ars, int64_t acs, int64_t ar, int64_t n, int64_t s,  \
                              int64_t N, const int64_t *op, const uint8_t *signs,          \
                              double scale, int64_t bsize, double alpha, double beta) {    \
    ORC_T *pad = (ORC_T *)malloc(sizeof(ORC_T) * N * bsize);                               \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t r0 = 0; r0 < ar; r0 += bsize) {                                           \
        int64_t bw = ar - r0 < bsize ? ar - r0 : bsize;                                    \
        memset(pad, 0, sizeof(ORC_T) * N * bsize);                                         \
        /* pad is column-major (bsize x N): element (i, j) at i + j*bsize */               \
        for (int64_t j = 0; j < n; ++j)                                                    \
            for (int64_t i = 0; i < bw; ++i) pad[i + j * bsize] = A[(r0 + i) * ars + j * acs]; \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_signed_##ORC_S(pad + i, N, bsize, signs, N, scale); \
        for (int64_t k = 0; k < s; ++k)                                                    \
            for (int64_t i = 0; i < bw; ++i) {                                             \
                ORC_T *c = &C[(r0 + i) * crs + k * ccs];                                   \
                *c = (ORC_T)(beta * *c + alpha * pad[i + op[k] * bsize]);                  \
            }                                                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, S::SRHTRecipe{Right}, A, alpha, beta) -- src/Compressors/srht.jl:432-504.       \
 * S (n x s); A (s x ac), C (n x ac). */                                                   \
int orc_srht_right_SA_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,         \
                              int64_t ars, int64_t acs, int64_t n, int64_t ac, int64_t s,  \
                              int64_t N, const int64_t *op, const uint8_t *signs,          \
                              double scale, int64_t bsize, double alpha, double beta) {    \
    ORC_T *pad = (ORC_T *)malloc(sizeof(ORC_T) * N * bsize);                               \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t c0 = 0; c0 < ac; c0 += bsize) {                                           \
        int64_t bw = ac - c0 < bsize ? ac - c0 : bsize;                                    \
        memset(pad, 0, sizeof(ORC_T) * N * bsize);                                         \
        for (int64_t k = 0; k < s; ++k)                                                    \
            for (int64_t i = 0; i < bw; ++i)                                               \
                pad[i + op[k] * bsize] = (ORC_T)(alpha * A[k * ars + (c0 + i) * acs]);     \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_##ORC_S(pad + i, N, bsize, scale);       \
        for (int64_t j = 0; j < N; ++j)                                                    \
            if (!signs[j])                                                                 \
                for (int64_t i = 0; i < bsize; ++i) pad[i + j * bsize] = -pad[i + j * bsize]; \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t j = 0; j < n; ++j) {                                              \
                ORC_T *c = &C[j * crs + (c0 + i) * ccs];                                   \
                *c = (ORC_T)(pad[i + j * bsize] + beta * *c);                              \
            }                                                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, S::FJLTRecipe{Left}, A, alpha, beta) -- src/Compressors/fjlt.jl:257-323.        \
 * K = S.op is an (s x N) CSC matrix. */                                                   \
int orc_fjlt_left_SA_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,          \
                             int64_t ars, int64_t acs, int64_t m, int64_t n, int64_t s,    \
                             int64_t N, const int64_t *kcolptr, const int64_t *krowval,    \
                             const ORC_T *knzval, const uint8_t *signs, double scale,      \
                             int64_t bsize, double alpha, double beta) {                   \
    ORC_T *pad = (ORC_T *)malloc(sizeof(ORC_T) * N * bsize);                               \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t c0 = 0; c0 < n; c0 += bsize) {                                            \
        int64_t bw = n - c0 < bsize ? n - c0 : bsize;                                      \
        memset(pad, 0, sizeof(ORC_T) * N * bsize);                                         \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t r = 0; r < m; ++r) pad[r + i * N] = A[r * ars + (c0 + i) * acs];  \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_signed_##ORC_S(pad + i * N, N, 1, signs, N, scale); \
        orc_csc_mul_##ORC_S(C + c0 * ccs, crs, ccs, s, N, kcolptr, krowval, knzval, pad, 1, N, \
                            bw, alpha, beta);                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, A, S::FJLTRecipe{Left}, alpha, beta) -- src/Compressors/fjlt.jl:326-397.        \
 * A (ar x s), C (ar x m); K (s x N) CSC. */                                               \
int orc_fjlt_left_AS_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,          \
                             int64_t ars, int64_t acs, int64_t ar, int64_t m, int64_t s,   \
                             int64_t N, const int64_t *kcolptr, const int64_t *krowval,    \
                             const ORC_T *knzval, const uint8_t *signs, double scale,      \
                             int64_t bsize, double alpha, double beta) {                   \
    ORC_T *pad = (ORC_T *)calloc((size_t)(N * bsize), sizeof(ORC_T));                      \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t r0 = 0; r0 < ar; r0 += bsize) {                                           \
        int64_t bw = ar - r0 < bsize ? ar - r0 : bsize;                                    \
        /* mul!(pv', Av, S.op, alpha, 0): pv' is (bw x N), row-major view of pad */        \
        orc_dense_mul_csc_##ORC_S(pad, N, 1, A + r0 * ars, ars, acs, bw, s, N, kcolptr,     \
                                  krowval, knzval, alpha, 0.0);                            \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_##ORC_S(pad + i * N, N, 1, scale);       \
        for (int64_t i = 0; i < bsize; ++i)                                                \
            for (int64_t r = 0; r < N; ++r)                                                \
                if (!signs[r]) pad[r + i * N] = -pad[r + i * N];                           \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t j = 0; j < m; ++j) {                                              \
                ORC_T *c = &C[(r0 + i) * crs + j * ccs];                                   \
                *c = (ORC_T)(pad[j + i * N] + beta * *c);                                  \
            }                                                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, A, S::FJLTRecipe{Right}, alpha, beta) -- src/Compressors/fjlt.jl:400-463.       \
 * A (ar x n), C (ar x s); K (N x s) CSC. */                                               \
int orc_fjlt_right_AS_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,         \
                              int64_t ars, int64_t acs, int64_t ar, int64_t n, int64_t s,  \
                              int64_t N, const int64_t *kcolptr, const int64_t *krowval,   \
                              const ORC_T *knzval, const uint8_t *signs, double scale,     \
                              int64_t bsize, double alpha, double beta) {                  \
    ORC_T *pad = (ORC_T *)malloc(sizeof(ORC_T) * N * bsize);                               \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t r0 = 0; r0 < ar; r0 += bsize) {                                           \
        int64_t bw = ar - r0 < bsize ? ar - r0 : bsize;                                    \
        memset(pad, 0, sizeof(ORC_T) * N * bsize);                                         \
        for (int64_t j = 0; j < n; ++j)                                                    \
            for (int64_t i = 0; i < bw; ++i) pad[i + j * bsize] = A[(r0 + i) * ars + j * acs]; \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_signed_##ORC_S(pad + i, N, bsize, signs, N, scale); \
        orc_dense_mul_csc_##ORC_S(C + r0 * crs, crs, ccs, pad, 1, bsize, bw, N, s, kcolptr, \
                                  krowval, knzval, alpha, beta);                           \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}                                                                                          \
                                                                                           \
/* mul!(C, S::FJLTRecipe{Right}, A, alpha, beta) -- src/Compressors/fjlt.jl:465-535.       \
 * S (n x s); A (s x ac), C (n x ac); K (N x s) CSC. */                                    \
int orc_fjlt_right_SA_##ORC_S(ORC_T *C, int64_t crs, int64_t ccs, const ORC_T *A,         \
                              int64_t ars, int64_t acs, int64_t n, int64_t ac, int64_t s,  \
                              int64_t N, const int64_t *kcolptr, const int64_t *krowval,   \
                              const ORC_T *knzval, const uint8_t *signs, double scale,     \
                              int64_t bsize, double alpha, double beta) {                  \
    ORC_T *pad = (ORC_T *)calloc((size_t)(N * bsize), sizeof(ORC_T));                      \
    if (!pad) return ORC_E_OOM;                                                            \
    for (int64_t c0 = 0; c0 < ac; c0 += bsize) {                                           \
        int64_t bw = ac - c0 < bsize ? ac - c0 : bsize;                                    \
        /* mul!(pv', S.op, Av, alpha, 0): pv' is (N x bw), view of pad with rs = bsize */  \
        orc_csc_mul_##ORC_S(pad, bsize, 1, N, s, kcolptr, krowval, knzval,                 \
                            A + c0 * acs, ars, acs, bw, alpha, 0.0);                       \
        for (int64_t i = 0; i < bw; ++i) orc_fwht_##ORC_S(pad + i, N, bsize, scale);       \
        for (int64_t j = 0; j < N; ++j)                                                    \
            if (!signs[j])                                                                 \
                for (int64_t i = 0; i < bsize; ++i) pad[i + j * bsize] = -pad[i + j * bsize]; \
        for (int64_t i = 0; i < bw; ++i)                                                   \
            for (int64_t j = 0; j < n; ++j) {                                              \
                ORC_T *c = &C[j * crs + (c0 + i) * ccs];                                   \
                *c = (ORC_T)(pad[i + j * bsize] + beta * *c);                              \
            }                                                                              \
    }                                                                                      \
    free(pad);                                                                             \
    return 0;                                                                              \
}

ORC_DEFINE(float, f)
ORC_DEFINE(double, d)

/* Version tag so the Python side can check it loaded the matching build. */
int orc_version(void) { return 1; }
