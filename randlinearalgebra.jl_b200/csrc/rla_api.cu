// rla_api.cu -- mul! for every compressor and orientation.
//
// Every orientation of mul! reduces to one of two operators on vectors:
//   compress  P   : R^L -> R^s   (S for Left cardinality, S' for Right)
//   expand    P'  : R^s -> R^L
// applied to the columns (side Left) or rows (side Right) of A.  A Left S applied from
// the left compresses columns; the adjoint routes of src/Compressors.jl:363-384 flip the
// operator.  Vectors are "contiguous" when their elements are adjacent in memory
// (columns of a column-major matrix) and "strided" otherwise.
#include "rla_internal.cuh"
#include "rla_kernels.cuh"
#include "rla_tc.cuh"

namespace rla {

static int dimcheck(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s, int64_t c_rows, int64_t c_cols,
                    int64_t a_rows, int64_t a_cols) {
    const int64_t nr = sk->n_rows, nc = sk->n_cols;
    // src/helpers/mul_dim_checks.jl:41-64 and :110-133, reached directly or through the
    // transposes of the adjoint routes (src/Compressors.jl:363-384).
    auto left = [&](int64_t cr, int64_t cc, int64_t sr, int64_t sc, int64_t ar, int64_t ac) {
        if (ar != sc)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)ar, (long long)sc);
        if (ac != cc)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while C has %lld columns.", (long long)ac, (long long)cc);
        if (cr != sr)
            return set_error(ctx, RLA_E_DIM, "Matrix C has %lld rows while S has %lld rows.", (long long)cr, (long long)sr);
        return RLA_OK;
    };
    auto right = [&](int64_t cr, int64_t cc, int64_t ar, int64_t ac, int64_t sr, int64_t sc) {
        if (ac != sr)
            return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while S has %lld rows.", (long long)ac, (long long)sr);
        if (cc != sc)
            return set_error(ctx, RLA_E_DIM, "Matrix C has %lld columns while S has %lld columns.", (long long)cc, (long long)sc);
        if (cr != ar)
            return set_error(ctx, RLA_E_DIM, "Matrix C has %lld rows while A has %lld rows.", (long long)cr, (long long)ar);
        return RLA_OK;
    };
    if (side == RLA_SIDE_LEFT)
        return trans_s ? right(c_cols, c_rows, a_cols, a_rows, nr, nc) : left(c_rows, c_cols, nr, nc, a_rows, a_cols);
    return trans_s ? left(c_cols, c_rows, nr, nc, a_cols, a_rows) : right(c_rows, c_cols, a_rows, a_cols, nr, nc);
}

// Dense products of the Gaussian sketch: Float32 on the 5th-generation tensor cores (three
// BF16 terms per operand, FP64 accumulation across k-chunks: an FP32-accurate product),
// Float64 on the FP64 tensor cores.
template <class T>
static int dense_gemm(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const T *A, int64_t lda, int ta, const T *B,
                      int64_t ldb, int tb, T *C, int64_t ldc, double alpha, double beta) {
    if constexpr (std::is_same<T, float>::value)
        return gemm_f32_tc<float>(ctx, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, alpha, beta);
    else
        return gemm<T, T, T, double>(ctx, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, alpha, beta);
}

template <class T>
static int dispatch(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s, int64_t c_rows, int64_t c_cols, T *C,
                    int64_t ldc, int trans_c, int64_t a_rows, int64_t a_cols, const T *A, int64_t lda, int trans_a,
                    double alpha, double beta) {
    const int kind = sk->p.kind;
    if (kind == RLA_GAUSSIAN) {
        const T *S = (const T *)sk->dense;
        const int64_t lds = sk->n_rows;
        if (side == RLA_SIDE_LEFT) {
            const int64_t K = trans_s ? sk->n_rows : sk->n_cols;
            if (!trans_c) return dense_gemm<T>(ctx, c_rows, c_cols, K, S, lds, trans_s, A, lda, trans_a, C, ldc, alpha, beta);
            return dense_gemm<T>(ctx, c_cols, c_rows, K, A, lda, !trans_a, S, lds, !trans_s, C, ldc, alpha, beta);
        }
        const int64_t K = a_cols;
        if (!trans_c) return dense_gemm<T>(ctx, c_rows, c_cols, K, A, lda, trans_a, S, lds, trans_s, C, ldc, alpha, beta);
        return dense_gemm<T>(ctx, c_cols, c_rows, K, S, lds, !trans_s, A, lda, !trans_a, C, ldc, alpha, beta);
    }
    const bool compress = side == RLA_SIDE_LEFT ? ((sk->p.card == RLA_LEFT) != (trans_s != 0))
                                                : ((sk->p.card == RLA_RIGHT) != (trans_s != 0));
    const int64_t nv = side == RLA_SIDE_LEFT ? a_cols : a_rows;
    const bool in_contig = (side == RLA_SIDE_LEFT) == (trans_a == 0);
    const bool out_contig = (side == RLA_SIDE_LEFT) == (trans_c == 0);
    const int64_t x_es = in_contig ? 1 : lda, x_vs = in_contig ? lda : 1;
    const int64_t y_es = out_contig ? 1 : ldc, y_vs = out_contig ? ldc : 1;
    switch (kind) {
        case RLA_SPARSE_SIGN:
        case RLA_COUNT_SKETCH:
            return compress ? sparse_compress<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta)
                            : sparse_expand<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta);
        case RLA_SRHT:
            return compress ? srht_compress<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta)
                            : srht_expand<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta);
        case RLA_FJLT:
            return compress ? fjlt_compress<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta)
                            : fjlt_expand<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta);
        case RLA_SAMPLING:
            return compress ? sampling_compress<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta)
                            : sampling_expand<T>(ctx, sk, A, x_es, x_vs, nv, C, y_es, y_vs, alpha, beta);
    }
    return set_error(ctx, RLA_E_ARG, "unknown compressor kind");
}

int sketch_mul_impl(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s, int64_t c_rows, int64_t c_cols,
                    void *C, int64_t ldc, int trans_c, int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                    int trans_a, double alpha, double beta) {
    if (!ctx) return RLA_E_ARG;
    if (!sk) return set_error(ctx, RLA_E_ARG, "NULL compressor recipe.");
    if (sk->device != ctx->device) return set_error(ctx, RLA_E_ARG, "Compressor lives on device %d, context on %d.", sk->device, ctx->device);
    if ((side != 0 && side != 1) || (trans_s != 0 && trans_s != 1) || (trans_a != 0 && trans_a != 1) ||
        (trans_c != 0 && trans_c != 1))
        return set_error(ctx, RLA_E_ARG, "side/trans flags must be 0 or 1.");
    if (c_rows < 0 || c_cols < 0 || a_rows < 0 || a_cols < 0) return set_error(ctx, RLA_E_ARG, "Negative dimension.");
    RLA_TRY(dimcheck(ctx, sk, side, trans_s, c_rows, c_cols, a_rows, a_cols));
    if (c_rows == 0 || c_cols == 0) return RLA_OK;
    const int64_t a_stored_rows = trans_a ? a_cols : a_rows;
    const int64_t c_stored_rows = trans_c ? c_cols : c_rows;
    if (lda < std::max<int64_t>(1, a_stored_rows) || ldc < std::max<int64_t>(1, c_stored_rows))
        return set_error(ctx, RLA_E_ARG, "Leading dimension smaller than the stored row count.");
    if (!C || (!A && a_rows * a_cols > 0)) return set_error(ctx, RLA_E_ARG, "NULL matrix pointer.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    if (sk->p.dtype == RLA_F32)
        return dispatch<float>(ctx, sk, side, trans_s, c_rows, c_cols, (float *)C, ldc, trans_c, a_rows, a_cols,
                               (const float *)A, lda, trans_a, alpha, beta);
    return dispatch<double>(ctx, sk, side, trans_s, c_rows, c_cols, (double *)C, ldc, trans_c, a_rows, a_cols,
                            (const double *)A, lda, trans_a, alpha, beta);
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_sketch_mul(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s, int64_t c_rows, int64_t c_cols,
                   void *C, int64_t ldc, int trans_c, int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                   int trans_a, double alpha, double beta) {
    RLA_TRY(sketch_mul_impl(ctx, sk, side, trans_s, c_rows, c_cols, C, ldc, trans_c, a_rows, a_cols, A, lda, trans_a,
                            alpha, beta));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

int rla_sketch_mul_async(rla_ctx *ctx, const rla_sketch *sk, int side, int trans_s, int64_t c_rows, int64_t c_cols,
                         void *C, int64_t ldc, int trans_c, int64_t a_rows, int64_t a_cols, const void *A,
                         int64_t lda, int trans_a, double alpha, double beta) {
    return sketch_mul_impl(ctx, sk, side, trans_s, c_rows, c_cols, C, ldc, trans_c, a_rows, a_cols, A, lda, trans_a,
                           alpha, beta);
}

}  // extern "C"
