// rla_sparse_op.cu -- SparseSign / CountSketch applied from the left to a sparse operand.
//
// The reference has one method for a sparse A: mul!(C, S, transpose(B), alpha, beta) with a
// Left SparseSign or CountSketch recipe S (s x m) and B an n x m SparseMatrixCSC
// (sparse_sign.jl:364-442, count_sketch.jl:215-262).  transpose(B) is A (m x n) stored by
// rows: rowptr = B.colptr, colidx = B.rowval, vals = B.nzval (0-based here).  C (s x n) is
// dense.  Row j of A adds sign * scale * A(j, :) to the nnz rows of C that j hashes to.
//
// Deterministic, without atomics: a per-recipe plan lists, for every row i of C, the long
// indices j that hash to it in increasing j (a stable radix sort of the bucket array, built
// once per draw).  A warp owns one row i of C and a tile of up to SPT_TILE of its columns in
// shared memory; it walks the plan's j in order, and its lanes add the nonzeros of row j of
// A (their columns are distinct, so no two lanes touch one slot).  Every C(i, c) is thus
// summed in increasing j, the order of the reference's loops.
#include <cub/device/device_radix_sort.cuh>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

constexpr int SPT_WARPS = 4;
constexpr int SPT_TILE = 1024;  // columns of C per warp tile

__global__ void iota_kernel(int32_t *x, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) x[i] = (int32_t)i;
}

// ptr[b] = first position of bucket b in the sorted keys (ptr[s] = n)
__global__ void bucket_offsets_kernel(const int32_t *keys, int64_t n, int64_t s, int64_t *ptr) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p > n) return;
    const int64_t hi = p < n ? (int64_t)keys[p] : s;
    const int64_t lo = p == 0 ? -1 : (int64_t)keys[p - 1];
    for (int64_t b = lo + 1; b <= hi; ++b) ptr[b] = p;
}

template <class T>
__global__ void __launch_bounds__(SPT_WARPS * 32)
sparse_t_kernel(const int64_t *__restrict__ plan_ptr, const int32_t *__restrict__ plan_idx,
                const uint8_t *__restrict__ negative, int nnz, int64_t s, const int64_t *__restrict__ rowptr,
                const int64_t *__restrict__ colidx, const T *__restrict__ vals, int64_t ncols, T *C, int64_t ldc,
                T alpha, T beta, int beta_zero) {
    __shared__ T acc_s[SPT_WARPS][SPT_TILE];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * SPT_WARPS + w;
    if (i >= s) return;  // warp-uniform
    const int64_t c0 = (int64_t)blockIdx.y * SPT_TILE;
    const int64_t cw = min((int64_t)SPT_TILE, ncols - c0);
    T *acc = acc_s[w];
    for (int64_t c = lane; c < cw; c += 32) acc[c] = T(0);
    __syncwarp();
    for (int64_t q = plan_ptr[i]; q < plan_ptr[i + 1]; ++q) {
        const int32_t e = plan_idx[q];
        const int64_t j = e / nnz;
        const bool neg = negative[e] != 0;
        for (int64_t k = rowptr[j] + lane; k < rowptr[j + 1]; k += 32) {
            const int64_t c = colidx[k] - c0;
            if (c >= 0 && c < cw) {
                const T v = vals[k];
                acc[c] += neg ? -v : v;
            }
        }
        __syncwarp();
    }
    for (int64_t c = lane; c < cw; c += 32) {
        T *cp = C + i + (c0 + c) * ldc;
        T r = alpha * acc[c];
        if (!beta_zero) r += beta * *cp;
        *cp = r;
    }
}

// Bucket-major plan of a SparseSign / CountSketch recipe: plan_idx lists the entries
// e = j*nnz + slot by bucket, j increasing within a bucket.  Rebuilt after every redraw.
static int sparse_t_plan(rla_ctx *ctx, rla_sketch *sk) {
    if (sk->tp_ptr && sk->tp_version == sk->draw_count) return RLA_OK;
    const int64_t n = sk->L * sk->nnz, s = sk->s;
    if (n >= (1ll << 31)) return set_error(ctx, RLA_E_UNSUPPORTED, "sparse operand: more than 2^31 sketch entries");
    if (!sk->tp_ptr) {
        RLA_CUDA_TRY(ctx, cudaMalloc(&sk->tp_ptr, sizeof(int64_t) * (s + 1)));
        RLA_CUDA_TRY(ctx, cudaMalloc(&sk->tp_idx, sizeof(int32_t) * std::max<int64_t>(n, 1)));
    }
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < s) ++end_bit;
    int32_t *keys_out = nullptr, *vals_in = nullptr;
    size_t temp = 0;
    RLA_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(nullptr, temp, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                                      (const int32_t *)nullptr, (int32_t *)nullptr, (int)n, 0, end_bit,
                                                      ctx->stream));
    const size_t off_vals = ((size_t)n * 4 + 255) / 256 * 256, off_temp = off_vals + off_vals;
    void *ws = nullptr;
    RLA_TRY(scratch_get(ctx, off_temp + temp, &ws));
    keys_out = (int32_t *)ws;
    vals_in = (int32_t *)((char *)ws + off_vals);
    if (n > 0) {
        iota_kernel<<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(vals_in, n);
        RLA_TRY(check_launch(ctx, "iota"));
        RLA_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs((char *)ws + off_temp, temp, (const uint32_t *)sk->bucket,
                                                          (uint32_t *)keys_out, vals_in, sk->tp_idx, (int)n, 0, end_bit,
                                                          ctx->stream));
    }
    bucket_offsets_kernel<<<ceil_div_i(n + 1, 256), 256, 0, ctx->stream>>>(keys_out, n, s, sk->tp_ptr);
    RLA_TRY(check_launch(ctx, "bucket_offsets"));
    sk->tp_version = sk->draw_count;
    return RLA_OK;
}

template <class T>
static int sparse_t_apply(rla_ctx *ctx, rla_sketch *sk, int64_t ncols, T *C, int64_t ldc, const int64_t *rowptr,
                          const int64_t *colidx, const T *vals, double alpha, double beta) {
    RLA_TRY(sparse_t_plan(ctx, sk));
    const dim3 grid((unsigned)ceil_div(sk->s, SPT_WARPS), (unsigned)ceil_div(ncols, SPT_TILE));
    if (grid.y > 65535) return set_error(ctx, RLA_E_UNSUPPORTED, "sparse operand: more than 65535 column tiles");
    sparse_t_kernel<T><<<grid, SPT_WARPS * 32, 0, ctx->stream>>>(sk->tp_ptr, sk->tp_idx, sk->negative, (int)sk->nnz,
                                                                 sk->s, rowptr, colidx, vals, ncols, C, ldc,
                                                                 (T)(alpha * sk->scale), (T)beta, beta == 0.0);
    return check_launch(ctx, "sparse_t");
}

}  // namespace rla

using namespace rla;

extern "C" int rla_sketch_mul_sparse_t(rla_ctx *ctx, rla_sketch *sk, int64_t c_rows, int64_t c_cols, void *C,
                                       int64_t ldc, int64_t a_rows, int64_t a_cols, int64_t a_nnz,
                                       const int64_t *a_rowptr, const int64_t *a_colidx, const void *a_vals,
                                       double alpha, double beta) {
    if (!ctx) return RLA_E_ARG;
    if (!sk) return set_error(ctx, RLA_E_ARG, "NULL compressor recipe.");
    if (sk->device != ctx->device) return set_error(ctx, RLA_E_ARG, "Compressor lives on another device.");
    if ((sk->p.kind != RLA_SPARSE_SIGN && sk->p.kind != RLA_COUNT_SKETCH) || sk->p.card != RLA_LEFT)
        return set_error(ctx, RLA_E_ARG,
                         "A sparse operand is taken by Left SparseSign and CountSketch recipes only (S * transpose(B)).");
    if (c_rows < 0 || c_cols < 0 || a_rows < 0 || a_cols < 0 || a_nnz < 0)
        return set_error(ctx, RLA_E_ARG, "Negative dimension.");
    // left_mul_dimcheck (src/helpers/mul_dim_checks.jl:41-64)
    if (a_rows != sk->n_cols)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)a_rows, (long long)sk->n_cols);
    if (a_cols != c_cols)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while C has %lld columns.", (long long)a_cols, (long long)c_cols);
    if (c_rows != sk->n_rows)
        return set_error(ctx, RLA_E_DIM, "Matrix C has %lld rows while S has %lld rows.", (long long)c_rows, (long long)sk->n_rows);
    if (c_rows == 0 || c_cols == 0) return RLA_OK;
    if (!C || ldc < c_rows) return set_error(ctx, RLA_E_ARG, "NULL C or leading dimension smaller than the row count.");
    if (!a_rowptr || (a_nnz > 0 && (!a_colidx || !a_vals)))
        return set_error(ctx, RLA_E_ARG, "NULL sparse operand array.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    int rc;
    if (sk->p.dtype == RLA_F32)
        rc = sparse_t_apply<float>(ctx, sk, c_cols, (float *)C, ldc, a_rowptr, a_colidx, (const float *)a_vals, alpha,
                                   beta);
    else
        rc = sparse_t_apply<double>(ctx, sk, c_cols, (double *)C, ldc, a_rowptr, a_colidx, (const double *)a_vals,
                                    alpha, beta);
    RLA_TRY(rc);
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}
