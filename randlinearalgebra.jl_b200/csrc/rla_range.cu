// rla_range.cu -- rapproximate! for RangeFinder and RandSVD.
//
// rand_power_it / rand_ortho_it (power_its.jl:15-80) with the products on the GPU and
// every `Array(qr!(Y).Q)` replaced by CholeskyQR2:
//   G = Y'Y (FP64 accumulate), D = diag(G)^-1/2, R = chol(D G D), Q = Y D R^-1, twice;
// shifted CholeskyQR3 (Fukaya et al., SIAM J. Sci. Comput. 2020) when a Cholesky pivot
// breaks down.  The column signs of Q are then set to what LAPACK's Householder QR of Y
// returns: for orthonormal Q, Householder QR yields R = diag(+-1), and those signs follow
// from an LU elimination of the top l x l block (Ballard et al., "Reconstructing
// Householder vectors from tall-skinny QR", 2015), so Q matches qr!(Y).Q column by column.
//
// RandSVD (randsvd.jl:174-189): Bt = A'Q (n x l, FP64), Bt = Qb Rb (CholeskyQR2 in FP64),
// one-sided Jacobi on Rb' gives Rb' J = W Sigma, so B = Q'A = W Sigma (Qb J)' and
// U = Q W, V = Qb J, S = Sigma.
#include <math.h>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"
#include "rla_tc.cuh"

namespace rla {

// dscale[i] = 1/sqrt(G_ii)
__global__ void diag_rsqrt_kernel(const double *G, int64_t l, double *dscale) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= l) return;
    const double g = G[i + i * l];
    dscale[i] = g > 0 ? rsqrt(g) : 1.0;
}

// G <- D G D
__global__ void sym_scale_kernel(double *G, int64_t l, const double *dscale) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= l * l) return;
    G[idx] *= dscale[idx % l] * dscale[idx / l];
}

static int equilibrate(rla_ctx *ctx, double *G, int64_t l, double *dscale) {
    diag_rsqrt_kernel<<<ceil_div_i(l, 256), 256, 0, ctx->stream>>>(G, l, dscale);
    sym_scale_kernel<<<ceil_div_i(l * l, 256), 256, 0, ctx->stream>>>(G, l, dscale);
    return check_launch(ctx, "equilibrate");
}

// Rinv <- D * Rinv (row scaling)
__global__ void row_scale_kernel(double *M, int64_t l, const double *d) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= l * l) return;
    M[idx] *= d[idx % l];
}

__global__ void copy_diag_kernel(const double *G, int64_t l, double *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < l) out[i] = G[i + i * l];
}

// Householder column signs of orthonormal Q (m x l, ld ldq) from its top block.
template <class T>
__global__ void __launch_bounds__(1024) house_signs_kernel(T *Q, int64_t m, int64_t l, int64_t ldq, double *W) {
    __shared__ double piv_s;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int64_t idx = tid; idx < l * l; idx += nt) W[idx] = (double)Q[(idx % l) + (idx / l) * ldq];
    __syncthreads();
    double *S = W + l * l;
    for (int64_t k = 0; k < l; ++k) {
        if (tid == 0) {
            const double piv = W[k + k * l];
            const double sk = (k == m - 1) ? (piv >= 0 ? 1.0 : -1.0) : (piv >= 0 ? -1.0 : 1.0);
            S[k] = sk;
            W[k + k * l] = piv - sk;
            piv_s = W[k + k * l];
        }
        __syncthreads();
        for (int64_t i = k + 1 + tid; i < l; i += nt) W[i + k * l] /= piv_s;
        __syncthreads();
        const int64_t n = l - k - 1;
        for (int64_t idx = tid; idx < n * n; idx += nt) {
            const int64_t i = k + 1 + idx % n, j = k + 1 + idx / n;
            W[i + j * l] -= W[i + k * l] * W[k + j * l];
        }
        __syncthreads();
    }
    for (int64_t idx = tid; idx < m * l; idx += nt) {
        const int64_t r = idx % m, c = idx / m;
        if (S[c] < 0) Q[r + c * ldq] = -Q[r + c * ldq];
    }
}

template <class T>
__global__ void transpose_to_kernel(const T *X, int64_t rows, int64_t cols, int64_t ldx, T *Y, int64_t ldy) {
    // Y (cols x rows) = X'
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const int64_t r = idx % rows, c = idx / rows;
    Y[c + r * ldy] = X[r + c * ldx];
}

template <class TI, class TO>
__global__ void convert_kernel(const TI *X, int64_t rows, int64_t cols, int64_t ldx, TO *Y, int64_t ldy) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const int64_t r = idx % rows, c = idx / rows;
    Y[r + c * ldy] = (TO)X[r + c * ldx];
}

// ---- tall-skinny Gram matrix G = Y'Y (l x l, FP64 accumulation) ------------------------
template <class T>
int gram_fp64(rla_ctx *ctx, const T *Y, int64_t rows, int64_t l, int64_t ldy, double *G) {
    // symmetric FP64 product on the FP64 tensor cores: upper tiles, split over row chunks
    return dgemm<T, T, double>(ctx, l, l, rows, Y, ldy, 1, Y, ldy, 0, G, l, 1.0, 0.0, 0, 1);
}

template int gram_fp64<float>(rla_ctx *, const float *, int64_t, int64_t, int64_t, double *);
template int gram_fp64<double>(rla_ctx *, const double *, int64_t, int64_t, int64_t, double *);

struct OrthWork {
    double *G, *Rinv, *dscale, *diag, *hw;
    double *cw = nullptr;  // chol_inv working copy (null: separate Cholesky and inverse)
    int *flag;
    void *tmp;  // rows x l of T
};

// In-place orthonormalisation of Y (rows x l, ld ldy).  With `signs` the columns of Q get
// the signs LAPACK's Householder QR of Y gives them (needed only where Q itself is
// returned: column signs of intermediate bases cancel out of the final factors).
// `passes` CholeskyQR passes: 2 (CholeskyQR2) for a basis that must be orthonormal to
// working precision; 1 for an intermediate basis of the power iterations, which only has
// to span range(Y) and be well conditioned (one pass with the FP64 Gram matrix leaves
// ||Q'Q - I|| ~ u * cond(Y) for Float32 Y, ~ u * cond(Y)^2 for Float64).
//
// Passes alternate between Y and w.tmp (rows x l, ld rows).  With `owned` (Y is a library
// buffer with ld == rows) a result that ends in w.tmp is not copied back: Y and w.tmp trade
// places.
template <class T>
static int orth(rla_ctx *ctx, T *&Y, int64_t rows, int64_t l, int64_t ldy, OrthWork &w, bool signs = true,
                int passes = 2, bool owned = false) {
    if (l > rows)
        return set_error(ctx, RLA_E_UNSUPPORTED, "compression dimension %lld exceeds the %lld rows being orthogonalised",
                         (long long)l, (long long)rows);
    T *tmp = (T *)w.tmp;
    // the current basis: cur (ld ldc), the product goes to the other buffer
    T *cur = Y;
    int64_t ldc = ldy;
    bool shifted_done = false;
    auto finish = [&]() -> int {
        if (cur != Y) {
            if (owned && ldy == rows) {
                w.tmp = Y;
                Y = cur;
            } else {
                convert_kernel<T, T><<<ceil_div_i(rows * l, 256), 256, 0, ctx->stream>>>(cur, rows, l, rows, Y, ldy);
                RLA_TRY(check_launch(ctx, "copy_back"));
            }
        }
        return RLA_OK;
    };
    for (int pass = 0; pass < passes; ++pass) {
        RLA_TRY(gram_fp64<T>(ctx, cur, rows, l, ldc, w.G));
        double shift = 0.0;
        RLA_TRY(equilibrate(ctx, w.G, l, w.dscale));
        if (w.cw) RLA_TRY(chol_inv(ctx, w.G, l, shift, w.flag, w.Rinv, w.cw));
        else RLA_TRY(cholesky_upper(ctx, w.G, l, shift, w.flag));
        int bad = 0;
        RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&bad, w.flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        if (bad && shifted_done) {
            // numerically rank-deficient block: Householder QR gives an orthonormal basis
            // (and LAPACK's Q) whatever the rank
            RLA_TRY(finish());
            return householder_q<T>(ctx, Y, rows, l, ldy, w.diag);
        }
        if (bad) {
            // Shifted CholeskyQR: on the equilibrated Gram matrix (unit diagonal, so
            // ||Y D||_F^2 = l) the shift is 11 (rows*l + l(l+1)) u ||Y D||_2^2 <= ... * l.
            RLA_TRY(gram_fp64<T>(ctx, cur, rows, l, ldc, w.G));
            RLA_TRY(equilibrate(ctx, w.G, l, w.dscale));
            const double u = sizeof(T) == 4 ? 5.96e-8 : 1.11e-16;
            shift = 11.0 * ((double)rows * l + (double)l * (l + 1)) * u * (double)l;
            if (w.cw) RLA_TRY(chol_inv(ctx, w.G, l, shift, w.flag, w.Rinv, w.cw));
            else RLA_TRY(cholesky_upper(ctx, w.G, l, shift, w.flag));
            RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&bad, w.flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
            if (bad) {
                RLA_TRY(finish());
                return householder_q<T>(ctx, Y, rows, l, ldy, w.diag);
            }
            shifted_done = true;
            passes = pass + 3;  // shifted pass followed by two plain passes
        }
        if (!w.cw) RLA_TRY(tri_inv_upper(ctx, w.G, l, w.Rinv));
        row_scale_kernel<<<ceil_div_i(l * l, 256), 256, 0, ctx->stream>>>(w.Rinv, l, w.dscale);
        RLA_TRY(check_launch(ctx, "row_scale"));
        // the product goes to the buffer the basis is not in (Y or tmp)
        T *dst = cur == Y ? tmp : Y;
        const int64_t ldd = cur == Y ? rows : ldy;
        RLA_TRY((gemm<T, double, T, double>(ctx, rows, l, l, cur, ldc, 0, w.Rinv, l, 0, dst, ldd, 1.0, 0.0, 1)));
        cur = dst;
        ldc = ldd;
    }
    RLA_TRY(finish());
    if (!signs) return RLA_OK;
    house_signs_kernel<T><<<1, 1024, 0, ctx->stream>>>(Y, rows, l, ldy, w.hw);
    return check_launch(ctx, "house_signs");
}

template <class T>
static int alloc_orth(rla_ctx *ctx, OrthWork &w, int64_t rows, int64_t l, std::vector<void *> &owned) {
    auto get = [&](size_t bytes, void **p) -> int {
        RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, p, std::max<size_t>(bytes, 16), ctx->stream));
        owned.push_back(*p);
        return RLA_OK;
    };
    RLA_TRY(get(sizeof(double) * l * l, (void **)&w.G));
    RLA_TRY(get(sizeof(double) * l * l, (void **)&w.Rinv));
    RLA_TRY(get(sizeof(double) * l, (void **)&w.dscale));
    RLA_TRY(get(sizeof(double) * l, (void **)&w.diag));
    RLA_TRY(get(sizeof(double) * (l * l + l), (void **)&w.hw));
    RLA_TRY(get(sizeof(int), (void **)&w.flag));
    RLA_TRY(get(sizeof(T) * rows * l, &w.tmp));
    if (chol_inv_supported(ctx, l)) RLA_TRY(get(sizeof(double) * chol_inv_work_doubles(l), (void **)&w.cw));
    return RLA_OK;
}

struct Owned {
    rla_ctx *ctx;
    std::vector<void *> ptrs;
    ~Owned() {
        for (void *p : ptrs) cudaFreeAsync(p, ctx->stream);
    }
};

// Operands of the tensor-core products with A (Float32 data): A split once into NT BF16
// terms (NT = 2 for RLA_PREC_SPLIT_BF16, about 16 bits; NT = 3 with FP64 accumulation across
// k-chunks for RLA_PREC_NATIVE, an FP32-accurate product); one buffer set reused for the
// terms of the thin factor of each product (Omega, Q or Z).
struct TcOps {
    int nt = 2;
    bf16 *a[3] = {nullptr, nullptr, nullptr};
    int64_t lda = 0;
    bf16 *x[3] = {nullptr, nullptr, nullptr};
};

static int tc_ops_make(rla_ctx *ctx, const float *A, int64_t m, int64_t n, int64_t lda, int64_t l, int nt, TcOps &ops,
                       Owned &own) {
    ops.nt = nt;
    ops.lda = ceil_div(m, 8) * 8;
    const size_t na = (size_t)ops.lda * n, nx = (size_t)ceil_div(std::max(m, n), 8) * 8 * l;
    bf16 *buf = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&buf, sizeof(bf16) * nt * (na + nx), ctx->stream));
    own.ptrs.push_back(buf);
    for (int t = 0; t < nt; ++t) {
        ops.a[t] = buf + t * na;
        ops.x[t] = buf + nt * na + t * nx;
    }
    return nt == 2 ? split_terms_launch<2>(ctx, A, m, n, lda, 0, ops.a, ops.lda)
                   : split_terms_launch<3>(ctx, A, m, n, lda, 0, ops.a, ops.lda);
}

// out (rows_out x l) = op(A) * X with X (k x l, ld ldx) FP32; op(A) = A' when at.
template <class TO>
static int tc_apply(rla_ctx *ctx, const TcOps &ops, int at, int64_t m, int64_t n, const float *X, int64_t ldx,
                    int64_t l, TO *out, int64_t ldo) {
    const int64_t k = at ? m : n, rows_out = at ? n : m;
    const int64_t ldxs = ceil_div(k, 8) * 8;
    const bf16 *a[3] = {ops.a[0], ops.a[1], ops.a[2]}, *x[3] = {ops.x[0], ops.x[1], ops.x[2]};
    if (ops.nt == 2) {
        RLA_TRY(split_terms_launch<2>(ctx, X, k, l, ldx, 0, ops.x, ldxs));
        return tc_gemm_split<2, TO>(ctx, rows_out, l, k, a, ops.lda, at, x, ldxs, out, ldo, 1.0, 0.0, 0);
    }
    RLA_TRY(split_terms_launch<3>(ctx, X, k, l, ldx, 0, ops.x, ldxs));
    return tc_gemm_f64acc<TO>(ctx, rows_out, l, k, a, ops.lda, at, x, ldxs, out, ldo, 1.0, 0.0);
}

// Q (m x l, ld ldq) <- range of A*Omega after the power iterations.  With `tc` (FP32 data
// only) the products with A run on the tensor cores in split BF16.
template <class T>
static int range_core(rla_ctx *ctx, const rla_sketch *om, int64_t m, int64_t n, const T *A, int64_t lda,
                      const rla_range_params *pr, T *&Q, int64_t ldq, Owned &own, const TcOps *tc = nullptr,
                      bool q_signs = true, bool q_owned = false) {
    const int64_t l = om->n_cols;
    // Z = A'Q, Q = A Z
    auto at_q = [&](const T *Qp, T *Zp) -> int {
        if constexpr (std::is_same<T, float>::value)
            if (tc) return tc_apply<float>(ctx, *tc, 1, m, n, Qp, ldq, l, Zp, n);
        return gemm<T, T, T, double>(ctx, n, l, m, A, lda, 1, Qp, ldq, 0, Zp, n, 1.0, 0.0);
    };
    auto a_z = [&](const T *Zp, T *Qp) -> int {
        if constexpr (std::is_same<T, float>::value)
            if (tc) return tc_apply<float>(ctx, *tc, 0, m, n, Zp, n, l, Qp, ldq);
        return gemm<T, T, T, double>(ctx, m, l, n, A, lda, 0, Zp, n, 0, Qp, ldq, 1.0, 0.0);
    };
    OrthWork wq{}, wz{};
    RLA_TRY(alloc_orth<T>(ctx, wq, m, l, own.ptrs));
    T *Z = nullptr;
    if (pr->power_its > 0) {
        RLA_TRY(alloc_orth<T>(ctx, wz, n, l, own.ptrs));
        RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&Z, sizeof(T) * n * l, ctx->stream));
        own.ptrs.push_back(Z);
    }
    // Y = A * Omega (power_its.jl:21 / :59); a dense Gaussian Omega is a GEMM
    bool done = false;
    if constexpr (std::is_same<T, float>::value) {
        if (tc && om->p.kind == RLA_GAUSSIAN) {
            RLA_TRY(tc_apply<float>(ctx, *tc, 0, m, n, (const float *)om->dense, om->n_rows, l, Q, ldq));
            done = true;
        }
    }
    if (!done) RLA_TRY(sketch_mul_impl(ctx, om, RLA_SIDE_RIGHT, 0, m, l, Q, ldq, 0, m, n, A, lda, 0, 1.0, 0.0));
    if (pr->orthogonalize) {
        // intermediate bases (every one but the last Q) take one CholeskyQR pass
        RLA_TRY(orth<T>(ctx, Q, m, l, ldq, wq, q_signs && pr->power_its == 0, pr->power_its == 0 ? 2 : 1, q_owned));
        for (int64_t it = 0; it < pr->power_its; ++it) {
            const bool last = it + 1 == pr->power_its;
            RLA_TRY(at_q(Q, Z));
            RLA_TRY(orth<T>(ctx, Z, n, l, n, wz, false, 1, true));
            RLA_TRY(a_z(Z, Q));
            RLA_TRY(orth<T>(ctx, Q, m, l, ldq, wq, q_signs && last, last ? 2 : 1, q_owned));
        }
    } else {
        for (int64_t it = 0; it < pr->power_its; ++it) {
            RLA_TRY(at_q(Q, Z));
            RLA_TRY(a_z(Z, Q));
        }
        RLA_TRY(orth<T>(ctx, Q, m, l, ldq, wq, q_signs, 2, q_owned));
    }
    return RLA_OK;
}

static int check_range_args(rla_ctx *ctx, const rla_sketch *om, int dtype, int64_t m, int64_t n, const void *A,
                             int64_t lda, const rla_range_params *pr) {
    if (!ctx) return RLA_E_ARG;
    if (!om || !pr || !A) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    if (pr->power_its < 0) return set_error(ctx, RLA_E_ARG, "Field `power_its` must be non-negative.");
    if (dtype != om->p.dtype) return set_error(ctx, RLA_E_ARG, "Compressor type and matrix type differ.");
    if (m <= 0 || n <= 0 || lda < m) return set_error(ctx, RLA_E_ARG, "Bad matrix dimensions.");
    if (pr->precision != RLA_PREC_NATIVE && pr->precision != RLA_PREC_SPLIT_BF16)
        return set_error(ctx, RLA_E_ARG, "Unknown precision mode %d.", pr->precision);
    if (pr->precision == RLA_PREC_SPLIT_BF16 && dtype != RLA_F32)
        return set_error(ctx, RLA_E_ARG, "Split-BF16 products take Float32 data.");
    return RLA_OK;
}

template <class T, class TO>
static int randsvd_t(rla_ctx *ctx, const rla_sketch *om, int64_t m, int64_t n, const T *A, int64_t lda,
                     const rla_range_params *pr, TO *U, int64_t ldu, double *S, TO *V, int64_t ldv) {
    const int64_t l = om->n_cols;
    Owned own{ctx, {}};
    T *Q;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&Q, sizeof(T) * m * l, ctx->stream));
    own.ptrs.push_back(Q);
    TcOps tc;
    // Float32 products with A run on the tensor cores: split BF16 (2 terms) when asked,
    // otherwise three terms with FP64 accumulation (FP32 accuracy)
    const bool use_tc = std::is_same<T, float>::value;
    if constexpr (std::is_same<T, float>::value)
        RLA_TRY(tc_ops_make(ctx, A, m, n, lda, l, pr->precision == RLA_PREC_SPLIT_BF16 ? 2 : 3, tc, own));
    RLA_TRY(range_core<T>(ctx, om, m, n, A, lda, pr, Q, m, own, use_tc ? &tc : nullptr, false, true));
    // Bt = A'Q (n x l) in FP64 (randsvd.jl:183-185 forms QA in Float64)
    double *Bt, *X, *J, *sig, *jw;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&Bt, sizeof(double) * n * l, ctx->stream));
    own.ptrs.push_back(Bt);
    bool bt_done = false;
    if constexpr (std::is_same<T, float>::value) {
        if (use_tc) {
            RLA_TRY(tc_apply<double>(ctx, tc, 1, m, n, Q, m, l, Bt, n));
            bt_done = true;
        }
    }
    if (!bt_done) RLA_TRY((gemm<T, T, double, double>(ctx, n, l, m, A, lda, 1, Q, m, 0, Bt, n, 1.0, 0.0)));
    double *Qb;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&Qb, sizeof(double) * n * l, ctx->stream));
    own.ptrs.push_back(Qb);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(Qb, Bt, sizeof(double) * n * l, cudaMemcpyDeviceToDevice, ctx->stream));
    OrthWork wb{};
    RLA_TRY(alloc_orth<double>(ctx, wb, n, l, own.ptrs));
    RLA_TRY(orth<double>(ctx, Qb, n, l, n, wb, false, 2, true));
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&X, sizeof(double) * l * l, ctx->stream));
    own.ptrs.push_back(X);
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&J, sizeof(double) * l * l, ctx->stream));
    own.ptrs.push_back(J);
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&sig, sizeof(double) * l, ctx->stream));
    own.ptrs.push_back(sig);
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&jw, sizeof(double) * (2 * l * l + 2 * l), ctx->stream));
    own.ptrs.push_back(jw);
    // X = Rb' = Bt' Qb (l x l)
    RLA_TRY((gemm<double, double, double, double>(ctx, l, l, n, Bt, n, 1, Qb, n, 0, X, l, 1.0, 0.0)));
    // Float32 data resolves singular triplets to about 1e-7: pairs orthogonal to 1e-10 are
    // converged there (the last sweeps of the quadratic phase are skipped); Float64 data
    // keeps 1e-15
    RLA_TRY(jacobi_svd(ctx, X, J, sig, l, jw, sizeof(T) == 4 ? 1e-10 : 1e-15));
    // U = Q W, V = Qb J
    RLA_TRY((gemm<T, double, TO, double>(ctx, m, l, l, Q, m, 0, X, l, 0, U, ldu, 1.0, 0.0)));
    RLA_TRY((gemm<double, double, TO, double>(ctx, n, l, l, Qb, n, 0, J, l, 0, V, ldv, 1.0, 0.0)));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(S, sig, sizeof(double) * l, cudaMemcpyDeviceToDevice, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return use_tc ? tc_status_check(ctx) : RLA_OK;
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_rangefinder(rla_ctx *ctx, const rla_sketch *om, int dtype, int64_t m, int64_t n, const void *A, int64_t lda,
                    const rla_range_params *pr, void *Q, int64_t ldq) {
    RLA_TRY(check_range_args(ctx, om, dtype, m, n, A, lda, pr));
    if (!Q || ldq < m) return set_error(ctx, RLA_E_ARG, "Bad Q buffer.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    Owned own{ctx, {}};
    int rc;
    if (dtype == RLA_F32) {
        TcOps tc;
        RLA_TRY(tc_ops_make(ctx, (const float *)A, m, n, lda, om->n_cols, pr->precision == RLA_PREC_SPLIT_BF16 ? 2 : 3,
                            tc, own));
        float *Qf = (float *)Q;  // the caller's buffer: results are copied into it
        rc = range_core<float>(ctx, om, m, n, (const float *)A, lda, pr, Qf, ldq, own, &tc);
        RLA_TRY(rc);
        RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        return tc_status_check(ctx);
    }
    double *Qd = (double *)Q;
    rc = range_core<double>(ctx, om, m, n, (const double *)A, lda, pr, Qd, ldq, own);
    RLA_TRY(rc);
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

int rla_randsvd(rla_ctx *ctx, const rla_sketch *om, int dtype, int64_t m, int64_t n, const void *A, int64_t lda,
                const rla_range_params *pr, int out_dtype, void *U, int64_t ldu, double *S, void *V, int64_t ldv) {
    RLA_TRY(check_range_args(ctx, om, dtype, m, n, A, lda, pr));
    const int64_t l = om->n_cols;
    if (!U || !S || !V || ldu < m || ldv < n) return set_error(ctx, RLA_E_ARG, "Bad U/S/V buffers.");
    if (l > n) return set_error(ctx, RLA_E_UNSUPPORTED, "compression dimension %lld exceeds n = %lld", (long long)l, (long long)n);
    if (out_dtype != RLA_F32 && out_dtype != RLA_F64) return set_error(ctx, RLA_E_ARG, "out_dtype must be RLA_F32 or RLA_F64.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    if (dtype == RLA_F32) {
        if (out_dtype == RLA_F64)
            return randsvd_t<float, double>(ctx, om, m, n, (const float *)A, lda, pr, (double *)U, ldu, S, (double *)V, ldv);
        return randsvd_t<float, float>(ctx, om, m, n, (const float *)A, lda, pr, (float *)U, ldu, S, (float *)V, ldv);
    }
    if (out_dtype == RLA_F64)
        return randsvd_t<double, double>(ctx, om, m, n, (const double *)A, lda, pr, (double *)U, ldu, S, (double *)V, ldv);
    return randsvd_t<double, float>(ctx, om, m, n, (const double *)A, lda, pr, (float *)U, ldu, S, (float *)V, ldv);
}

}  // extern "C"
