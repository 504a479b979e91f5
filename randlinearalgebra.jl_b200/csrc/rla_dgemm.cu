// rla_dgemm.cu -- FP64-accumulating GEMM on the FP64 tensor cores (DMMA, mma.m8n8k4.f64).
//
// C = alpha * op(A) * op(B) + beta * C with FP64 products and FP64 accumulation, for
// Float32 or Float64 operands (Float32 inputs are widened exactly when staged): the Gram
// matrices, triangular-factor products and small-SVD products of CholeskyQR2 / RandSVD,
// and every other product the library accumulates in FP64.  tcgen05 has no FP64 kind, so
// these use the warp-level FP64 MMA.
//
//   * CTA tile 64 x 64, BK = 16, 128 threads as 2 x 2 warps of 32 x 32 (4 x 4 MMAs of 8 x 8,
//     16 MMAs per k4 step from 4 A and 4 B fragments);
//   * operands copied global -> shared in their own type by cp.async (one element per copy,
//     zero-filled outside the matrix and below the diagonal of an upper-triangular op(B)),
//     DG_STAGES k-tiles in flight; Float32 elements are widened when a fragment is read;
//   * a K-major source is staged [mn][k] with a row stride of 20 elements, an MN-major one
//     [k][mn] with a row stride of 72: the fragment loads (8 mn x 4 k) are conflict-free;
//   * split-K over blockIdx.z with FP64 partial tiles added in split order (deterministic);
//     symmetric products (Gram matrices) compute the upper tiles only and write the upper
//     elements, mirrored; a warp whose 32 x 32 tile lies outside C, below the diagonal, or
//     past the nonzero rows of an upper-triangular op(B) skips those k-steps.
#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

constexpr int DG_BM = 64, DG_BN = 64, DG_BK = 16, DG_THREADS = 128, DG_STAGES = 4;
constexpr int DG_LDK = 20, DG_LDM = 72;  // staged row strides (elements): [mn][k] and [k][mn]
constexpr int DG_TILE = 64 * DG_LDK;      // elements per staged tile (>= DG_BK * DG_LDM)

struct DgParams {
    int64_t M, N, K;
    const void *A;
    int64_t lda;
    const void *B;
    int64_t ldb;
    void *C;
    int64_t ldc;
    double alpha, beta;
    int beta_zero;
    int b_upper;   // op(B) upper triangular: k > n entries are zero and not read
    int sym;       // op(A) * op(B) symmetric: tiles below the diagonal skipped
    int64_t kps;   // K per split
    double *part;  // split partials [split][M x N] (ld M), or null: write C directly
};

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// One element copy global -> shared (4 or 8 bytes); src_bytes = 0 fills zero.
template <class T>
__device__ __forceinline__ void cp_elem(T *dst, const T *src, bool in) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(in ? 4 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(in ? 8 : 0) : "memory");
}

// Stage the 64 (mn) x 16 (k) tile at (mn0, k0) of a source with MN x K extent (k < kmax read):
// 8 elements per thread, consecutive threads along the contiguous dimension.  `upper`:
// entries with k > mn are zero (not read).
template <class T, bool K_MAJOR>
__device__ __forceinline__ void stage_tile(T *s, const T *src, int64_t ld, int64_t mn0, int64_t k0, int64_t MN,
                                           int64_t kmax, int t, bool upper) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int idx = t + DG_THREADS * r;
        const int mn = K_MAJOR ? idx / DG_BK : idx % DG_BM;
        const int k = K_MAJOR ? idx % DG_BK : idx / DG_BM;
        const int64_t gm = mn0 + mn, gk = k0 + k;
        const bool in = gm < MN && gk < kmax && !(upper && gk > gm);
        const T *g = src + (in ? (K_MAJOR ? gk + gm * ld : gm + gk * ld) : 0);
        cp_elem<T>(s + (K_MAJOR ? mn * DG_LDK + k : k * DG_LDM + mn), g, in);
    }
}

template <class T, bool K_MAJOR>
__device__ __forceinline__ double frag(const T *s, int mn, int k) {
    return (double)(K_MAJOR ? s[mn * DG_LDK + k] : s[k * DG_LDM + mn]);
}

template <class TA, class TB, class TC, bool A_KM, bool B_KM>
__global__ void __launch_bounds__(DG_THREADS) dgemm_kernel(DgParams p) {
    extern __shared__ __align__(16) unsigned char dg_sm[];
    TA *As = reinterpret_cast<TA *>(dg_sm);
    TB *Bs = reinterpret_cast<TB *>(dg_sm + sizeof(TA) * DG_STAGES * DG_TILE);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int64_t m0 = (int64_t)blockIdx.x * DG_BM, n0 = (int64_t)blockIdx.y * DG_BN;
    if (p.sym && m0 > n0) return;
    const int64_t kb = (int64_t)blockIdx.z * p.kps;
    int64_t ke = min(p.K, kb + p.kps);
    if (p.b_upper) ke = min(ke, n0 + DG_BN);  // rows k > n of an upper-triangular op(B) are zero
    const TA *A = (const TA *)p.A;
    const TB *B = (const TB *)p.B;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int nkt = kb < ke ? (int)((ke - kb + DG_BK - 1) / DG_BK) : 0;
    auto issue = [&](int kt) {
        if (kt < nkt) {
            const int st = kt % DG_STAGES;
            const int64_t k0 = kb + (int64_t)kt * DG_BK;
            stage_tile<TA, A_KM>(As + st * DG_TILE, A, p.lda, m0, k0, p.M, ke, t, false);
            stage_tile<TB, B_KM>(Bs + st * DG_TILE, B, p.ldb, n0, k0, p.N, ke, t, p.b_upper != 0);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
#pragma unroll
    for (int kt = 0; kt < DG_STAGES - 1; ++kt) issue(kt);
    const int fr = lane >> 2, fk = lane & 3;
    const int64_t wm0 = m0 + wm * 32, wn0 = n0 + wn * 32, wn_last = wn0 + 31;
    const bool warp_live = wm0 < p.M && wn0 < p.N && !(p.sym && wm0 > wn_last);
    for (int kt = 0; kt < nkt; ++kt) {
        asm volatile("cp.async.wait_group %0;" ::"n"(DG_STAGES - 2) : "memory");
        __syncthreads();
        issue(kt + DG_STAGES - 1);  // into the stage every thread finished with at the barrier
        const TA *as = As + (kt % DG_STAGES) * DG_TILE;
        const TB *bs = Bs + (kt % DG_STAGES) * DG_TILE;
        const int64_t k0 = kb + (int64_t)kt * DG_BK;
#pragma unroll
        for (int kk = 0; kk < DG_BK; kk += 4) {
            // a warp whose 32 x 32 tile has nothing to add skips the step (warp-uniform):
            // outside C, below the diagonal of a symmetric product, or past the last nonzero
            // row of an upper-triangular op(B)
            if (!warp_live || (p.b_upper && k0 + kk > wn_last)) continue;
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = frag<TA, A_KM>(as, wm * 32 + i * 8 + fr, kk + fk);
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = frag<TB, B_KM>(bs, wn * 32 + j * 8 + fr, kk + fk);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j], a[i], b[j]);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // acc[i][j][e] holds C(m0 + wm*32 + i*8 + fr, n0 + wn*32 + j*8 + 2*fk + e)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t m = m0 + wm * 32 + i * 8 + fr;
        if (m >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int64_t n = n0 + wn * 32 + j * 8 + 2 * fk + e;
                if (n >= p.N) continue;
                if (p.sym && m > n) continue;  // a symmetric product keeps its upper elements
                if (p.part) {
                    p.part[(int64_t)blockIdx.z * p.M * p.N + m + n * p.M] = acc[i][j][e];
                } else {
                    TC *cp = (TC *)p.C + m + n * p.ldc;
                    double r = p.alpha * acc[i][j][e];
                    if (!p.beta_zero) r += p.beta * (double)*cp;
                    *cp = (TC)r;
                    if (p.sym && m != n) {
                        TC *cq = (TC *)p.C + n + m * p.ldc;
                        double q = p.alpha * acc[i][j][e];
                        if (!p.beta_zero) q += p.beta * (double)*cq;
                        *cq = (TC)q;
                    }
                }
            }
        }
    }
}

// C = alpha * sum_s part[s] + beta * C, splits in order; symmetric: upper tiles mirrored.
template <class TC>
__global__ void dgemm_reduce_kernel(const double *__restrict__ part, int splits, int64_t M, int64_t N, TC *C,
                                    int64_t ldc, double alpha, double beta, int beta_zero, int sym) {
    const int64_t MN = M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < MN; idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t m = idx % M, n = idx / M;
        // a symmetric product computed only its upper elements: read the mirrored element
        int64_t sm = m, sn = n;
        if (sym && m > n) {
            sm = n;
            sn = m;
        }
        double acc = 0.0;
        for (int s = 0; s < splits; ++s) acc += part[s * MN + sm + sn * M];
        TC *cp = C + m + n * ldc;
        double r = alpha * acc;
        if (!beta_zero) r += beta * (double)*cp;
        *cp = (TC)r;
    }
}

template <class TA, class TB, class TC>
int dgemm(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const TA *A, int64_t lda, int ta, const TB *B, int64_t ldb,
          int tb, TC *C, int64_t ldc, double alpha, double beta, int b_upper, int sym) {
    if (M <= 0 || N <= 0) return RLA_OK;
    const int64_t mt = ceil_div(M, DG_BM), nt = ceil_div(N, DG_BN);
    if (mt > 65535 * 1024ll || nt > 65535) return set_error(ctx, RLA_E_UNSUPPORTED, "FP64 GEMM: grid too large");
    const size_t smem = (sizeof(TA) + sizeof(TB)) * DG_STAGES * DG_TILE;
    auto kern = ta ? (tb ? dgemm_kernel<TA, TB, TC, true, false> : dgemm_kernel<TA, TB, TC, true, true>)
                   : (tb ? dgemm_kernel<TA, TB, TC, false, false> : dgemm_kernel<TA, TB, TC, false, true>);
    RLA_CUDA_TRY(ctx, set_smem_max(kern));
    int occ = 1;
    RLA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, DG_THREADS, smem));
    // split K so that the grid fills the resident CTA slots once (no SM runs one CTA more
    // than the others), with at least 256 rows per split
    const int64_t tiles = sym ? nt * (nt + 1) / 2 + (mt - nt > 0 ? (mt - nt) * nt : 0) : mt * nt;
    const int64_t slots = (int64_t)ctx->sm_count * std::max(occ, 1);
    int64_t splits = 1;
    if (K > 0 && tiles < slots) splits = std::max<int64_t>(1, std::min<int64_t>(slots / tiles, K / 256));
    splits = std::max<int64_t>(1, std::min<int64_t>(splits, 1024));
    const int64_t kps = K > 0 ? ceil_div(ceil_div(K, splits), DG_BK) * DG_BK : DG_BK;
    splits = K > 0 ? ceil_div(K, kps) : 1;
    DgParams p{M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, beta == 0.0, b_upper, sym, kps, nullptr};
    if (splits > 1 || (sym && mt != nt)) {
        void *ws = nullptr;
        RLA_TRY(scratch_get(ctx, sizeof(double) * (size_t)splits * M * N, &ws));
        p.part = (double *)ws;
    }
    const dim3 grid((unsigned)mt, (unsigned)nt, (unsigned)splits);
    kern<<<grid, DG_THREADS, smem, ctx->stream>>>(p);
    RLA_TRY(check_launch(ctx, "dgemm"));
    if (p.part) {
        const int64_t MN = M * N;
        const unsigned g = (unsigned)std::min<int64_t>(ceil_div(MN, 256), (int64_t)ctx->sm_count * 16);
        dgemm_reduce_kernel<TC><<<g, 256, 0, ctx->stream>>>(p.part, (int)splits, M, N, C, ldc, alpha, beta, beta == 0.0,
                                                            sym);
        RLA_TRY(check_launch(ctx, "dgemm_reduce"));
    }
    return RLA_OK;
}

#define RLA_INST_DG(TA, TB, TC)                                                                                      \
    template int dgemm<TA, TB, TC>(rla_ctx *, int64_t, int64_t, int64_t, const TA *, int64_t, int, const TB *,      \
                                   int64_t, int, TC *, int64_t, double, double, int, int);
RLA_INST_DG(float, float, float)
RLA_INST_DG(float, float, double)
RLA_INST_DG(float, double, float)
RLA_INST_DG(float, double, double)
RLA_INST_DG(double, float, float)
RLA_INST_DG(double, float, double)
RLA_INST_DG(double, double, float)
RLA_INST_DG(double, double, double)
#undef RLA_INST_DG

}  // namespace rla
