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
//   * both operands staged in shared memory as [k][mn] with a row stride of 68 doubles, so
//     the fragment loads (8 rows x 4 k per phase) hit 16 distinct bank pairs;
//   * the next k-tile is loaded into registers while the current one is multiplied;
//   * split-K over blockIdx.z with FP64 partial tiles added in split order (deterministic);
//     symmetric products (Gram matrices) compute the upper tiles only and mirror them.
#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

constexpr int DG_BM = 64, DG_BN = 64, DG_BK = 16, DG_LD = 68, DG_THREADS = 128;

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

// Element (mn, k) of a K x MN tile source: K_MAJOR: src[k + mn*ld]; else src[mn + k*ld].
template <class T, bool K_MAJOR>
__device__ __forceinline__ double ld_op(const T *src, int64_t ld, int64_t mn, int64_t k, int64_t MN, int64_t K) {
    if (mn >= MN || k >= K) return 0.0;
    return K_MAJOR ? (double)src[k + mn * ld] : (double)src[mn + k * ld];
}

// 8 elements per thread of a 64 (mn) x 16 (k) tile; (i, q) -> element index t + 128 q.
// K-major sources walk k fastest (16-element runs), MN-major sources walk mn fastest.
// `upper`: the source is upper triangular in (k, mn) (entries with k > mn read as zero).
template <class T, bool K_MAJOR>
__device__ __forceinline__ void load_tile(const T *src, int64_t ld, int64_t mn0, int64_t k0, int64_t MN, int64_t K,
                                          int64_t kmax, int t, bool upper, double (&r)[8]) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = t + DG_THREADS * q;
        const int mn = K_MAJOR ? idx / DG_BK : idx % DG_BM;
        const int k = K_MAJOR ? idx % DG_BK : idx / DG_BM;
        r[q] = (upper && k0 + k > mn0 + mn) ? 0.0 : ld_op<T, K_MAJOR>(src, ld, mn0 + mn, k0 + k, MN, kmax);
    }
}

template <bool K_MAJOR>
__device__ __forceinline__ void store_tile(double *s, int t, const double (&r)[8]) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = t + DG_THREADS * q;
        const int mn = K_MAJOR ? idx / DG_BK : idx % DG_BM;
        const int k = K_MAJOR ? idx % DG_BK : idx / DG_BM;
        s[k * DG_LD + mn] = r[q];
    }
}

template <class TA, class TB, class TC, bool A_KM, bool B_KM>
__global__ void __launch_bounds__(DG_THREADS) dgemm_kernel(DgParams p) {
    __shared__ __align__(16) double As[2][DG_BK * DG_LD];
    __shared__ __align__(16) double Bs[2][DG_BK * DG_LD];
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
    double ra[8], rb[8];
    int buf = 0;
    if (kb < ke) {
        load_tile<TA, A_KM>(A, p.lda, m0, kb, p.M, p.K, ke, t, false, ra);
        load_tile<TB, B_KM>(B, p.ldb, n0, kb, p.N, p.K, ke, t, p.b_upper != 0, rb);
        store_tile<A_KM>(As[0], t, ra);
        store_tile<B_KM>(Bs[0], t, rb);
    }
    __syncthreads();
    const int fr = lane >> 2, fk = lane & 3;
    for (int64_t k0 = kb; k0 < ke; k0 += DG_BK) {
        const bool next = k0 + DG_BK < ke;
        if (next) {
            load_tile<TA, A_KM>(A, p.lda, m0, k0 + DG_BK, p.M, p.K, ke, t, false, ra);
            load_tile<TB, B_KM>(B, p.ldb, n0, k0 + DG_BK, p.N, p.K, ke, t, p.b_upper != 0, rb);
        }
        const double *as = As[buf], *bs = Bs[buf];
#pragma unroll
        for (int kk = 0; kk < DG_BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = as[(kk + fk) * DG_LD + wm * 32 + i * 8 + fr];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = bs[(kk + fk) * DG_LD + wn * 32 + j * 8 + fr];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j], a[i], b[j]);
        }
        if (next) {
            store_tile<A_KM>(As[buf ^ 1], t, ra);
            store_tile<B_KM>(Bs[buf ^ 1], t, rb);
        }
        __syncthreads();
        buf ^= 1;
    }
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
                if (p.part) {
                    p.part[(int64_t)blockIdx.z * p.M * p.N + m + n * p.M] = acc[i][j][e];
                } else {
                    TC *cp = (TC *)p.C + m + n * p.ldc;
                    double r = p.alpha * acc[i][j][e];
                    if (!p.beta_zero) r += p.beta * (double)*cp;
                    *cp = (TC)r;
                    if (p.sym && m != n && n0 != m0) {
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
        // a symmetric product computed only its upper tiles: read the mirrored element
        int64_t sm = m, sn = n;
        if (sym && (m / DG_BM) > (n / DG_BN)) {
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
    // split K until the grid covers the GPU about twice, with at least 256 rows per split
    const int64_t tiles = sym ? nt * (nt + 1) / 2 + (mt - nt > 0 ? (mt - nt) * nt : 0) : mt * nt;
    int64_t splits = 1;
    const int64_t want = 2 * (int64_t)ctx->sm_count;
    if (K > 0 && tiles < want) splits = std::min<int64_t>(ceil_div(want, tiles), std::max<int64_t>(1, K / 256));
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
    auto go = [&](auto kern) { kern<<<grid, DG_THREADS, 0, ctx->stream>>>(p); };
    if (ta) {
        if (tb) go(dgemm_kernel<TA, TB, TC, true, false>);
        else go(dgemm_kernel<TA, TB, TC, true, true>);
    } else {
        if (tb) go(dgemm_kernel<TA, TB, TC, false, false>);
        else go(dgemm_kernel<TA, TB, TC, false, true>);
    }
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
