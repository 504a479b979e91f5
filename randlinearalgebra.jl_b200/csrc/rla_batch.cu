// rla_batch.cu -- batched RandSVD: many uneven instances in grouped launches.
//
// rapproximate! of randsvd.jl:174-189 (with power_its.jl:15-80) for a list of Float32
// problems (A_i m_i x n_i, rank k_i <= 128, Gaussian sketch, compression_dim = k_i, the
// reference's defaults p = 0) without one launch sequence per instance: every phase is one
// grouped launch per rank class (k <= 16, 32, 64, 128) whose CTAs map to (instance, tile)
// through a prefix table of tile counts.  Phases:
//   Omega_i (Philox draws, identical to a Gaussian sketch with the instance's seed),
//   Y = A*Omega, CholeskyQR2(Y) [FP64 Gram split over row chunks, Cholesky + triangular
//   inverse of the equilibrated Gram per instance in shared memory, Y <- Y*R^-1 in place],
//   Bt = A'Q (split over row chunks, partial sums added in FP64), CholeskyQR2(Bt) in FP64,
//   X = Bt'Qb (= Rb'), one-sided Jacobi SVD of X per instance in shared memory, U = Q*W,
//   V = Qb*J.
// Products with A accumulate in FP32 on the CUDA cores (the instances are short and wide:
// n <= 1024 per dot); the Gram matrices, Cholesky, inverses and the SVD are FP64.  The
// tile shapes of the two products with A come from an autotuner that times the candidate
// shapes on the actual problem set.  The launch sequence is captured once as a CUDA graph
// and replayed.  An instance whose Cholesky breaks down (numerically rank-deficient Y) is
// flagged and recomputed afterwards by the single-instance path, which has the shifted
// and Householder fallbacks.
#include <math.h>

#include <array>
#include <map>
#include <tuple>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"
#include "rla_tc.cuh"

namespace rla {

constexpr int B_THREADS = 256;
constexpr int B_NCLASS = 4;
static inline int b_kclass(int64_t k) { return k <= 16 ? 0 : k <= 32 ? 1 : k <= 64 ? 2 : 3; }
static inline int b_kt(int c) { return 16 << c; }

struct BProb {
    int64_t m, n, k;
    const float *A;
    int64_t lda;
    float *U;
    int64_t ldu;
    double *S;
    float *V;
    int64_t ldv;
    uint64_t seed;
    // workspace
    float *Om, *Y, *Z;
    double *G, *Rinv, *Bt, *Bt0, *X, *J;
    void *part;
    int *flag;
};

__device__ __forceinline__ int b_find(const int *tstart, int count, int t) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tstart[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---- Omega: element e of instance i (column-major n x k) from the Gaussian stream ----------
__global__ void b_omega_kernel(BProb *P, const int *idx, const int *tstart, int count, float scale_unused) {
    const int t = blockIdx.x;
    const int q = b_find(tstart, count, t);
    BProb &p = P[idx[q]];
    const int64_t npairs = (p.n * p.k + 1) / 2;
    const int64_t i = (int64_t)(t - tstart[q]) * B_THREADS + threadIdx.x;
    if (i >= npairs) return;
    Rng rng;
    rng.k0 = (uint32_t)p.seed;
    rng.k1 = (uint32_t)(p.seed >> 32);
    rng.epoch = 0;
    WordStream ws{rng, STREAM_GAUSS, (uint64_t)i};
    double z2;
    const double z1 = normal_pair(ws, &z2);
    const float sc = (float)(1.0 / sqrt((double)p.k));
    const int64_t tot = p.n * p.k;
    p.Om[2 * i] = sc * (float)z1;
    if (2 * i + 1 < tot) p.Om[2 * i + 1] = sc * (float)z2;
}

// ---- operand selectors -------------------------------------------------------------------
// AX products out(r, j) = sum_c X(r, c) W(c, j) over rows of X:
enum AxKind { AX_A_OM, AX_A_Z, AX_Y_RINV, AX_BT_RINV, AX_Q_W, AX_QB_J };
// Xᵀ·Y products out(i, j) = sum_r X(r, i) Y(r, j), split over row chunks:
enum XtyKind { XT_GRAM_Y, XT_GRAM_BT, XT_A_Q, XT_A_Q_Z, XT_BT0_QB };

template <int KIND>
struct AxOps;
template <>
struct AxOps<AX_A_OM> {
    using TX = float; using TW = float; using TAcc = float; using TO = float;
    __device__ static int64_t rows(const BProb &p) { return p.m; }
    __device__ static int64_t K(const BProb &p) { return p.n; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.lda; return p.A; }
    __device__ static const TW *W(const BProb &p, int64_t &ld) { ld = p.n; return p.Om; }
    __device__ static TO *O(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
};
template <>
struct AxOps<AX_A_Z> : AxOps<AX_A_OM> {
    __device__ static const float *W(const BProb &p, int64_t &ld) { ld = p.n; return p.Z; }
};
template <>
struct AxOps<AX_Y_RINV> {
    using TX = float; using TW = double; using TAcc = double; using TO = float;
    __device__ static int64_t rows(const BProb &p) { return p.m; }
    __device__ static int64_t K(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
    __device__ static const TW *W(const BProb &p, int64_t &ld) { ld = p.k; return p.Rinv; }
    __device__ static TO *O(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
};
template <>
struct AxOps<AX_BT_RINV> {
    using TX = double; using TW = double; using TAcc = double; using TO = double;
    __device__ static int64_t rows(const BProb &p) { return p.n; }
    __device__ static int64_t K(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt; }
    __device__ static const TW *W(const BProb &p, int64_t &ld) { ld = p.k; return p.Rinv; }
    __device__ static TO *O(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt; }
};
template <>
struct AxOps<AX_Q_W> {
    using TX = float; using TW = double; using TAcc = double; using TO = float;
    __device__ static int64_t rows(const BProb &p) { return p.m; }
    __device__ static int64_t K(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
    __device__ static const TW *W(const BProb &p, int64_t &ld) { ld = p.k; return p.X; }
    __device__ static TO *O(const BProb &p, int64_t &ld) { ld = p.ldu; return p.U; }
};
template <>
struct AxOps<AX_QB_J> {
    using TX = double; using TW = double; using TAcc = double; using TO = float;
    __device__ static int64_t rows(const BProb &p) { return p.n; }
    __device__ static int64_t K(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt; }
    __device__ static const TW *W(const BProb &p, int64_t &ld) { ld = p.k; return p.J; }
    __device__ static TO *O(const BProb &p, int64_t &ld) { ld = p.ldv; return p.V; }
};

// Register tiling shared by the grouped products: a CTA computes a BM x KT output tile with
// B_THREADS threads, KT/4 threads across the columns (4 consecutive columns each) and the rest
// down the rows (TM rows each, strided so a warp's shared-memory reads are broadcasts or
// consecutive).  The reduction runs over BK-deep slices staged in shared memory; the next
// slice is read from global memory into registers while the current one is multiplied.
template <class TAcc, int KT, int BM>
struct Tile {
    static constexpr int TN = 4, TXN = KT / TN, TYM = B_THREADS / TXN, TM = BM / TYM;
    static constexpr int BK = (sizeof(TAcc) == 8 && (KT >= 128 || BM >= 128)) ? 16 : 32;
    static constexpr int NP = BK * BM / B_THREADS;  // P-slice elements per thread
    static constexpr int NW = (BK * KT + B_THREADS - 1) / B_THREADS;
    static_assert(TM >= 1 && TYM * TM == BM, "tile shape");
    static_assert(NP * B_THREADS == BK * BM, "slice shape");
};

// FP64 tensor-core form of the slice product for the FP64-accumulating kinds: the CTA's R x KT
// output tile as 8 x 8 mma.m8n8k4.f64 blocks, 8 warps in a WM x WN grid (each warp 16 columns,
// R / WM rows).  Operands as staged: A(mn, k) = SA[k * LDA + mn], B(k, n) = SB[k * LDB + n]
// (row strides 4 mod 16 doubles: conflict-free fragment loads).  Fragment (i, j, e) of a lane
// (g = lane >> 2, q = lane & 3) is element (wm*RW + 8i + g, wn*16 + 8j + 2q + e).
__device__ __forceinline__ void b_dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}
template <int R, int KT, int BK, int LDA, int LDB>
struct BDmma {
    static constexpr int WN = KT / 16, WM = (B_THREADS / 32) / WN, RW = R / WM, MB = RW / 8;
    static_assert(KT % 16 == 0 && WN >= 1 && WM * WN == B_THREADS / 32 && RW % 8 == 0 && MB >= 1, "dmma tile");
    double acc[MB][2][2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < MB; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    }
    __device__ __forceinline__ void slice(const double *SA, const double *SB, int warp, int lane) {
        const int wm = warp / WN, wn = warp % WN, g = lane >> 2, q = lane & 3;
#pragma unroll
        for (int k0 = 0; k0 < BK; k0 += 4) {
            double a[MB], b[2];
#pragma unroll
            for (int i = 0; i < MB; ++i) a[i] = SA[(k0 + q) * LDA + wm * RW + 8 * i + g];
#pragma unroll
            for (int j = 0; j < 2; ++j) b[j] = SB[(k0 + q) * LDB + wn * 16 + 8 * j + g];
#pragma unroll
            for (int i = 0; i < MB; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) b_dmma(acc[i][j], a[i], b[j]);
        }
    }
    __device__ static int row(int warp, int lane, int i) { return (warp / WN) * RW + 8 * i + (lane >> 2); }
    __device__ static int col(int warp, int lane, int j, int e) { return (warp % WN) * 16 + 8 * j + 2 * (lane & 3) + e; }
};

// out (rows x k) = X (rows x K) * W (K x k); CTA = BM rows of one instance, all k columns.
// In-place use (out == X) is safe: a CTA reads all of its rows before it writes them.
template <int KIND, int KT, int BM>
__global__ void __launch_bounds__(B_THREADS) b_ax_kernel(BProb *P, const int *idx, const int *tstart, int count) {
    using O = AxOps<KIND>;
    using TX = typename O::TX;
    using TW = typename O::TW;
    using TAcc = typename O::TAcc;
    using TO = typename O::TO;
    using Tl = Tile<TAcc, KT, BM>;
    constexpr int BK = Tl::BK, TM = Tl::TM, TN = Tl::TN, TXN = Tl::TXN, TYM = Tl::TYM, NP = Tl::NP, NW = Tl::NW;
    __shared__ __align__(16) TAcc Xs[BK][BM + 4];
    __shared__ __align__(16) TAcc Ws[BK][KT + 4];
    constexpr bool TC = sizeof(TAcc) == 8;  // FP64 accumulation: on the FP64 tensor cores
    using Dm = BDmma<BM, KT, BK, BM + 4, KT + 4>;
    Dm dm;
    const int t = blockIdx.x;
    const int q = b_find(tstart, count, t);
    const BProb &p = P[idx[q]];
    const int64_t rows = O::rows(p), K = O::K(p), kk = p.k;
    int64_t ldx, ldw, ldo;
    const TX *X = O::X(p, ldx);
    const TW *W = O::W(p, ldw);
    TO *Out = O::O(p, ldo);
    const int64_t r0 = (int64_t)(t - tstart[q]) * BM;
    const int tid = threadIdx.x, tx = tid % TXN, ty = tid / TXN;
    TAcc acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = TAcc(0);
    TAcc px[NP], pw[NW];
    auto fetch = [&](int64_t c0) {
#pragma unroll
        for (int u = 0; u < NP; ++u) {
            const int e = tid + u * B_THREADS, r = e % BM, c = e / BM;
            const int64_t gr = r0 + r, gc = c0 + c;
            px[u] = (gr < rows && gc < K) ? (TAcc)X[gr + gc * ldx] : TAcc(0);
        }
#pragma unroll
        for (int u = 0; u < NW; ++u) {
            const int e = tid + u * B_THREADS, c = e % BK, j = e / BK;
            const int64_t gc = c0 + c;
            pw[u] = (e < BK * KT && gc < K && j < kk) ? (TAcc)W[gc + j * ldw] : TAcc(0);
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int u = 0; u < NP; ++u) {
            const int e = tid + u * B_THREADS;
            Xs[e / BM][e % BM] = px[u];
        }
#pragma unroll
        for (int u = 0; u < NW; ++u) {
            const int e = tid + u * B_THREADS;
            if (e < BK * KT) Ws[e % BK][e / BK] = pw[u];
        }
    };
    if constexpr (TC) dm.zero();
    fetch(0);
    for (int64_t c0 = 0; c0 < K; c0 += BK) {
        stash();
        __syncthreads();
        if (c0 + BK < K) fetch(c0 + BK);
        if constexpr (TC) {
            dm.slice(reinterpret_cast<const double *>(&Xs[0][0]), reinterpret_cast<const double *>(&Ws[0][0]), tid >> 5,
                     tid & 31);
        } else {
#pragma unroll 8
            for (int c = 0; c < BK; ++c) {
                TAcc a[TM], b[TN];
#pragma unroll
                for (int i = 0; i < TM; ++i) a[i] = Xs[c][ty + TYM * i];
#pragma unroll
                for (int j = 0; j < TN; ++j) b[j] = Ws[c][tx * TN + j];
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
        }
        __syncthreads();
    }
    if constexpr (TC) {
        const int w = tid >> 5, l = tid & 31;
#pragma unroll
        for (int i = 0; i < Dm::MB; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int64_t gr = r0 + Dm::row(w, l, i), gj = Dm::col(w, l, j, e);
                    if (gr < rows && gj < kk) Out[gr + gj * ldo] = (TO)dm.acc[i][j][e];
                }
        return;
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
        const int64_t gj = tx * TN + j;
        if (gj >= kk) continue;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int64_t gr = r0 + ty + TYM * i;
            if (gr < rows) Out[gr + gj * ldo] = (TO)acc[i][j];
        }
    }
}

template <int KIND>
struct XtyOps;
template <>
struct XtyOps<XT_GRAM_Y> {
    using TX = float; using TAcc = double;
    __device__ static int64_t rows(const BProb &p) { return p.m; }
    __device__ static int64_t nx(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
    __device__ static const TX *Y(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
};
template <>
struct XtyOps<XT_GRAM_BT> {
    using TX = double; using TAcc = double;
    __device__ static int64_t rows(const BProb &p) { return p.n; }
    __device__ static int64_t nx(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt; }
    __device__ static const TX *Y(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt; }
};
template <>
struct XtyOps<XT_A_Q> {
    using TX = float; using TAcc = float;
    __device__ static int64_t rows(const BProb &p) { return p.m; }
    __device__ static int64_t nx(const BProb &p) { return p.n; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.lda; return p.A; }
    __device__ static const TX *Y(const BProb &p, int64_t &ld) { ld = p.m; return p.Y; }
};
template <>
struct XtyOps<XT_A_Q_Z> : XtyOps<XT_A_Q> {};
template <>
struct XtyOps<XT_BT0_QB> {
    using TX = double; using TAcc = double;
    __device__ static int64_t rows(const BProb &p) { return p.n; }
    __device__ static int64_t nx(const BProb &p) { return p.k; }
    __device__ static const TX *X(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt0; }
    __device__ static const TX *Y(const BProb &p, int64_t &ld) { ld = p.n; return p.Bt; }
};

// part[s][i][j] = sum over rows r of chunk s of X(r, i) Y(r, j), i in a BR-column block of
// X, j < k.  Tiles of an instance: (column block, chunk), chunk-major.  Same register tiling
// and slice prefetch as b_ax_kernel, with the X slice transposed into shared memory.
template <int KIND, int KT, int BR>
__global__ void __launch_bounds__(B_THREADS) b_xty_kernel(BProb *P, const int *idx, const int *tstart, int count,
                                                          int64_t chunk) {
    using O = XtyOps<KIND>;
    using TX = typename O::TX;
    using TAcc = typename O::TAcc;
    using Tl = Tile<TAcc, KT, BR>;
    constexpr int BK = Tl::BK, TM = Tl::TM, TN = Tl::TN, TXN = Tl::TXN, TYM = Tl::TYM, NP = Tl::NP, NW = Tl::NW;
    __shared__ __align__(16) TAcc Xs[BK][BR + 4];
    __shared__ __align__(16) TAcc Ys[BK][KT + 4];
    constexpr bool TC = sizeof(TAcc) == 8;  // FP64 accumulation: on the FP64 tensor cores
    using Dm = BDmma<BR, KT, BK, BR + 4, KT + 4>;
    Dm dm;
    const int t = blockIdx.x;
    const int q = b_find(tstart, count, t);
    const BProb &p = P[idx[q]];
    const int64_t rows = O::rows(p), nx = O::nx(p), kk = p.k;
    int64_t ldx, ldy;
    const TX *X = O::X(p, ldx);
    const TX *Yp = O::Y(p, ldy);
    const int64_t ncb = (nx + BR - 1) / BR;
    const int64_t lt = t - tstart[q];
    const int64_t cb = lt % ncb, split = lt / ncb;
    const int64_t i0 = cb * BR, rs = split * chunk, re = min(rows, rs + chunk);
    const int tid = threadIdx.x, tx = tid % TXN, ty = tid / TXN;
    TAcc acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = TAcc(0);
    TAcc px[NP], py[NW];
    auto fetch = [&](int64_t r0) {
#pragma unroll
        for (int u = 0; u < NP; ++u) {
            const int e = tid + u * B_THREADS, r = e % BK, c = e / BK;
            const int64_t gr = r0 + r, gc = i0 + c;
            px[u] = (gr < re && gc < nx) ? (TAcc)X[gr + gc * ldx] : TAcc(0);
        }
#pragma unroll
        for (int u = 0; u < NW; ++u) {
            const int e = tid + u * B_THREADS, r = e % BK, j = e / BK;
            const int64_t gr = r0 + r;
            py[u] = (e < BK * KT && gr < re && j < kk) ? (TAcc)Yp[gr + j * ldy] : TAcc(0);
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int u = 0; u < NP; ++u) {
            const int e = tid + u * B_THREADS;
            Xs[e % BK][e / BK] = px[u];
        }
#pragma unroll
        for (int u = 0; u < NW; ++u) {
            const int e = tid + u * B_THREADS;
            if (e < BK * KT) Ys[e % BK][e / BK] = py[u];
        }
    };
    if constexpr (TC) dm.zero();
    if (rs < re) fetch(rs);
    for (int64_t r0 = rs; r0 < re; r0 += BK) {
        stash();
        __syncthreads();
        if (r0 + BK < re) fetch(r0 + BK);
        if constexpr (TC) {
            dm.slice(reinterpret_cast<const double *>(&Xs[0][0]), reinterpret_cast<const double *>(&Ys[0][0]), tid >> 5,
                     tid & 31);
        } else {
#pragma unroll 8
            for (int r = 0; r < BK; ++r) {
                TAcc a[TM], b[TN];
#pragma unroll
                for (int i = 0; i < TM; ++i) a[i] = Xs[r][ty + TYM * i];
#pragma unroll
                for (int j = 0; j < TN; ++j) b[j] = Ys[r][tx * TN + j];
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
        }
        __syncthreads();
    }
    TAcc *part = reinterpret_cast<TAcc *>(p.part) + split * nx * kk;
    if constexpr (TC) {
        const int w = tid >> 5, l = tid & 31;
#pragma unroll
        for (int i = 0; i < Dm::MB; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int64_t gi = i0 + Dm::row(w, l, i), gj = Dm::col(w, l, j, e);
                    if (gi < nx && gj < kk) part[gi * kk + gj] = dm.acc[i][j][e];
                }
        return;
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int64_t gi = i0 + ty + TYM * i;
        if (gi >= nx) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int64_t gj = tx * TN + j;
            if (gj < kk) part[gi * kk + gj] = acc[i][j];
        }
    }
}

// out(i, j) (ld ldo) = sum_s part[s][i][j] added in split order in FP64.  KIND selects the
// target: Gram (G, k x k), Bt (n x k, also copied to Bt0), X (k x k).
enum RedKind { RED_G_M, RED_G_N, RED_BT, RED_X, RED_Z };
template <int KIND, class TP>
__global__ void b_reduce_kernel(BProb *P, const int *idx, int64_t chunk_m, int64_t chunk_n) {
    const BProb &p = P[idx[blockIdx.y]];
    const int64_t kk = p.k;
    int64_t nx, rows, chunk;
    if (KIND == RED_G_M) { nx = kk; rows = p.m; chunk = chunk_m; }
    else if (KIND == RED_G_N || KIND == RED_X) { nx = kk; rows = p.n; chunk = chunk_n; }
    else { nx = p.n; rows = p.m; chunk = chunk_m; }
    const int64_t ns = (rows + chunk - 1) / chunk;
    const TP *part = reinterpret_cast<const TP *>(p.part);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nx * kk; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / kk, j = e % kk;
        double acc = 0.0;
        for (int64_t s = 0; s < ns; ++s) acc += (double)part[s * nx * kk + e];
        if (KIND == RED_BT) {
            p.Bt[i + j * p.n] = acc;
            p.Bt0[i + j * p.n] = acc;
        } else if (KIND == RED_Z) {
            p.Z[i + j * p.n] = (float)acc;
        } else if (KIND == RED_X) {
            p.X[i + j * kk] = acc;
        } else {
            p.G[i + j * kk] = acc;
        }
    }
}

__device__ inline double b_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Per instance (one CTA): D = diag(G)^-1/2, R'R = D G D (upper Cholesky in shared memory),
// Rinv = D R^-1 (so that Y Rinv = Q).  A non-positive pivot sets *flag.
__global__ void __launch_bounds__(512) b_chol_inv_kernel(BProb *P, const int *idx) {
    extern __shared__ double b_sm[];
    const BProb &p = P[idx[blockIdx.x]];
    const int k = (int)p.k;
    double *Gs = b_sm;                  // k x k
    double *d = Gs + (int64_t)k * k;    // k
    double *xs = d + k;                 // 16 warps x k
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    if (tid == 0) bad = 0;
    for (int i = tid; i < k; i += nt) {
        const double g = p.G[i + (int64_t)i * k];
        d[i] = g > 0.0 ? rsqrt(g) : 1.0;
    }
    __syncthreads();
    for (int e = tid; e < k * k; e += nt) {
        const int i = e % k, j = e / k;
        Gs[e] = p.G[e] * d[i] * d[j];
    }
    __syncthreads();
    for (int c = 0; c < k; ++c) {
        if (tid == 0) {
            double v = Gs[c + c * k];
            if (!(v > 0.0) || !isfinite(v)) {
                bad = 1;
                v = 1.0;
            }
            Gs[c + c * k] = sqrt(v);
        }
        __syncthreads();
        const double rcc = Gs[c + c * k];
        for (int j = c + 1 + tid; j < k; j += nt) Gs[c + j * k] /= rcc;
        __syncthreads();
        const int n2 = k - c - 1;
        for (int e = tid; e < n2 * n2; e += nt) {
            const int a = c + 1 + e % n2, b = c + 1 + e / n2;
            if (a <= b) Gs[a + b * k] -= Gs[c + a * k] * Gs[c + b * k];
        }
        __syncthreads();
    }
    // Rinv columns: back substitution, one warp per column
    for (int j = warp; j < k; j += nw) {
        double *x = xs + (int64_t)warp * k;
        for (int i = lane; i < k; i += 32) x[i] = 0.0;
        __syncwarp();
        if (lane == 0) x[j] = 1.0 / Gs[j + j * k];
        __syncwarp();
        for (int i = j - 1; i >= 0; --i) {
            double s = 0.0;
            for (int c = i + 1 + lane; c <= j; c += 32) s += Gs[i + c * k] * x[c];
            s = b_warp_sum(s);
            if (lane == 0) x[i] = -s / Gs[i + i * k];
            __syncwarp();
        }
        for (int i = lane; i < k; i += 32) p.Rinv[i + (int64_t)j * k] = d[i] * x[i];
        __syncwarp();
    }
    if (tid == 0 && bad) *p.flag = 1;
}

__device__ inline void b_pair(int r, int pidx, int n2, int *i, int *j) {
    const int mm = n2 - 1;
    if (pidx == 0) {
        *i = r % mm;
        *j = mm;
    } else {
        *i = (r + pidx) % mm;
        *j = (r - pidx + mm) % mm;
    }
    if (*i > *j) {
        const int t = *i;
        *i = *j;
        *j = t;
    }
}

// One-sided Jacobi SVD of X (k x k) per instance, X and J in shared memory; on return X
// holds W (normalised columns sorted by descending sigma), J the matching rotations and
// S the singular values.
__global__ void __launch_bounds__(512) b_jacobi_kernel(BProb *P, const int *idx, double tol, int max_sweeps,
                                                       int j_in_smem) {
    extern __shared__ double b_sm[];
    const BProb &p = P[idx[blockIdx.x]];
    const int k = (int)p.k;
    // J stays in global memory (L2) when X and J together exceed shared memory
    double *Xs = b_sm, *sg = Xs + (int64_t)k * k;
    int *perm = reinterpret_cast<int *>(sg + k);
    double *Js = j_in_smem ? reinterpret_cast<double *>(perm + k + (k & 1)) : p.Bt0;
    __shared__ unsigned long long off_bits;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int e = tid; e < k * k; e += nt) {
        Xs[e] = p.X[e];
        Js[e] = (e % k == e / k) ? 1.0 : 0.0;
    }
    __syncthreads();
    const int n2 = k + (k & 1);
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        if (tid == 0) off_bits = 0ull;
        __syncthreads();
        for (int r = 0; r < n2 - 1; ++r) {
            for (int pp = warp; pp < n2 / 2; pp += nw) {
                int i, j;
                b_pair(r, pp, n2, &i, &j);
                if (j >= k) continue;
                double *xi = Xs + (int64_t)i * k, *xj = Xs + (int64_t)j * k;
                double a = 0, b = 0, g = 0;
                for (int e = lane; e < k; e += 32) {
                    const double u = xi[e], w = xj[e];
                    a = fma(u, u, a);
                    b = fma(w, w, b);
                    g = fma(u, w, g);
                }
                a = b_warp_sum(a);
                b = b_warp_sum(b);
                g = b_warp_sum(g);
                const double nrm = sqrt(a * b);
                if (g != 0.0 && fabs(g) > tol * nrm) {
                    if (lane == 0) atomicMax(&off_bits, (unsigned long long)__double_as_longlong(fabs(g) / nrm));
                    const double zeta = (b - a) / (2.0 * g);
                    const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
                    double *ji = Js + (int64_t)i * k, *jj = Js + (int64_t)j * k;
                    for (int e = lane; e < k; e += 32) {
                        const double u = xi[e], w = xj[e];
                        xi[e] = cs * u - sn * w;
                        xj[e] = sn * u + cs * w;
                        const double uj = ji[e], wj = jj[e];
                        ji[e] = cs * uj - sn * wj;
                        jj[e] = sn * uj + cs * wj;
                    }
                }
            }
            __syncthreads();
        }
        const bool done = __longlong_as_double((long long)off_bits) <= tol;
        __syncthreads();
        if (done) break;
    }
    for (int c = warp; c < k; c += nw) {
        double a = 0;
        for (int e = lane; e < k; e += 32) a += Xs[e + (int64_t)c * k] * Xs[e + (int64_t)c * k];
        a = b_warp_sum(a);
        if (lane == 0) sg[c] = sqrt(a);
    }
    __syncthreads();
    if (tid == 0) {
        for (int c = 0; c < k; ++c) perm[c] = c;
        for (int a = 1; a < k; ++a) {
            const int v = perm[a];
            int b = a - 1;
            while (b >= 0 && sg[perm[b]] < sg[v]) {
                perm[b + 1] = perm[b];
                --b;
            }
            perm[b + 1] = v;
        }
    }
    __syncthreads();
    for (int e = tid; e < k * k; e += nt) {
        const int r = e % k, c = e / k, src = perm[c];
        const double sv = sg[src];
        p.X[e] = sv > 0.0 ? Xs[r + (int64_t)src * k] / sv : 0.0;
        p.J[e] = Js[r + (int64_t)src * k];
    }
    for (int c = tid; c < k; c += nt) p.S[c] = sg[perm[c]];
}

}  // namespace rla

// ------------------------------------------------------------------------------------
// host side: plan, autotuner, graph
// ------------------------------------------------------------------------------------
struct rla_batch {
    rla_ctx *ctx = nullptr;   // allocations come from this context's pool
    int device = 0;
    int flags = 0;
    int count = 0;
    std::vector<rla_svd_problem> probs;
    rla_range_params params{};
    rla::BProb *d_probs = nullptr;
    std::vector<rla::BProb> h_probs;
    void *work = nullptr;
    int *flagbuf = nullptr;
    // per rank class: instance list (device) and host copy
    std::vector<int> cls_h[rla::B_NCLASS];
    int *cls_d[rla::B_NCLASS] = {nullptr, nullptr, nullptr, nullptr};
    // tile prefix tables keyed by (class, kind, tile size)
    std::map<std::tuple<int, int, int64_t>, int *> maps;
    std::map<std::tuple<int, int, int64_t>, int> map_total;
    int64_t chunk_m = 4096, chunk_n = 1 << 20;
    int bm_ax[rla::B_NCLASS] = {256, 256, 256, 128};  // rows per CTA of A*Omega / A*Z (64, 128, 256)
    int br_aq[rla::B_NCLASS] = {256, 256, 256, 128};  // columns of A per CTA of A'Q (64, 128, 256)
    int64_t chunk_aq[rla::B_NCLASS] = {8192, 8192, 8192, 8192};
    bool tuned = false;
    cudaStream_t cs = nullptr;
    cudaStream_t side[rla::B_NCLASS] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[rla::B_NCLASS] = {nullptr, nullptr, nullptr, nullptr};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void *> owned;
    // RLA_PREC_SPLIT_BF16 (classes with k <= 64): the passes over A as grouped tensor-core
    // products, A split once per run into BF16 hi/lo, the thin factor split per product
    bool tc = false;
    rla::SplitGroup s_a[rla::B_NCLASS], s_om[rla::B_NCLASS], s_y[rla::B_NCLASS], s_z[rla::B_NCLASS];
    rla::TcGroup g_ax[rla::B_NCLASS], g_atq_z[rla::B_NCLASS], g_atq_bt[rla::B_NCLASS];
};

namespace rla {

enum MapKind { MK_OMEGA, MK_ROWS_M, MK_ROWS_N, MK_XTY_GRAM_M, MK_XTY_GRAM_N, MK_XTY_AQ };

// Tiles of instance p for a map kind; `sz` is the tile parameter (BM, BR or elements).
static int64_t tiles_of(const rla_batch *b, const BProb &p, int kind, int64_t sz, int64_t chunk) {
    switch (kind) {
        case MK_OMEGA: return ceil_div((p.n * p.k + 1) / 2, B_THREADS);
        case MK_ROWS_M: return ceil_div(p.m, sz);
        case MK_ROWS_N: return ceil_div(p.n, sz);
        case MK_XTY_GRAM_M: return ceil_div(p.k, sz) * ceil_div(p.m, chunk);
        case MK_XTY_GRAM_N: return ceil_div(p.k, sz) * ceil_div(p.n, chunk);
        case MK_XTY_AQ: return ceil_div(p.n, sz) * ceil_div(p.m, chunk);
    }
    return 0;
}

static int get_map(rla_ctx *ctx, rla_batch *b, int cls, int kind, int64_t sz, int64_t chunk, int **out, int *total) {
    const auto key = std::make_tuple(cls, kind * 1000003 + (int)(chunk % 1000003), sz);
    auto it = b->maps.find(key);
    if (it != b->maps.end()) {
        *out = it->second;
        *total = b->map_total[key];
        return RLA_OK;
    }
    const auto &ids = b->cls_h[cls];
    std::vector<int> ts(ids.size() + 1, 0);
    int64_t acc = 0;
    for (size_t q = 0; q < ids.size(); ++q) {
        ts[q] = (int)acc;
        acc += tiles_of(b, b->h_probs[ids[q]], kind, sz, chunk);
    }
    ts[ids.size()] = (int)acc;
    if (acc >= (1ll << 31)) return set_error(ctx, RLA_E_UNSUPPORTED, "batch too large for one grouped launch");
    int *d = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(b->ctx, &d, sizeof(int) * ts.size(), b->ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(d, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice, b->ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(b->ctx->stream));
    b->owned.push_back(d);
    b->maps[key] = d;
    b->map_total[key] = (int)acc;
    *out = d;
    *total = (int)acc;
    return RLA_OK;
}

template <int KIND, int KT, int BM>
static int launch_ax(rla_ctx *ctx, rla_batch *b, int cls, cudaStream_t st) {
    const int kind = (KIND == AX_BT_RINV || KIND == AX_QB_J) ? MK_ROWS_N : MK_ROWS_M;
    int *ts, tot;
    RLA_TRY(get_map(ctx, b, cls, kind, BM, 0, &ts, &tot));
    if (tot == 0) return RLA_OK;
    b_ax_kernel<KIND, KT, BM><<<tot, B_THREADS, 0, st>>>(b->d_probs, b->cls_d[cls], ts, (int)b->cls_h[cls].size());
    return check_launch(ctx, "batch_ax");
}

// Rows per CTA of the A*X products: candidates 64, 128, 256 (256 only while the register tile
// stays small, KT <= 64).
template <int KIND, int KT>
static int launch_ax_bm(rla_ctx *ctx, rla_batch *b, int cls, int bm, cudaStream_t st) {
    if (bm <= 64) return launch_ax<KIND, KT, 64>(ctx, b, cls, st);
    if constexpr (KT <= 64) {
        if (bm > 128) return launch_ax<KIND, KT, 256>(ctx, b, cls, st);
    }
    return launch_ax<KIND, KT, 128>(ctx, b, cls, st);
}

// Smallest column block of an X'Y product with a full register tile (Tile<.., KT, BR>).
template <int KT>
constexpr int min_br() { return 1024 / KT > KT ? 1024 / KT : KT; }

template <int KIND, int KT, int BR>
static int launch_xty(rla_ctx *ctx, rla_batch *b, int cls, int64_t chunk, cudaStream_t st);

// Columns of A per CTA of A'Q: candidates 64, 128, 256 (256 only while the register tile stays
// small, KT <= 64).
template <int KIND, int KT>
static int launch_xty_br(rla_ctx *ctx, rla_batch *b, int cls, int br, int64_t chunk, cudaStream_t st) {
    if (br <= 64) return launch_xty<KIND, KT, 64>(ctx, b, cls, chunk, st);
    if constexpr (KT <= 64) {
        if (br > 128) return launch_xty<KIND, KT, 256>(ctx, b, cls, chunk, st);
    }
    return launch_xty<KIND, KT, 128>(ctx, b, cls, chunk, st);
}

template <int KIND, int KT, int BR>
static int launch_xty(rla_ctx *ctx, rla_batch *b, int cls, int64_t chunk, cudaStream_t st) {
    const int kind = KIND == XT_GRAM_Y ? MK_XTY_GRAM_M : (KIND == XT_A_Q || KIND == XT_A_Q_Z) ? MK_XTY_AQ : MK_XTY_GRAM_N;
    int *ts, tot;
    RLA_TRY(get_map(ctx, b, cls, kind, BR, chunk, &ts, &tot));
    if (tot == 0) return RLA_OK;
    b_xty_kernel<KIND, KT, BR><<<tot, B_THREADS, 0, st>>>(b->d_probs, b->cls_d[cls], ts, (int)b->cls_h[cls].size(), chunk);
    return check_launch(ctx, "batch_xty");
}

template <int KIND, class TP>
static int launch_reduce(rla_ctx *ctx, rla_batch *b, int cls, int64_t chunk_m, int64_t chunk_n, cudaStream_t st) {
    const int nq = (int)b->cls_h[cls].size();
    if (nq == 0) return RLA_OK;
    b_reduce_kernel<KIND, TP><<<dim3(8, nq), 256, 0, st>>>(b->d_probs, b->cls_d[cls], chunk_m, chunk_n);
    return check_launch(ctx, "batch_reduce");
}

template <int KT>
static int run_class(rla_ctx *ctx, rla_batch *b, int cls, cudaStream_t st) {
    const int nq = (int)b->cls_h[cls].size();
    if (nq == 0) return RLA_OK;
    int *ts, tot;
    // Omega
    RLA_TRY(get_map(ctx, b, cls, MK_OMEGA, B_THREADS, 0, &ts, &tot));
    b_omega_kernel<<<tot, B_THREADS, 0, st>>>(b->d_probs, b->cls_d[cls], ts, nq, 0.f);
    RLA_TRY(check_launch(ctx, "batch_omega"));
    const int kt = KT;
    const size_t chol_smem = sizeof(double) * ((size_t)kt * kt + kt + 16 * kt);
    const size_t jac_x = sizeof(double) * ((size_t)kt * kt + kt) + sizeof(int) * (kt + 2);
    const size_t jac_xj = jac_x + sizeof(double) * (size_t)kt * kt;
    const int j_in_smem = jac_xj <= (size_t)ctx->smem_optin - 1024 ? 1 : 0;
    const size_t jac_smem = j_in_smem ? jac_xj : jac_x;
    // (dynamic shared-memory limits of b_chol_inv_kernel / b_jacobi_kernel are raised at plan creation)
    auto orth_m = [&]() -> int {  // CholeskyQR2 of Y (m x k, FP32 data, FP64 Gram)
        for (int pass = 0; pass < 2; ++pass) {
            RLA_TRY((launch_xty<XT_GRAM_Y, KT, min_br<KT>()>(ctx, b, cls, b->chunk_m, st)));
            RLA_TRY((launch_reduce<RED_G_M, double>(ctx, b, cls, b->chunk_m, b->chunk_n, st)));
            b_chol_inv_kernel<<<nq, 512, chol_smem, st>>>(b->d_probs, b->cls_d[cls]);
            RLA_TRY(check_launch(ctx, "batch_chol"));
            RLA_TRY((launch_ax<AX_Y_RINV, KT, 64>(ctx, b, cls, st)));
        }
        return RLA_OK;
    };
    const bool tc = b->tc && KT <= 64;
    // Y = A * Omega
    if (tc) {
        RLA_TRY(split_group_run(ctx, b->s_a[cls], st));
        RLA_TRY(split_group_run(ctx, b->s_om[cls], st));
        RLA_TRY(tc_group_run(ctx, b->g_ax[cls], st));
    } else {
        RLA_TRY((launch_ax_bm<AX_A_OM, KT>(ctx, b, cls, b->bm_ax[cls], st)));
    }
    const bool ortho = b->params.orthogonalize != 0;
    if (ortho || b->params.power_its == 0) RLA_TRY(orth_m());
    for (int64_t it = 0; it < b->params.power_its; ++it) {
        // Z = A'Q, optionally orthonormalised, then Q = A Z
        if (tc) {
            RLA_TRY(split_group_run(ctx, b->s_y[cls], st));
            RLA_TRY(tc_group_run(ctx, b->g_atq_z[cls], st));
            RLA_TRY(split_group_run(ctx, b->s_z[cls], st));
            RLA_TRY(tc_group_run(ctx, b->g_ax[cls], st));
        } else {
            RLA_TRY((launch_xty_br<XT_A_Q_Z, KT>(ctx, b, cls, b->br_aq[cls], b->chunk_aq[cls], st)));
            RLA_TRY((launch_reduce<RED_Z, float>(ctx, b, cls, b->chunk_aq[cls], b->chunk_n, st)));
            RLA_TRY((launch_ax_bm<AX_A_Z, KT>(ctx, b, cls, b->bm_ax[cls], st)));
        }
        if (ortho || it + 1 == b->params.power_its) RLA_TRY(orth_m());
    }
    // Bt = A'Q in FP64 (CUDA cores: FP32 partials added in FP64; tensor cores: FP64
    // accumulation across k-chunks, written to Bt and its copy Bt0)
    if (tc) {
        RLA_TRY(split_group_run(ctx, b->s_y[cls], st));
        RLA_TRY(tc_group_run(ctx, b->g_atq_bt[cls], st));
    } else {
        RLA_TRY((launch_xty_br<XT_A_Q, KT>(ctx, b, cls, b->br_aq[cls], b->chunk_aq[cls], st)));
        RLA_TRY((launch_reduce<RED_BT, float>(ctx, b, cls, b->chunk_aq[cls], b->chunk_n, st)));
    }
    // CholeskyQR2 of Bt (n x k, FP64)
    for (int pass = 0; pass < 2; ++pass) {
        RLA_TRY((launch_xty<XT_GRAM_BT, KT, min_br<KT>()>(ctx, b, cls, b->chunk_n, st)));
        RLA_TRY((launch_reduce<RED_G_N, double>(ctx, b, cls, b->chunk_m, b->chunk_n, st)));
        b_chol_inv_kernel<<<nq, 512, chol_smem, st>>>(b->d_probs, b->cls_d[cls]);
        RLA_TRY(check_launch(ctx, "batch_chol"));
        RLA_TRY((launch_ax<AX_BT_RINV, KT, 64>(ctx, b, cls, st)));
    }
    // X = Bt0' Qb = Rb', SVD, U = Q W, V = Qb J
    RLA_TRY((launch_xty<XT_BT0_QB, KT, min_br<KT>()>(ctx, b, cls, b->chunk_n, st)));
    RLA_TRY((launch_reduce<RED_X, double>(ctx, b, cls, b->chunk_m, b->chunk_n, st)));
    b_jacobi_kernel<<<nq, 512, jac_smem, st>>>(b->d_probs, b->cls_d[cls], 1e-15, 60, j_in_smem);
    RLA_TRY(check_launch(ctx, "batch_jacobi"));
    RLA_TRY((launch_ax<AX_Q_W, KT, 64>(ctx, b, cls, st)));
    RLA_TRY((launch_ax<AX_QB_J, KT, 64>(ctx, b, cls, st)));
    return RLA_OK;
}

// The rank classes share nothing, so each runs on its own stream forked from `st` (their
// launch tails overlap); `st` waits for all of them.
static int enqueue_all(rla_ctx *ctx, rla_batch *b, cudaStream_t st) {
    RLA_CUDA_TRY(ctx, cudaEventRecord(b->fork, st));
    for (int c = 0; c < B_NCLASS; ++c) {
        if (b->cls_h[c].empty()) continue;
        cudaStream_t sc = b->side[c];
        RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(sc, b->fork, 0));
        switch (c) {
            case 0: RLA_TRY(run_class<16>(ctx, b, 0, sc)); break;
            case 1: RLA_TRY(run_class<32>(ctx, b, 1, sc)); break;
            case 2: RLA_TRY(run_class<64>(ctx, b, 2, sc)); break;
            default: RLA_TRY(run_class<128>(ctx, b, 3, sc));
        }
        RLA_CUDA_TRY(ctx, cudaEventRecord(b->join[c], sc));
        RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(st, b->join[c], 0));
    }
    return RLA_OK;
}

// Time one enqueue of class `cls` with the current tile choices (ms).
static int time_class(rla_ctx *ctx, rla_batch *b, int cls, float *ms) {
    cudaStream_t st = b->cs;
    auto go = [&]() -> int {
        switch (cls) {
            case 0: return run_class<16>(ctx, b, 0, st);
            case 1: return run_class<32>(ctx, b, 1, st);
            case 2: return run_class<64>(ctx, b, 2, st);
            default: return run_class<128>(ctx, b, 3, st);
        }
    };
    RLA_TRY(go());  // warm
    RLA_CUDA_TRY(ctx, cudaEventRecord(b->ev0, st));
    RLA_TRY(go());
    RLA_CUDA_TRY(ctx, cudaEventRecord(b->ev1, st));
    RLA_CUDA_TRY(ctx, cudaEventSynchronize(b->ev1));
    RLA_CUDA_TRY(ctx, cudaEventElapsedTime(ms, b->ev0, b->ev1));
    return RLA_OK;
}

// Autotuner: per rank class, the rows per CTA of A*Omega and the column block and row chunk
// of A'Q, chosen by timing the class's whole launch sequence on the actual problems.
static int autotune(rla_ctx *ctx, rla_batch *b) {
    for (int c = 0; c < B_NCLASS; ++c) {
        if (b->cls_h[c].empty()) continue;
        float best = 1e30f;
        int bbm = b->bm_ax[c], bbr = b->br_aq[c];
        int64_t bch = b->chunk_aq[c];
        for (int bm : {64, 128, 256}) {
            b->bm_ax[c] = bm;
            float ms;
            RLA_TRY(time_class(ctx, b, c, &ms));
            if (ms < best) { best = ms; bbm = bm; }
        }
        b->bm_ax[c] = bbm;
        for (int br : {64, 128, 256})
            for (int64_t ch : {2048, 8192, 32768}) {
                b->br_aq[c] = br;
                b->chunk_aq[c] = ch;
                float ms;
                RLA_TRY(time_class(ctx, b, c, &ms));
                if (ms < best) { best = ms; bbr = br; bch = ch; }
            }
        b->br_aq[c] = bbr;
        b->chunk_aq[c] = bch;
    }
    b->tuned = true;
    return RLA_OK;
}

static size_t part_bytes(const rla_batch *b, const BProb &p) {
    // largest of: Gram partials over m, A'Q partials over m (any tuned chunk), Gram over n
    size_t g = sizeof(double) * (size_t)ceil_div(p.m, b->chunk_m) * p.k * p.k;
    size_t a = sizeof(float) * (size_t)ceil_div(p.m, 2048) * p.n * p.k;
    size_t n = sizeof(double) * (size_t)ceil_div(p.n, b->chunk_n) * p.k * p.k;
    return std::max(g, std::max(a, n));
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_randsvd_batch_create(rla_ctx *ctx, int count, const rla_svd_problem *probs, const rla_range_params *params,
                             int flags, rla_batch **out) {
    if (!ctx) return RLA_E_ARG;
    if (!out || (count > 0 && !probs) || !params) return set_error(ctx, RLA_E_ARG, "NULL argument.");
    *out = nullptr;
    if (count < 0) return set_error(ctx, RLA_E_ARG, "Negative problem count.");
    if (params->power_its < 0) return set_error(ctx, RLA_E_ARG, "Field `power_its` must be non-negative.");
    for (int i = 0; i < count; ++i) {
        const rla_svd_problem &q = probs[i];
        if (q.m <= 0 || q.n <= 0 || q.k <= 0 || q.k > 128 || q.k > q.n || q.k > q.m)
            return set_error(ctx, RLA_E_ARG, "problem %d: need 0 < k <= min(m, n, 128)", i);
        if (!q.A || !q.U || !q.S || !q.V || q.lda < q.m || q.ldu < q.m || q.ldv < q.n)
            return set_error(ctx, RLA_E_ARG, "problem %d: bad buffer or leading dimension", i);
    }
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    rla_batch *b = new rla_batch();
    b->ctx = ctx;
    b->flags = flags;
    b->device = ctx->device;
    b->count = count;
    b->probs.assign(probs, probs + count);
    b->params = *params;
    b->h_probs.resize(count);
    size_t total = 0;
    auto add = [&](size_t bytes) {
        const size_t off = total;
        total += (bytes + 255) & ~size_t(255);
        return off;
    };
    std::vector<std::array<size_t, 12>> offs(count);
    for (int i = 0; i < count; ++i) {
        const rla_svd_problem &q = probs[i];
        BProb &p = b->h_probs[i];
        p.m = q.m; p.n = q.n; p.k = q.k;
        p.A = q.A; p.lda = q.lda; p.U = q.U; p.ldu = q.ldu; p.S = q.S; p.V = q.V; p.ldv = q.ldv; p.seed = q.seed;
        auto &o = offs[i];
        o[0] = add(sizeof(float) * q.n * q.k);   // Om
        o[1] = add(sizeof(float) * q.m * q.k);   // Y
        o[2] = add(params->power_its > 0 ? sizeof(float) * q.n * q.k : 16);  // Z
        o[3] = add(sizeof(double) * q.k * q.k);  // G
        o[4] = add(sizeof(double) * q.k * q.k);  // Rinv
        o[5] = add(sizeof(double) * q.n * q.k);  // Bt
        o[6] = add(sizeof(double) * q.n * q.k);  // Bt0
        o[7] = add(sizeof(double) * q.k * q.k);  // X
        o[8] = add(sizeof(double) * q.k * q.k);  // J
        o[9] = add(part_bytes(b, p));            // partials
        const bool tci = params->precision == RLA_PREC_SPLIT_BF16 && q.k <= 64;
        o[10] = add(tci ? sizeof(bf16) * 2 * (size_t)ceil_div(q.m, 8) * 8 * q.n : 16);                // A hi, lo
        o[11] = add(tci ? sizeof(bf16) * 2 * (size_t)ceil_div(std::max(q.m, q.n), 8) * 8 * q.k : 16);  // factor hi, lo
        b->cls_h[b_kclass(q.k)].push_back(i);
    }
    b->tc = params->precision == RLA_PREC_SPLIT_BF16;
    int rc = RLA_OK;
    auto fail = [&](int r) {
        rla_randsvd_batch_destroy(b);
        return r;
    };
    if (pool_malloc_s(ctx, &b->work, std::max<size_t>(total, 256), ctx->stream) != cudaSuccess)
        return fail(set_error(ctx, RLA_E_OOM, "batch workspace of %zu bytes", total));
    if (pool_malloc_s(ctx, &b->flagbuf, sizeof(int) * std::max(count, 1), ctx->stream) != cudaSuccess)
        return fail(set_error(ctx, RLA_E_OOM, "batch flags"));
    char *w = (char *)b->work;
    for (int i = 0; i < count; ++i) {
        BProb &p = b->h_probs[i];
        auto &o = offs[i];
        p.Om = (float *)(w + o[0]); p.Y = (float *)(w + o[1]); p.Z = (float *)(w + o[2]);
        p.G = (double *)(w + o[3]); p.Rinv = (double *)(w + o[4]); p.Bt = (double *)(w + o[5]);
        p.Bt0 = (double *)(w + o[6]); p.X = (double *)(w + o[7]); p.J = (double *)(w + o[8]);
        p.part = w + o[9];
        p.flag = b->flagbuf + i;
    }
    if (b->tc) {
        // grouped split and product tables per rank class (k <= 64), over fixed buffers
        for (int c = 0; c < B_NCLASS - 1; ++c) {
            if (b->cls_h[c].empty()) continue;
            std::vector<SplitSpec> sa, so, sy, sz;
            std::vector<TcGroupSpec> gx, gz, gb;
            for (int i : b->cls_h[c]) {
                const BProb &p = b->h_probs[i];
                const int64_t lda2 = ceil_div(p.m, 8) * 8, ldn = ceil_div(p.n, 8) * 8, ldm = ceil_div(p.m, 8) * 8;
                bf16 *ahi = (bf16 *)(w + offs[i][10]), *alo = ahi + lda2 * p.n;
                bf16 *bhi = (bf16 *)(w + offs[i][11]), *blo = bhi + ceil_div(std::max(p.m, p.n), 8) * 8 * p.k;
                sa.push_back(SplitSpec{p.A, p.m, p.n, p.lda, ahi, alo, lda2});
                so.push_back(SplitSpec{p.Om, p.n, p.k, p.n, bhi, blo, ldn});
                sy.push_back(SplitSpec{p.Y, p.m, p.k, p.m, bhi, blo, ldm});
                sz.push_back(SplitSpec{p.Z, p.n, p.k, p.n, bhi, blo, ldn});
                gx.push_back(TcGroupSpec{{ahi, alo}, lda2, 0, {bhi, blo}, ldn, p.m, p.k, p.n, p.Y, nullptr, p.m, 0});
                gz.push_back(TcGroupSpec{{ahi, alo}, lda2, 1, {bhi, blo}, ldm, p.n, p.k, p.m, p.Z, nullptr, p.n, 0});
                gb.push_back(TcGroupSpec{{ahi, alo}, lda2, 1, {bhi, blo}, ldm, p.n, p.k, p.m, p.Bt, p.Bt0, p.n, 1});
            }
            int r = split_group_build(ctx, sa, &b->s_a[c]);
            if (r == RLA_OK) r = split_group_build(ctx, so, &b->s_om[c]);
            if (r == RLA_OK) r = split_group_build(ctx, sy, &b->s_y[c]);
            if (r == RLA_OK && params->power_its > 0) r = split_group_build(ctx, sz, &b->s_z[c]);
            if (r == RLA_OK) r = tc_group_build(ctx, gx, &b->g_ax[c]);
            if (r == RLA_OK && params->power_its > 0) r = tc_group_build(ctx, gz, &b->g_atq_z[c]);
            if (r == RLA_OK) r = tc_group_build(ctx, gb, &b->g_atq_bt[c]);
            if (r != RLA_OK) return fail(r);
        }
    }
    if (pool_malloc_s(ctx, &b->d_probs, sizeof(BProb) * std::max(count, 1), ctx->stream) != cudaSuccess)
        return fail(set_error(ctx, RLA_E_OOM, "batch table"));
    if (count)
        cudaMemcpyAsync(b->d_probs, b->h_probs.data(), sizeof(BProb) * count, cudaMemcpyHostToDevice, ctx->stream);
    for (int c = 0; c < B_NCLASS; ++c) {
        if (b->cls_h[c].empty()) continue;
        if (pool_malloc_s(ctx, &b->cls_d[c], sizeof(int) * b->cls_h[c].size(), ctx->stream) != cudaSuccess)
            return fail(set_error(ctx, RLA_E_OOM, "batch class table"));
        cudaMemcpyAsync(b->cls_d[c], b->cls_h[c].data(), sizeof(int) * b->cls_h[c].size(), cudaMemcpyHostToDevice,
                        ctx->stream);
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(set_error(ctx, RLA_E_CUDA, "batch tables"));
    {
        const int lim = ctx->smem_optin - 1024;
        if (set_smem_max(b_chol_inv_kernel) != cudaSuccess ||
            set_smem_max(b_jacobi_kernel) != cudaSuccess)
            return fail(set_error(ctx, RLA_E_CUDA, "batch kernel attributes"));
    }
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(set_error(ctx, RLA_E_CUDA, "batch events"));
    for (int c = 0; c < B_NCLASS; ++c)
        if (cudaStreamCreateWithFlags(&b->side[c], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[c], cudaEventDisableTiming) != cudaSuccess)
            return fail(set_error(ctx, RLA_E_CUDA, "batch class streams"));
    if (!(flags & RLA_BATCH_EAGER) || (flags & RLA_BATCH_AUTOTUNE)) {
        if (cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
            return fail(set_error(ctx, RLA_E_CUDA, "batch stream/events"));
    }
    if (flags & RLA_BATCH_AUTOTUNE) {
        rc = autotune(ctx, b);
        if (rc != RLA_OK) return fail(rc);
    }
    *out = b;
    return RLA_OK;
}

int rla_randsvd_batch_tiles(const rla_batch *b, int cls, int *rows_a_omega, int *cols_at_q, int64_t *chunk_at_q) {
    if (!b || cls < 0 || cls >= B_NCLASS || !rows_a_omega || !cols_at_q || !chunk_at_q) return RLA_E_ARG;
    *rows_a_omega = b->bm_ax[cls];
    *cols_at_q = b->br_aq[cls];
    *chunk_at_q = b->chunk_aq[cls];
    return RLA_OK;
}

int rla_randsvd_batch_run(rla_ctx *ctx, rla_batch *b) {
    if (!ctx || !b) return RLA_E_ARG;
    if (b->device != ctx->device) return set_error(ctx, RLA_E_ARG, "Batch lives on device %d, context on %d.", b->device, ctx->device);
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    if (b->count == 0) return RLA_OK;
    if (b->flags & RLA_BATCH_EAGER) {
        RLA_CUDA_TRY(ctx, cudaMemsetAsync(b->flagbuf, 0, sizeof(int) * b->count, ctx->stream));
        RLA_TRY(enqueue_all(ctx, b, ctx->stream));
    } else {
    if (!b->exec) {
        // first run: capture the grouped launch sequence (prefix tables and attributes are
        // created outside the capture by a dry enqueue)
        RLA_TRY(enqueue_all(ctx, b, b->cs));
        RLA_CUDA_TRY(ctx, cudaStreamSynchronize(b->cs));
        RLA_CUDA_TRY(ctx, cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_all(ctx, b, b->cs);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->cs, &g);
        RLA_TRY(rc);
        if (e != cudaSuccess) return set_error(ctx, RLA_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
        b->graph = g;
        RLA_CUDA_TRY(ctx, cudaGraphInstantiate(&b->exec, g, 0));
    }
    RLA_CUDA_TRY(ctx, cudaMemsetAsync(b->flagbuf, 0, sizeof(int) * b->count, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaEventRecord(b->ev0, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(b->cs, b->ev0, 0));
    RLA_CUDA_TRY(ctx, cudaGraphLaunch(b->exec, b->cs));
    RLA_CUDA_TRY(ctx, cudaEventRecord(b->ev1, b->cs));
    RLA_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, b->ev1, 0));
    }
    // instances whose Cholesky broke down: the single-instance path (shifted CholeskyQR /
    // Householder fallback) recomputes them with the same draws
    std::vector<int> fl(b->count);
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(fl.data(), b->flagbuf, sizeof(int) * b->count, cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (b->tc) RLA_TRY(tc_status_check(ctx));
    for (int i = 0; i < b->count; ++i) {
        if (!fl[i]) continue;
        const rla_svd_problem &q = b->probs[i];
        rla_sketch_params sp{RLA_GAUSSIAN, RLA_RIGHT, RLA_F32, q.k, q.n, 0, 0, 0.0, q.seed};
        rla_sketch *om = nullptr;
        RLA_TRY(rla_sketch_create(ctx, &sp, &om));
        rla_range_params pr = b->params;
        pr.precision = RLA_PREC_NATIVE;
        const int rc = rla_randsvd(ctx, om, RLA_F32, q.m, q.n, q.A, q.lda, &pr, RLA_F32, q.U, q.ldu, q.S, q.V, q.ldv);
        rla_sketch_destroy(om);
        RLA_TRY(rc);
    }
    return RLA_OK;
}

int rla_randsvd_batch_destroy(rla_batch *b) {
    if (!b) return RLA_OK;
    cudaSetDevice(b->device);
    if (b->cs) cudaStreamSynchronize(b->cs);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->cs) cudaStreamDestroy(b->cs);
    for (int c = 0; c < B_NCLASS; ++c) {
        if (b->side[c]) {
            cudaStreamSynchronize(b->side[c]);
            cudaStreamDestroy(b->side[c]);
        }
        if (b->join[c]) cudaEventDestroy(b->join[c]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    for (int c = 0; c < B_NCLASS; ++c) {
        split_group_free(&b->s_a[c]);
        split_group_free(&b->s_om[c]);
        split_group_free(&b->s_y[c]);
        split_group_free(&b->s_z[c]);
        tc_group_free(&b->g_ax[c]);
        tc_group_free(&b->g_atq_z[c]);
        tc_group_free(&b->g_atq_bt[c]);
    }
    cudaStream_t st = b->ctx->stream;
    for (void *p : b->owned) cudaFreeAsync(p, st);
    for (int c = 0; c < B_NCLASS; ++c)
        if (b->cls_d[c]) cudaFreeAsync(b->cls_d[c], st);
    if (b->d_probs) cudaFreeAsync(b->d_probs, st);
    if (b->flagbuf) cudaFreeAsync(b->flagbuf, st);
    if (b->work) cudaFreeAsync(b->work, st);
    delete b;
    return RLA_OK;
}

int rla_randsvd_grouped(rla_ctx *ctx, int count, const rla_svd_problem *probs, const rla_range_params *params) {
    rla_batch *b = nullptr;
    RLA_TRY(rla_randsvd_batch_create(ctx, count, probs, params, 0, &b));
    const int rc = rla_randsvd_batch_run(ctx, b);
    if (rc == RLA_OK) cudaStreamSynchronize(ctx->stream);
    rla_randsvd_batch_destroy(b);
    return rc;
}

}  // extern "C"
