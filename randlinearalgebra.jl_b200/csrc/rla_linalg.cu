// rla_linalg.cu -- small dense FP64 kernels for CholeskyQR2 and the SVD of B = Q'A.
//
// The reference orthogonalises with Householder QR (power_its.jl:35,60,70,73) and calls
// LAPACK's svd (randsvd.jl:186).  Here the tall-skinny orthogonalisation is CholeskyQR2
// (Gram matrix, Cholesky and triangular solve in FP64), and the SVD of the small l x l
// triangular factor is a one-sided (Hestenes) Jacobi iteration in FP64.
#include <math.h>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Upper Cholesky factor, left-looking by rows of R: step j forms r_jj from column j of R
// and then row j, r_ji = (g_ji - R(0:j, j)' R(0:j, i)) / r_jj, one warp per column i with
// the dot product split over the lanes.  Column j of R is staged in shared memory.
__global__ void __launch_bounds__(1024) chol_upper_kernel(double *G, int64_t l, double shift, int *breakdown) {
    extern __shared__ double colj[];
    __shared__ double rjj_s;
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    if (tid == 0) bad = 0;
    for (int64_t i = tid; i < l; i += nt) G[i + i * l] += shift;
    __syncthreads();
    for (int64_t j = 0; j < l; ++j) {
        for (int64_t k = tid; k < j; k += nt) colj[k] = G[k + j * l];
        __syncthreads();
        if (warp == 0) {
            double d = 0.0;
            for (int64_t k = lane; k < j; k += 32) d += colj[k] * colj[k];
            d = warp_sum(d);
            if (lane == 0) {
                double v = G[j + j * l] - d;
                if (!(v > 0.0) || !isfinite(v)) {
                    bad = 1;
                    v = 1.0;
                }
                rjj_s = sqrt(v);
                G[j + j * l] = rjj_s;
            }
        }
        __syncthreads();
        const double rjj = rjj_s;
        // four columns per warp at a time, so their loads overlap
        for (int64_t i0 = j + 1 + 4 * warp; i0 < l; i0 += 4 * nwarps) {
            double d[4] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t k = lane; k < j; k += 32) {
                const double cj = colj[k];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (i0 + q < l) d[q] = fma(cj, G[k + (i0 + q) * l], d[q]);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) d[q] = warp_sum(d[q]);
            if (lane < 4 && i0 + lane < l) {
                const double dq = lane == 0 ? d[0] : lane == 1 ? d[1] : lane == 2 ? d[2] : d[3];
                G[j + (i0 + lane) * l] = (G[j + (i0 + lane) * l] - dq) / rjj;
            }
        }
        __syncthreads();
    }
    for (int64_t idx = tid; idx < l * l; idx += nt) {
        const int64_t r = idx % l, c = idx / l;
        if (r > c) G[idx] = 0.0;
    }
    if (tid == 0) *breakdown = bad;
}

// Blocked right-looking upper Cholesky in one CTA for l <= CB_MAXL.  Per panel of CB
// columns: (1) the diagonal block is factored by one warp in shared memory, (2) the panel's
// rows of R, R(p, p+CB:l) = R_pp^-T G(p, p+CB:l), by forward substitution with one thread
// per column (the column in registers), staged in shared memory, (3) the trailing upper
// triangle G(a, b) -= R(p, a)' R(p, b), one 4x4 block of entries per thread.
constexpr int CB = 32, CB_MAXL = 512, CB_THREADS = 512;

__global__ void __launch_bounds__(CB_THREADS) chol_blocked_kernel(double *G, int64_t l, double shift, int *breakdown,
                                                                  int ldp) {
    extern __shared__ double cb_sm[];
    double *D = cb_sm;             // CB x CB, column-major (ld CB)
    double *P = cb_sm + CB * CB;   // panel rows: P[c + t*ldp] = R(p+t, p+CB+c)
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) bad = 0;
    for (int64_t i = tid; i < l; i += nt) G[i + i * l] += shift;
    __syncthreads();
    for (int64_t p = 0; p < l; p += CB) {
        const int pb = (int)(l - p < CB ? l - p : CB);
        const int64_t c0 = p + pb, rest = l - c0;
        for (int e = tid; e < pb * pb; e += nt) {
            const int r = e % pb, c = e / pb;
            D[r + c * CB] = r <= c ? G[(p + r) + (p + c) * l] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int t = 0; t < pb; ++t) {
                double v = D[t + t * CB];
                if (!(v > 0.0) || !isfinite(v)) {
                    if (lane == 0) bad = 1;
                    v = 1.0;
                }
                const double piv = sqrt(v);
                __syncwarp();
                if (lane == t) D[t + t * CB] = piv;
                if (lane > t && lane < pb) D[t + lane * CB] /= piv;
                __syncwarp();
                if (lane > t && lane < pb)
                    for (int a = t + 1; a <= lane; ++a) D[a + lane * CB] -= D[t + a * CB] * D[t + lane * CB];
                __syncwarp();
            }
        }
        __syncthreads();
        for (int e = tid; e < pb * pb; e += nt) {
            const int r = e % pb, c = e / pb;
            if (r <= c) G[(p + r) + (p + c) * l] = D[r + c * CB];
        }
        for (int64_t c = tid; c < rest; c += nt) {
            double y[CB];
#pragma unroll
            for (int t = 0; t < CB; ++t) y[t] = t < pb ? G[(p + t) + (c0 + c) * l] : 0.0;
#pragma unroll
            for (int t = 0; t < CB; ++t) {
                if (t < pb) {
                    double acc = y[t];
#pragma unroll
                    for (int q = 0; q < t; ++q) acc -= D[q + t * CB] * y[q];
                    y[t] = acc / D[t + t * CB];
                }
            }
#pragma unroll
            for (int t = 0; t < CB; ++t)
                if (t < pb) {
                    G[(p + t) + (c0 + c) * l] = y[t];
                    P[c + (int64_t)t * ldp] = y[t];
                }
        }
        __syncthreads();
        const int nb = (int)((rest + 3) / 4);
        for (int blk = tid; blk < nb * nb; blk += nt) {
            const int ia = blk % nb, ib = blk / nb;
            if (ia > ib) continue;
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            for (int t = 0; t < pb; ++t) {
                const double *pt = P + (int64_t)t * ldp;
                const double2 a01 = *reinterpret_cast<const double2 *>(pt + 4 * ia);
                const double2 a23 = *reinterpret_cast<const double2 *>(pt + 4 * ia + 2);
                const double2 b01 = *reinterpret_cast<const double2 *>(pt + 4 * ib);
                const double2 b23 = *reinterpret_cast<const double2 *>(pt + 4 * ib + 2);
                const double a[4] = {a01.x, a01.y, a23.x, a23.y}, b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t a = 4 * ia + i, b = 4 * ib + j;
                    if (a <= b && b < rest) G[(c0 + a) + (c0 + b) * l] -= acc[i][j];
                }
        }
        __syncthreads();
    }
    for (int64_t idx = tid; idx < l * l; idx += nt) {
        const int64_t r = idx % l, c = idx / l;
        if (r > c) G[idx] = 0.0;
    }
    if (tid == 0) *breakdown = bad;
}

// Column j of R^-1 (R upper triangular, l x l, ld l) by back substitution in column form:
// x = e_j; for i = j .. 0: x_i *= 1/R_ii, then x_r -= x_i R_ri for r < i.  Each step reads
// column i of R (contiguous), one warp per column of the inverse (wpc warps per CTA), x and
// the reciprocal diagonal in shared memory.  Used for orders too large for the staged
// variant below.
__global__ void __launch_bounds__(256) tri_inv_upper_kernel(const double *R, int64_t l, double *Ri, int wpc) {
    extern __shared__ double xs_all[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *dinv = xs_all + (int64_t)wpc * l;
    for (int64_t i = threadIdx.x; i < l; i += blockDim.x) dinv[i] = 1.0 / R[i + i * l];
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * wpc + wib;
    if (j >= l) return;
    double *x = xs_all + (int64_t)wib * l;
    for (int64_t i = lane; i <= j; i += 32) x[i] = i == j ? 1.0 : 0.0;
    __syncwarp();
    for (int64_t i = j; i >= 0; --i) {
        const double xi = x[i] * dinv[i];
        __syncwarp();
        if (lane == 0) x[i] = xi;
        const double *ri = R + i * l;
        for (int64_t r = lane; r < i; r += 32) x[r] = fma(-xi, ri[r], x[r]);
        __syncwarp();
    }
    double *out = Ri + j * l;
    for (int64_t i = lane; i < l; i += 32) out[i] = i <= j ? x[i] : 0.0;
}


// The same back substitution with the columns of R staged in shared memory: the warps of a
// CTA take consecutive columns j of the inverse and walk i together, so column i of R is read
// from global memory once per CTA, TI_CH columns at a time by cp.async into one half of a
// two-chunk ring while the warps work on the other half (two barriers per chunk instead of
// an L2 round trip per step).
constexpr int TI_WARPS = 8, TI_CH = 16;

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(TI_WARPS * 32) tri_inv_ring_kernel(const double *R, int64_t l, double *Ri) {
    extern __shared__ __align__(16) double ti_sm[];
    const int li = (int)l;
    double *ring = ti_sm;                  // [2][TI_CH][l]: column q of a chunk at q*l
    double *xs = ring + 2 * TI_CH * li;    // [TI_WARPS][l]: the warps' columns x
    double *dinv = xs + TI_WARPS * li;     // [l]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j0 = blockIdx.x * TI_WARPS, j = j0 + warp;
    const int j_hi = min(li, j0 + TI_WARPS) - 1, c_hi = j_hi / TI_CH;
    // chunk c (columns c*TI_CH .. c*TI_CH + TI_CH - 1, rows above the diagonal) into half h
    auto issue = [&](int c, int h) {
        if (c >= 0) {
            double *dst = ring + h * TI_CH * li;
            for (int q = 0; q < TI_CH; ++q) {
                const int i = c * TI_CH + q;
                if (i > j_hi) break;
                for (int r = tid; r < i; r += TI_WARPS * 32) cp_async8(dst + q * li + r, R + r + (int64_t)i * l);
            }
        }
        cp_async_commit();
    };
    issue(c_hi, 0);
    issue(c_hi - 1, 1);
    for (int i = tid; i <= j_hi; i += TI_WARPS * 32) dinv[i] = 1.0 / R[i + (int64_t)i * l];
    double *x = xs + warp * li;
    if (j < li)
        for (int r = lane; r <= j; r += 32) x[r] = r == j ? 1.0 : 0.0;
    for (int k = 0, c = c_hi; c >= 0; ++k, --c) {
        cp_async_wait<1>();  // every chunk but the newest has landed
        __syncthreads();
        const double *cols = ring + (k & 1) * TI_CH * li;
        if (j < li) {
            for (int q = TI_CH - 1; q >= 0; --q) {
                const int i = c * TI_CH + q;
                if (i > j) continue;
                const double xi = x[i] * dinv[i];
                __syncwarp();
                if (lane == 0) x[i] = xi;
                const double *ci = cols + q * li;
                for (int r = lane; r < i; r += 32) x[r] = fma(-xi, ci[r], x[r]);
                __syncwarp();
            }
        }
        __syncthreads();      // every warp is done with half (k & 1)
        issue(c - 2, k & 1);  // chunk k + 2 takes its place
    }
    cp_async_wait<0>();
    if (j < li) {
        double *out = Ri + (int64_t)j * l;
        for (int r = lane; r < li; r += 32) out[r] = r <= j ? x[r] : 0.0;
    }
}

// Circle-method pairing: round r (0..n2-2), pair p (0..n2/2-1) over players 0..n2-1.
__device__ inline void tourney_pair(int r, int p, int n2, int *i, int *j) {
    const int m = n2 - 1;
    if (p == 0) {
        *i = r % m;
        *j = m;
    } else {
        *i = (r + p) % m;
        *j = (r - p + m) % m;
    }
}

__global__ void __launch_bounds__(1024) jacobi_kernel(double *X, double *J, double *sigma, int64_t l, double *work,
                                                      int max_sweeps, double tol) {
    __shared__ unsigned long long off_bits;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    for (int64_t idx = tid; idx < l * l; idx += nt) J[idx] = (idx % l == idx / l) ? 1.0 : 0.0;
    __syncthreads();
    const int n2 = (int)(l + (l & 1));
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        if (tid == 0) off_bits = 0ull;
        __syncthreads();
        for (int r = 0; r < n2 - 1; ++r) {
            for (int p = warp; p < n2 / 2; p += nwarps) {
                int i, j;
                tourney_pair(r, p, n2, &i, &j);
                if (i >= l || j >= l) continue;
                if (i > j) {
                    int t = i;
                    i = j;
                    j = t;
                }
                double *xi = X + (int64_t)i * l, *xj = X + (int64_t)j * l;
                double a = 0, b = 0, g = 0;
                for (int64_t k = lane; k < l; k += 32) {
                    const double u = xi[k], w = xj[k];
                    a += u * u;
                    b += w * w;
                    g += u * w;
                }
                a = warp_sum(a);
                b = warp_sum(b);
                g = warp_sum(g);
                const double nrm = sqrt(a * b);
                if (g != 0.0 && fabs(g) > tol * nrm) {
                    const double off = fabs(g) / nrm;
                    if (lane == 0) atomicMax(&off_bits, (unsigned long long)__double_as_longlong(off));
                    const double zeta = (b - a) / (2.0 * g);
                    const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                    double *ji = J + (int64_t)i * l, *jj = J + (int64_t)j * l;
                    for (int64_t k = lane; k < l; k += 32) {
                        const double u = xi[k], w = xj[k];
                        xi[k] = c * u - s * w;
                        xj[k] = s * u + c * w;
                        const double uj = ji[k], wj = jj[k];
                        ji[k] = c * uj - s * wj;
                        jj[k] = s * uj + c * wj;
                    }
                }
            }
            __syncthreads();
        }
        if (__longlong_as_double((long long)off_bits) <= tol) break;
        __syncthreads();
    }
    __syncthreads();
}

// Column norms -> sigma, columns sorted by descending sigma (stable), X normalised, J
// permuted alongside.  work: 2*l*l + 2*l doubles.  jacobi_rank_kernel (one CTA) forms the
// norms and the permutation -- the rank of column c is the number of columns with a larger
// norm plus the earlier ones with an equal norm (NaN norms sort last) -- and
// jacobi_permute_kernel (one CTA per output column) writes the permuted columns to work.
__global__ void __launch_bounds__(1024) jacobi_rank_kernel(const double *X, double *sigma, int64_t l, double *work) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    double *sg = work + 2 * l * l;
    int *perm = reinterpret_cast<int *>(work + 2 * l * l + l);
    for (int c = warp; c < l; c += nwarps) {
        const double *xc = X + (int64_t)c * l;
        double a = 0;
        for (int64_t k = lane; k < l; k += 32) a += xc[k] * xc[k];
        a = warp_sum(a);
        if (lane == 0) sg[c] = sqrt(a);
    }
    __syncthreads();
    for (int64_t c = tid; c < l; c += nt) {
        const double v = sg[c], kv = isnan(v) ? -1.0 : v;
        int64_t rank = 0;
        for (int64_t d = 0; d < l; ++d) {
            const double w = sg[d], kw = isnan(w) ? -1.0 : w;
            rank += (kw > kv) || (kw == kv && d < c);
        }
        perm[rank] = (int)c;
        sigma[rank] = v;
    }
}

__global__ void __launch_bounds__(256) jacobi_permute_kernel(const double *X, const double *J, int64_t l,
                                                             double *work) {
    const double *sg = work + 2 * l * l;
    const int *perm = reinterpret_cast<const int *>(work + 2 * l * l + l);
    double *Xt = work, *Jt = work + l * l;
    const int64_t c = blockIdx.x;
    const int src = perm[c];
    const double sv = sg[src];
    for (int64_t r = threadIdx.x; r < l; r += blockDim.x) {
        Xt[r + c * l] = sv > 0.0 ? X[r + (int64_t)src * l] / sv : 0.0;
        Jt[r + c * l] = J[r + (int64_t)src * l];
    }
}


// ---- block one-sided Jacobi -------------------------------------------------------------
// Columns in blocks of BJ_B; an outer round pairs blocks (circle method) and each CTA takes
// one pair: it stages the pair's columns of X and J in shared memory (row stride rounded up
// to an even count, zero padded, so the column loops run on 16-byte vectors), runs inner
// one-sided (Hestenes) sweeps over them (one warp per column pair, circle-method rounds)
// until they are mutually orthogonal to `tol` or BJ_INNER sweeps, and writes them back.
// Small blocks spread each outer round over many SMs: the rotations of a sweep are the same
// work whatever the blocking, and a pair's inner rounds are bound by the latency of one
// warp's rotation.  The largest relative off-diagonal seen in a CTA's first inner sweep goes
// to *off (max over the outer sweep), which the host reads to stop.
constexpr int BJ_B = 8, BJ_INNER = 1, BJ_THREADS = 32 * BJ_B;

__global__ void jacobi_identity_kernel(double *J, int64_t l) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx < l * l) J[idx] = (idx % l == idx / l) ? 1.0 : 0.0;
}

__global__ void __launch_bounds__(BJ_THREADS) block_jacobi_round_kernel(double *X, double *J, int64_t l, int nbp,
                                                                        int round, double tol,
                                                                        unsigned long long *off) {
    extern __shared__ __align__(16) double bj_smem[];
    __shared__ unsigned long long inner_off;
    __shared__ int cols[2 * BJ_B];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = BJ_THREADS / 32;
    const int li = (int)l, ls = (li + 1) & ~1;  // padded column stride
    const int nb = (li + BJ_B - 1) / BJ_B;
    int bi, bj;
    tourney_pair(round, blockIdx.x, nbp, &bi, &bj);
    int c = 0;
    for (int q = 0; q < 2; ++q) {
        const int blk = q == 0 ? bi : bj;
        if (blk >= nb) continue;
        const int c0 = blk * BJ_B, c1 = min(li, c0 + BJ_B);
        for (int cc = c0; cc < c1; ++cc) {
            if (tid == 0) cols[c] = cc;
            ++c;
        }
    }
    __syncthreads();
    if (c < 2) return;
    double *Xs = bj_smem, *Js = bj_smem + 2 * BJ_B * ls;
    for (int idx = tid; idx < c * ls; idx += BJ_THREADS) {
        const int q = idx / ls, r = idx - q * ls;
        const int64_t g = r + (int64_t)cols[q] * l;
        Xs[idx] = r < li ? X[g] : 0.0;
        Js[idx] = r < li ? J[g] : 0.0;
    }
    __syncthreads();
    const int cp = c + (c & 1);
    for (int sweep = 0; sweep < BJ_INNER; ++sweep) {
        if (tid == 0) inner_off = 0ull;
        __syncthreads();
        for (int r = 0; r < cp - 1; ++r) {
            for (int p = warp; p < cp / 2; p += nwarps) {
                int i, j;
                tourney_pair(r, p, cp, &i, &j);
                if (i >= c || j >= c) continue;
                if (i > j) {
                    const int t = i;
                    i = j;
                    j = t;
                }
                double2 *xi = reinterpret_cast<double2 *>(Xs + i * ls), *xj = reinterpret_cast<double2 *>(Xs + j * ls);
                double a = 0, b = 0, g = 0;
                for (int k = lane; k < ls / 2; k += 32) {
                    const double2 u = xi[k], w = xj[k];
                    a = fma(u.x, u.x, fma(u.y, u.y, a));
                    b = fma(w.x, w.x, fma(w.y, w.y, b));
                    g = fma(u.x, w.x, fma(u.y, w.y, g));
                }
                a = warp_sum(a);
                b = warp_sum(b);
                g = warp_sum(g);
                const double nrm = sqrt(a * b);
                if (g != 0.0 && fabs(g) > tol * nrm) {
                    if (lane == 0) atomicMax(&inner_off, (unsigned long long)__double_as_longlong(fabs(g) / nrm));
                    const double zeta = (b - a) / (2.0 * g);
                    const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                    double2 *ji = reinterpret_cast<double2 *>(Js + i * ls), *jj = reinterpret_cast<double2 *>(Js + j * ls);
                    for (int k = lane; k < ls / 2; k += 32) {
                        const double2 u = xi[k], w = xj[k];
                        xi[k] = make_double2(cs * u.x - sn * w.x, cs * u.y - sn * w.y);
                        xj[k] = make_double2(sn * u.x + cs * w.x, sn * u.y + cs * w.y);
                        const double2 uj = ji[k], wj = jj[k];
                        ji[k] = make_double2(cs * uj.x - sn * wj.x, cs * uj.y - sn * wj.y);
                        jj[k] = make_double2(sn * uj.x + cs * wj.x, sn * uj.y + cs * wj.y);
                    }
                }
            }
            __syncthreads();
        }
        if (sweep == 0 && tid == 0 && inner_off) atomicMax(off, inner_off);
        const bool done = __longlong_as_double((long long)inner_off) <= tol;
        __syncthreads();
        if (done) break;
    }
    for (int idx = tid; idx < c * ls; idx += BJ_THREADS) {
        const int q = idx / ls, r = idx - q * ls;
        if (r >= li) continue;
        const int64_t g = r + (int64_t)cols[q] * l;
        X[g] = Xs[idx];
        J[g] = Js[idx];
    }
}

// Gram-based variant of the pair step (Float32 data, stopping tolerance >= 1e-13).  The CTA
// forms the FP64 Gram matrix G = Xp'Xp of the pair's 16 columns on the FP64 tensor cores
// (mma.m8n8k4.f64), measures the relative off-diagonal on it (fresh dot products of the
// actual columns), runs the pair's rotations on G itself -- a rotation costs O(16) operations
// on G instead of O(l) on the columns -- accumulates V = prod R, and applies V to the columns
// of X and J once (Xp <- Xp V, Jp <- Jp V, again on the tensor cores).  The next visit
// recomputes G from the columns, so rounding in the updated G does not accumulate.
//
// Ordering: every pair of columns is rotated once per sweep.  The 64 cross pairs of the two
// blocks (a, 8 + (a + r) mod 8), r = 0..7, are done at the visit of the two blocks; the pairs
// inside a block (circle method, 7 rounds) are done in outer round 0, where every block is
// visited once.  An inner round applies 8 disjoint rotations, G <- R'GR and V <- VR, with one
// thread per entry of G and V and one barrier.
constexpr int BJX_THREADS = 256;  // 16 x 16: thread (x, y) owns G(x, y) and V(x, y)

__device__ __forceinline__ void dmma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Partner of index x (0..15) in inner round r: inside each 8-index half by the circle method
// (intra), or across the halves, pairs (a, 8 + (a + r) mod 8).
__device__ __forceinline__ int bjx_partner(int x, int r, bool intra) {
    if (intra) {
        const int u = x & 7, r7 = r % 7;
        const int p = u == 7 ? r7 : (u == r7 ? 7 : (2 * r7 - u + 14) % 7);
        return (x & 8) | p;
    }
    return x < 8 ? 8 + ((x + r) & 7) : ((x - 8 - r) & 7);
}

// Rotation R = [cs sn; -sn cs] on columns (i, j) that makes them orthogonal, from their Gram
// entries a = |x_i|^2, b = |x_j|^2, g = x_i'x_j: the smaller angle, tan = sign(b - a) 2g /
// (|b - a| + h) with h = sqrt((b - a)^2 + 4g^2).  With w = h + |b - a| and r = 1/sqrt(2hw):
// cs = w r and sn = sign(b - a) 2g r (cs^2 + sn^2 = (w^2 + 4g^2) / (2hw) = 1), two reciprocal
// square roots and no division.  No overflow for Gram entries of Float32 data.  Identity when
// g^2 <= tol^2 a b.
__device__ __forceinline__ bool bjx_rot(double a, double b, double g, double tol, double &cs, double &sn) {
    if (g == 0.0 || g * g <= tol * tol * a * b) {
        cs = 1.0;
        sn = 0.0;
        return false;
    }
    const double d = b - a, q = fma(d, d, 4.0 * g * g);
    const double h = q * rsqrt(q), w = h + fabs(d);
    const double r = rsqrt(2.0 * h * w);
    cs = w * r;
    sn = (d >= 0.0 ? 2.0 * g : -2.0 * g) * r;
    return true;
}

__global__ void __launch_bounds__(BJX_THREADS) block_jacobi_gram_round_kernel(double *X, double *J, int64_t l, int nbp,
                                                                              int round, double tol,
                                                                              unsigned long long *off) {
    extern __shared__ __align__(16) double bj_smem[];
    __shared__ double G[2][16][17], V[2][16][17];  // ping-pong across inner rounds
    __shared__ double part[8][3][64];              // per-warp partial Gram tiles
    __shared__ double wmax[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int li = (int)l, kp = (li + 31) & ~31, ls = kp + 4;  // ls = 4 mod 16: conflict-free fragments
    const int nb = (li + BJ_B - 1) / BJ_B;
    int bi, bj;
    tourney_pair(round, blockIdx.x, nbp, &bi, &bj);
    const bool vi = bi < nb, vj = bj < nb;
    if ((!vi && !vj) || (round > 0 && !(vi && vj))) return;  // nothing to rotate in this visit
    auto col_of = [&](int s) -> int {
        const int blk = s < 8 ? bi : bj, c = blk * BJ_B + (s & 7);
        return (blk < nb && c < li) ? c : -1;
    };
    double *Xs = bj_smem, *Js = bj_smem + 16 * ls;
    int cs_[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) cs_[s] = col_of(s);
    // all 32 loads of a row in flight before the shared stores (a store between two loads
    // would order them: one L2 round trip per element)
    for (int r0 = 0; r0 < kp; r0 += BJX_THREADS) {
        const int r = r0 + tid;
        double vx[16], vj[16];
#pragma unroll
        for (int s = 0; s < 16; ++s) {
            const bool in = cs_[s] >= 0 && r < li;
            vx[s] = in ? X[r + (int64_t)cs_[s] * l] : 0.0;
            vj[s] = in ? J[r + (int64_t)cs_[s] * l] : 0.0;
        }
        if (r < kp) {
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                Xs[s * ls + r] = vx[s];
                Js[s * ls + r] = vj[s];
            }
        }
    }
    __syncthreads();
    // G = Xp'Xp: warp w sums rows [w kp/8, (w+1) kp/8); the fragment of columns 0..7 (8..15)
    // serves as both the A operand (Xp') and the B operand (Xp).
    {
        double acc[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        const int k_lo = warp * (kp / 8), k_hi = k_lo + kp / 8;
        for (int k0 = k_lo; k0 < k_hi; k0 += 4) {
            const int kk = k0 + (lane & 3);
            const double f0 = Xs[(lane >> 2) * ls + kk], f1 = Xs[(8 + (lane >> 2)) * ls + kk];
            dmma_f64(acc[0], f0, f0);
            dmma_f64(acc[1], f0, f1);
            dmma_f64(acc[2], f1, f1);
        }
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            part[warp][t][(lane >> 2) * 8 + 2 * (lane & 3)] = acc[t][0];
            part[warp][t][(lane >> 2) * 8 + 2 * (lane & 3) + 1] = acc[t][1];
        }
    }
    __syncthreads();
    if (tid < 192) {
        const int t = tid >> 6, e = tid & 63, r = e >> 3, c = e & 7;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) s += part[w][t][e];
        if (t == 0) {
            G[0][r][c] = s;
        } else if (t == 1) {
            G[0][r][8 + c] = s;
            G[0][8 + c][r] = s;
        } else {
            G[0][8 + r][8 + c] = s;
        }
    }
    const int x = tid >> 4, y = tid & 15;
    V[0][x][y] = x == y ? 1.0 : 0.0;
    __syncthreads();
    // largest relative off-diagonal (squared) over the pairs this visit rotates
    {
        double m2 = 0.0;
        if (x < y && (round == 0 || (x < 8 && y >= 8))) {
            const double a = G[0][x][x], b = G[0][y][y], g = G[0][x][y];
            if (g != 0.0 && a * b > 0.0) m2 = g * g / (a * b);
        }
        for (int o = 16; o > 0; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(FULL, m2, o));
        if (lane == 0) wmax[warp] = m2;
    }
    int cur = 0;
    bool rotated = false;  // block-uniform: every warp computes the same rotations
    const int n_intra = round == 0 ? 7 : 0, n_in = n_intra + ((vi && vj) ? 8 : 0);
    for (int r = 0; r < n_in; ++r) {
        const bool intra = r < n_intra;
        const int rr = intra ? r : r - n_intra;
        // lanes 0..15 of every warp: the rotation of the pair holding index `lane`, as the
        // diagonal entry e and the partner's coefficient f of that column of R
        double e = 1.0, f = 0.0;
        if (lane < 16) {
            const int p = bjx_partner(lane, rr, intra), i = min(lane, p), j = max(lane, p);
            double cs, sn;
            if (bjx_rot(G[cur][i][i], G[cur][j][j], G[cur][i][j], tol, cs, sn)) {
                e = cs;
                f = lane == i ? -sn : sn;
            }
        }
        // a round that rotates no pair leaves G and V as they are
        if (!__any_sync(FULL, f != 0.0)) continue;
        rotated = true;
        const double ex = __shfl_sync(FULL, e, x), fx = __shfl_sync(FULL, f, x);
        const double ey = __shfl_sync(FULL, e, y), fy = __shfl_sync(FULL, f, y);
        const int xp = bjx_partner(x, rr, intra), yp = bjx_partner(y, rr, intra);
        // (R'GR)(x, y), summed as (t1 + t4) + (t2 + t3) so that (y, x) rounds identically
        const double t1 = (ex * ey) * G[cur][x][y], t4 = (fx * fy) * G[cur][xp][yp];
        const double t2 = (ex * fy) * G[cur][x][yp], t3 = (fx * ey) * G[cur][xp][y];
        G[cur ^ 1][x][y] = (t1 + t4) + (t2 + t3);
        V[cur ^ 1][x][y] = ey * V[cur][x][y] + fy * V[cur][x][yp];
        cur ^= 1;
        __syncthreads();
    }
    __syncthreads();  // wmax (also when no round ran its barrier)
    if (tid == 0) {
        double m2 = 0.0;
        for (int w = 0; w < 8; ++w) m2 = fmax(m2, wmax[w]);
        if (m2 > 0.0) atomicMax(off, (unsigned long long)__double_as_longlong(sqrt(m2)));
    }
    if (!rotated) return;  // V = I: the columns of X and J are unchanged
    // Xp <- Xp V, Jp <- Jp V: 8-row tiles round-robin over the warps, k = the 16 columns
    double vb[4][2];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) vb[ks][nt] = V[cur][4 * ks + (lane & 3)][8 * nt + (lane >> 2)];
    const int nmt = (li + 7) >> 3;
    for (int mt = warp; mt < nmt; mt += 8) {
        const int row = 8 * mt + (lane >> 2);
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const double *S = w ? Js : Xs;
            double *D = w ? J : X;
            double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const double a = S[(4 * ks + (lane & 3)) * ls + 8 * mt + (lane >> 2)];
                dmma_f64(acc[0], a, vb[ks][0]);
                dmma_f64(acc[1], a, vb[ks][1]);
            }
            if (row < li) {
#pragma unroll
                for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int c = col_of(8 * nt + 2 * (lane & 3) + q);
                        if (c >= 0) D[row + (int64_t)c * l] = acc[nt][q];
                    }
            }
        }
    }
}


// ---- Householder QR with LAPACK's conventions (dgeqr2 + dlarfg + dorg2r) --------------
// Used when CholeskyQR breaks down (numerically rank-deficient blocks, e.g. a compression
// dimension above rank(A)); the explicit Q it forms has LAPACK's column signs.
__device__ inline double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = threadIdx.x < nw ? red[threadIdx.x] : 0.0;
    if (warp == 0) t = warp_sum(t);
    if (threadIdx.x == 0) red[0] = t;
    __syncthreads();
    return red[0];
}

// dlarfg on column k of Y: v stored below the diagonal, beta on the diagonal.
template <class T>
__global__ void __launch_bounds__(1024) house_reflector_kernel(T *Y, int64_t m, int64_t ldy, int64_t k, double *tau) {
    __shared__ double red[32];
    T *col = Y + k * ldy;
    double ss = 0.0;
    for (int64_t i = k + 1 + threadIdx.x; i < m; i += blockDim.x) {
        const double x = (double)col[i];
        ss += x * x;
    }
    ss = block_sum(ss, red);
    const double alpha = (double)col[k];
    if (ss == 0.0) {
        if (threadIdx.x == 0) tau[k] = 0.0;
        return;
    }
    const double beta = -copysign(sqrt(alpha * alpha + ss), alpha);
    const double sc = 1.0 / (alpha - beta);
    for (int64_t i = k + 1 + threadIdx.x; i < m; i += blockDim.x) col[i] = (T)((double)col[i] * sc);
    if (threadIdx.x == 0) {
        tau[k] = (beta - alpha) / beta;
        col[k] = (T)beta;
    }
}

// Apply H = I - tau v v' (v_k = 1, v below the diagonal of column k of V) to columns
// j0.. of X from the left, rows k..m-1.  One block per column.
template <class T>
__global__ void __launch_bounds__(1024) house_apply_kernel(const T *V, T *X, int64_t m, int64_t ld, int64_t k,
                                                           int64_t j0, const double *tau) {
    __shared__ double red[32];
    const double t = tau[k];
    if (t == 0.0) return;
    const int64_t j = j0 + blockIdx.x;
    const T *v = V + k * ld;
    T *x = X + j * ld;
    double w = 0.0;
    for (int64_t i = k + threadIdx.x; i < m; i += blockDim.x) w += (i == k ? 1.0 : (double)v[i]) * (double)x[i];
    w = block_sum(w, red) * t;
    for (int64_t i = k + threadIdx.x; i < m; i += blockDim.x) x[i] = (T)((double)x[i] - w * (i == k ? 1.0 : (double)v[i]));
}

// dorg2r step for column i (after H(i) was applied to the columns to its right).
template <class T>
__global__ void house_form_col_kernel(T *Y, int64_t m, int64_t ld, int64_t i, const double *tau) {
    const double t = tau[i];
    T *col = Y + i * ld;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
        if (r < i) col[r] = T(0);
        else if (r == i) col[r] = (T)(1.0 - t);
        else col[r] = (T)(-t * (double)col[r]);
    }
}

template <class T>
int householder_q(rla_ctx *ctx, T *Y, int64_t m, int64_t l, int64_t ldy, double *tau) {
    for (int64_t k = 0; k < l; ++k) {
        house_reflector_kernel<T><<<1, 1024, 0, ctx->stream>>>(Y, m, ldy, k, tau);
        if (k + 1 < l) house_apply_kernel<T><<<(unsigned)(l - k - 1), 1024, 0, ctx->stream>>>(Y, Y, m, ldy, k, k + 1, tau);
    }
    RLA_TRY(check_launch(ctx, "householder_qr"));
    for (int64_t i = l - 1; i >= 0; --i) {
        if (i + 1 < l) house_apply_kernel<T><<<(unsigned)(l - i - 1), 1024, 0, ctx->stream>>>(Y, Y, m, ldy, i, i + 1, tau);
        house_form_col_kernel<T><<<ceil_div_i(m, 256) < 1024 ? ceil_div_i(m, 256) : 1024, 256, 0, ctx->stream>>>(Y, m, ldy, i, tau);
    }
    return check_launch(ctx, "householder_org2r");
}

template int householder_q<float>(rla_ctx *, float *, int64_t, int64_t, int64_t, double *);
template int householder_q<double>(rla_ctx *, double *, int64_t, int64_t, int64_t, double *);

// ---- blocked right-looking Cholesky over several CTAs (l >= MC_MIN) ------------------------
// Panel step p (MB columns): chol_panel_kernel factors the diagonal block in every CTA
// (redundantly; CTA 0 writes it back) and solves R_pp' X = G(p:p+pb, cols) for the CTA's
// 256 columns of the panel rows (one thread per column), zeroing the mirrored lower entries
// G(cols, p:p+pb); chol_syrk_kernel then updates the trailing upper triangle,
// G(I, J) -= R(p, I)' R(p, J), in 64 x 64 tiles (I <= J) spread over the GPU.
constexpr int MB = 64, MC_MIN = 33, MP_THREADS = 256;

// Upper Cholesky of the diagonal block G(p:p+pb, p:p+pb) (+ shift on its diagonal) into R
// (shared, ld MB+2, rows t < pb, zero below the diagonal) and rinv[t] = 1/R(t,t).  The 256
// threads form a 16 x 16 grid; thread (ty, tx) keeps the block's entries (4ty+i, 4tx+j) in
// registers.  Step t: the owners of row t publish it in a double-buffered shared row, then
// every thread applies the rank-1 update to its entries -- one barrier per step.
__device__ void chol_diag_block(const double *G, int64_t l, int64_t p, int pb, double shift, double (*R)[MB + 2],
                                double *rinv, double *rowbuf, int *bad) {
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    double d[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = 4 * ty + i, c = 4 * tx + j;
            double v = 0.0;
            if (r < pb && c < pb && r <= c) v = G[(p + r) + (p + c) * l] + (r == c ? shift : 0.0);
            d[i][j] = v;
        }
    for (int t = 0; t < pb; ++t) {
        double *buf = rowbuf + (t & 1) * MB;
        if (ty == (t >> 2)) {
            const int i = t & 3;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                buf[4 * tx + j] = i == 0 ? d[0][j] : i == 1 ? d[1][j] : i == 2 ? d[2][j] : d[3][j];
        }
        __syncthreads();
        double v = buf[t];
        if (!(v > 0.0) || !isfinite(v)) {
            if (tid == 0) *bad = 1;
            v = 1.0;
        }
        const double rp = rsqrt(v), piv = v * rp, rp2 = rp * rp;
        if (tid < MB) {
            const int c = tid;
            if (c >= t && c < pb) R[t][c] = c == t ? piv : buf[c] * rp;
            if (c == t) rinv[t] = rp;
        }
        double ba[4], bc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ba[q] = buf[4 * ty + q] * rp2;
            bc[q] = buf[4 * tx + q];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int a = 4 * ty + i, c = 4 * tx + j;
                if (t < a && a <= c) d[i][j] -= ba[i] * bc[j];
            }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(MP_THREADS) chol_panel_kernel(double *G, int64_t l, int64_t p, double shift,
                                                                int *breakdown) {
    extern __shared__ double mc_sm[];
    double(*R)[MB + 2] = reinterpret_cast<double(*)[MB + 2]>(mc_sm);
    double *rinv = mc_sm + MB * (MB + 2);
    double *rowbuf = rinv + MB;
    __shared__ int bad;
    const int tid = threadIdx.x;
    const int pb = (int)min((int64_t)MB, l - p);
    if (tid == 0) bad = 0;
    for (int e = tid; e < MB * (MB + 2); e += blockDim.x) (&R[0][0])[e] = 0.0;
    __syncthreads();
    chol_diag_block(G, l, p, pb, shift, R, rinv, rowbuf, &bad);
    if (blockIdx.x == 0) {
        for (int e = tid; e < pb * pb; e += blockDim.x) {
            const int r = e % pb, c = e / pb;
            G[(p + r) + (p + c) * l] = r <= c ? R[r][c] : 0.0;
        }
        if (tid == 0 && bad) *breakdown = 1;
    }
    // panel rows X = R_pp^-T G(p, cols) for the CTA's <= 256 trailing columns: staged in
    // shared memory (Ys[t][c], ld MP_THREADS + 1) so that G is read and written along its
    // columns; then thread c solves column c, column-oriented (y_t = y_t / r_tt, then
    // y_q -= r_tq y_t for q > t) so that the updates of one step are independent.
    const int64_t cb = p + pb + (int64_t)blockIdx.x * MP_THREADS;
    const int nc = (int)max((int64_t)0, min((int64_t)MP_THREADS, l - cb));
    if (nc == 0) return;
    constexpr int LDY = MP_THREADS + 1;
    double *Ys = rowbuf + 2 * MB;
    const int lane = tid & 31, warp = tid >> 5;
    // 16 loads per lane in flight before the shared stores
    for (int c0 = warp; c0 < nc; c0 += 8 * (MP_THREADS / 32)) {
        double v[8][2];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = c0 + u * (MP_THREADS / 32), t = lane + 32 * h;
                v[u][h] = (c < nc && t < pb) ? G[(p + t) + (cb + c) * l] : 0.0;
            }
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = c0 + u * (MP_THREADS / 32), t = lane + 32 * h;
                if (c < nc && t < pb) Ys[t * LDY + c] = v[u][h];
            }
    }
    __syncthreads();
    if (tid < nc) {
        double y[MB];
#pragma unroll
        for (int t = 0; t < MB; ++t) y[t] = t < pb ? Ys[t * LDY + tid] : 0.0;
#pragma unroll
        for (int t = 0; t < MB; ++t) {
            if (t < pb) {
                y[t] *= rinv[t];
#pragma unroll
                for (int q = t + 1; q < MB; ++q) y[q] -= R[t][q] * y[t];
            }
        }
#pragma unroll
        for (int t = 0; t < MB; ++t)
            if (t < pb) Ys[t * LDY + tid] = y[t];
    }
    __syncthreads();
    for (int c = warp; c < nc; c += MP_THREADS / 32)
        for (int t = lane; t < pb; t += 32) G[(p + t) + (cb + c) * l] = Ys[t * LDY + c];
    // the mirrored lower entries G(cols, p:p+pb), along columns of G
    for (int e = tid; e < nc * pb; e += MP_THREADS) {
        const int t = e / nc, c = e - t * nc;
        G[(cb + c) + (p + t) * l] = 0.0;
    }
}

__global__ void __launch_bounds__(256) chol_syrk_kernel(double *G, int64_t l, int64_t p, int pb) {
    extern __shared__ double mc_sm[];
    double(*As)[MB + 1] = reinterpret_cast<double(*)[MB + 1]>(mc_sm);
    double(*Bs)[MB + 1] = reinterpret_cast<double(*)[MB + 1]>(mc_sm + MB * (MB + 1));
    // tile (ti, tj), ti <= tj, from the linear index over the upper triangle (by columns)
    int idx = blockIdx.x, tj = 0;
    while (idx >= tj + 1) {
        idx -= tj + 1;
        ++tj;
    }
    const int ti = idx;
    const int64_t c0 = p + pb, I0 = c0 + (int64_t)ti * MB, J0 = c0 + (int64_t)tj * MB;
    const int tid = threadIdx.x;
    {
        // all 32 loads of a thread in flight before the shared stores
        constexpr int PER = MB * MB / 256;
        double va[PER], vb[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int e = tid + 256 * u, t = e % MB, i = e / MB;
            va[u] = (t < pb && I0 + i < l) ? G[(p + t) + (I0 + i) * l] : 0.0;
            vb[u] = (t < pb && J0 + i < l) ? G[(p + t) + (J0 + i) * l] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int e = tid + 256 * u, t = e % MB, i = e / MB;
            As[t][i] = va[u];
            Bs[t][i] = vb[u];
        }
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;  // outputs (4tx + ii, 4ty + jj)
    double acc[4][4];
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = 0.0;
    for (int t = 0; t < pb; ++t) {
        double a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            a[q] = As[t][4 * tx + q];
            b[q] = Bs[t][4 * ty + q];
        }
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = fma(a[ii], b[jj], acc[ii][jj]);
    }
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int64_t r = I0 + 4 * tx + ii, c = J0 + 4 * ty + jj;
            if (r < l && c < l) G[r + c * l] -= acc[ii][jj];
        }
}

static int cholesky_upper_mc(rla_ctx *ctx, double *G, int64_t l, double shift, int *breakdown) {
    RLA_CUDA_TRY(ctx, cudaMemsetAsync(breakdown, 0, sizeof(int), ctx->stream));
    const size_t smem = sizeof(double) * 2 * MB * (MB + 1);
    const size_t smem_panel = sizeof(double) * (MB * (MB + 2) + 3 * MB + (size_t)MB * (MP_THREADS + 1));
    RLA_CUDA_TRY(ctx, set_smem_max(chol_panel_kernel));
    RLA_CUDA_TRY(ctx, set_smem_max(chol_syrk_kernel));
    for (int64_t p = 0; p < l; p += MB) {
        const int pb = (int)std::min<int64_t>(MB, l - p);
        const int64_t rest = l - p - pb;
        const unsigned gp = (unsigned)std::max<int64_t>(1, ceil_div(rest, MP_THREADS));
        chol_panel_kernel<<<gp, MP_THREADS, smem_panel, ctx->stream>>>(G, l, p, shift, breakdown);
        if (rest > 0) {
            const int T = (int)ceil_div(rest, MB);
            chol_syrk_kernel<<<(unsigned)(T * (T + 1) / 2), 256, smem, ctx->stream>>>(G, l, p, pb);
        }
    }
    return check_launch(ctx, "chol_multi_cta");
}

int cholesky_upper(rla_ctx *ctx, double *G, int64_t l, double shift, int *breakdown) {
    if (l >= MC_MIN) return cholesky_upper_mc(ctx, G, l, shift, breakdown);
    if (l <= CB_MAXL) {
        // panel rows padded so every 4-entry group is a whole 16-byte pair
        const int ldp = (int)(ceil_div(std::max<int64_t>(l, 1), 4) * 4 + 4);
        const size_t smem = sizeof(double) * ((size_t)CB * CB + (size_t)CB * ldp);
        RLA_CUDA_TRY(ctx, set_smem_max(chol_blocked_kernel));
        chol_blocked_kernel<<<1, CB_THREADS, smem, ctx->stream>>>(G, l, shift, breakdown, ldp);
        return check_launch(ctx, "chol_blocked");
    }
    const size_t smem = sizeof(double) * (size_t)std::max<int64_t>(l, 1);
    if (smem > (size_t)ctx->smem_optin - 1024)
        return set_error(ctx, RLA_E_UNSUPPORTED, "Cholesky of order %lld exceeds shared memory", (long long)l);
    RLA_CUDA_TRY(ctx, set_smem_max(chol_upper_kernel));
    chol_upper_kernel<<<1, 1024, smem, ctx->stream>>>(G, l, shift, breakdown);
    return check_launch(ctx, "chol_upper");
}

int tri_inv_upper(rla_ctx *ctx, const double *R, int64_t l, double *Rinv) {
    const int64_t per = sizeof(double) * std::max<int64_t>(l, 1);
    const size_t ring_smem = (size_t)per * (2 * TI_CH + TI_WARPS + 1);
    if (ring_smem <= (size_t)ctx->smem_optin - 1024) {
        RLA_CUDA_TRY(ctx, set_smem_max(tri_inv_ring_kernel));
        tri_inv_ring_kernel<<<ceil_div_i(l, TI_WARPS), TI_WARPS * 32, ring_smem, ctx->stream>>>(R, l, Rinv);
        return check_launch(ctx, "tri_inv_ring");
    }
    // per warp one column of x, plus the reciprocal diagonal shared by the CTA
    const int wpc = (int)std::max<int64_t>(1, std::min<int64_t>(8, (ctx->smem_optin - 1024) / per - 1));
    if (2 * per > ctx->smem_optin - 1024)
        return set_error(ctx, RLA_E_UNSUPPORTED, "triangular inverse of order %lld exceeds shared memory", (long long)l);
    const size_t smem = (size_t)per * (wpc + 1);
    RLA_CUDA_TRY(ctx, set_smem_max(tri_inv_upper_kernel));
    tri_inv_upper_kernel<<<ceil_div_i(l, wpc), 32 * wpc, smem, ctx->stream>>>(R, l, Rinv, wpc);
    return check_launch(ctx, "tri_inv_upper");
}

// Largest relative off-diagonal sqrt(g_ij^2 / (g_ii g_jj)) of a Gram matrix G (l x l), to *out.
__global__ void __launch_bounds__(1024) jacobi_offdiag_kernel(const double *G, int64_t l, double *out) {
    __shared__ double wm[32];
    double m2 = 0.0;
    for (int64_t idx = threadIdx.x; idx < l * l; idx += blockDim.x) {
        const int64_t i = idx % l, j = idx / l;
        if (i >= j) continue;
        const double g = G[idx], a = G[i + i * l], b = G[j + j * l];
        if (g != 0.0 && a * b > 0.0) m2 = fmax(m2, g * g / (a * b));
    }
    for (int o = 16; o > 0; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(FULL, m2, o));
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m2;
    __syncthreads();
    if (threadIdx.x < 32) {
        m2 = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(FULL, m2, o));
        if (threadIdx.x == 0) *out = sqrt(m2);
    }
}

int jacobi_svd(rla_ctx *ctx, double *X, double *J, double *sigma, int64_t l, double *work, double tol) {
    // Float32 data (tolerance >= 1e-13): the Gram-based pair step
    const bool gram = tol >= 1e-13;
    const size_t smem = gram ? sizeof(double) * 32 * (size_t)(((l + 31) & ~31) + 4)
                             : sizeof(double) * 4 * BJ_B * (size_t)((l + 1) & ~1);
    // the Gram kernel also holds 21 KB of static shared memory
    if (l <= 2 * BJ_B || smem > (size_t)ctx->smem_optin - (gram ? 24576 : 2048)) {
        jacobi_kernel<<<1, 1024, 0, ctx->stream>>>(X, J, sigma, l, work, 60, tol);
        RLA_TRY(check_launch(ctx, "jacobi_svd"));
    } else {
        const int nb = (int)ceil_div(l, BJ_B), nbp = nb + (nb & 1);
        jacobi_identity_kernel<<<ceil_div_i(l * l, 256), 256, 0, ctx->stream>>>(J, l);
        RLA_TRY(check_launch(ctx, "jacobi_identity"));
        auto kern = gram ? block_jacobi_gram_round_kernel : block_jacobi_round_kernel;
        const int threads = gram ? BJX_THREADS : BJ_THREADS;
        RLA_CUDA_TRY(ctx, set_smem_max(kern));
        unsigned long long *off = reinterpret_cast<unsigned long long *>(work + 2 * l * l);
        for (int sweep = 0; sweep < 40; ++sweep) {
            RLA_CUDA_TRY(ctx, cudaMemsetAsync(off, 0, sizeof(unsigned long long), ctx->stream));
            for (int r = 0; r < nbp - 1; ++r)
                kern<<<nbp / 2, threads, smem, ctx->stream>>>(X, J, l, nbp, r, tol, off);
            RLA_TRY(check_launch(ctx, "block_jacobi_round"));
            unsigned long long h = 0;
            RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&h, off, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
            RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
            double v;
            memcpy(&v, &h, sizeof(v));
            if (v <= tol) break;
            // Quadratic convergence: once every pair measured below sqrt(tol) this sweep, the
            // next sweep is most likely one that rotates nothing.  Check that on the Gram matrix
            // of X (every pair at once, fresh FP64 dot products) instead of running it: if all
            // pairs are within tol, that sweep would leave X and J unchanged.
            if (v <= sqrt(tol)) {
                double *Gx = work;  // l x l, free until the final sort
                RLA_TRY((dgemm<double, double, double>(ctx, l, l, l, X, l, 1, X, l, 0, Gx, l, 1.0, 0.0, 0, 1)));
                double *dev_v = work + l * l;
                jacobi_offdiag_kernel<<<1, 1024, 0, ctx->stream>>>(Gx, l, dev_v);
                RLA_TRY(check_launch(ctx, "jacobi_offdiag"));
                double g = 0.0;
                RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&g, dev_v, sizeof(g), cudaMemcpyDeviceToHost, ctx->stream));
                RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
                if (g <= tol) break;
            }
        }
    }
    jacobi_rank_kernel<<<1, 1024, 0, ctx->stream>>>(X, sigma, l, work);
    jacobi_permute_kernel<<<(unsigned)l, 256, 0, ctx->stream>>>(X, J, l, work);
    RLA_TRY(check_launch(ctx, "jacobi_finish"));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(X, work, sizeof(double) * l * l, cudaMemcpyDeviceToDevice, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(J, work + l * l, sizeof(double) * l * l, cudaMemcpyDeviceToDevice, ctx->stream));
    return RLA_OK;
}

}  // namespace rla
