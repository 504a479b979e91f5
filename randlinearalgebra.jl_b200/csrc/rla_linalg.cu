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

__global__ void __launch_bounds__(1024) chol_upper_kernel(double *G, int64_t l, double shift, int *breakdown) {
    __shared__ double rkk;
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) bad = 0;
    for (int64_t i = tid; i < l; i += nt) G[i + i * l] += shift;
    __syncthreads();
    for (int64_t k = 0; k < l; ++k) {
        if (tid == 0) {
            double d = G[k + k * l];
            if (!(d > 0.0) || !isfinite(d)) {
                bad = 1;
                d = 1.0;
            }
            rkk = sqrt(d);
            G[k + k * l] = rkk;
        }
        __syncthreads();
        for (int64_t j = k + 1 + tid; j < l; j += nt) G[k + j * l] /= rkk;
        __syncthreads();
        const int64_t n = l - k - 1;
        for (int64_t idx = tid; idx < n * n; idx += nt) {
            const int64_t a = k + 1 + idx % n, b = k + 1 + idx / n;
            if (a <= b) G[a + b * l] -= G[k + a * l] * G[k + b * l];
        }
        __syncthreads();
    }
    for (int64_t idx = tid; idx < l * l; idx += nt) {
        const int64_t r = idx % l, c = idx / l;
        if (r > c) G[idx] = 0.0;
    }
    if (tid == 0) *breakdown = bad;
}

__global__ void tri_inv_upper_kernel(const double *R, int64_t l, double *Ri) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= l) return;
    double *x = Ri + j * l;
    for (int64_t i = j + 1; i < l; ++i) x[i] = 0.0;
    x[j] = 1.0 / R[j + j * l];
    for (int64_t i = j - 1; i >= 0; --i) {
        double s = 0.0;
        for (int64_t k = i + 1; k <= j; ++k) s += R[i + k * l] * x[k];
        x[i] = -s / R[i + i * l];
    }
}

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
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
    __shared__ int perm_done;
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
    // column norms
    for (int c = warp; c < l; c += nwarps) {
        const double *xc = X + (int64_t)c * l;
        double a = 0;
        for (int64_t k = lane; k < l; k += 32) a += xc[k] * xc[k];
        a = warp_sum(a);
        if (lane == 0) work[2 * l * l + c] = sqrt(a);
    }
    __syncthreads();
    // descending order (stable), one thread
    int *perm = reinterpret_cast<int *>(work + 2 * l * l + l);
    if (tid == 0) {
        const double *sg = work + 2 * l * l;
        for (int64_t c = 0; c < l; ++c) perm[c] = (int)c;
        for (int64_t a = 1; a < l; ++a) {
            int v = perm[a];
            int64_t b = a - 1;
            while (b >= 0 && sg[perm[b]] < sg[v]) {
                perm[b + 1] = perm[b];
                --b;
            }
            perm[b + 1] = v;
        }
        perm_done = 1;
    }
    __syncthreads();
    const double *sg = work + 2 * l * l;
    double *Xt = work, *Jt = work + l * l;
    for (int64_t idx = tid; idx < l * l; idx += nt) {
        const int64_t r = idx % l, c = idx / l;
        const int src = perm[c];
        const double sv = sg[src];
        Xt[idx] = sv > 0.0 ? X[r + (int64_t)src * l] / sv : 0.0;
        Jt[idx] = J[r + (int64_t)src * l];
    }
    __syncthreads();
    for (int64_t idx = tid; idx < l * l; idx += nt) {
        X[idx] = Xt[idx];
        J[idx] = Jt[idx];
    }
    for (int64_t c = tid; c < l; c += nt) sigma[c] = sg[perm[c]];
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

int cholesky_upper(rla_ctx *ctx, double *G, int64_t l, double shift, int *breakdown) {
    chol_upper_kernel<<<1, 1024, 0, ctx->stream>>>(G, l, shift, breakdown);
    return check_launch(ctx, "chol_upper");
}

int tri_inv_upper(rla_ctx *ctx, const double *R, int64_t l, double *Rinv) {
    tri_inv_upper_kernel<<<ceil_div_i(l, 128), 128, 0, ctx->stream>>>(R, l, Rinv);
    return check_launch(ctx, "tri_inv_upper");
}

int jacobi_svd(rla_ctx *ctx, double *X, double *J, double *sigma, int64_t l, double *work) {
    jacobi_kernel<<<1, 1024, 0, ctx->stream>>>(X, J, sigma, l, work, 60, 1e-15);
    return check_launch(ctx, "jacobi_svd");
}

}  // namespace rla
