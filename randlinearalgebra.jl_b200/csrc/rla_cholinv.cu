// rla_cholinv.cu -- Cholesky factor R (R'R = G) and its inverse for the l x l Gram matrices of
// CholeskyQR (l <= 384), blocked by 16 on the FP64 tensor cores.
//
// The reference orthogonalises with Householder QR (power_its.jl:35,60,70,73); CholeskyQR
// needs R and R^-1 (Q = Y R^-1).
//
//  * chol_blocked16_kernel: ONE CTA of 16 warps, right-looking over 16-column blocks J, two
//    barriers per block.  Warps 1 .. 15 form the block row R(J, K) = R_JJ^-T G(J, K); then all
//    warps apply the trailing update G(K1, K2) -= R(J, K1)' R(J, K2) (J < K1 <= K2, one warp
//    per block pair, the next pair's tile in flight while the current one is computed), both
//    as 8 x 8 tiles of mma.m8n8k4.f64 with the block row staged in shared memory.  Warp 0
//    updates the next diagonal block first and factors it during the rest of the update:
//    register shuffles (lane c holds column c, R_JJ to shared memory), then its inverse (lane i
//    forms row i of R_JJ^-1).  G is a zero-padded lp x lp working copy
//    (lp = l rounded up to 16, identity on the padded diagonal) that stays in L2.
//  * tri_inv_block_kernel: one CTA per 16-column block K of Z = R^-1, block back substitution
//    Z(J, K) = -Z_JJ sum_{I=J+1..K} R(J, I) Z(I, K) for J = K-1 .. 0, with Z(:, K) in shared
//    memory, the block row R(J, :) and Z_JJ double-buffered by cp.async one step ahead, and
//    the sum over I split over the warps (partial sums added in warp order).
//
// mma.m8n8k4.f64 fragments (per lane, g = lane >> 2, q = lane & 3): A (8 x 4, row) holds
// A[g][q]; B (4 x 8, col) holds B[q][g]; C/D (8 x 8) hold C[g][2q] and C[g][2q+1].
#include <math.h>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"

namespace rla {

namespace {

constexpr int CI_WARPS = 16, CI_THREADS = 32 * CI_WARPS, TB_WARPS = 8, TB_CS = 20;  // TB_CS: column stride of R rows

__device__ __forceinline__ void dmma8(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Padded working copy: W = [G + shift I, 0; 0, I] (lp x lp, ld lp), Z = 0.
__global__ void chol_pad_kernel(const double *G, int64_t l, int64_t lp, double shift, double *W, double *Z) {
    const int64_t n = lp * lp;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx % lp, c = idx / lp;
        double v = r == c ? 1.0 : 0.0;
        if (r < l && c < l) v = G[r + c * l] + (r == c ? shift : 0.0);
        W[idx] = v;
        Z[idx] = 0.0;
    }
}

// Triangular index p (0 .. T(T+1)/2 - 1) -> (k1, k2), k1 <= k2, ordered by k2 then k1.
__device__ __forceinline__ void tri_decode(int p, int &k1, int &k2) {
    int c = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
    while ((c + 1) * (c + 2) / 2 <= p) ++c;
    while (c * (c + 1) / 2 > p) --c;
    k2 = c;
    k1 = p - c * (c + 1) / 2;
}

// the 8 x 8 tiles (ta, tb) of block (r0, c0) of W as C fragments
__device__ __forceinline__ void load_ctile(const double *W, int lp, int r0, int c0, int g, int q, double (&c)[2][2][2]) {
#pragma unroll
    for (int ta = 0; ta < 2; ++ta)
#pragma unroll
        for (int tb = 0; tb < 2; ++tb)
#pragma unroll
            for (int e = 0; e < 2; ++e) c[ta][tb][e] = W[(r0 + 8 * ta + g) + (int64_t)(c0 + 8 * tb + 2 * q + e) * lp];
}

// Warp 0: 16 x 16 Cholesky of W(J, J) (lane c mod 16 owns column c), R_JJ into W and Rs,
// R_JJ^-1 into Di and Dg (column-major 16 x 16 per block).
__device__ __forceinline__ void chol_diag16(double *W, int lp, int J, int lane, double (*Rs)[17], double (*Di)[17],
                                            double *rinv_s, double *Dg, int *breakdown) {
    const int j0 = 16 * J, c = lane & 15;
    double d[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) d[r] = W[(j0 + r) + (int64_t)(j0 + c) * lp];
    bool bad = false;
#pragma unroll
    for (int t = 0; t < 16; ++t) {
        double piv = __shfl_sync(FULL, d[t], t);
        if (!(piv > 0.0) || !isfinite(piv)) {
            bad = true;
            piv = 1.0;
        }
        const double ri = rsqrt(piv);
        const double v = c == t ? piv * ri : (c > t ? d[t] * ri : 0.0);  // R(t, c)
        if (lane < 16) Rs[t][c] = v;
        if (lane == t) rinv_s[t] = ri;
#pragma unroll
        for (int r = t + 1; r < 16; ++r) d[r] = fma(-__shfl_sync(FULL, v, r), v, d[r]);
    }
    __syncwarp();
    // row i = c of R_JJ^-1 (Z R = I, columns in order)
    double z[16];
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
        double s = c == jj ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < jj; ++k) s = fma(-z[k], Rs[k][jj], s);
        z[jj] = s * rinv_s[jj];
    }
    if (lane < 16) {
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            W[(j0 + t) + (int64_t)(j0 + c) * lp] = Rs[t][c];
            Di[c][t] = z[t];
            Dg[(int64_t)J * 256 + c + 16 * t] = z[t];
        }
    }
    if (__any_sync(FULL, bad) && lane == 0) *breakdown = 1;
}

// One trailing-update tile pair: cur -= R(J, c1 block)' R(J, c2 block) from the panel P, then
// the upper part written back to W.
__device__ __forceinline__ void chol_update_pair(double *W, int lp, const double *P, int ps, int c1, int c2, bool diag,
                                                 int g, int q, double (&cur)[2][2][2]) {
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        const int kk = 4 * ks + q;
        const double a0 = -P[kk * ps + c1 + g], a1 = -P[kk * ps + c1 + 8 + g];
        const double b0 = P[kk * ps + c2 + g], b1 = P[kk * ps + c2 + 8 + g];
        dmma8(cur[0][0], a0, b0);
        dmma8(cur[0][1], a0, b1);
        dmma8(cur[1][0], a1, b0);
        dmma8(cur[1][1], a1, b1);
    }
#pragma unroll
    for (int ta = 0; ta < 2; ++ta)
#pragma unroll
        for (int tb = 0; tb < 2; ++tb) {
            if (diag && ta > tb) continue;  // below the diagonal of a diagonal block
#pragma unroll
            for (int e = 0; e < 2; ++e) W[(c1 + 8 * ta + g) + (int64_t)(c2 + 8 * tb + 2 * q + e) * lp] = cur[ta][tb][e];
        }
}

__global__ void __launch_bounds__(CI_THREADS) chol_blocked16_kernel(double *W, int64_t lp64, int *breakdown,
                                                                    double *Dg) {
    extern __shared__ __align__(16) double ci_sm[];
    const int lp = (int)lp64, nb = lp / 16, ps = lp + 4;  // panel row stride = 4 mod 16 doubles
    double *P = ci_sm;                                    // [16][ps]: block row R(J, :)
    __shared__ double Rs[16][17], Di[16][17], rinv_s[16];  // R_JJ, R_JJ^-1, 1 / R_JJ(t, t)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
    if (warp == 0) chol_diag16(W, lp, 0, lane, Rs, Di, rinv_s, Dg, breakdown);
    __syncthreads();
    for (int J = 0; J < nb; ++J) {
        const int j0 = 16 * J, T = nb - J - 1, np = T * (T + 1) / 2;
        // trailing pairs: warp 0 takes pair 0 (the next diagonal block, then factors it);
        // warps 1 .. take pairs warp, warp + (CI_WARPS - 1), ...
        int p = warp, t1 = 0, t2 = 0;
        const int pstep = warp == 0 ? np : CI_WARPS - 1;
        double cur[2][2][2];
        if (p < np) {
            tri_decode(p, t1, t2);
            load_ctile(W, lp, 16 * (J + 1 + t1), 16 * (J + 1 + t2), g, q, cur);
        }
        // ---- block row R(J, K) = R_JJ^-T W(J, K), K = J + warp, J + warp + (CI_WARPS - 1), ... ----
        for (int kb = J + warp; warp >= 1 && kb < nb; kb += CI_WARPS - 1) {
            double bp[4][2];
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int kk = 4 * ks + q;
                bp[ks][0] = W[(j0 + kk) + (int64_t)(16 * kb + g) * lp];
                bp[ks][1] = W[(j0 + kk) + (int64_t)(16 * kb + 8 + g) * lp];
            }
            const int k0 = 16 * kb;
            double acc[2][2][2] = {};
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int kk = 4 * ks + q;
                const double a0 = Di[kk][g], a1 = Di[kk][8 + g];  // A[i][k] = R_JJ^-1(k, i)
                dmma8(acc[0][0], a0, bp[ks][0]);
                dmma8(acc[0][1], a0, bp[ks][1]);
                dmma8(acc[1][0], a1, bp[ks][0]);
                dmma8(acc[1][1], a1, bp[ks][1]);
            }
#pragma unroll
            for (int ta = 0; ta < 2; ++ta)
#pragma unroll
                for (int tb = 0; tb < 2; ++tb)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int row = 8 * ta + g, col = k0 + 8 * tb + 2 * q + e;
                        P[row * ps + col] = acc[ta][tb][e];
                        W[(j0 + row) + (int64_t)col * lp] = acc[ta][tb][e];
                    }
        }
        __syncthreads();
        // ---- trailing update W(K1, K2) -= R(J, K1)' R(J, K2), J < K1 <= K2, next tile in flight ----
        while (p < np) {
            const int pn = p + pstep;
            int n1 = 0, n2 = 0;
            double nxt[2][2][2];
            if (pn < np) {
                tri_decode(pn, n1, n2);
                load_ctile(W, lp, 16 * (J + 1 + n1), 16 * (J + 1 + n2), g, q, nxt);
            }
            chol_update_pair(W, lp, P, ps, 16 * (J + 1 + t1), 16 * (J + 1 + t2), t1 == t2, g, q, cur);
            if (pn < np) {
#pragma unroll
                for (int ta = 0; ta < 2; ++ta)
#pragma unroll
                    for (int tb = 0; tb < 2; ++tb)
#pragma unroll
                        for (int e = 0; e < 2; ++e) cur[ta][tb][e] = nxt[ta][tb][e];
            }
            p = pn;
            t1 = n1;
            t2 = n2;
        }
        // warp 0: the next diagonal block is final (its own pair 0): factor it now, while the
        // other warps finish the trailing update
        if (warp == 0 && J + 1 < nb) {
            __syncwarp();
            chol_diag16(W, lp, J + 1, lane, Rs, Di, rinv_s, Dg, breakdown);
        }
        __syncthreads();
    }
}

// Block column K of Z = R^-1 (R = upper triangle of W, lp x lp).  Zc holds Z(0 : 16K+16, K)
// (column c at Zc + c * zs); Rb[b] the block row R(J, J+1 : K+1) (column c of W at
// Rb[b] + c * TB_CS, 16 rows); Db[b] Z_JJ (column-major 16 x 16).
__global__ void __launch_bounds__(32 * TB_WARPS) tri_inv_block_kernel(const double *W, int64_t lp64, const double *Dg,
                                                                      double *Z) {
    extern __shared__ __align__(16) double tb_sm[];
    const int lp = (int)lp64, zs = lp + 4;
    const int K = blockIdx.x, k0 = 16 * K;
    double *Zc = tb_sm;                       // [16][zs]
    double *Rb = Zc + 16 * zs;                // [2][lp * TB_CS]
    double *Db = Rb + 2 * (size_t)lp * TB_CS;  // [2][256]
    double *part = Db + 512;                  // [TB_WARPS][256]
    __shared__ double Tm[16][17];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
    // block row J of R (columns j0+16 .. k0+15) and Z_JJ into buffer b
    auto issue = [&](int J, int b) {
        if (J >= 0) {
            const int j0 = 16 * J, nc = k0 + 16 - (j0 + 16);
            double *rb = Rb + (size_t)b * lp * TB_CS;
            for (int e = tid; e < nc * 8; e += blockDim.x) {
                const int c = j0 + 16 + (e >> 3), h = e & 7;
                cp_async16(rb + (size_t)c * TB_CS + 2 * h, W + (j0 + 2 * h) + (int64_t)c * lp);
            }
            for (int e = tid; e < 128; e += blockDim.x) cp_async16(Db + b * 256 + 2 * e, Dg + (int64_t)J * 256 + 2 * e);
        }
        cp_commit();
    };
    issue(K - 1, 0);
    for (int e = tid; e < 256; e += blockDim.x) {
        const int r = e & 15, c = e >> 4;
        Zc[c * zs + k0 + r] = Dg[(int64_t)K * 256 + r + 16 * c];  // Z(K, K) = Z_KK
    }
    for (int J = K - 1, it = 0; J >= 0; --J, ++it) {
        const int j0 = 16 * J, b = it & 1;
        issue(J - 1, b ^ 1);
        cp_wait1();
        __syncthreads();
        const double *rb = Rb + (size_t)b * lp * TB_CS, *db = Db + b * 256;
        // partial T = sum over this warp's I of R(J, I) Z(I, K)
        double acc[2][2][2] = {};
        for (int I = J + 1 + warp; I <= K; I += TB_WARPS) {
            const int i0 = 16 * I;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int kk = 4 * ks + q;
                const double a0 = rb[(i0 + kk) * TB_CS + g], a1 = rb[(i0 + kk) * TB_CS + 8 + g];
                const double b0 = Zc[g * zs + i0 + kk], b1 = Zc[(8 + g) * zs + i0 + kk];
                dmma8(acc[0][0], a0, b0);
                dmma8(acc[0][1], a0, b1);
                dmma8(acc[1][0], a1, b0);
                dmma8(acc[1][1], a1, b1);
            }
        }
#pragma unroll
        for (int ta = 0; ta < 2; ++ta)
#pragma unroll
            for (int tb = 0; tb < 2; ++tb)
#pragma unroll
                for (int e = 0; e < 2; ++e) part[warp * 256 + (8 * ta + g) + 16 * (8 * tb + 2 * q + e)] = acc[ta][tb][e];
        __syncthreads();
        if (tid < 256) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < TB_WARPS; ++w) s += part[w * 256 + tid];
            Tm[tid & 15][tid >> 4] = s;
        }
        __syncthreads();
        // Z(J, K) = -Z_JJ T (warp 0)
        if (warp == 0) {
            double za[2][2][2] = {};
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int kk = 4 * ks + q;
                const double a0 = -db[g + 16 * kk], a1 = -db[8 + g + 16 * kk];
                const double b0 = Tm[kk][g], b1 = Tm[kk][8 + g];
                dmma8(za[0][0], a0, b0);
                dmma8(za[0][1], a0, b1);
                dmma8(za[1][0], a1, b0);
                dmma8(za[1][1], a1, b1);
            }
#pragma unroll
            for (int ta = 0; ta < 2; ++ta)
#pragma unroll
                for (int tb = 0; tb < 2; ++tb)
#pragma unroll
                    for (int e = 0; e < 2; ++e) Zc[(8 * tb + 2 * q + e) * zs + j0 + 8 * ta + g] = za[ta][tb][e];
        }
        __syncthreads();
    }
    cp_wait1();
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    // Z(0 : k0 + 16, K); the rows below stay zero
    for (int e = tid; e < 16 * (k0 + 16); e += blockDim.x) {
        const int c = e / (k0 + 16), r = e - c * (k0 + 16);
        Z[r + (int64_t)(k0 + c) * lp] = Zc[c * zs + r];
    }
}

// Unpad: G <- R (upper, zero below), Rinv <- Z, both l x l with ld l.
__global__ void chol_unpad_kernel(const double *W, const double *Z, int64_t l, int64_t lp, double *G, double *Rinv) {
    const int64_t n = l * l;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx % l, c = idx / l;
        G[idx] = r <= c ? W[r + c * lp] : 0.0;
        Rinv[idx] = r <= c ? Z[r + c * lp] : 0.0;
    }
}

size_t inv_smem_bytes(int64_t lp) {
    return sizeof(double) * (16 * (size_t)(lp + 4) + 2 * (size_t)lp * TB_CS + 512 + 256 * TB_WARPS);
}

}  // namespace

size_t chol_inv_work_doubles(int64_t l) {
    const int64_t lp = (l + 15) / 16 * 16;
    return (size_t)(2 * lp * lp + 256 * (lp / 16));
}

bool chol_inv_supported(const rla_ctx *ctx, int64_t l) {
    const int64_t lp = (l + 15) / 16 * 16;
    const size_t chol_smem = sizeof(double) * 16 * (size_t)(lp + 4);
    return l >= 1 && l <= 384 && chol_smem + 8192 <= (size_t)ctx->smem_optin &&
           inv_smem_bytes(lp) + 4096 <= (size_t)ctx->smem_optin;
}

int chol_inv(rla_ctx *ctx, double *G, int64_t l, double shift, int *breakdown, double *Rinv, double *work) {
    const int64_t lp = (l + 15) / 16 * 16, nb = lp / 16;
    double *W = work, *Z = work + lp * lp, *Dg = work + 2 * lp * lp;
    RLA_CUDA_TRY(ctx, cudaMemsetAsync(breakdown, 0, sizeof(int), ctx->stream));
    const unsigned gpad = (unsigned)std::min<int64_t>(ceil_div(lp * lp, 256), 1024);
    chol_pad_kernel<<<gpad, 256, 0, ctx->stream>>>(G, l, lp, shift, W, Z);
    RLA_CUDA_TRY(ctx, set_smem_max(chol_blocked16_kernel));
    chol_blocked16_kernel<<<1, CI_THREADS, sizeof(double) * 16 * (size_t)(lp + 4), ctx->stream>>>(W, lp, breakdown, Dg);
    RLA_CUDA_TRY(ctx, set_smem_max(tri_inv_block_kernel));
    tri_inv_block_kernel<<<(unsigned)nb, 32 * TB_WARPS, inv_smem_bytes(lp), ctx->stream>>>(W, lp, Dg, Z);
    const unsigned gun = (unsigned)std::min<int64_t>(ceil_div(l * l, 256), 1024);
    chol_unpad_kernel<<<gun, 256, 0, ctx->stream>>>(W, Z, l, lp, G, Rinv);
    return check_launch(ctx, "chol_inv");
}

}  // namespace rla
