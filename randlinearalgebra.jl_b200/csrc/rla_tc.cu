// rla_tc.cu -- split-BF16 GEMM on the 5th-generation tensor cores (tcgen05 + TMEM + TMA).
//
// C = alpha * op(A) * B + beta * C for FP32 data on BF16 tensor cores.  Every FP32 operand
// x is split into NT BF16 terms t0 = bf16(x), t1 = bf16(x - t0), t2 = bf16(x - t0 - t1) and
// the product keeps the term pairs of order below NT, all into one FP32 accumulator in
// tensor memory (tcgen05.mma.kind::f16):
//   NT = 2: t0*t0 + t0*t1 + t1*t0 (3 MMAs per k-step, about 16 mantissa bits; the
//           split-BF16 precision mode of RandSVD);
//   NT = 3: t0*t0 + t0*t1 + t1*t0 + t0*t2 + t1*t1 + t2*t0 (6 MMAs, about 24 bits: an FP32
//           product, used for the Gaussian sketch and native-precision Float32 products).
//
//   * tile: 128 rows of op(A) x BN columns of B per CTA (BN <= 288 for NT = 2, <= 160 for
//     NT = 3), so a tall A is read from HBM once per output tile; BK = 32 (64-byte rows,
//     64-byte swizzle) so that 4 stages of the NT terms of both operands fit in shared memory;
//   * op(A) is K-major (A' * X: A column-major, K = rows of A) or MN-major (A * X), both
//     loaded by TMA and described to the MMA by shared-memory descriptors; B is K-major;
//   * warp 0 lane 0 issues TMA loads, warp 1 lane 0 issues the MMAs and commits them to
//     the stage's "empty" mbarrier; after the last k-block all four warps read the
//     accumulator (tcgen05.ld, one TMEM lane quarter per warp) and store FP32 rows;
//   * long K is split over CTAs (split-K); partial tiles are added in split order by a
//     reduction kernel, so results are deterministic;
//   * every mbarrier wait is bounded (2 s of %globaltimer); a wait that runs out sets a
//     device status word that the host turns into RLA_E_TIMEOUT.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "rla_internal.cuh"
#include "rla_kernels.cuh"
#include "rla_tc.cuh"

namespace rla {

// ------------------------------------------------------------------------------------
// FP32 -> NT BF16 terms; element (r, c) of X at X[r + c*ldx], outputs at [r + c*ldo]
// (or, transposed, at [c + r*ldo])
// ------------------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void split_terms(float v, bf16 (&t)[NT]) {
    float rem = v;
#pragma unroll
    for (int q = 0; q < NT; ++q) {
        t[q] = __float2bfloat16_rn(rem);
        rem -= __bfloat162float(t[q]);
    }
}

template <int NT>
__global__ void split_terms_kernel(const float *__restrict__ X, int64_t rows, int64_t cols, int64_t ldx, bf16 *o0,
                                   bf16 *o1, bf16 *o2, int64_t ldo, int vec) {
    bf16 *outs[3] = {o0, o1, o2};
    const int64_t groups = (rows + 7) / 8;
    for (int64_t c = blockIdx.y; c < cols; c += gridDim.y) {
        const float *xc = X + c * ldx;
        for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < groups; g += (int64_t)gridDim.x * blockDim.x) {
            const int64_t r0 = g * 8;
            float v[8];
            if (vec && r0 + 8 <= rows) {
                const float4 a = __ldg(reinterpret_cast<const float4 *>(xc + r0));
                const float4 b = __ldg(reinterpret_cast<const float4 *>(xc + r0 + 4));
                v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
                v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = (r0 + i < rows) ? __ldg(xc + r0 + i) : 0.f;
            }
            __align__(16) bf16 t[NT][8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                bf16 ti[NT];
                split_terms<NT>(v[i], ti);
#pragma unroll
                for (int q = 0; q < NT; ++q) t[q][i] = ti[q];
            }
            // ldo is a multiple of 8 and r0 + 8 <= ldo, so whole 16-byte groups are written
#pragma unroll
            for (int q = 0; q < NT; ++q)
                *reinterpret_cast<uint4 *>(outs[q] + r0 + c * ldo) = *reinterpret_cast<const uint4 *>(t[q]);
        }
    }
}

// Transposed split: output element (c, r) at [c + r*ldo] (rows x cols in, cols x rows out),
// through 32 x 32 shared-memory tiles so reads and writes are both coalesced.  Output rows
// cols .. ldo-1 of a 32-row block that reaches them are written as zeros.
template <int NT>
__global__ void split_terms_t_kernel(const float *__restrict__ X, int64_t rows, int64_t cols, int64_t ldx, bf16 *o0,
                                     bf16 *o1, bf16 *o2, int64_t ldo) {
    __shared__ float tile[32][33];
    bf16 *outs[3] = {o0, o1, o2};
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int64_t cb = blockIdx.y; cb * 32 < cols; cb += gridDim.y) {
        for (int64_t rb = blockIdx.x; rb * 32 < rows; rb += gridDim.x) {
            const int64_t r0 = rb * 32, c0 = cb * 32;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int64_t r = r0 + tx, c = c0 + ty + 8 * k;
                tile[ty + 8 * k][tx] = (r < rows && c < cols) ? __ldg(X + r + c * ldx) : 0.f;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                // output column r = r0 + ty + 8k, output row c = c0 + tx
                const int64_t r = r0 + ty + 8 * k, c = c0 + tx;
                if (r < rows && c < ldo) {
                    bf16 t[NT];
                    split_terms<NT>(c < cols ? tile[tx][ty + 8 * k] : 0.f, t);
#pragma unroll
                    for (int q = 0; q < NT; ++q) outs[q][c + r * ldo] = t[q];
                }
            }
            __syncthreads();
        }
    }
}

template <int NT>
int split_terms_launch(rla_ctx *ctx, const float *X, int64_t rows, int64_t cols, int64_t ldx, int transpose,
                       bf16 *const *out, int64_t ldo) {
    if (rows <= 0 || cols <= 0) return RLA_OK;
    const int64_t out_rows = transpose ? cols : rows;
    uintptr_t al = 0;
    for (int q = 0; q < NT; ++q) al |= (uintptr_t)out[q];
    if (ldo % 8 != 0 || ldo < out_rows || al % 16 != 0)
        return set_error(ctx, RLA_E_ARG, "split: output leading dimension must be a multiple of 8");
    bf16 *o0 = out[0], *o1 = out[1], *o2 = NT > 2 ? out[2] : nullptr;
    if (!transpose) {
        const int vec = (ldx % 4 == 0) && ((uintptr_t)X % 16 == 0);
        const int64_t groups = (rows + 7) / 8;
        const unsigned gx = (unsigned)std::min<int64_t>(ceil_div(groups, 256), 4096);
        const unsigned gy = (unsigned)std::min<int64_t>(cols, 65535);
        split_terms_kernel<NT><<<dim3(gx, gy), 256, 0, ctx->stream>>>(X, rows, cols, ldx, o0, o1, o2, ldo, vec);
    } else {
        const unsigned gx = (unsigned)std::min<int64_t>(ceil_div(rows, 32), 65535);
        const unsigned gy = (unsigned)std::min<int64_t>(ceil_div(cols, 32), 65535);
        split_terms_t_kernel<NT><<<dim3(gx, gy), dim3(32, 8), 0, ctx->stream>>>(X, rows, cols, ldx, o0, o1, o2, ldo);
    }
    return check_launch(ctx, "split_terms");
}

int split_bf16(rla_ctx *ctx, const float *X, int64_t rows, int64_t cols, int64_t ldx, bf16 *hi, bf16 *lo, int64_t ldo) {
    bf16 *out[2] = {hi, lo};
    return split_terms_launch<2>(ctx, X, rows, cols, ldx, 0, out, ldo);
}

// ------------------------------------------------------------------------------------
// PTX wrappers (sm_100a)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the phase of parity `parity` to complete; gives up after limit_ns (and 2^26
// polls) or once another CTA has recorded a failure, records the failure in *status and
// returns false.
__device__ __noinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *status, uint64_t limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < (1u << 26) && limit_ns > 0; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63u) == 0u && (global_ns() - t0 > limit_ns || *(volatile int *)status != 0)) break;
    }
    atomicExch(status, 1);
    return false;
}

// Drain wait before a CTA releases its shared memory or tensor memory: waits for copies or
// MMAs already issued, whatever the pipeline limit, for at most 2 s (and 2^26 polls).
constexpr uint64_t TC_DRAIN_NS = 2000000000ull;
__device__ __noinline__ bool mbar_drain(uint32_t bar, uint32_t parity, int *status) {
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63u) == 0u && global_ns() - t0 > TC_DRAIN_NS) break;
    }
    atomicExch(status, 2);
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor, 64-byte swizzle (Blackwell descriptor version 1).
__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}

// Instruction descriptor of kind::f16 with BF16 inputs and an FP32 accumulator.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn_major, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ------------------------------------------------------------------------------------
// GEMM kernel
// ------------------------------------------------------------------------------------
constexpr int TC_BM = 128, TC_BK = 32, TC_THREADS = 128;
constexpr uint32_t TC_A_BYTES = TC_BM * TC_BK * 2;  // 8 KB per operand term

// Tensor maps of the NT BF16 terms of both operands.
template <int NT>
struct TcMaps {
    CUtensorMap a[NT], b[NT];
    CUtensorMap b_rem[NT];  // NT = 2: boxes of the remainder columns (rows main .. main+rem of B)
};

// Term pairs (A term, B term) of the product, largest first.
__host__ __device__ constexpr int tc_pairs(int NT) { return NT == 2 ? 3 : 6; }
__device__ __forceinline__ void tc_pair(int i, int &ta, int &tb) {
    constexpr int PA[6] = {0, 0, 1, 0, 1, 2}, PB[6] = {0, 1, 0, 2, 1, 0};
    ta = PA[i];
    tb = PB[i];
}

struct TcParams {
    int M, N, K;      // op(A) is M x K, B is K x N
    int BN;           // tile columns (multiple of 16; NT = 3: > 256 only as two halves of a multiple of 32)
    int nch;          // MMA column chunks (1 or 2)
    int a_kmajor;     // 1: op(A) = A' with A column-major K x M; 0: A column-major M x K
    int nkb;          // k-blocks of TC_BK in total
    int kbps;         // k-blocks per split
    int stages;
    uint32_t tmem_cols;
    float *out;       // FP32 tile output: out + split*split_stride + row + col*ldo
    int64_t ldo, split_stride;
    int *status;
    uint64_t wait_ns;  // limit of one pipeline wait
    // NT = 2: columns [0, main_cols) take the three term products as MMAs of N = main_cols;
    // the remainder [main_cols, BN) takes two: A_hi x [B_hi | B_lo] (N = 2 rem, the rows of
    // the two terms adjacent in shared memory) and A_lo x B_hi (N = rem), summed in the
    // epilogue.  An MMA costs the same for every N <= 256, so this issues 5 MMAs per k-step
    // at BN = 272 instead of 6, and 2 instead of 3 when BN <= 128.
    int main_cols, rem_cols;
};

template <int NT>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm_kernel(const __grid_constant__ TcMaps<NT> maps, TcParams p) {
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t b_bytes = (uint32_t)p.BN * TC_BK * 2;
    const uint32_t stage_bytes = NT * TC_A_BYTES + NT * b_bytes;
    const uint32_t bar_base = base + (uint32_t)p.stages * stage_bytes;  // full[s], empty[s], done
    auto full_bar = [&](int s) { return bar_base + 8u * (uint32_t)s; };
    auto empty_bar = [&](int s) { return bar_base + 8u * (uint32_t)(p.stages + s); };
    const uint32_t done_bar = bar_base + 16u * (uint32_t)p.stages;
    const uint32_t tmem_slot = done_bar + 8u;
    unsigned char *gen_base = smem_raw + (base - raw);
    volatile uint32_t *tmem_slot_ptr = reinterpret_cast<volatile uint32_t *>(gen_base + (tmem_slot - base));

    const int m0 = blockIdx.x * TC_BM;
    const int split = blockIdx.y;
    const int kb0 = split * p.kbps;
    const int nkb = max(0, min(p.nkb - kb0, p.kbps));

    if (threadIdx.x == 0) {
        for (int s = 0; s < p.stages; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
#pragma unroll
        for (int q = 0; q < NT; ++q) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.a[q])) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.b[q])) : "memory");
            if (NT == 2 && p.rem_cols)
                asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.b_rem[q])) : "memory");
        }
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tmem_slot),
                     "r"(p.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot_ptr;

    const uint32_t chunk_cols = (uint32_t)(p.BN / p.nch);
    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            const uint32_t tx = stage_bytes;
            int issued = 0;
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb % p.stages;
                const uint32_t ph = (uint32_t)(kb / p.stages) & 1u;
                if (!mbar_wait(empty_bar(s), ph ^ 1u, p.status, p.wait_ns)) break;
                issued = kb + 1;
                const uint32_t st = base + (uint32_t)s * stage_bytes;
                const int k0 = (kb0 + kb) * TC_BK;
                mbar_arrive_expect_tx(full_bar(s), tx);
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    const uint32_t a_t = st + (uint32_t)t * TC_A_BYTES;
                    const uint32_t b_t = st + NT * TC_A_BYTES + (uint32_t)t * b_bytes;
                    if (p.a_kmajor) {
                        tma_load_2d(a_t, &maps.a[t], full_bar(s), k0, m0);
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; ++q) tma_load_2d(a_t + q * 2048u, &maps.a[t], full_bar(s), m0 + 32 * q, k0);
                    }
                    if constexpr (NT == 2) {
                        // B region: [B_hi main][B_hi rem][B_lo rem][B_lo main], rows of 64 B
                        const uint32_t b0 = st + NT * TC_A_BYTES, mc = (uint32_t)p.main_cols, rc = (uint32_t)p.rem_cols;
                        const uint32_t main_off = t == 0 ? 0u : (mc + 2u * rc) * TC_BK * 2;
                        const uint32_t rem_off = (mc + (uint32_t)t * rc) * TC_BK * 2;
                        if (mc) tma_load_2d(b0 + main_off, &maps.b[t], full_bar(s), k0, 0);
                        if (rc) tma_load_2d(b0 + rem_off, &maps.b_rem[t], full_bar(s), k0, (int)mc);
                    } else {
                        for (int c = 0; c < p.nch; ++c) {
                            const uint32_t off = (uint32_t)c * chunk_cols * TC_BK * 2;
                            tma_load_2d(b_t + off, &maps.b[t], full_bar(s), k0, c * (int)chunk_cols);
                        }
                    }
                }
            }
            // No copy into this CTA's shared memory may be outstanding when it exits: wait for
            // the last phase issued on every stage (earlier phases of a stage completed before
            // its slot was reissued).  Immediate on the normal path.
            for (int kb = max(0, issued - p.stages); kb < issued; ++kb)
                mbar_drain(full_bar(kb % p.stages), (uint32_t)(kb / p.stages) & 1u, p.status);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            const uint32_t idesc = idesc_bf16(TC_BM, (int)chunk_cols, p.a_kmajor ? 0 : 1, 0);
            const uint32_t idesc_main = idesc_bf16(TC_BM, p.main_cols > 0 ? p.main_cols : 16, p.a_kmajor ? 0 : 1, 0);
            const uint32_t idesc_rem2 = idesc_bf16(TC_BM, p.rem_cols > 0 ? 2 * p.rem_cols : 16, p.a_kmajor ? 0 : 1, 0);
            const uint32_t idesc_rem = idesc_bf16(TC_BM, p.rem_cols > 0 ? p.rem_cols : 16, p.a_kmajor ? 0 : 1, 0);
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb % p.stages;
                const uint32_t ph = (uint32_t)(kb / p.stages) & 1u;
                if (!mbar_wait(full_bar(s), ph, p.status, p.wait_ns)) break;
                tc_fence_after();
                const uint32_t st = base + (uint32_t)s * stage_bytes;
#pragma unroll
                for (int kk = 0; kk < TC_BK / 16; ++kk) {
                    uint64_t da[NT];
#pragma unroll
                    for (int t = 0; t < NT; ++t) {
                        const uint32_t a_t = st + (uint32_t)t * TC_A_BYTES;
                        // K-major: 128 rows of 64 B, 8-row groups 512 B apart; k-step = 32 B.
                        // MN-major: 32-row blocks of 2 KB; k rows 64 B apart; k-step = 16 rows.
                        da[t] = p.a_kmajor ? sdesc_sw64(a_t + kk * 32u, 16u, 512u) : sdesc_sw64(a_t + kk * 1024u, 2048u, 512u);
                    }
                    if constexpr (NT == 2) {
                        const uint32_t b0 = st + NT * TC_A_BYTES + kk * 32u, mc = (uint32_t)p.main_cols,
                                       rc = (uint32_t)p.rem_cols;
                        const uint32_t first = (kb | kk) != 0 ? 1u : 0u;
                        if (mc) {
                            const uint64_t bh = sdesc_sw64(b0, 16u, 512u), bl = sdesc_sw64(b0 + (mc + 2u * rc) * TC_BK * 2, 16u, 512u);
                            mma_bf16(tmem, da[0], bh, idesc_main, first);
                            mma_bf16(tmem, da[0], bl, idesc_main, 1u);
                            mma_bf16(tmem, da[1], bh, idesc_main, 1u);
                        }
                        if (rc) {
                            const uint64_t br = sdesc_sw64(b0 + mc * TC_BK * 2, 16u, 512u);  // [B_hi rem][B_lo rem]
                            mma_bf16(tmem + mc, da[0], br, idesc_rem2, first);
                            mma_bf16(tmem + mc + 2u * rc, da[1], br, idesc_rem, first);
                        }
                    } else {
                        for (int c = 0; c < p.nch; ++c) {
                            const uint32_t off = (uint32_t)c * chunk_cols * TC_BK * 2 + kk * 32u;
                            uint64_t db[NT];
#pragma unroll
                            for (int t = 0; t < NT; ++t) db[t] = sdesc_sw64(st + NT * TC_A_BYTES + (uint32_t)t * b_bytes + off, 16u, 512u);
                            const uint32_t d = tmem + (uint32_t)c * chunk_cols;
#pragma unroll
                            for (int i = 0; i < tc_pairs(NT); ++i) {
                                int ta, tb;
                                tc_pair(i, ta, tb);
                                mma_bf16(d, da[ta], db[tb], idesc, (i > 0 || (kb | kk) != 0) ? 1u : 0u);
                            }
                        }
                    }
                }
                mma_commit(empty_bar(s));
            }
            mma_commit(done_bar);
        }
        __syncwarp();
    }
    // ---- epilogue: all four warps; warp w owns TMEM lanes 32w .. 32w+31 ----
    bool ok = nkb > 0 && mbar_wait(done_bar, 0u, p.status, p.wait_ns);
    // the MMAs issued before a failed wait still write tensor memory: drain them before the
    // accumulator is read and released (done_bar is committed on every path)
    if (!ok) mbar_drain(done_bar, 0u, p.status);
    __syncwarp();
    tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    float *out = p.out + (int64_t)split * p.split_stride;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    const int direct = NT == 2 ? p.main_cols : p.BN;  // columns read straight from TMEM
    for (int c0 = 0; c0 < direct; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(lane_base + (uint32_t)c0, r);
        if (row < p.M) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = c0 + j;
                if (col < p.N) out[row + (int64_t)col * p.ldo] = ok ? __uint_as_float(r[j]) : 0.f;
            }
        }
    }
    if constexpr (NT == 2) {
        // remainder column main + c: hi.hi at main + c, hi.lo at main + rem + c, lo.hi at main + 2 rem + c
        const int mc = p.main_cols, rc = p.rem_cols;
        for (int c0 = 0; c0 < rc; c0 += 16) {
            uint32_t r0[16], r1[16], r2[16];
            tmem_ld16(lane_base + (uint32_t)(mc + c0), r0);
            tmem_ld16(lane_base + (uint32_t)(mc + rc + c0), r1);
            tmem_ld16(lane_base + (uint32_t)(mc + 2 * rc + c0), r2);
            if (row < p.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = mc + c0 + j;
                    const float v = __uint_as_float(r0[j]) + __uint_as_float(r1[j]) + __uint_as_float(r2[j]);
                    if (col < p.N) out[row + (int64_t)col * p.ldo] = ok ? v : 0.f;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols) : "memory");
    }
}

// ------------------------------------------------------------------------------------
// FP32-accurate products: NT = 3 terms with FP64 accumulation across k-chunks.
// The tensor cores accumulate in FP32, and over a long K that running sum drifts well above
// the FP32 rounding of the result.  Here the MMAs of every TC_CHUNK k-blocks go into one of
// two TMEM accumulators (ping-pong); four epilogue warps add each finished chunk into FP64
// registers while the MMAs fill the other one (the NT term products of A_t with all the B
// terms of lower order form one MMA each: 3 MMAs per k-step for NT = 3, 2 for NT = 2).
// Warps: 0 TMA producer (lane 0), 1 MMA
// issuer (lane 0), 2 TMEM allocator, 4..7 chunk drain / epilogue (warp 4+q reads TMEM
// lanes 32q .. 32q+31, the tile rows of its quarter).  Tiles are 128 x 64; the grid is
// (N tiles, M tiles, splits), N fastest, so the CTAs that share an A tile run together and
// A comes from HBM about once.  Output: FP64 partial tiles, one per split.
constexpr int TC64_THREADS = 256, TC64_BN = 64, TC_CHUNK = 4;
// TMEM columns of the two chunk accumulators (64 NT columns each), a power of two
constexpr uint32_t tc64_tmem_cols(int NT) { return NT >= 3 ? 512u : (NT == 2 ? 256u : 128u); }

// One CTA of the FP64-accumulating pipeline: the 128 x 64 tile (m0, n0) of op(A) * B over
// k-blocks kb0 .. kb0+nkb-1 with MMAs mma_n columns wide, written as FP64 sums (or rounded to
// Float32) to out[row + col*ldo].  ma / mb: the NT tensor maps of A and B (kernel parameter
// or global memory).
template <int NT>
__device__ __forceinline__ void f64acc_cta(const CUtensorMap *ma, const CUtensorMap *mb, const TcParams &p, int m0,
                                           int n0, int kb0, int nkb, uint32_t mma_n, void *out, int64_t ldo,
                                           int out_f64, void *out2 = nullptr) {
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t b_bytes = (uint32_t)TC64_BN * TC_BK * 2;
    const uint32_t stage_bytes = NT * TC_A_BYTES + NT * b_bytes;
    const uint32_t bar_base = base + (uint32_t)p.stages * stage_bytes;
    auto full_bar = [&](int s) { return bar_base + 8u * (uint32_t)s; };
    auto empty_bar = [&](int s) { return bar_base + 8u * (uint32_t)(p.stages + s); };
    auto accf_bar = [&](int x) { return bar_base + 16u * (uint32_t)p.stages + 8u * (uint32_t)x; };
    auto acce_bar = [&](int x) { return bar_base + 16u * (uint32_t)p.stages + 16u + 8u * (uint32_t)x; };
    const uint32_t done_bar = bar_base + 16u * (uint32_t)p.stages + 32u;
    const uint32_t tmem_slot = done_bar + 8u;
    unsigned char *gen_base = smem_raw + (base - raw);
    volatile uint32_t *tmem_slot_ptr = reinterpret_cast<volatile uint32_t *>(gen_base + (tmem_slot - base));

    const int nchunks = (nkb + TC_CHUNK - 1) / TC_CHUNK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < p.stages; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int x = 0; x < 2; ++x) {
            mbar_init(accf_bar(x), 1);
            mbar_init(acce_bar(x), 4);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
#pragma unroll
        for (int q = 0; q < NT; ++q) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(ma + q)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(mb + q)) : "memory");
        }
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tmem_slot),
                     "r"(p.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot_ptr;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            int issued = 0;
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb % p.stages;
                const uint32_t ph = (uint32_t)(kb / p.stages) & 1u;
                if (!mbar_wait(empty_bar(s), ph ^ 1u, p.status, p.wait_ns)) break;
                issued = kb + 1;
                const uint32_t st = base + (uint32_t)s * stage_bytes;
                const int k0 = (kb0 + kb) * TC_BK;
                mbar_arrive_expect_tx(full_bar(s), stage_bytes);
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    const uint32_t a_t = st + (uint32_t)t * TC_A_BYTES;
                    const uint32_t b_t = st + NT * TC_A_BYTES + (uint32_t)t * b_bytes;
                    if (p.a_kmajor) {
                        tma_load_2d(a_t, ma + t, full_bar(s), k0, m0);
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; ++q) tma_load_2d(a_t + q * 2048u, ma + t, full_bar(s), m0 + 32 * q, k0);
                    }
                    tma_load_2d(b_t, mb + t, full_bar(s), k0, n0);
                }
            }
            for (int kb = max(0, issued - p.stages); kb < issued; ++kb)
                mbar_drain(full_bar(kb % p.stages), (uint32_t)(kb / p.stages) & 1u, p.status);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer: chunk c accumulates into TMEM columns (c & 1) * 64 NT ----
            // The B terms' 64-row tiles are adjacent in shared memory, so A_t x [B_0 | .. |
            // B_(NT-1-t)] is one MMA (an MMA costs the same for every N <= 256); column group u
            // of the accumulator collects the products with B_u, the drain adds the groups.
            const uint32_t a_mn = p.a_kmajor ? 0 : 1;
            const uint32_t idesc_n[3] = {idesc_bf16(TC_BM, TC64_BN * (NT >= 1 ? NT : 1), a_mn, 0),
                                         idesc_bf16(TC_BM, TC64_BN * (NT >= 2 ? NT - 1 : 1), a_mn, 0),
                                         idesc_bf16(TC_BM, TC64_BN * (NT >= 3 ? NT - 2 : 1), a_mn, 0)};
            (void)mma_n;
            for (int kb = 0; kb < nkb; ++kb) {
                const int c = kb / TC_CHUNK, x = c & 1;
                const bool first = kb % TC_CHUNK == 0;
                if (first) {
                    // the epilogue has drained this buffer's previous chunk (c - 2)
                    if (!mbar_wait(acce_bar(x), ((uint32_t)(c >> 1) & 1u) ^ 1u, p.status, p.wait_ns)) break;
                    tc_fence_after();
                }
                const int s = kb % p.stages;
                const uint32_t ph = (uint32_t)(kb / p.stages) & 1u;
                if (!mbar_wait(full_bar(s), ph, p.status, p.wait_ns)) break;
                tc_fence_after();
                const uint32_t st = base + (uint32_t)s * stage_bytes;
                const uint32_t d = tmem + (uint32_t)x * TC64_BN * NT;
#pragma unroll
                for (int kk = 0; kk < TC_BK / 16; ++kk) {
                    const uint64_t db = sdesc_sw64(st + NT * TC_A_BYTES + kk * 32u, 16u, 512u);  // from B_0 on
#pragma unroll
                    for (int t = 0; t < NT; ++t) {
                        const uint32_t a_t = st + (uint32_t)t * TC_A_BYTES;
                        const uint64_t da = p.a_kmajor ? sdesc_sw64(a_t + kk * 32u, 16u, 512u)
                                                       : sdesc_sw64(a_t + kk * 1024u, 2048u, 512u);
                        mma_bf16(d, da, db, idesc_n[t], (first && kk == 0 && t == 0) ? 0u : 1u);
                    }
                }
                mma_commit(empty_bar(s));
                if (kb % TC_CHUNK == TC_CHUNK - 1 || kb == nkb - 1) mma_commit(accf_bar(x));
            }
            mma_commit(done_bar);
        }
        __syncwarp();
    } else if (warp >= 4) {
        // ---- chunk drain: FP64 sums of the rows of this warp's TMEM lane quarter ----
        const int q = warp - 4;
        double acc[TC64_BN];
#pragma unroll
        for (int j = 0; j < TC64_BN; ++j) acc[j] = 0.0;
        bool ok = true;
        for (int c = 0; c < nchunks && ok; ++c) {
            const int x = c & 1;
            ok = mbar_wait(accf_bar(x), (uint32_t)(c >> 1) & 1u, p.status, p.wait_ns);
            __syncwarp();
            if (!ok) break;
            tc_fence_after();
#pragma unroll
            for (int c0 = 0; c0 < TC64_BN; c0 += 16) {
#pragma unroll
                for (int u = 0; u < NT; ++u) {
                    uint32_t r[16];
                    tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(x * TC64_BN * NT + u * TC64_BN + c0), r);
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[c0 + j] += (double)__uint_as_float(r[j]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acce_bar(x)) : "memory");
        }
        const int row = m0 + q * 32 + lane;
        if (row < p.M) {
            if (out_f64) {
                double *o = (double *)out + row;
                double *o2 = out2 ? (double *)out2 + row : nullptr;
#pragma unroll
                for (int j = 0; j < TC64_BN; ++j)
                    if (n0 + j < p.N) {
                        o[(int64_t)(n0 + j) * ldo] = ok ? acc[j] : 0.0;
                        if (o2) o2[(int64_t)(n0 + j) * ldo] = ok ? acc[j] : 0.0;
                    }
            } else {
                float *o = (float *)out + row;
#pragma unroll
                for (int j = 0; j < TC64_BN; ++j)
                    if (n0 + j < p.N) o[(int64_t)(n0 + j) * ldo] = ok ? (float)acc[j] : 0.f;
            }
        }
    }
    // every MMA issued (done_bar is committed on every path) has finished before the
    // accumulators are released
    if (threadIdx.x == 64) mbar_drain(done_bar, 0u, p.status);
    tc_fence_before();
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols) : "memory");
    }
}

template <int NT>
__global__ void __launch_bounds__(TC64_THREADS, 1)
tc_gemm_f64acc_kernel(const __grid_constant__ TcMaps<NT> maps, TcParams p, double *out64) {
    const int n0 = blockIdx.x * TC64_BN;
    const int m0 = blockIdx.y * TC_BM;
    const int split = blockIdx.z;
    const int kb0 = split * p.kbps;
    const int nkb = max(0, min(p.nkb - kb0, p.kbps));
    f64acc_cta<NT>(maps.a, maps.b, p, m0, n0, kb0, nkb, TC64_BN, out64 + (int64_t)split * p.split_stride, p.ldo, 1);
}

// ---- grouped products: many instances, one launch ------------------------------------
// Item q: op(A_q) (M x K) * B_q (K x N, N <= 64) from NT BF16 terms, FP64 accumulation across
// k-chunks, written to out (Float32 or Float64, ld ldo) and, when out2 is set, to out2 too.  CTA t takes M tile t - tstart[q]
// of the item with tstart[q] <= t < tstart[q+1]; the tensor maps live in the item table in
// global memory (written before the launch).
template <int NT>
struct alignas(64) TcGroupItem {
    CUtensorMap a[NT], b[NT];
    int M, N, K, a_kmajor;
    int nkb, mma_n;
    void *out, *out2;
    int64_t ldo;
    int out_f64;
};

template <int NT>
__global__ void __launch_bounds__(TC64_THREADS, 1)
tc_group_f64acc_kernel(const TcGroupItem<NT> *items, const int *tstart, int count, TcParams p) {
    const int t = blockIdx.x;
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tstart[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    const TcGroupItem<NT> &it = items[lo];
    p.M = it.M;
    p.N = it.N;
    p.K = it.K;
    p.a_kmajor = it.a_kmajor;
    f64acc_cta<NT>(it.a, it.b, p, (t - tstart[lo]) * TC_BM, 0, 0, it.nkb, (uint32_t)it.mma_n, it.out, it.ldo,
                   it.out_f64, it.out2);
}

// Grouped split: item q converts X_q (rows x cols, ld ldx, FP32) into NT BF16 terms (ld ldo);
// CTA t takes 256 groups of 8 rows of item q with bstart[q] <= t < bstart[q+1].
struct SplitItem {
    const float *X;
    int64_t rows, cols, ldx;
    bf16 *t[3];
    int64_t ldo;
};

template <int NT>
__global__ void split_group_kernel(const SplitItem *items, const int *bstart, int count) {
    const int blk = blockIdx.x;
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bstart[mid] <= blk) lo = mid;
        else hi = mid - 1;
    }
    const SplitItem &it = items[lo];
    const int64_t groups = (it.rows + 7) / 8;
    const int64_t u = (int64_t)(blk - bstart[lo]) * blockDim.x + threadIdx.x;
    if (u >= groups * it.cols) return;
    const int64_t c = u / groups, r0 = (u - c * groups) * 8;
    const float *xc = it.X + c * it.ldx;
    float v[8];
    if (r0 >= 4 && r0 + 12 <= it.rows) {
        // three 16-byte loads of the aligned window around the 8 elements (columns of an
        // instance need not start on a 16-byte boundary); the window stays inside the column
        const uintptr_t addr = reinterpret_cast<uintptr_t>(xc + r0);
        const int a = (int)((addr >> 2) & 3u);
        const float4 *w = reinterpret_cast<const float4 *>(addr - 4u * (uintptr_t)a);
        const float4 f0 = __ldg(w), f1 = __ldg(w + 1), f2 = __ldg(w + 2);
        const float win[12] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w};
        switch (a) {
#define RLA_WIN(A)                                   \
    case A:                                          \
        _Pragma("unroll") for (int i = 0; i < 8; ++i) v[i] = win[A + i]; \
        break;
            RLA_WIN(0)
            RLA_WIN(1)
            RLA_WIN(2)
            RLA_WIN(3)
#undef RLA_WIN
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = r0 + i < it.rows ? __ldg(xc + r0 + i) : 0.f;
    }
    __align__(16) bf16 t[NT][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        bf16 ti[NT];
        split_terms<NT>(v[i], ti);
#pragma unroll
        for (int q = 0; q < NT; ++q) t[q][i] = ti[q];
    }
#pragma unroll
    for (int q = 0; q < NT; ++q)
        *reinterpret_cast<uint4 *>(it.t[q] + r0 + c * it.ldo) = *reinterpret_cast<const uint4 *>(t[q]);
}

// C(i, j) = alpha * sum_s P[s](i, j) + beta * C(i, j), splits added in order.
template <class TC, class TP = float>
__global__ void splitk_reduce_kernel(const TP *__restrict__ P, int splits, int64_t split_stride, int64_t ldp,
                                     int64_t M, int64_t N, TC *C, int64_t ldc, double alpha, double beta,
                                     int beta_zero) {
    // four consecutive rows per thread: 16-byte partial loads (ldp and split_stride are
    // multiples of 4 floats), and 16-byte stores when C's columns allow them
    constexpr bool V4 = sizeof(TP) == 4;
    const bool c_vec = V4 && sizeof(TC) == 4 && ldc % 4 == 0 && ((uintptr_t)C & 15u) == 0;
    const int64_t M4 = V4 ? (M + 3) / 4 : M;
    for (int64_t j = blockIdx.y; j < N; j += gridDim.y) {
        for (int64_t i4 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i4 < M4; i4 += (int64_t)gridDim.x * blockDim.x) {
            if (V4 && 4 * i4 + 4 <= M) {
                const int64_t i = 4 * i4;
                double acc[4] = {0.0, 0.0, 0.0, 0.0};
                for (int s = 0; s < splits; ++s) {
                    const float4 v = *reinterpret_cast<const float4 *>(P + s * split_stride + i + j * ldp);
                    acc[0] += (double)v.x;
                    acc[1] += (double)v.y;
                    acc[2] += (double)v.z;
                    acc[3] += (double)v.w;
                }
                TC *cp = C + i + j * ldc;
                TC r[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) r[e] = (TC)(alpha * acc[e] + (beta_zero ? 0.0 : beta * (double)cp[e]));
                if (c_vec) {
                    *reinterpret_cast<float4 *>(cp) = make_float4((float)r[0], (float)r[1], (float)r[2], (float)r[3]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) cp[e] = r[e];
                }
            } else {
                for (int64_t i = V4 ? 4 * i4 : i4; i < (V4 ? min(M, 4 * i4 + 4) : i4 + 1); ++i) {
                    double acc = 0.0;
                    for (int s = 0; s < splits; ++s) acc += (double)P[s * split_stride + i + j * ldp];
                    TC *cp = C + i + j * ldc;
                    double r = alpha * acc;
                    if (!beta_zero) r += beta * (double)*cp;
                    *cp = (TC)r;
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2-D BF16 map over a column-major array: inner dimension `inner` (contiguous), outer
// dimension `outer` with stride ld elements; 64-byte swizzle, zero fill outside.
static int make_map(rla_ctx *ctx, CUtensorMap *map, const bf16 *ptr, int64_t inner, int64_t outer, int64_t ld,
                    uint32_t box_inner, uint32_t box_outer) {
    auto fn = encode_fn();
    if (!fn) return set_error(ctx, RLA_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    if (((uintptr_t)ptr & 15u) != 0 || (ld * 2) % 16 != 0)
        return set_error(ctx, RLA_E_ARG, "tensor-core operands need 16-byte aligned columns");
    cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(ptr), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(ctx, RLA_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return RLA_OK;
}

int tc_status_get(rla_ctx *ctx, int **out) {
    if (!ctx->tc_status) {
        RLA_CUDA_TRY(ctx, cudaMalloc((void **)&ctx->tc_status, 256));
        RLA_CUDA_TRY(ctx, cudaMemsetAsync(ctx->tc_status, 0, 256, ctx->stream));
    }
    *out = ctx->tc_status;
    return RLA_OK;
}

int tc_status_check(rla_ctx *ctx) {
    if (!ctx->tc_status) return RLA_OK;
    int st = 0;
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(&st, ctx->tc_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (st) {
        RLA_CUDA_TRY(ctx, cudaMemsetAsync(ctx->tc_status, 0, sizeof(int), ctx->stream));
        return set_error(ctx, RLA_E_TIMEOUT, "tensor-core GEMM pipeline wait timed out");
    }
    return RLA_OK;
}

TcPlan tc_plan(const rla_ctx *ctx, int64_t M, int64_t N, int64_t K, int splits, int NT) {
    TcPlan pl;
    const int64_t nb = std::min<int64_t>(N, tc_max_bn(NT));
    if (NT == 2) {
        // one MMA of N = main for the three term products, two packed MMAs for the remainder
        pl.BN = (int)(ceil_div(nb, 16) * 16);
        pl.main_cols = pl.BN > 256 ? 256 : (pl.BN > 128 ? pl.BN : 0);
        pl.rem_cols = pl.BN - pl.main_cols;
        pl.nch = 1;
    } else {
        pl.BN = (int)(nb <= 256 ? ceil_div(nb, 16) * 16 : ceil_div(nb, 32) * 32);
        pl.nch = pl.BN > 256 ? 2 : 1;
    }
    const int64_t b_bytes = (int64_t)pl.BN * TC_BK * 2;
    const int64_t stage = NT * TC_A_BYTES + NT * b_bytes;
    const int64_t budget = ctx->smem_optin - 1024 - 256;
    pl.stages = (int)std::max<int64_t>(2, std::min<int64_t>(8, budget / stage));
    pl.smem = (size_t)(pl.stages * stage + 1024 + 256);
    pl.tmem_cols = 32;
    const int acc_cols = NT == 2 ? pl.main_cols + 3 * pl.rem_cols : pl.BN;
    while ((int)pl.tmem_cols < acc_cols) pl.tmem_cols <<= 1;
    const int64_t mt = ceil_div(M, TC_BM), nkb = ceil_div(K, TC_BK);
    pl.mt = (int)mt;
    pl.nkb = (int)nkb;
    if (splits <= 0) {
        // model: waves x k-blocks per split x MMA time per k-block, plus partial-tile traffic
        // an MMA of M = 128 costs the same for every N <= 256: time per k-block ~ MMA count
        const int mmas = NT == 2 ? (pl.main_cols ? 3 : 0) + (pl.rem_cols ? 2 : 0) : tc_pairs(NT) * pl.nch;
        const double t_kb = 0.25e-6 * mmas, bw = 6.0e12;
        double best = 1e30;
        splits = 1;
        for (int s = 1; s <= std::min<int64_t>(nkb, 64); ++s) {
            const int64_t kbps = ceil_div(nkb, s);
            if (s > 1 && kbps < 8) break;
            const double waves = (double)ceil_div(mt * s, ctx->sm_count);
            const double t = waves * (double)kbps * t_kb + (s > 1 ? (double)s * M * pl.BN * 8.0 / bw : 0.0);
            if (t < best * 0.98) {
                best = t;
                splits = s;
            }
        }
    }
    pl.kbps = (int)ceil_div(nkb, splits);
    pl.splits = (int)ceil_div(nkb, pl.kbps);
    return pl;
}

template <int NT, class TC>
int tc_gemm_split(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *const *A, int64_t lda, int a_kmajor,
                  const bf16 *const *B, int64_t ldb, TC *C, int64_t ldc, double alpha, double beta, int splits) {
    if (M <= 0 || N <= 0) return RLA_OK;
    if (M >= (1ll << 31) || K >= (1ll << 31)) return set_error(ctx, RLA_E_UNSUPPORTED, "tensor-core GEMM: dimension above 2^31");
    int *status = nullptr;
    RLA_TRY(tc_status_get(ctx, &status));
    const int max_bn = tc_max_bn(NT);
    for (int64_t n0 = 0; n0 < N; n0 += max_bn) {
        const int64_t nb = std::min<int64_t>(max_bn, N - n0);
        TcPlan pl = tc_plan(ctx, M, nb, K, splits, NT);
        TcMaps<NT> maps;
        const uint32_t box_n = (uint32_t)(NT == 2 ? pl.main_cols : pl.BN / pl.nch);
        for (int t = 0; t < NT; ++t) {
            if (a_kmajor) RLA_TRY(make_map(ctx, &maps.a[t], A[t], K, M, lda, TC_BK, TC_BM));
            else RLA_TRY(make_map(ctx, &maps.a[t], A[t], M, K, lda, 32, TC_BK));
            if (box_n) RLA_TRY(make_map(ctx, &maps.b[t], B[t] + n0 * ldb, K, nb, ldb, TC_BK, box_n));
            if (NT == 2 && pl.rem_cols)
                RLA_TRY(make_map(ctx, &maps.b_rem[t], B[t] + n0 * ldb, K, nb, ldb, TC_BK, (uint32_t)pl.rem_cols));
        }
        TC *Cn = C + n0 * ldc;
        const bool direct = pl.splits == 1 && std::is_same<TC, float>::value && alpha == 1.0 && beta == 0.0;
        float *out;
        int64_t ldo, sstride;
        if (direct) {
            out = reinterpret_cast<float *>(Cn);
            ldo = ldc;
            sstride = 0;
        } else {
            ldo = ceil_div(M, 4) * 4;
            sstride = ldo * nb;
            void *ws = nullptr;
            RLA_TRY(scratch_get(ctx, sizeof(float) * (size_t)sstride * pl.splits, &ws));
            out = (float *)ws;
        }
        TcParams p{(int)M, (int)nb, (int)K, pl.BN, pl.nch, a_kmajor, pl.nkb, pl.kbps, pl.stages, pl.tmem_cols,
                   out, ldo, sstride, status, ctx->wait_ns, pl.main_cols, pl.rem_cols};
        RLA_CUDA_TRY(ctx, set_smem_max(tc_gemm_kernel<NT>));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (ctx->timing) {
            RLA_CUDA_TRY(ctx, cudaEventCreate(&e0));
            RLA_CUDA_TRY(ctx, cudaEventCreate(&e1));
            RLA_CUDA_TRY(ctx, cudaEventRecord(e0, ctx->stream));
        }
        tc_gemm_kernel<NT><<<dim3(pl.mt, pl.splits), TC_THREADS, pl.smem, ctx->stream>>>(maps, p);
        RLA_TRY(check_launch(ctx, "tc_gemm"));
        if (ctx->timing) {
            RLA_CUDA_TRY(ctx, cudaEventRecord(e1, ctx->stream));
            ctx->timed[0].emplace_back(e0, e1);
        }
        if (!direct) {
            const unsigned gx = (unsigned)std::min<int64_t>(ceil_div(M, 1024), 1024);  // 4 rows per thread
            const unsigned gy = (unsigned)std::min<int64_t>(nb, 65535);
            splitk_reduce_kernel<TC><<<dim3(gx, gy), 256, 0, ctx->stream>>>(out, pl.splits, sstride, ldo, M, nb, Cn, ldc,
                                                                            alpha, beta, beta == 0.0);
            RLA_TRY(check_launch(ctx, "splitk_reduce"));
        }
    }
    return RLA_OK;
}

template int split_terms_launch<2>(rla_ctx *, const float *, int64_t, int64_t, int64_t, int, bf16 *const *, int64_t);
template int split_terms_launch<3>(rla_ctx *, const float *, int64_t, int64_t, int64_t, int, bf16 *const *, int64_t);
#define RLA_INST_TC(NT, TC)                                                                                          \
    template int tc_gemm_split<NT, TC>(rla_ctx *, int64_t, int64_t, int64_t, const bf16 *const *, int64_t, int,     \
                                       const bf16 *const *, int64_t, TC *, int64_t, double, double, int);
RLA_INST_TC(2, float)
RLA_INST_TC(2, double)
RLA_INST_TC(3, float)
RLA_INST_TC(3, double)
#undef RLA_INST_TC

template <class TC>
int tc_gemm_bf16x3(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *Ahi, const bf16 *Alo, int64_t lda,
                   int a_kmajor, const bf16 *Bhi, const bf16 *Blo, int64_t ldb, TC *C, int64_t ldc, double alpha,
                   double beta, int splits) {
    const bf16 *a[2] = {Ahi, Alo}, *b[2] = {Bhi, Blo};
    return tc_gemm_split<2, TC>(ctx, M, N, K, a, lda, a_kmajor, b, ldb, C, ldc, alpha, beta, splits);
}

template int tc_gemm_bf16x3<float>(rla_ctx *, int64_t, int64_t, int64_t, const bf16 *, const bf16 *, int64_t, int,
                                   const bf16 *, const bf16 *, int64_t, float *, int64_t, double, double, int);
template int tc_gemm_bf16x3<double>(rla_ctx *, int64_t, int64_t, int64_t, const bf16 *, const bf16 *, int64_t, int,
                                    const bf16 *, const bf16 *, int64_t, double *, int64_t, double, double, int);

// ---- grouped products and splits (host side) ---------------------------------------------
int tc_group_build(rla_ctx *ctx, const std::vector<TcGroupSpec> &specs, TcGroup *g) {
    constexpr int NT = 2;
    g->count = (int)specs.size();
    g->tiles = 0;
    if (specs.empty()) return RLA_OK;
    std::vector<TcGroupItem<NT>> items(specs.size());
    std::vector<int> ts(specs.size() + 1);
    for (size_t q = 0; q < specs.size(); ++q) {
        const TcGroupSpec &sp = specs[q];
        TcGroupItem<NT> &it = items[q];
        if (sp.N > TC64_BN || sp.M <= 0 || sp.N <= 0 || sp.K <= 0 || sp.M >= (1ll << 31) || sp.K >= (1ll << 31))
            return set_error(ctx, RLA_E_UNSUPPORTED, "grouped tensor-core product: shape %lld x %lld x %lld",
                             (long long)sp.M, (long long)sp.N, (long long)sp.K);
        for (int t = 0; t < NT; ++t) {
            if (sp.a_kmajor) RLA_TRY(make_map(ctx, &it.a[t], sp.a[t], sp.K, sp.M, sp.lda, TC_BK, TC_BM));
            else RLA_TRY(make_map(ctx, &it.a[t], sp.a[t], sp.M, sp.K, sp.lda, 32, TC_BK));
            RLA_TRY(make_map(ctx, &it.b[t], sp.b[t], sp.K, sp.N, sp.ldb, TC_BK, TC64_BN));
        }
        it.M = (int)sp.M;
        it.N = (int)sp.N;
        it.K = (int)sp.K;
        it.a_kmajor = sp.a_kmajor;
        it.nkb = (int)ceil_div(sp.K, TC_BK);
        it.mma_n = (int)ceil_div(sp.N, 16) * 16;
        it.out = sp.out;
        it.out2 = sp.out2;
        it.ldo = sp.ldo;
        it.out_f64 = sp.out_f64;
        ts[q] = g->tiles;
        g->tiles += (int)ceil_div(sp.M, TC_BM);
    }
    ts[specs.size()] = g->tiles;
    void *di = nullptr, *dt = nullptr;
    g->stream = ctx->stream;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &di, sizeof(TcGroupItem<NT>) * items.size(), ctx->stream));
    g->items = di;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &dt, sizeof(int) * ts.size(), ctx->stream));
    g->tstart = (int *)dt;
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(di, items.data(), sizeof(TcGroupItem<NT>) * items.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(dt, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice, ctx->stream));
    const int64_t stage = NT * TC_A_BYTES + NT * (int64_t)TC64_BN * TC_BK * 2;
    const int64_t budget = ctx->smem_optin - 1024 - 256;
    g->stages = (int)std::max<int64_t>(2, std::min<int64_t>(8, budget / stage));
    g->smem = (size_t)(g->stages * stage + 1024 + 256);
    RLA_CUDA_TRY(ctx, set_smem_max(tc_group_f64acc_kernel<NT>));
    return tc_status_get(ctx, &g->status);
}

int tc_group_run(rla_ctx *ctx, const TcGroup &g, cudaStream_t st) {
    if (g.tiles == 0) return RLA_OK;
    TcParams p{};
    p.BN = TC64_BN;
    p.nch = 1;
    p.stages = g.stages;
    p.tmem_cols = tc64_tmem_cols(2);  // grouped products are split-BF16 (NT = 2)
    p.status = g.status;
    p.wait_ns = ctx->wait_ns;
    tc_group_f64acc_kernel<2><<<g.tiles, TC64_THREADS, g.smem, st>>>((const TcGroupItem<2> *)g.items, g.tstart, g.count,
                                                                     p);
    return check_launch(ctx, "tc_group_f64acc");
}

int split_group_build(rla_ctx *ctx, const std::vector<SplitSpec> &specs, SplitGroup *g) {
    g->count = (int)specs.size();
    g->blocks = 0;
    if (specs.empty()) return RLA_OK;
    std::vector<SplitItem> items(specs.size());
    std::vector<int> bs(specs.size() + 1);
    for (size_t q = 0; q < specs.size(); ++q) {
        const SplitSpec &sp = specs[q];
        if (sp.ldo % 8 != 0 || sp.ldo < sp.rows || (((uintptr_t)sp.hi | (uintptr_t)sp.lo) & 15u))
            return set_error(ctx, RLA_E_ARG, "grouped split: output leading dimension must be a multiple of 8");
        items[q] = SplitItem{sp.X, sp.rows, sp.cols, sp.ldx, {sp.hi, sp.lo, nullptr}, sp.ldo};
        bs[q] = g->blocks;
        g->blocks += (int)ceil_div(ceil_div(sp.rows, 8) * sp.cols, 256);
    }
    bs[specs.size()] = g->blocks;
    void *di = nullptr, *db = nullptr;
    g->stream = ctx->stream;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &di, sizeof(SplitItem) * items.size(), ctx->stream));
    g->items = di;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &db, sizeof(int) * bs.size(), ctx->stream));
    g->bstart = (int *)db;
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(di, items.data(), sizeof(SplitItem) * items.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
    RLA_CUDA_TRY(ctx, cudaMemcpyAsync(db, bs.data(), sizeof(int) * bs.size(), cudaMemcpyHostToDevice, ctx->stream));
    return RLA_OK;
}

int split_group_run(rla_ctx *ctx, const SplitGroup &g, cudaStream_t st) {
    if (g.blocks == 0) return RLA_OK;
    split_group_kernel<2><<<g.blocks, 256, 0, st>>>((const SplitItem *)g.items, g.bstart, g.count);
    return check_launch(ctx, "split_group");
}

// Released after the work queued on the building stream; launches on other streams that read
// the tables are joined into that stream (or synchronised) before the free is issued.
void tc_group_free(TcGroup *g) {
    if (g->items) cudaFreeAsync(g->items, g->stream);
    if (g->tstart) cudaFreeAsync(g->tstart, g->stream);
    *g = TcGroup{};
}

void split_group_free(SplitGroup *g) {
    if (g->items) cudaFreeAsync(g->items, g->stream);
    if (g->bstart) cudaFreeAsync(g->bstart, g->stream);
    *g = SplitGroup{};
}

// C (M x N, ld ldc) = alpha * op(A) * B + beta * C from three BF16 terms of each operand,
// FP64 accumulation across k-chunks (tc_gemm_f64acc_kernel); split-K partials in FP64.
template <class TC>
int tc_gemm_f64acc(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *const *A, int64_t lda, int a_kmajor,
                   const bf16 *const *B, int64_t ldb, TC *C, int64_t ldc, double alpha, double beta) {
    constexpr int NT = 3;
    if (M <= 0 || N <= 0) return RLA_OK;
    if (M >= (1ll << 31) || K >= (1ll << 31) || N >= (1ll << 31))
        return set_error(ctx, RLA_E_UNSUPPORTED, "tensor-core GEMM: dimension above 2^31");
    int *status = nullptr;
    RLA_TRY(tc_status_get(ctx, &status));
    const int64_t mt = ceil_div(M, TC_BM), ntl = ceil_div(N, TC64_BN), nkb = ceil_div(K, TC_BK);
    if (mt > 65535 || ntl > 65535) return set_error(ctx, RLA_E_UNSUPPORTED, "tensor-core GEMM: grid too large");
    const int64_t stage = NT * TC_A_BYTES + NT * (int64_t)TC64_BN * TC_BK * 2;
    const int64_t budget = ctx->smem_optin - 1024 - 256;
    const int stages = (int)std::max<int64_t>(2, std::min<int64_t>(8, budget / stage));
    const size_t smem = (size_t)(stages * stage + 1024 + 256);
    // split K until the grid covers the GPU, keeping whole chunks per split
    int64_t splits = 1;
    const int64_t tiles = mt * ntl;
    if (tiles < ctx->sm_count) splits = std::min<int64_t>(ceil_div(ctx->sm_count, tiles), std::max<int64_t>(1, nkb / (2 * TC_CHUNK)));
    const int64_t kbps = ceil_div(ceil_div(nkb, splits), TC_CHUNK) * TC_CHUNK;
    splits = ceil_div(nkb, kbps);
    TcMaps<NT> maps;
    for (int t = 0; t < NT; ++t) {
        if (a_kmajor) RLA_TRY(make_map(ctx, &maps.a[t], A[t], K, M, lda, TC_BK, TC_BM));
        else RLA_TRY(make_map(ctx, &maps.a[t], A[t], M, K, lda, 32, TC_BK));
        RLA_TRY(make_map(ctx, &maps.b[t], B[t], K, N, ldb, TC_BK, TC64_BN));
    }
    const int64_t ldo = M, sstride = M * N;
    void *ws = nullptr;
    RLA_TRY(scratch_get(ctx, sizeof(double) * (size_t)sstride * splits, &ws));
    TcParams p{(int)M, (int)N, (int)K, TC64_BN, 1, a_kmajor, (int)nkb, (int)kbps, stages, tc64_tmem_cols(NT),
               nullptr, ldo, sstride, status, ctx->wait_ns};
    RLA_CUDA_TRY(ctx, set_smem_max(tc_gemm_f64acc_kernel<NT>));
    cudaEvent_t e0 = timing_begin(ctx);
    tc_gemm_f64acc_kernel<NT><<<dim3((unsigned)ntl, (unsigned)mt, (unsigned)splits), TC64_THREADS, smem, ctx->stream>>>(
        maps, p, (double *)ws);
    RLA_TRY(check_launch(ctx, "tc_gemm_f64acc"));
    timing_end(ctx, 0, e0);
    const unsigned gx = (unsigned)std::min<int64_t>(ceil_div(M, 256), 1024);
    const unsigned gy = (unsigned)std::min<int64_t>(N, 65535);
    splitk_reduce_kernel<TC, double><<<dim3(gx, gy), 256, 0, ctx->stream>>>((const double *)ws, (int)splits, sstride,
                                                                              ldo, M, N, C, ldc, alpha, beta, beta == 0.0);
    return check_launch(ctx, "splitk_reduce");
}

// C (M x N, ld ldc, TC) = alpha * op(A) * op(B) + beta * C for Float32 A and B on the
// tensor cores with three BF16 terms per operand and FP64 accumulation across k-chunks (an
// FP32-accurate product).  op(A) may be
// A or A' (both layouts are read by TMA); op(B) must be K-major for the MMA, so B' (tb = 1)
// is transposed while it is split.  The split copies come from the context's memory pool.
template <class TC>
int gemm_f32_tc(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const float *A, int64_t lda, int ta, const float *B,
                int64_t ldb, int tb, TC *C, int64_t ldc, double alpha, double beta) {
    if (M <= 0 || N <= 0) return RLA_OK;
    if (K <= 0) return gemm<float, float, TC, double>(ctx, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, alpha, beta);
    const int64_t a_rows = ta ? K : M, a_cols = ta ? M : K;
    const int64_t lda2 = ceil_div(a_rows, 8) * 8, ldb2 = ceil_div(K, 8) * 8;
    const size_t na = (size_t)lda2 * a_cols, nb = (size_t)ldb2 * N;
    bf16 *buf = nullptr;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&buf, sizeof(bf16) * 3 * (na + nb) + 256, ctx->stream));
    bf16 *a3[3] = {buf, buf + na, buf + 2 * na};
    bf16 *b3[3] = {buf + 3 * na, buf + 3 * na + nb, buf + 3 * na + 2 * nb};
    int rc = split_terms_launch<3>(ctx, A, a_rows, a_cols, lda, 0, a3, lda2);
    if (rc == RLA_OK) rc = tb ? split_terms_launch<3>(ctx, B, N, K, ldb, 1, b3, ldb2)
                              : split_terms_launch<3>(ctx, B, K, N, ldb, 0, b3, ldb2);
    if (rc == RLA_OK) {
        const bf16 *ac[3] = {a3[0], a3[1], a3[2]}, *bc[3] = {b3[0], b3[1], b3[2]};
        rc = tc_gemm_f64acc<TC>(ctx, M, N, K, ac, lda2, ta, bc, ldb2, C, ldc, alpha, beta);
    }
    cudaFreeAsync(buf, ctx->stream);
    return rc;
}

template int gemm_f32_tc<float>(rla_ctx *, int64_t, int64_t, int64_t, const float *, int64_t, int, const float *,
                                int64_t, int, float *, int64_t, double, double);
template int gemm_f32_tc<double>(rla_ctx *, int64_t, int64_t, int64_t, const float *, int64_t, int, const float *,
                                 int64_t, int, double *, int64_t, double, double);

}  // namespace rla

using namespace rla;

extern "C" {

int rla_gemm_bf16x3(rla_ctx *ctx, int trans_a, int64_t m, int64_t n, int64_t k, const float *A, int64_t lda,
                    const float *B, int64_t ldb, float *C, int64_t ldc, double alpha, double beta) {
    if (!ctx) return RLA_E_ARG;
    if (m < 0 || n < 0 || k < 0) return set_error(ctx, RLA_E_ARG, "Negative dimension.");
    if (trans_a != 0 && trans_a != 1) return set_error(ctx, RLA_E_ARG, "trans_a must be 0 or 1.");
    const int64_t a_rows = trans_a ? k : m;
    if (lda < std::max<int64_t>(1, a_rows) || ldb < std::max<int64_t>(1, k) || ldc < std::max<int64_t>(1, m))
        return set_error(ctx, RLA_E_ARG, "Leading dimension smaller than the stored row count.");
    if (m == 0 || n == 0) return RLA_OK;
    if (!A || !B || !C) return set_error(ctx, RLA_E_ARG, "NULL matrix pointer.");
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    const int64_t a_cols = trans_a ? m : k;
    const int64_t lda2 = ceil_div(std::max<int64_t>(a_rows, 1), 8) * 8, ldb2 = ceil_div(std::max<int64_t>(k, 1), 8) * 8;
    bf16 *buf = nullptr;
    const size_t na = (size_t)lda2 * a_cols, nb = (size_t)ldb2 * n;
    if (k > 0) {
        RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, (void **)&buf, sizeof(bf16) * 2 * (na + nb) + 64, ctx->stream));
    }
    int rc = RLA_OK;
    if (k == 0) {
        // C = beta * C
        rc = gemm<float, float, float, double>(ctx, m, n, 0, A, lda, 0, B, ldb, 0, C, ldc, alpha, beta);
    } else {
        bf16 *ahi = buf, *alo = buf + na, *bhi = buf + 2 * na, *blo = buf + 2 * na + nb;
        rc = split_bf16(ctx, A, a_rows, a_cols, lda, ahi, alo, lda2);
        if (rc == RLA_OK) rc = split_bf16(ctx, B, k, n, ldb, bhi, blo, ldb2);
        if (rc == RLA_OK)
            rc = tc_gemm_bf16x3<float>(ctx, m, n, k, ahi, alo, lda2, trans_a, bhi, blo, ldb2, C, ldc, alpha, beta, 0);
        cudaFreeAsync(buf, ctx->stream);
    }
    RLA_TRY(rc);
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return tc_status_check(ctx);
}

}  // extern "C"
