// rla_tc.cu -- split-BF16 GEMM on the 5th-generation tensor cores (tcgen05 + TMEM + TMA).
//
// C = alpha * op(A) * B + beta * C for FP32 data whose products must keep about 16
// mantissa bits: every FP32 operand x is split into hi = bf16(x) and lo = bf16(x - hi) and
// the product is hi*hi + hi*lo + lo*hi, three tcgen05.mma.kind::f16 per k-step into one
// FP32 accumulator in tensor memory (lo*lo is below FP32 rounding of the result).
//
//   * tile: 128 rows of op(A) x BN <= 288 columns of B per CTA, so a tall A is read from
//     HBM once per output tile; BK = 32 (64-byte rows, 64-byte swizzle) so that 4 stages
//     of {A_hi, A_lo, B_hi, B_lo} fit in shared memory;
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
// FP32 -> (hi, lo) BF16 split; element (r, c) of X at X[r + c*ldx], outputs at [r + c*ldo]
// ------------------------------------------------------------------------------------
__global__ void split_bf16_kernel(const float *__restrict__ X, int64_t rows, int64_t cols, int64_t ldx,
                                  bf16 *__restrict__ hi, bf16 *__restrict__ lo, int64_t ldo, int vec) {
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
            __align__(16) bf16 h[8], l[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                h[i] = __float2bfloat16_rn(v[i]);
                l[i] = __float2bfloat16_rn(v[i] - __bfloat162float(h[i]));
            }
            // ldo is a multiple of 8 and r0 + 8 <= ldo, so whole 16-byte groups are written
            *reinterpret_cast<uint4 *>(hi + r0 + c * ldo) = *reinterpret_cast<const uint4 *>(h);
            *reinterpret_cast<uint4 *>(lo + r0 + c * ldo) = *reinterpret_cast<const uint4 *>(l);
        }
    }
}

int split_bf16(rla_ctx *ctx, const float *X, int64_t rows, int64_t cols, int64_t ldx, bf16 *hi, bf16 *lo, int64_t ldo) {
    if (rows <= 0 || cols <= 0) return RLA_OK;
    if (ldo % 8 != 0 || ldo < rows || ((uintptr_t)hi | (uintptr_t)lo) % 16 != 0)
        return set_error(ctx, RLA_E_ARG, "split_bf16: output leading dimension must be a multiple of 8");
    const int vec = (ldx % 4 == 0) && ((uintptr_t)X % 16 == 0);
    const int64_t groups = (rows + 7) / 8;
    const unsigned gx = (unsigned)std::min<int64_t>(ceil_div(groups, 256), 4096);
    const unsigned gy = (unsigned)std::min<int64_t>(cols, 65535);
    split_bf16_kernel<<<dim3(gx, gy), 256, 0, ctx->stream>>>(X, rows, cols, ldx, hi, lo, ldo, vec);
    return check_launch(ctx, "split_bf16");
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
constexpr uint32_t TC_A_BYTES = TC_BM * TC_BK * 2;  // 8 KB per operand half

struct TcParams {
    int M, N, K;      // op(A) is M x K, B is K x N
    int BN;           // tile columns (multiple of 16; > 256 only as two halves of a multiple of 32)
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
};

__global__ void __launch_bounds__(TC_THREADS, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
               const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo, TcParams p) {
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t b_bytes = (uint32_t)p.BN * TC_BK * 2;
    const uint32_t stage_bytes = 2 * TC_A_BYTES + 2 * b_bytes;
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
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_ahi)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_alo)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_bhi)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_blo)) : "memory");
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
                const uint32_t a_hi = st, a_lo = st + TC_A_BYTES, b_hi = st + 2 * TC_A_BYTES, b_lo = b_hi + b_bytes;
                const int k0 = (kb0 + kb) * TC_BK;
                mbar_arrive_expect_tx(full_bar(s), tx);
                if (p.a_kmajor) {
                    tma_load_2d(a_hi, &map_ahi, full_bar(s), k0, m0);
                    tma_load_2d(a_lo, &map_alo, full_bar(s), k0, m0);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        tma_load_2d(a_hi + q * 2048u, &map_ahi, full_bar(s), m0 + 32 * q, k0);
                        tma_load_2d(a_lo + q * 2048u, &map_alo, full_bar(s), m0 + 32 * q, k0);
                    }
                }
                for (int c = 0; c < p.nch; ++c) {
                    const uint32_t off = (uint32_t)c * chunk_cols * TC_BK * 2;
                    tma_load_2d(b_hi + off, &map_bhi, full_bar(s), k0, c * (int)chunk_cols);
                    tma_load_2d(b_lo + off, &map_blo, full_bar(s), k0, c * (int)chunk_cols);
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
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb % p.stages;
                const uint32_t ph = (uint32_t)(kb / p.stages) & 1u;
                if (!mbar_wait(full_bar(s), ph, p.status, p.wait_ns)) break;
                tc_fence_after();
                const uint32_t st = base + (uint32_t)s * stage_bytes;
                const uint32_t a_hi = st, a_lo = st + TC_A_BYTES, b_hi = st + 2 * TC_A_BYTES, b_lo = b_hi + b_bytes;
#pragma unroll
                for (int kk = 0; kk < TC_BK / 16; ++kk) {
                    uint64_t dah, dal;
                    if (p.a_kmajor) {  // 128 rows of 64 B, 8-row groups 512 B apart; k-step = 32 B
                        dah = sdesc_sw64(a_hi + kk * 32u, 16u, 512u);
                        dal = sdesc_sw64(a_lo + kk * 32u, 16u, 512u);
                    } else {           // 32-row blocks of 2 KB; k rows 64 B apart; k-step = 16 rows
                        dah = sdesc_sw64(a_hi + kk * 1024u, 2048u, 512u);
                        dal = sdesc_sw64(a_lo + kk * 1024u, 2048u, 512u);
                    }
                    for (int c = 0; c < p.nch; ++c) {
                        const uint32_t off = (uint32_t)c * chunk_cols * TC_BK * 2 + kk * 32u;
                        const uint64_t dbh = sdesc_sw64(b_hi + off, 16u, 512u);
                        const uint64_t dbl = sdesc_sw64(b_lo + off, 16u, 512u);
                        const uint32_t d = tmem + (uint32_t)c * chunk_cols;
                        mma_bf16(d, dah, dbh, idesc, (kb | kk) != 0 ? 1u : 0u);
                        mma_bf16(d, dah, dbl, idesc, 1u);
                        mma_bf16(d, dal, dbh, idesc, 1u);
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
    for (int c0 = 0; c0 < p.BN; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
        if (row < p.M) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = c0 + j;
                if (col < p.N) out[row + (int64_t)col * p.ldo] = ok ? __uint_as_float(r[j]) : 0.f;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols) : "memory");
    }
}

// C(i, j) = alpha * sum_s P[s](i, j) + beta * C(i, j), splits added in order.
template <class TC>
__global__ void splitk_reduce_kernel(const float *__restrict__ P, int splits, int64_t split_stride, int64_t ldp,
                                     int64_t M, int64_t N, TC *C, int64_t ldc, double alpha, double beta,
                                     int beta_zero) {
    for (int64_t j = blockIdx.y; j < N; j += gridDim.y) {
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
            double acc = 0.0;
            for (int s = 0; s < splits; ++s) acc += (double)P[s * split_stride + i + j * ldp];
            TC *cp = C + i + j * ldc;
            double r = alpha * acc;
            if (!beta_zero) r += beta * (double)*cp;
            *cp = (TC)r;
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

TcPlan tc_plan(const rla_ctx *ctx, int64_t M, int64_t N, int64_t K, int splits) {
    TcPlan pl;
    const int64_t nb = std::min<int64_t>(N, 288);
    pl.BN = (int)(nb <= 256 ? ceil_div(nb, 16) * 16 : ceil_div(nb, 32) * 32);
    pl.nch = pl.BN > 256 ? 2 : 1;
    const int64_t b_bytes = (int64_t)pl.BN * TC_BK * 2;
    const int64_t stage = 2 * TC_A_BYTES + 2 * b_bytes;
    const int64_t budget = ctx->smem_optin - 1024 - 256;
    pl.stages = (int)std::max<int64_t>(2, std::min<int64_t>(8, budget / stage));
    pl.smem = (size_t)(pl.stages * stage + 1024 + 256);
    pl.tmem_cols = 32;
    while ((int)pl.tmem_cols < pl.BN) pl.tmem_cols <<= 1;
    const int64_t mt = ceil_div(M, TC_BM), nkb = ceil_div(K, TC_BK);
    pl.mt = (int)mt;
    pl.nkb = (int)nkb;
    if (splits <= 0) {
        // model: waves x k-blocks per split x MMA time per k-block, plus partial-tile traffic
        const double t_kb = 0.45e-6 * (double)pl.BN / 288.0, bw = 6.0e12;
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

template <class TC>
int tc_gemm_bf16x3(rla_ctx *ctx, int64_t M, int64_t N, int64_t K, const bf16 *Ahi, const bf16 *Alo, int64_t lda,
                   int a_kmajor, const bf16 *Bhi, const bf16 *Blo, int64_t ldb, TC *C, int64_t ldc, double alpha,
                   double beta, int splits) {
    if (M <= 0 || N <= 0) return RLA_OK;
    if (M >= (1ll << 31) || K >= (1ll << 31)) return set_error(ctx, RLA_E_UNSUPPORTED, "tensor-core GEMM: dimension above 2^31");
    int *status = nullptr;
    RLA_TRY(tc_status_get(ctx, &status));
    for (int64_t n0 = 0; n0 < N; n0 += 288) {
        const int64_t nb = std::min<int64_t>(288, N - n0);
        TcPlan pl = tc_plan(ctx, M, nb, K, splits);
        CUtensorMap mah, mal, mbh, mbl;
        if (a_kmajor) {
            RLA_TRY(make_map(ctx, &mah, Ahi, K, M, lda, TC_BK, TC_BM));
            RLA_TRY(make_map(ctx, &mal, Alo, K, M, lda, TC_BK, TC_BM));
        } else {
            RLA_TRY(make_map(ctx, &mah, Ahi, M, K, lda, 32, TC_BK));
            RLA_TRY(make_map(ctx, &mal, Alo, M, K, lda, 32, TC_BK));
        }
        const uint32_t box_n = (uint32_t)(pl.BN / pl.nch);
        RLA_TRY(make_map(ctx, &mbh, Bhi + n0 * ldb, K, nb, ldb, TC_BK, box_n));
        RLA_TRY(make_map(ctx, &mbl, Blo + n0 * ldb, K, nb, ldb, TC_BK, box_n));
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
                   out, ldo, sstride, status, ctx->wait_ns};
        RLA_CUDA_TRY(ctx, set_smem_max(tc_gemm_kernel));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (ctx->timing) {
            RLA_CUDA_TRY(ctx, cudaEventCreate(&e0));
            RLA_CUDA_TRY(ctx, cudaEventCreate(&e1));
            RLA_CUDA_TRY(ctx, cudaEventRecord(e0, ctx->stream));
        }
        tc_gemm_kernel<<<dim3(pl.mt, pl.splits), TC_THREADS, pl.smem, ctx->stream>>>(mah, mal, mbh, mbl, p);
        RLA_TRY(check_launch(ctx, "tc_gemm"));
        if (ctx->timing) {
            RLA_CUDA_TRY(ctx, cudaEventRecord(e1, ctx->stream));
            ctx->timed[0].emplace_back(e0, e1);
        }
        if (!direct) {
            const unsigned gx = (unsigned)std::min<int64_t>(ceil_div(M, 256), 1024);
            const unsigned gy = (unsigned)std::min<int64_t>(nb, 65535);
            splitk_reduce_kernel<TC><<<dim3(gx, gy), 256, 0, ctx->stream>>>(out, pl.splits, sstride, ldo, M, nb, Cn, ldc,
                                                                            alpha, beta, beta == 0.0);
            RLA_TRY(check_launch(ctx, "splitk_reduce"));
        }
    }
    return RLA_OK;
}

template int tc_gemm_bf16x3<float>(rla_ctx *, int64_t, int64_t, int64_t, const bf16 *, const bf16 *, int64_t, int,
                                   const bf16 *, const bf16 *, int64_t, float *, int64_t, double, double, int);
template int tc_gemm_bf16x3<double>(rla_ctx *, int64_t, int64_t, int64_t, const bf16 *, const bf16 *, int64_t, int,
                                    const bf16 *, const bf16 *, int64_t, double *, int64_t, double, double, int);

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
