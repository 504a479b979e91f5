// rla_internal.cuh -- shared internals of librla_b200 (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <utility>
#include <string>
#include <vector>

#include "rla_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "librla_b200 is written for sm_100a (B200) only"
#endif

namespace rla {

constexpr unsigned FULL = 0xffffffffu;

// ------------------------------------------------------------------------------------
// Context
// ------------------------------------------------------------------------------------
struct Scratch {
    void *ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace rla

struct rla_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    int sm_count = 148;
    int smem_optin = 227 * 1024;
    std::string last_error;
    rla::Scratch scratch;    // grow-only workspace (partials, transposes, WHT buffers)
    rla::Scratch counters;   // zero-initialised ints for last-arriver fix-ups (self-resetting)
    int64_t scratch_high_water = 0;
    cudaMemPool_t pool = nullptr;  // context-owned stream-ordered pool, keeps freed memory mapped
    int *tc_status = nullptr;  // non-zero after a tensor-core kernel's bounded wait ran out
    uint64_t wait_ns = 2000000000ull;  // limit of a device-side pipeline wait (rla_ctx_set_wait_limit)
    bool timing = false;       // record CUDA events around timed kernel classes
    // classes: 0 tensor-core GEMM, 1 IHS fused pass over A, 2 IHS compressor apply,
    // 3 Sampling L2Norm weights pass over A
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed[4];
};

namespace rla {

int set_error(rla_ctx *ctx, int code, const char *fmt, ...);

#define RLA_CUDA_TRY(ctx, expr)                                                            \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess) {                                                           \
            return ::rla::set_error((ctx), (_e == cudaErrorMemoryAllocation) ? RLA_E_OOM   \
                                                                             : RLA_E_CUDA, \
                                    "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e),       \
                                    __FILE__, __LINE__);                                   \
        }                                                                                  \
    } while (0)

#define RLA_TRY(expr)                 \
    do {                              \
        int _rc = (expr);             \
        if (_rc != RLA_OK) return _rc; \
    } while (0)

// Workspace of at least `bytes` bytes on the context's stream (grow-only).
int scratch_get(rla_ctx *ctx, size_t bytes, void **out);
// Zero-initialised int32 counters (at least n); kernels leave them at zero on exit.
int counters_get(rla_ctx *ctx, size_t n, int **out);
int check_launch(rla_ctx *ctx, const char *what);
// Largest dynamic shared memory a block may use on this device (set by rla_ctx_create).
// Kernels' MaxDynamicSharedMemorySize attribute is process-wide and shared by every host
// thread, so set_smem_max always raises it to the most the kernel can take (never to a
// per-call size another thread could lower before its own launch).
extern int g_smem_optin;
template <class K>
inline cudaError_t set_smem_max(K kern) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, reinterpret_cast<const void *>(kern));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, g_smem_optin - (int)a.sharedSizeBytes);
}
// Stream-ordered allocation from the context's pool (memory stays mapped between calls, so
// repeated calls of the same size do not remap device memory).
template <class P>
inline cudaError_t pool_malloc_s(rla_ctx *ctx, P **p, size_t bytes, cudaStream_t s) {
    return cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, ctx->pool, s);
}

inline int ceil_div_i(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t next_pow2(int64_t n) {
    int64_t p = 1;
    while (p < n) p <<= 1;
    return p;
}
inline int ilog2(int64_t n) {
    int k = 0;
    while ((int64_t(1) << k) < n) ++k;
    return k;
}

// ------------------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw: "Parallel random
// numbers: as easy as 1, 2, 3", SC'11).  key = seed, counter = (stream, index).
// ------------------------------------------------------------------------------------
struct P4 {
    uint32_t x, y, z, w;
};

__host__ __device__ inline P4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                            uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c0;
        uint64_t p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    return P4{c0, c1, c2, c3};
}

// Draw streams: distinct counter words so different draw kinds never share numbers.
enum : uint32_t {
    STREAM_SPARSE = 1,
    STREAM_COUNT = 2,
    STREAM_SRHT_SIGNS = 3,
    STREAM_SRHT_ROWS = 4,
    STREAM_FJLT_K = 5,
    STREAM_FJLT_SIGNS = 6,
    STREAM_GAUSS = 7,
};

struct Rng {
    uint32_t k0, k1;  // seed
    uint32_t epoch;   // draw count (update_compressor! advances it)
    __host__ __device__ P4 at(uint32_t stream, uint64_t index) const {
        return philox4x32_10((uint32_t)index, (uint32_t)(index >> 32), epoch, stream, k0, k1);
    }
};

// Uniform integer in [0, range) by Lemire's multiply-shift with rejection.  `next`
// yields 32-bit words; the rejection loop is bounded (probability of 64 rejections in a
// row is below 2^-64 for any range).
template <class Next>
__host__ __device__ inline uint32_t uniform_below(uint32_t range, Next &&next) {
    uint64_t m = (uint64_t)next() * range;
    uint32_t l = (uint32_t)m;
    if (l < range) {
        uint32_t t = (uint32_t)(-range) % range;
        for (int it = 0; it < 64 && l < t; ++it) {
            m = (uint64_t)next() * range;
            l = (uint32_t)m;
        }
    }
    return (uint32_t)(m >> 32);
}

__host__ __device__ inline double u01_open_d(uint32_t a, uint32_t b) {
    // 53-bit uniform in (0, 1]
    uint64_t v = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return ((double)v + 1.0) * (1.0 / 9007199254740992.0);
}

// Per-thread word source over one Philox stream position.
struct WordStream {
    Rng rng;
    uint32_t stream;
    uint64_t base;   // index of the first block
    uint64_t block = 0;
    int used = 4;
    P4 cur{};
    __device__ uint32_t operator()() {
        if (used == 4) {
            cur = rng.at(stream, base + block++);
            used = 0;
        }
        uint32_t w = used == 0 ? cur.x : used == 1 ? cur.y : used == 2 ? cur.z : cur.w;
        ++used;
        return w;
    }
};

// Two N(0,1) draws by Box-Muller from four 32-bit words (53-bit uniforms in (0, 1]).
__device__ inline double normal_pair(WordStream &ws, double *second) {
    double u1 = u01_open_d(ws(), ws());
    double u2 = u01_open_d(ws(), ws());
    double r = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    *second = r * sn;
    return r * cs;
}

// ------------------------------------------------------------------------------------
// Element-type helpers
// ------------------------------------------------------------------------------------
template <class T>
struct Vec4;
template <>
struct Vec4<float> {
    using type = float4;
};
template <>
struct Vec4<double> {
    using type = double4;
};

inline size_t dtype_size(int dtype) { return dtype == RLA_F64 ? 8 : 4; }

// Contiguous split of `total` work units over W workers (stream-K style): worker g owns
// [start(g), start(g+1)); the first `rem` workers take base+1 units, the rest base.
struct Split {
    int64_t total = 0, base = 0, rem = 0;
    int W = 1;
    static Split make(int64_t total, int W) {
        Split s;
        s.total = total;
        s.W = W;
        s.base = total / W;
        s.rem = total % W;
        return s;
    }
    __host__ __device__ int64_t start(int g) const { return (int64_t)g * base + (g < rem ? g : rem); }
    __host__ __device__ int owner(int64_t u) const {
        const int64_t cut = rem * (base + 1);
        if (u < cut) return (int)(u / (base + 1));
        return (int)(rem + (u - cut) / base);  // base >= 1 whenever u >= cut
    }
    // Partial-sum slot of worker g for a segment [vbeg, vbeg+len) it shares: a worker's
    // first segment uses slot 2g, its last (when it started in an earlier segment) 2g+1.
    __host__ __device__ int slot(int g, int64_t vbeg) const { return 2 * g + (start(g) < vbeg ? 1 : 0); }
};


// CUDA events around a timed launch (rla_ctx_set_timing); no-ops while timing is off.
inline cudaEvent_t timing_begin(rla_ctx *ctx) {
    cudaEvent_t e0 = nullptr;
    if (ctx->timing && cudaEventCreate(&e0) == cudaSuccess) cudaEventRecord(e0, ctx->stream);
    return e0;
}
inline void timing_end(rla_ctx *ctx, int cls, cudaEvent_t e0) {
    if (!e0) return;
    cudaEvent_t e1 = nullptr;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return;
    }
    cudaEventRecord(e1, ctx->stream);
    ctx->timed[cls].emplace_back(e0, e1);
}

}  // namespace rla

// ------------------------------------------------------------------------------------
// Sketch state (device-resident draws and derived tables)
// ------------------------------------------------------------------------------------
struct rla_sketch {
    rla_sketch_params p{};
    int64_t n_rows = 0, n_cols = 0;
    int64_t s = 0, L = 0;     // compression dim, long dim
    int64_t nnz = 1;          // entries per long index (SparseSign / CountSketch)
    int64_t N = 0;            // padded size (SRHT / FJLT)
    double scale = 1.0;       // see rla_sketch_info
    double sparsity = 0.0;
    uint64_t draw_count = 0;
    int device = 0;

    // SparseSign / CountSketch
    int32_t *bucket = nullptr;     // [L*nnz] compress-side bucket per (j, e), sorted within j
    uint8_t *negative = nullptr;   // [L*nnz] 1 when the value is -scale
    uint32_t *meta = nullptr;      // tile-blocked (bucket | deferred << 30 | neg << 31)
    uint32_t *tile_flags = nullptr;  // per 128-element tile: 0, SLOW, or (first extra round << 8) | rounds
    uint32_t *extra = nullptr;     // deferred items: 32 words (one per lane) per extra round
    int64_t extra_rounds_cap = 0;
    int batch_mode = 0;            // 1: CountSketch schedule over 512-element batches (see rla_sketch.cu)
    int64_t *tp_ptr = nullptr;     // sparse-operand plan (rla_sparse_op.cu): [s+1] offsets per bucket
    int32_t *tp_idx = nullptr;     // [L*nnz] entries j*nnz+slot by bucket, j increasing
    uint64_t tp_version = 0;       // draw_count the plan was built for
    // SRHT
    int32_t *rows = nullptr;       // [s] sampled padded rows (op)
    uint32_t *signbits = nullptr;  // [ceil(N/32)] bit r = 1 means +1
    uint4 *sign_tl = nullptr;      // fused compress kernel: per (chunk, thread) sign bits in register order (FP32: 64 as uint2, FP64: 128)
    int32_t *p2_ptr = nullptr;     // expand tables: per low-bit position, samples sorted
    int32_t *p2_list = nullptr;
    int64_t chunk = 0;             // WHT chunk length used by the expand tables
    // FJLT: compress matrix Kc (s x N) in CSR, and its transpose (N x s) in CSR
    int32_t *k_ptr = nullptr, *k_col = nullptr;
    void *k_val = nullptr;
    int32_t *kt_ptr = nullptr, *kt_row = nullptr;
    void *kt_val = nullptr;
    int64_t k_nnz = 0;
    // Gaussian: op, column-major n_rows x n_cols
    void *dense = nullptr;
    // Sampling (rla_sampling.cu)
    int s_dist = 0;                // RLA_DIST_*
    bool s_replace = false;
    int64_t s_beta = 1;            // Agmon subset size
    int64_t *sidx = nullptr;       // [s] sampled indices (0-based), the recipe's idx
    int64_t *splan = nullptr;      // expand plan: [s] targets, [s+1] run offsets, [s] positions, U
    int64_t *s_err = nullptr;      // precondition flags of the last draw (0: none)
    double *sweights = nullptr;    // [L] L2Norm weights of the last update
    bool s_has_weights = false;
};
