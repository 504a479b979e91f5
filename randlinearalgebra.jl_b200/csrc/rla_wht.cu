// rla_wht.cu -- Walsh-Hadamard based sketches (SRHT, FJLT).
//
// The reference applies SRHT block by block: zero a padding buffer, copy A, run the
// natural-order fwht! per column (log2 N passes over the column), gather the sampled
// rows (srht.jl:220-286, fwht.jl:21-70).  Here the left compress (S*A on column-major A)
// is one pass over A:
//
//   N = N1 * 2^CH with CH = 14 (FP32) / 13 (FP64).  For a padded column x,
//   y[r] = sum_c (-1)^popc(r1 & c) * Z_c[r2],  r = r1*2^CH + r2,
//   where Z_c = H_{2^CH} (D x)[c*2^CH : (c+1)*2^CH] is the natural-order WHT of chunk c.
//
// A CTA of 256 threads holds one chunk in registers (16 16-byte vectors per thread) and
// transforms its bits in three register passes, moving between them through a
// bank-conflict-free swizzled 64 KB shared buffer (sign flip fused into the first pass);
// each sampled row then accumulates +-Z_c[r2].  Columns are split over the persistent grid
// (stream-K); a column shared by several CTAs is finished by the last CTA to arrive, which
// adds the partial accumulators in CTA order, so results are reproducible bit for bit.
#include <mutex>

#include "rla_internal.cuh"

namespace rla {

template <class T>
struct WhtCfg;
// The fused compress kernel's CTA: NT = 256 threads; a 16-byte vector holds 2^VB elements;
// a chunk has CH = VB + 12 bits (2^14 FP32 or 2^13 FP64 elements, 64 KB either way), and each
// thread holds 16 vectors of it.
template <>
struct WhtCfg<float> {
    static constexpr int VB = 2, CH = 14, NT = 256;
    using V = float4;
    using SignW = uint2;  // 64 sign bits per thread and chunk
};
template <>
struct WhtCfg<double> {
    static constexpr int VB = 1, CH = 13, NT = 256;
    using V = double2;
    using SignW = uint32_t;  // 32 sign bits per thread and chunk
};

// Register storage of one thread's 2^TB chunk elements.  FP32 values live in float2
// pairs so that the butterflies over every register-index bit but the lowest use the
// packed sm_100 FP32x2 instructions (a+b as fadd2, a-b as ffma2(b, -1, a), both exact
// to one rounding like the scalar forms).
template <class T, int TB>
struct Regs;

template <int TB>
struct Regs<float, TB> {
    float2 d[(1 << TB) / 2];
    __device__ __forceinline__ float get(int q) const { return (q & 1) ? d[q >> 1].y : d[q >> 1].x; }
    __device__ __forceinline__ void set(int q, float v) {
        if (q & 1) d[q >> 1].y = v;
        else d[q >> 1].x = v;
    }
    __device__ __forceinline__ void wht() {
#pragma unroll
        for (int p = 0; p < (1 << TB) / 2; ++p) {
            const float a = d[p].x, b = d[p].y;
            d[p].x = a + b;
            d[p].y = a - b;
        }
        const float2 m1 = make_float2(-1.f, -1.f);
#pragma unroll
        for (int h = 0; h < TB - 1; ++h)
#pragma unroll
            for (int p = 0; p < (1 << TB) / 2; ++p)
                if (!(p & (1 << h))) {
                    const float2 a = d[p], b = d[p | (1 << h)];
                    d[p] = __fadd2_rn(a, b);
                    d[p | (1 << h)] = __ffma2_rn(b, m1, a);
                }
    }
};

template <int TB>
struct Regs<double, TB> {
    double d[1 << TB];
    __device__ __forceinline__ double get(int q) const { return d[q]; }
    __device__ __forceinline__ void set(int q, double v) { d[q] = v; }
    __device__ __forceinline__ void wht() {
#pragma unroll
        for (int h = 0; h < TB; ++h)
#pragma unroll
            for (int q = 0; q < (1 << TB); ++q)
                if (!(q & (1 << h))) {
                    const double a = d[q], b = d[q | (1 << h)];
                    d[q] = a + b;
                    d[q | (1 << h)] = a - b;
                }
    }
};

template <class T>
struct SrhtParams {
    const T *X;
    int64_t x_ld;  // element (j, v) at X[j + v*x_ld]
    int64_t L, N;
    const uint4 *sign_tl;  // per (chunk, thread): sign bits in pass-A register order
    const int32_t *rows;
    int64_t s_lo;
    int s_cnt;
    T *Y;
    int64_t y_es, y_vs;
    T alpha, beta;
    int beta_zero;
    T *partials;
    int *counters;
    int64_t cpv;  // chunks per column
    Split split;
};

template <class T>
__device__ __forceinline__ T flip(T x, uint32_t keep) {
    if constexpr (sizeof(T) == 4) {
        return __uint_as_float(__float_as_uint(x) ^ ((~keep & 1u) << 31));
    } else {
        return keep & 1u ? x : -x;
    }
}

// Element address of chunk element e in the shared buffer: the 16-byte slot bits
// [VB, VB+3) XOR bits [VB+4, VB+7).  Every 16-byte access of the kernel below then puts the
// 8 lanes of each quarter warp on 8 different slots of a 128-byte row: no bank conflicts.
template <int VB>
__device__ __forceinline__ int swzv(int e) { return e ^ (((e >> (VB + 4)) & 7) << VB); }

// Vector m (elements 2^VB*m ...) of a thread's registers.
__device__ __forceinline__ void set_vec(Regs<float, 6> &r, int m, float4 q) {
    r.d[2 * m] = make_float2(q.x, q.y);
    r.d[2 * m + 1] = make_float2(q.z, q.w);
}
__device__ __forceinline__ void set_vec(Regs<double, 5> &r, int m, double2 q) {
    r.d[2 * m] = q.x;
    r.d[2 * m + 1] = q.y;
}
__device__ __forceinline__ float4 get_vec(const Regs<float, 6> &r, int m) {
    return make_float4(r.d[2 * m].x, r.d[2 * m].y, r.d[2 * m + 1].x, r.d[2 * m + 1].y);
}
__device__ __forceinline__ double2 get_vec(const Regs<double, 5> &r, int m) {
    return make_double2(r.d[2 * m], r.d[2 * m + 1]);
}

__device__ __forceinline__ uint32_t sign_word(uint2 sg, int q) { return q < 32 ? sg.x : sg.y; }
__device__ __forceinline__ uint32_t sign_word(uint32_t sg, int) { return sg; }

// Radix-2 butterflies over bits 0..3 of the index of a thread's 16 vectors (the elements of
// a vector are carried through): packed FP32x2 adds and subtracts, or FP64 scalar ones.
__device__ __forceinline__ void wht_vec16(Regs<float, 6> &r) {
    const float2 m1 = make_float2(-1.f, -1.f);
#pragma unroll
    for (int h = 0; h < 4; ++h)
#pragma unroll
        for (int m = 0; m < 16; ++m)
            if (!(m & (1 << h))) {
#pragma unroll
                for (int o = 0; o < 2; ++o) {
                    const float2 a = r.d[2 * m + o], b = r.d[2 * (m | (1 << h)) + o];
                    r.d[2 * m + o] = __fadd2_rn(a, b);
                    r.d[2 * (m | (1 << h)) + o] = __ffma2_rn(b, m1, a);
                }
            }
}
__device__ __forceinline__ void wht_vec16(Regs<double, 5> &r) {
#pragma unroll
    for (int h = 0; h < 4; ++h)
#pragma unroll
        for (int m = 0; m < 16; ++m)
            if (!(m & (1 << h))) {
#pragma unroll
                for (int o = 0; o < 2; ++o) {
                    const double a = r.d[2 * m + o], b = r.d[2 * (m | (1 << h)) + o];
                    r.d[2 * m + o] = a + b;
                    r.d[2 * (m | (1 << h)) + o] = a - b;
                }
            }
}

// Pass-A loads of the chunk at cbase of column xv: register q = i | k<<VB (i < 2^VB, k < 16)
// holds element i | t<<VB | k<<(VB+8).
template <class T, bool VEC>
__device__ __forceinline__ void load_chunk(const T *__restrict__ xv, int64_t cbase, int64_t L, int t,
                                           Regs<T, WhtCfg<T>::VB + 4> &r) {
    constexpr int VB = WhtCfg<T>::VB, CH = WhtCfg<T>::CH, VW = 1 << VB;
    using V = typename WhtCfg<T>::V;
    if (VEC && cbase + (1 << CH) <= L) {  // whole chunk inside the column: no per-vector checks
        const V *src = reinterpret_cast<const V *>(xv + cbase) + t;
#pragma unroll
        for (int k = 0; k < 16; ++k) set_vec(r, k, __ldg(src + (k << 8)));
        return;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int64_t e0 = cbase + ((int64_t)t << VB) + ((int64_t)k << (VB + 8));
        if (VEC && e0 + VW <= L) {
            set_vec(r, k, __ldg(reinterpret_cast<const V *>(xv + e0)));
        } else {
#pragma unroll
            for (int i = 0; i < VW; ++i) r.set(k * VW + i, (e0 + i < L) ? __ldg(xv + e0 + i) : T(0));
        }
    }
}

// Fused compress, one CTA of 256 threads per chunk at a time.  Chunk element bits
// (e = 0..2^CH-1) by pass, lane l, warp w:
//   pass A (after the coalesced load): register q = i | k<<VB holds e = i | t<<VB | k<<(VB+8);
//          butterflies over e bits [0, VB) and [VB+8, VB+12);
//   pass B: vectors m hold e = m<<VB | t<<(VB+4); butterflies over e bits [VB, VB+4);
//   pass C: vectors m hold e = (l&15)<<VB | m<<(VB+4) | (l>>4)<<(VB+8) | w<<(VB+9);
//          butterflies over e bits [VB+4, VB+8).
// The chunk then holds H_c (D x) in natural order, and each thread's SPT sampled rows
// r = r1*2^CH + r2 add (-1)^popc(r1 & c) * Z_c[r2]:
//   y[r] = sum_c (-1)^popc(r1 & c) * Z_c[r2],  Z_c = H_{2^CH} (D x)[c*2^CH : (c+1)*2^CH].
// Columns are split over the persistent grid (stream-K); a column shared by several CTAs is
// finished by the last CTA to arrive, which adds the partial accumulators in CTA order, so
// results are reproducible bit for bit.
template <class T, bool VEC, int SPT>
__global__ void __launch_bounds__(256, 2) srht_fused_kernel(SrhtParams<T> p) {
    constexpr int VB = WhtCfg<T>::VB, CH = WhtCfg<T>::CH, NT = 256;
    using V = typename WhtCfg<T>::V;
    using SignW = typename WhtCfg<T>::SignW;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Z = reinterpret_cast<T *>(smem_raw);
    __shared__ int last_flag;
    const int t = threadIdx.x, lane = t & 31, wp = t >> 5;
    const int g = blockIdx.x;
    const int64_t u0 = p.split.start(g), u1 = p.split.start(g + 1);
    if (u0 >= u1) return;
    // With 16 samples per thread their packed rows live in shared memory (after the chunk),
    // which keeps the kernel within 128 registers; each thread reads only its own entries.
    constexpr bool SR_SMEM = SPT > 8;
    uint32_t *sr_s = reinterpret_cast<uint32_t *>(Z + (1 << CH));
    T acc[SPT];
    uint32_t sr[SR_SMEM ? 1 : SPT];
#pragma unroll
    for (int k = 0; k < SPT; ++k) {
        const int i = t + k * NT;
        acc[k] = T(0);
        const uint32_t row = i < p.s_cnt ? (uint32_t)__ldg(p.rows + p.s_lo + i) : 0u;
        const uint32_t packed = ((row >> CH) << CH) | (uint32_t)swzv<VB>((int)(row & ((1u << CH) - 1)));
        if constexpr (SR_SMEM) sr_s[k * NT + t] = packed;
        else sr[k] = packed;
    }
    // Per-thread bases.  The swizzle flips the slot bits only, so every address below is a
    // base (XOR a compile-time pattern) plus a compile-time offset:
    //   pass A, vector k: baseA + k<<(VB+8)
    //   pass B, vector m: baseB ^ (m&7)<<VB, + (m>>3)<<(VB+3)
    //   pass C, vector m: baseC ^ (m&7)<<VB, + m<<(VB+4)
    const int baseA = swzv<VB>(t << VB);
    const int baseB = (t << (VB + 4)) | ((t & 7) << VB);
    const int baseC = ((lane & 15) << VB) | ((lane >> 4) << (VB + 8)) | (wp << (VB + 9));
    Regs<T, VB + 4> r;
    SignW sg;
    const SignW *sign_tl = reinterpret_cast<const SignW *>(p.sign_tl);
    int64_t v = u0 / p.cpv, c = u0 - v * p.cpv;
    load_chunk<T, VEC>(p.X + v * p.x_ld, c << CH, p.L, t, r);
    sg = __ldg(sign_tl + c * NT + t);
    for (int64_t u = u0; u < u1; ++u) {
        // ---- pass A: sign flip, butterflies over the register bits, vector stores ----
#pragma unroll
        for (int q = 0; q < (16 << VB); ++q) r.set(q, flip<T>(r.get(q), sign_word(sg, q) >> (q & 31)));
        r.wht();
#pragma unroll
        for (int k = 0; k < 16; ++k) *reinterpret_cast<V *>(Z + baseA + (k << (VB + 8))) = get_vec(r, k);
        __syncthreads();
        // ---- passes B and C (each vector is read and written by one thread) ----
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            const int base = pass == 0 ? baseB : baseC;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int off = pass == 0 ? ((m >> 3) << (VB + 3)) : (m << (VB + 4));
                set_vec(r, m, *reinterpret_cast<const V *>(Z + (base ^ ((m & 7) << VB)) + off));
            }
            wht_vec16(r);
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int off = pass == 0 ? ((m >> 3) << (VB + 3)) : (m << (VB + 4));
                *reinterpret_cast<V *>(Z + (base ^ ((m & 7) << VB)) + off) = get_vec(r, m);
            }
            if (pass == 0) __syncthreads();
        }
        // ---- prefetch the next chunk while the sampled rows are accumulated ----
        const int64_t vcur = v, ccur = c;
        if (u + 1 < u1) {
            if (++c == p.cpv) {
                c = 0;
                ++v;
            }
            load_chunk<T, VEC>(p.X + v * p.x_ld, c << CH, p.L, t, r);
            sg = __ldg(sign_tl + c * NT + t);
        }
        __syncthreads();
        const uint32_t cc = (uint32_t)ccur;
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
            const uint32_t srk = SR_SMEM ? sr_s[k * NT + t] : sr[k % (SR_SMEM ? 1 : SPT)];
            const T z = Z[srk & ((1u << CH) - 1)];
            acc[k] += (__popc((srk >> CH) & cc) & 1) ? -z : z;
        }
        __syncthreads();
        const bool col_done = (u + 1 == u1) || (ccur + 1 == p.cpv);
        if (!col_done) continue;
        // ---- column finished in this CTA's range ----
        const int64_t vbeg = vcur * p.cpv;
        const bool exclusive = (u0 <= vbeg) && (vbeg + p.cpv <= u1);
        if (exclusive) {
#pragma unroll
            for (int k = 0; k < SPT; ++k) {
                const int i = t + k * NT;
                if (i < p.s_cnt) {
                    T *yp = p.Y + (p.s_lo + i) * p.y_es + vcur * p.y_vs;
                    T res = p.alpha * acc[k];
                    if (!p.beta_zero) res += p.beta * *yp;
                    *yp = res;
                }
                acc[k] = T(0);
            }
        } else {
            T *part = p.partials + (int64_t)p.split.slot(g, vbeg) * p.s_cnt;
#pragma unroll
            for (int k = 0; k < SPT; ++k) {
                const int i = t + k * NT;
                if (i < p.s_cnt) part[i] = acc[k];
                acc[k] = T(0);
            }
            __threadfence();
            __syncthreads();
            const int gf = p.split.owner(vbeg), gl = p.split.owner(vbeg + p.cpv - 1);
            if (t == 0) last_flag = (atomicAdd(&p.counters[vcur], 1) == gl - gf);
            __syncthreads();
            if (last_flag) {
                __threadfence();
                for (int i = t; i < p.s_cnt; i += NT) {
                    T a = __ldcg(p.partials + (int64_t)p.split.slot(gf, vbeg) * p.s_cnt + i);
#pragma unroll 4
                    for (int gg = gf + 1; gg <= gl; ++gg) a += __ldcg(p.partials + (int64_t)(2 * gg) * p.s_cnt + i);
                    T *yp = p.Y + (p.s_lo + i) * p.y_es + vcur * p.y_vs;
                    T res = p.alpha * a;
                    if (!p.beta_zero) res += p.beta * *yp;
                    *yp = res;
                }
                if (t == 0) p.counters[vcur] = 0;
            }
        }
        __syncthreads();
    }
}

// Launch the fused kernel with the smallest samples-per-thread that holds s_cnt samples.
template <class T, bool VEC>
static void launch_srht_fused(const SrhtParams<T> &p, int grid, size_t smem, cudaStream_t st) {
    // smem: the chunk buffer; room for the packed sample rows is added here when needed
    constexpr int NT = WhtCfg<T>::NT;
    auto go = [&](auto kern) {
        set_smem_max(kern);
        kern<<<grid, NT, smem, st>>>(p);
    };
    const int spt = (p.s_cnt + NT - 1) / NT;
    if (spt > 8) smem += (size_t)NT * 16 * sizeof(uint32_t);
    if (spt <= 1) go(srht_fused_kernel<T, VEC, 1>);
    else if (spt <= 2) go(srht_fused_kernel<T, VEC, 2>);
    else if (spt <= 4) go(srht_fused_kernel<T, VEC, 4>);
    else if (spt <= 8) go(srht_fused_kernel<T, VEC, 8>);
    else go(srht_fused_kernel<T, VEC, 16>);
}

// Largest samples window of one fused launch: 16 samples per thread (4096).
template <class T>
constexpr int srht_window() {
    return WhtCfg<T>::NT * 16;
}

// Per (chunk, thread) sign masks in pass-A register order: bit q is the sign of element
// (q & (2^VB-1)) | t<<VB | (q>>VB)<<(VB+8) of the chunk, so a thread reads its signs with one
// 8-byte (FP32) or 4-byte (FP64) load.
template <class T>
__global__ void sign_table_kernel(const uint32_t *signbits, int64_t nchunks, typename WhtCfg<T>::SignW *out) {
    constexpr int VB = WhtCfg<T>::VB, CH = WhtCfg<T>::CH, NT = WhtCfg<T>::NT;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= nchunks * NT) return;
    const int64_t c = idx / NT;
    const int t = (int)(idx % NT);
    uint32_t w[2] = {0u, 0u};
    for (int q = 0; q < (16 << VB); ++q) {
        const int64_t e = (c << CH) + (q & ((1 << VB) - 1)) + ((int64_t)t << VB) + ((int64_t)(q >> VB) << (VB + 8));
        w[q >> 5] |= ((signbits[e >> 5] >> (e & 31)) & 1u) << (q & 31);
    }
    if constexpr (sizeof(T) == 4) out[idx] = make_uint2(w[0], w[1]);
    else out[idx] = w[0];
}

int build_srht_sign_table(rla_ctx *ctx, rla_sketch *sk) {
    const bool f32 = sk->p.dtype == RLA_F32;
    const int CH = f32 ? WhtCfg<float>::CH : WhtCfg<double>::CH;
    const int NT = f32 ? WhtCfg<float>::NT : WhtCfg<double>::NT;
    if (sk->N < ((int64_t)1 << CH)) return RLA_OK;
    const int64_t nchunks = sk->N >> CH;
    const size_t bytes = (f32 ? sizeof(WhtCfg<float>::SignW) : sizeof(WhtCfg<double>::SignW)) * nchunks * NT;
    if (!sk->sign_tl) RLA_CUDA_TRY(ctx, cudaMalloc(&sk->sign_tl, bytes));
    const int64_t n = nchunks * NT;
    if (f32)
        sign_table_kernel<float><<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(
            sk->signbits, nchunks, reinterpret_cast<WhtCfg<float>::SignW *>(sk->sign_tl));
    else
        sign_table_kernel<double><<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(
            sk->signbits, nchunks, reinterpret_cast<WhtCfg<double>::SignW *>(sk->sign_tl));
    return check_launch(ctx, "sign_table");
}

// Small padded sizes (N < 2^CH): one CTA per column, the whole padded column in
// shared memory, log2(N) butterfly stages.
template <class T>
__global__ void srht_small_kernel(const T *X, int64_t x_ld, int64_t L, int64_t N, int64_t nv,
                                  const uint32_t *signbits, const int32_t *rows, int64_t s, T *Y, int64_t y_es,
                                  int64_t y_vs, T alpha, T beta, int beta_zero) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *z = reinterpret_cast<T *>(smem_raw);
    for (int64_t v = blockIdx.x; v < nv; v += gridDim.x) {
        const T *xv = X + v * x_ld;
        for (int64_t e = threadIdx.x; e < N; e += blockDim.x) {
            T x = e < L ? xv[e] : T(0);
            z[e] = ((signbits[e >> 5] >> (e & 31)) & 1u) ? x : -x;
        }
        __syncthreads();
        for (int64_t h = 1; h < N; h <<= 1) {
            for (int64_t q = threadIdx.x; q < N / 2; q += blockDim.x) {
                const int64_t i = (q / h) * 2 * h + (q % h);
                T a = z[i], b = z[i + h];
                z[i] = a + b;
                z[i + h] = a - b;
            }
            __syncthreads();
        }
        for (int64_t i = threadIdx.x; i < s; i += blockDim.x) {
            T *yp = Y + i * y_es + v * y_vs;
            T res = alpha * z[rows[i]];
            if (!beta_zero) res += beta * *yp;
            *yp = res;
        }
        __syncthreads();
    }
}

// Expand: out(r, v) = alpha*scale*d_r * sum_k H[r, rows_k] x(k, v) + beta*out(r, v), r < L.
// One CTA per (column, output chunk of `ch` rows).
template <class T>
__global__ void srht_expand_kernel(const T *X, int64_t x_es, int64_t x_vs, int64_t L, int64_t N, int64_t nv,
                                   const uint32_t *signbits, const int32_t *rows, const int32_t *p2_ptr,
                                   const int32_t *p2_list, int ch, int log_ch, T *Y, int64_t y_es, int64_t y_vs,
                                   T alpha, T beta, int beta_zero) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *z = reinterpret_cast<T *>(smem_raw);
    const int64_t nchunks = N >> log_ch;
    for (int64_t blk = blockIdx.x; blk < nv * nchunks; blk += gridDim.x) {
        const int64_t v = blk / nchunks, oc = blk % nchunks;
        if ((oc << log_ch) >= L) continue;  // block-uniform: chunk entirely in the padding
        for (int p2 = threadIdx.x; p2 < ch; p2 += blockDim.x) {
            T sum = T(0);
            for (int q = p2_ptr[p2]; q < p2_ptr[p2 + 1]; ++q) {
                const int k = p2_list[q];
                const int64_t r1 = (int64_t)rows[k] >> log_ch;
                const T x = X[(int64_t)k * x_es + v * x_vs];
                sum += (__popcll((unsigned long long)(r1 & oc)) & 1) ? -x : x;
            }
            z[p2] = sum;
        }
        __syncthreads();
        for (int h = 1; h < ch; h <<= 1) {
            for (int q = threadIdx.x; q < ch / 2; q += blockDim.x) {
                const int i = (q / h) * 2 * h + (q % h);
                T a = z[i], b = z[i + h];
                z[i] = a + b;
                z[i + h] = a - b;
            }
            __syncthreads();
        }
        for (int r2 = threadIdx.x; r2 < ch; r2 += blockDim.x) {
            const int64_t r = (oc << log_ch) + r2;
            if (r < L) {
                const T d = ((signbits[r >> 5] >> (r & 31)) & 1u) ? alpha : -alpha;
                T *yp = Y + r * y_es + v * y_vs;
                T res = d * z[r2];
                if (!beta_zero) res += beta * *yp;
                *yp = res;
            }
        }
        __syncthreads();
    }
}

// ---- generic full transform for FJLT: W (N x nv, ld = N) in place --------------------
template <class T>
__global__ void wht_chunk_kernel(T *W, int64_t N, int64_t nv, int ch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *z = reinterpret_cast<T *>(smem_raw);
    const int64_t nchunks = N / ch;
    for (int64_t blk = blockIdx.x; blk < nv * nchunks; blk += gridDim.x) {
        T *w = W + (blk / nchunks) * N + (blk % nchunks) * ch;
        for (int e = threadIdx.x; e < ch; e += blockDim.x) z[e] = w[e];
        __syncthreads();
        for (int h = 1; h < ch; h <<= 1) {
            for (int q = threadIdx.x; q < ch / 2; q += blockDim.x) {
                const int i = (q / h) * 2 * h + (q % h);
                T a = z[i], b = z[i + h];
                z[i] = a + b;
                z[i + h] = a - b;
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < ch; e += blockDim.x) w[e] = z[e];
        __syncthreads();
    }
}

template <class T>
__global__ void wht_stage_kernel(T *W, int64_t N, int64_t nv, int64_t h) {
    const int64_t half = N / 2;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < half * nv; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q / half, qq = q % half;
        const int64_t i = (qq / h) * 2 * h + (qq % h);
        T *w = W + v * N;
        T a = w[i], b = w[i + h];
        w[i] = a + b;
        w[i + h] = a - b;
    }
}

// W(r, v) = r < L ? d_r * X(r, v) : 0
template <class T>
__global__ void fjlt_pad_sign_kernel(const T *X, int64_t x_es, int64_t x_vs, int64_t L, int64_t N, int64_t nv,
                                     const uint32_t *signbits, T *W) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N * nv; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q / N, r = q % N;
        T x = r < L ? X[r * x_es + v * x_vs] : T(0);
        W[q] = ((signbits[r >> 5] >> (r & 31)) & 1u) ? x : -x;
    }
}

// Y(i, v) = alpha * sum_k val_k * W(col_k, v) + beta * Y(i, v), rows i of a CSR matrix.
template <class T>
__global__ void csr_gather_kernel(const int32_t *ptr, const int32_t *col, const T *val, int64_t nrows, const T *W,
                                  int64_t w_ld, int64_t nv, T *Y, int64_t y_es, int64_t y_vs, T alpha, T beta,
                                  int beta_zero) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nrows * nv; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q / nrows, i = q % nrows;
        T acc = T(0);
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) acc += val[k] * W[(int64_t)col[k] + v * w_ld];
        T *yp = Y + i * y_es + v * y_vs;
        T res = alpha * acc;
        if (!beta_zero) res += beta * *yp;
        *yp = res;
    }
}

// W(r, v) = sum_k val_k * X(row_k, v) for rows r of the transposed CSR (N rows).
template <class T>
__global__ void csr_t_gather_kernel(const int32_t *ptr, const int32_t *rowi, const T *val, int64_t N, const T *X,
                                    int64_t x_es, int64_t x_vs, int64_t nv, T *W) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N * nv; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q / N, r = q % N;
        T acc = T(0);
        for (int k = ptr[r]; k < ptr[r + 1]; ++k) acc += val[k] * X[(int64_t)rowi[k] * x_es + v * x_vs];
        W[q] = acc;
    }
}

template <class T>
__global__ void fjlt_expand_out_kernel(const T *W, int64_t N, int64_t L, int64_t nv, const uint32_t *signbits, T *Y,
                                       int64_t y_es, int64_t y_vs, T alpha, T beta, int beta_zero) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < L * nv; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = q / L, r = q % L;
        const T d = ((signbits[r >> 5] >> (r & 31)) & 1u) ? alpha : -alpha;
        T *yp = Y + r * y_es + v * y_vs;
        T res = d * W[r + v * N];
        if (!beta_zero) res += beta * *yp;
        *yp = res;
    }
}

// dst(k, v) = src(k, v) for a strided source, written as contiguous columns (ld = len).
template <class T>
__global__ void gather_columns_kernel(const T *src, int64_t s_es, int64_t s_vs, int64_t len, int64_t nv, T *dst) {
    __shared__ T tile[32][33];
    // tile over (k, v): threads read along the source's contiguous dimension
    const int64_t k0 = (int64_t)blockIdx.x * 32, v0 = (int64_t)blockIdx.y * 32;
    const bool src_v_contig = s_vs == 1;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        int64_t k = src_v_contig ? k0 + yy : k0 + threadIdx.x;
        int64_t v = src_v_contig ? v0 + threadIdx.x : v0 + yy;
        T x = (k < len && v < nv) ? src[k * s_es + v * s_vs] : T(0);
        if (src_v_contig) tile[yy][threadIdx.x] = x;   // tile[k][v]
        else tile[threadIdx.x][yy] = x;
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        int64_t v = v0 + yy, k = k0 + threadIdx.x;
        if (k < len && v < nv) dst[k + v * len] = tile[threadIdx.x][yy];
    }
}

// ------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------
template <class T>
static int to_contiguous(rla_ctx *ctx, const T *X, int64_t x_es, int64_t x_vs, int64_t len, int64_t nv, T *dst) {
    dim3 block(32, 8), grid(ceil_div_i(len, 32), ceil_div_i(nv, 32));
    if (grid.y > 65535) return set_error(ctx, RLA_E_UNSUPPORTED, "too many vectors for the strided path");
    gather_columns_kernel<T><<<grid, block, 0, ctx->stream>>>(X, x_es, x_vs, len, nv, dst);
    return check_launch(ctx, "gather_columns");
}

template <class T>
int srht_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                  int64_t y_es, int64_t y_vs, double alpha, double beta) {
    if (nv == 0) return RLA_OK;
    constexpr int CH = WhtCfg<T>::CH, VB = WhtCfg<T>::VB;
    const size_t es = sizeof(T);
    const int64_t L = sk->L, N = sk->N, s = sk->s;
    const T a = (T)(alpha * sk->scale);
    const bool beta_zero = beta == 0.0;
    // strided input: gather to contiguous columns first
    const T *Xc = X;
    int64_t ldx = x_vs;
    size_t off_partials = 0;
    char *scratch = nullptr;
    const int64_t cpv = N >> CH;
    const int cap = ctx->smem_optin - 2048;
    const int s_win = (int)std::min<int64_t>(s, srht_window<T>());
    const int64_t total = cpv * nv;
    const int blocks_per_sm = std::max(1, cap / (int)((es << CH) + 64));
    int64_t W = std::min<int64_t>((int64_t)ctx->sm_count * std::min(blocks_per_sm, 2), std::max<int64_t>(total, 1));
    const size_t need_t = x_es != 1 ? (size_t)L * nv * es : 0;
    const size_t need_p = N >= ((int64_t)1 << CH) ? (size_t)(2 * W) * s_win * es : 0;
    {
        void *p;
        RLA_TRY(scratch_get(ctx, ((need_t + 255) & ~size_t(255)) + need_p + 256, &p));
        scratch = (char *)p;
        off_partials = (need_t + 255) & ~size_t(255);
    }
    if (x_es != 1) {
        RLA_TRY(to_contiguous(ctx, X, x_es, x_vs, L, nv, (T *)scratch));
        Xc = (const T *)scratch;
        ldx = L;
    }
    if (N < ((int64_t)1 << CH)) {
        const size_t smem = (size_t)N * es;
        set_smem_max(srht_small_kernel<T>);
        const int grid = (int)std::min<int64_t>(nv, (int64_t)ctx->sm_count * 8);
        srht_small_kernel<T><<<grid, 256, smem, ctx->stream>>>(Xc, ldx, L, N, nv, sk->signbits, sk->rows, s, Y, y_es,
                                                               y_vs, a, (T)beta, beta_zero);
        return check_launch(ctx, "srht_small");
    }
    int *cnt = nullptr;
    RLA_TRY(counters_get(ctx, (size_t)nv, &cnt));
    const bool vec = (ldx % (int64_t)(1 << VB) == 0) && ((uintptr_t)Xc % 16 == 0);
    SrhtParams<T> p{Xc, ldx, L, N, sk->sign_tl, sk->rows, 0, s_win, Y, y_es, y_vs, a, (T)beta, beta_zero,
                    (T *)(scratch + off_partials), cnt, cpv, Split::make(total, (int)W)};
    const size_t smem = es << CH;
    for (int64_t lo = 0; lo < s; lo += s_win) {
        p.s_lo = lo;
        p.s_cnt = (int)std::min<int64_t>(s_win, s - lo);
        if (vec) launch_srht_fused<T, true>(p, (int)W, smem, ctx->stream);
        else launch_srht_fused<T, false>(p, (int)W, smem, ctx->stream);
        RLA_TRY(check_launch(ctx, "srht_fused"));
    }
    return RLA_OK;
}

template <class T>
int srht_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                int64_t y_es, int64_t y_vs, double alpha, double beta) {
    if (nv == 0) return RLA_OK;
    const int ch = (int)sk->chunk;
    const int log_ch = ilog2(ch);
    const int64_t nblk = nv * (sk->N >> log_ch);
    const int grid = (int)std::min<int64_t>(nblk, (int64_t)ctx->sm_count * 16);
    const size_t smem = (size_t)ch * sizeof(T);
    srht_expand_kernel<T><<<grid, 256, smem, ctx->stream>>>(X, x_es, x_vs, sk->L, sk->N, nv, sk->signbits, sk->rows,
                                                            sk->p2_ptr, sk->p2_list, ch, log_ch, Y, y_es, y_vs,
                                                            (T)(alpha * sk->scale), (T)beta, beta == 0.0);
    return check_launch(ctx, "srht_expand");
}

template <class T>
static int wht_full(rla_ctx *ctx, T *W, int64_t N, int64_t nv) {
    const int ch = (int)std::min<int64_t>(N, 4096);
    const int64_t nblk = nv * (N / ch);
    wht_chunk_kernel<T><<<(int)std::min<int64_t>(nblk, (int64_t)ctx->sm_count * 16), 256, ch * sizeof(T), ctx->stream>>>(
        W, N, nv, ch);
    RLA_TRY(check_launch(ctx, "wht_chunk"));
    for (int64_t h = ch; h < N; h <<= 1) {
        const int64_t work = (N / 2) * nv;
        wht_stage_kernel<T><<<(int)std::min<int64_t>(ceil_div(work, 256), (int64_t)ctx->sm_count * 32), 256, 0,
                              ctx->stream>>>(W, N, nv, h);
        RLA_TRY(check_launch(ctx, "wht_stage"));
    }
    return RLA_OK;
}

template <class T>
int fjlt_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                  int64_t y_es, int64_t y_vs, double alpha, double beta) {
    if (nv == 0) return RLA_OK;
    const int64_t N = sk->N;
    void *w;
    RLA_TRY(scratch_get(ctx, (size_t)N * nv * sizeof(T), &w));
    T *Wb = (T *)w;
    const int grid = (int)std::min<int64_t>(ceil_div(N * nv, 256), (int64_t)ctx->sm_count * 32);
    fjlt_pad_sign_kernel<T><<<grid, 256, 0, ctx->stream>>>(X, x_es, x_vs, sk->L, N, nv, sk->signbits, Wb);
    RLA_TRY(check_launch(ctx, "fjlt_pad_sign"));
    RLA_TRY(wht_full(ctx, Wb, N, nv));
    const int grid2 = (int)std::min<int64_t>(ceil_div(sk->s * nv, 256), (int64_t)ctx->sm_count * 32);
    csr_gather_kernel<T><<<std::max(grid2, 1), 256, 0, ctx->stream>>>(sk->k_ptr, sk->k_col, (const T *)sk->k_val, sk->s,
                                                                     Wb, N, nv, Y, y_es, y_vs, (T)(alpha * sk->scale),
                                                                     (T)beta, beta == 0.0);
    return check_launch(ctx, "fjlt_csr_gather");
}

template <class T>
int fjlt_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                int64_t y_es, int64_t y_vs, double alpha, double beta) {
    if (nv == 0) return RLA_OK;
    const int64_t N = sk->N;
    void *w;
    RLA_TRY(scratch_get(ctx, (size_t)N * nv * sizeof(T), &w));
    T *Wb = (T *)w;
    const int grid = (int)std::min<int64_t>(ceil_div(N * nv, 256), (int64_t)ctx->sm_count * 32);
    csr_t_gather_kernel<T><<<grid, 256, 0, ctx->stream>>>(sk->kt_ptr, sk->kt_row, (const T *)sk->kt_val, N, X, x_es,
                                                          x_vs, nv, Wb);
    RLA_TRY(check_launch(ctx, "fjlt_csr_t_gather"));
    RLA_TRY(wht_full(ctx, Wb, N, nv));
    const int grid2 = (int)std::min<int64_t>(ceil_div(sk->L * nv, 256), (int64_t)ctx->sm_count * 32);
    fjlt_expand_out_kernel<T><<<grid2, 256, 0, ctx->stream>>>(Wb, N, sk->L, nv, sk->signbits, Y, y_es, y_vs,
                                                              (T)(alpha * sk->scale), (T)beta, beta == 0.0);
    return check_launch(ctx, "fjlt_expand_out");
}

// ------------------------------------------------------------------------------------
// Allocation-free SRHT left apply.
//
// Some callers cannot call cudaMalloc: code that owns a fixed device-memory budget and
// hands every byte out itself (a serving process that partitions HBM up front), code whose
// device memory is managed by another runtime's pool allocator, and code on a path that
// must not touch the CUDA allocator at all (latency-critical request handling).  For them
// the partial-sum scratch of the stream-K SRHT kernel lives in fixed device arrays that the
// library defines; every GPU that loads the library holds them until the process exits.
// All calls share these arrays, so calls whose work overlaps on the GPU (different streams
// or host threads without ordering between them) race and give wrong results.
// ------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_partials[RLA_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) int g_noalloc_counters[RLA_NOALLOC_MAX_COLS];

struct NoallocDevice {
    bool ready = false;
    void *partials = nullptr;  // device address of g_noalloc_partials on this device
    int *counters = nullptr;   // device address of g_noalloc_counters on this device
};

static int noalloc_setup(rla_ctx *ctx, NoallocDevice **out) {
    static std::mutex mu;
    static NoallocDevice dev[64];
    if (ctx->device < 0 || ctx->device >= 64) return set_error(ctx, RLA_E_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    NoallocDevice &d = dev[ctx->device];
    if (!d.ready) {
        // In host code the array names are host-side stand-ins; the device addresses come
        // from the runtime, per device, with that device current (the caller made it so).
        RLA_CUDA_TRY(ctx, cudaGetSymbolAddress(&d.partials, g_noalloc_partials));
        RLA_CUDA_TRY(ctx, cudaGetSymbolAddress((void **)&d.counters, g_noalloc_counters));
        d.ready = true;
    }
    *out = &d;
    return RLA_OK;
}

template <class T>
static int srht_noalloc_t(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t ldx, int64_t nv, T *Y,
                          int64_t ldy, double alpha, double beta, const NoallocDevice &nd) {
    constexpr int CH = WhtCfg<T>::CH, VB = WhtCfg<T>::VB;
    const size_t es = sizeof(T);
    const int64_t L = sk->L, N = sk->N, s = sk->s;
    const T a = (T)(alpha * sk->scale);
    const bool beta_zero = beta == 0.0;
    if (N < ((int64_t)1 << CH)) {
        const size_t smem = (size_t)N * es;
        set_smem_max(srht_small_kernel<T>);
        const int grid = (int)std::min<int64_t>(nv, (int64_t)ctx->sm_count * 8);
        srht_small_kernel<T><<<grid, 256, smem, ctx->stream>>>(X, ldx, L, N, nv, sk->signbits, sk->rows, s, Y, 1, ldy,
                                                               a, (T)beta, beta_zero);
        return check_launch(ctx, "srht_small(noalloc)");
    }
    const int s_win = (int)std::min<int64_t>(s, srht_window<T>());
    const int64_t cpv = N >> CH, total = cpv * nv;
    int64_t W = std::min<int64_t>((int64_t)ctx->sm_count * 2, total);
    W = std::min<int64_t>(W, (int64_t)(RLA_NOALLOC_SCRATCH_BYTES / (2 * (size_t)s_win * es)));
    if (W < 1)
        return set_error(ctx, RLA_E_ARG, "compression dimension window %d does not fit the %u-byte allocation-free scratch",
                         s_win, (unsigned)RLA_NOALLOC_SCRATCH_BYTES);
    RLA_CUDA_TRY(ctx, cudaMemsetAsync(nd.counters, 0, sizeof(int) * (size_t)nv, ctx->stream));
    const bool vec = (ldx % (int64_t)(1 << VB) == 0) && ((uintptr_t)X % 16 == 0);
    SrhtParams<T> p{X, ldx, L, N, sk->sign_tl, sk->rows, 0, s_win, Y, 1, ldy, a, (T)beta, beta_zero,
                    (T *)nd.partials, nd.counters, cpv, Split::make(total, (int)W)};
    const size_t smem = es << CH;
    for (int64_t lo = 0; lo < s; lo += s_win) {
        p.s_lo = lo;
        p.s_cnt = (int)std::min<int64_t>(s_win, s - lo);
        if (vec) launch_srht_fused<T, true>(p, (int)W, smem, ctx->stream);
        else launch_srht_fused<T, false>(p, (int)W, smem, ctx->stream);
        RLA_TRY(check_launch(ctx, "srht_fused(noalloc)"));
    }
    return RLA_OK;
}

#define RLA_INST(T)                                                                                                  \
    template int srht_compress<T>(rla_ctx *, const rla_sketch *, const T *, int64_t, int64_t, int64_t, T *, int64_t,  \
                                  int64_t, double, double);                                                          \
    template int srht_expand<T>(rla_ctx *, const rla_sketch *, const T *, int64_t, int64_t, int64_t, T *, int64_t,    \
                                int64_t, double, double);                                                            \
    template int fjlt_compress<T>(rla_ctx *, const rla_sketch *, const T *, int64_t, int64_t, int64_t, T *, int64_t,  \
                                  int64_t, double, double);                                                          \
    template int fjlt_expand<T>(rla_ctx *, const rla_sketch *, const T *, int64_t, int64_t, int64_t, T *, int64_t,    \
                                int64_t, double, double);
RLA_INST(float)
RLA_INST(double)

}  // namespace rla

using namespace rla;

extern "C" int rla_srht_mul_noalloc(rla_ctx *ctx, const rla_sketch *sk, int64_t c_rows, int64_t c_cols, void *C,
                                    int64_t ldc, int64_t a_rows, int64_t a_cols, const void *A, int64_t lda,
                                    double alpha, double beta) {
    if (!ctx) return RLA_E_ARG;
    if (!sk || sk->p.kind != RLA_SRHT || sk->p.card != RLA_LEFT)
        return set_error(ctx, RLA_E_ARG, "rla_srht_mul_noalloc needs a Left-cardinality SRHT recipe.");
    if (c_rows < 0 || c_cols < 0 || a_rows < 0 || a_cols < 0) return set_error(ctx, RLA_E_ARG, "Negative dimension.");
    if (sk->device != ctx->device) return set_error(ctx, RLA_E_ARG, "Compressor lives on another device.");
    // left_mul_dimcheck (src/helpers/mul_dim_checks.jl:41-64)
    if (a_rows != sk->n_cols)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld rows while S has %lld columns.", (long long)a_rows, (long long)sk->n_cols);
    if (a_cols != c_cols)
        return set_error(ctx, RLA_E_DIM, "Matrix A has %lld columns while C has %lld columns.", (long long)a_cols, (long long)c_cols);
    if (c_rows != sk->n_rows)
        return set_error(ctx, RLA_E_DIM, "Matrix C has %lld rows while S has %lld rows.", (long long)c_rows, (long long)sk->n_rows);
    if (a_cols > RLA_NOALLOC_MAX_COLS)
        return set_error(ctx, RLA_E_ARG, "%lld columns exceed the allocation-free limit of %d columns per call.",
                         (long long)a_cols, RLA_NOALLOC_MAX_COLS);
    if (a_cols == 0) return RLA_OK;
    if (!A || !C || lda < std::max<int64_t>(1, a_rows) || ldc < std::max<int64_t>(1, c_rows))
        return set_error(ctx, RLA_E_ARG, "NULL pointer or leading dimension smaller than the row count.");
    // Every call runs on the context's device and hands the calling thread its own current
    // device back, whichever it was.
    int caller_dev = 0;
    RLA_CUDA_TRY(ctx, cudaGetDevice(&caller_dev));
    RLA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    NoallocDevice *nd = nullptr;
    int st = noalloc_setup(ctx, &nd);
    if (st == RLA_OK) {
        if (sk->p.dtype == RLA_F32)
            st = srht_noalloc_t<float>(ctx, sk, (const float *)A, lda, a_cols, (float *)C, ldc, alpha, beta, *nd);
        else
            st = srht_noalloc_t<double>(ctx, sk, (const double *)A, lda, a_cols, (double *)C, ldc, alpha, beta, *nd);
    }
    if (caller_dev != ctx->device) {
        const cudaError_t e = cudaSetDevice(caller_dev);
        if (st == RLA_OK && e != cudaSuccess)
            return set_error(ctx, RLA_E_CUDA, "restoring the caller's device %d: %s", caller_dev, cudaGetErrorString(e));
    }
    return st;
}
