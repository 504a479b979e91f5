// rla_sparse.cu -- SparseSign / CountSketch application kernels.
//
// A SparseSign (nnz per long index) or CountSketch (nnz = 1) operator is stored by its
// compress side P (s x L): long index j carries nnz (bucket, sign) entries with a common
// magnitude `scale`.  The reference applies it through SparseArrays' CSC kernels
// (sparse_sign.jl:339-361, count_sketch.jl:166-213); here:
//
//  * compress, contiguous vectors (S*A with Left S on column-major A, the sketch hot
//    path): each warp owns private shared-memory bins for one output vector and streams
//    its input vector with 16-byte loads.  Buckets that would collide inside a warp access
//    were scheduled away when the sketch was drawn (CountSketch: moved to a per-warp list
//    folded in by extra rounds; SparseSign: extra rounds), so no atomics are used and the
//    result is bit-for-bit reproducible.  Input batches are split over all warps of the
//    GPU (stream-K); a vector shared by several warps is finished by the last warp to
//    arrive, which adds the partial bins in warp order.
//  * compress, strided vectors (A*S with Right S: rows of column-major A): lane = vector,
//    the bucket is warp-uniform, bins are [bucket][lane] (conflict-free).
//  * expand (S'*A, A*S' ...): a gather, one thread per output element.
#include "rla_internal.cuh"

namespace rla {

template <class T>
struct CompressContigParams {
    const T *X;
    int64_t x_ld;  // vector stride; element (j, v) at X[j + v*x_ld]
    int64_t L, nv;
    const uint32_t *meta;
    const uint32_t *tile_flags;
    const uint32_t *extra;
    int nnz;
    int64_t bin_lo;
    int bin_cnt;
    T *Y;
    int64_t y_es, y_vs;  // element (i, v) of the output at Y[i*y_es + v*y_vs]
    T alpha, beta;
    int beta_zero;
    T *partials;
    int *counters;
    int64_t tpv;  // 128-element tiles per vector
    Split split;
};

// Sub-round with colliding buckets: lanes sharing a bucket are summed in lane order and
// the lowest lane adds the sum (rare for s >> 32, hence kept out of line).
template <class T>
__device__ __noinline__ void bin_add_collide(T *bins, T x, int b, bool inwin, int lane) {
    const unsigned key = inwin ? (unsigned)b : (0x80000000u | (unsigned)lane);
    const unsigned grp = __match_any_sync(FULL, key);
    const int cnt = __popc(grp);
    const int maxc = (int)__reduce_max_sync(FULL, (unsigned)cnt);
    T sum = T(0);
    for (int q = 0; q < maxc; ++q) {
        const int src = q < cnt ? (int)__fns(grp, 0, q + 1) : lane;
        const T y = __shfl_sync(FULL, x, src);
        if (q < cnt) sum += y;
    }
    if (inwin && (grp & ((1u << lane) - 1u)) == 0u) bins[b] += sum;
}

constexpr uint32_t TILE_SLOW = 0x80000000u;
constexpr uint32_t BUCKET_MASK = 0x3fffffu;  // bits 0..21
constexpr uint32_t BIT_DEFER = 1u << 30;     // main word: processed in an extra round
constexpr uint32_t BIT_VALID = 1u << 30;     // extra word: slot holds an item

template <class T>
__device__ __forceinline__ T apply_sign(T x, uint32_t w) {
    if constexpr (sizeof(T) == 4) return __uint_as_float(__float_as_uint(x) ^ (w & 0x80000000u));
    else return __longlong_as_double(__double_as_longlong(x) ^ ((long long)(w & 0x80000000u) << 32));
}

// Predicated read-modify-write of one bin; within a sub-round the active lanes' bins are
// distinct by construction (collisions were deferred when the sketch was drawn).
template <class T, bool WIN>
__device__ __forceinline__ void rmw(T *bins, T x, uint32_t w, bool on, int64_t bin_lo, int bin_cnt) {
    int b = (int)(w & BUCKET_MASK);
    if constexpr (WIN) {
        b -= (int)bin_lo;
        on = on && (unsigned)b < (unsigned)bin_cnt;
    }
    x = apply_sign(x, w);
    if (on) bins[b] += x;
}

// Run-time resolution for SLOW tiles: lanes sharing a bucket are summed in lane order.
template <class T, bool WIN>
__device__ __noinline__ void rmw_resolve(T *bins, T x, uint32_t w, bool valid, int64_t bin_lo, int bin_cnt, int lane) {
    int b = (int)(w & BUCKET_MASK);
    bool inwin = valid;
    if constexpr (WIN) {
        b -= (int)bin_lo;
        inwin = valid && (unsigned)b < (unsigned)bin_cnt;
    }
    x = apply_sign(x, w);
    bin_add_collide(bins, x, b, inwin, lane);
    __syncwarp();
}

template <class T, bool VEC>
__device__ __forceinline__ void load4(const T *xv, int64_t j0, int64_t L, bool tile_ok, T (&v)[4]) {
    if (VEC && tile_ok && j0 + 3 < L) {
        if constexpr (sizeof(T) == 4) {
            float4 q = __ldg(reinterpret_cast<const float4 *>(xv + j0));
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
        } else {
            double2 a = __ldg(reinterpret_cast<const double2 *>(xv + j0));
            double2 b = __ldg(reinterpret_cast<const double2 *>(xv + j0 + 2));
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
        }
    } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) v[t] = (tile_ok && j0 + t < L) ? __ldg(xv + j0 + t) : T(0);
    }
}

// 16-byte vector of T
template <class T>
struct V16 {
    using type = float4;
};
template <>
struct V16<double> {
    using type = double2;
};

// Finish this warp's share of output vector v: write it (alpha/beta epilogue) when the warp
// covered the whole vector, else store the partial bins and let the last warp to arrive add
// all partials in warp order.  Moves 16 bytes per access when the bin count allows it.
template <class T>
__device__ void flush_vector(const CompressContigParams<T> &p, T *bins, int g, int64_t v, bool exclusive, int lane) {
    constexpr int N = 16 / (int)sizeof(T);
    using V = typename V16<T>::type;
    __syncwarp();
    const int nvec = (p.bin_cnt % N == 0) ? p.bin_cnt / N : 0;
    T *y0 = p.Y + p.bin_lo * p.y_es + v * p.y_vs;
    const bool yvec = p.y_es == 1 && (reinterpret_cast<uintptr_t>(y0) & 15u) == 0;
    auto out = [&](int64_t i, T acc) {
        T *yp = y0 + i * p.y_es;
        T r = p.alpha * acc;
        if (!p.beta_zero) r += p.beta * *yp;
        *yp = r;
    };
    auto out_vec = [&](int q, V acc) {
        const T *a = reinterpret_cast<const T *>(&acc);
        if (yvec) {
            V y;
            T *ya = reinterpret_cast<T *>(&y);
            if (!p.beta_zero) y = *reinterpret_cast<const V *>(y0 + (int64_t)q * N);
#pragma unroll
            for (int e = 0; e < N; ++e) ya[e] = p.beta_zero ? p.alpha * a[e] : p.alpha * a[e] + p.beta * ya[e];
            *reinterpret_cast<V *>(y0 + (int64_t)q * N) = y;
        } else {
#pragma unroll
            for (int e = 0; e < N; ++e) out((int64_t)q * N + e, a[e]);
        }
    };
    V *bv = reinterpret_cast<V *>(bins);
    const V zero{};
    if (exclusive) {
        for (int q = lane; q < nvec; q += 32) {
            const V b = bv[q];
            bv[q] = zero;
            out_vec(q, b);
        }
        for (int i = nvec * N + lane; i < p.bin_cnt; i += 32) {
            out(i, bins[i]);
            bins[i] = T(0);
        }
        __syncwarp();
        return;
    }
    const int64_t vbeg = v * p.tpv;
    T *part = p.partials + (int64_t)p.split.slot(g, vbeg) * p.bin_cnt;
    for (int q = lane; q < nvec; q += 32) {
        reinterpret_cast<V *>(part)[q] = bv[q];
        bv[q] = zero;
    }
    for (int i = nvec * N + lane; i < p.bin_cnt; i += 32) {
        part[i] = bins[i];
        bins[i] = T(0);
    }
    __threadfence();
    __syncwarp();
    const int gf = p.split.owner(vbeg), gl = p.split.owner(vbeg + p.tpv - 1);
    int old = 0;
    if (lane == 0) old = atomicAdd(&p.counters[v], 1);
    old = __shfl_sync(FULL, old, 0);
    if (old == gl - gf) {
        __threadfence();
        const T *p0 = p.partials + (int64_t)p.split.slot(gf, vbeg) * p.bin_cnt;
        for (int q = lane; q < nvec; q += 32) {
            V acc = __ldcg(reinterpret_cast<const V *>(p0) + q);
            T *a = reinterpret_cast<T *>(&acc);
#pragma unroll 4
            for (int gg = gf + 1; gg <= gl; ++gg) {
                const V x = __ldcg(reinterpret_cast<const V *>(p.partials + (int64_t)(2 * gg) * p.bin_cnt) + q);
                const T *xe = reinterpret_cast<const T *>(&x);
#pragma unroll
                for (int e = 0; e < N; ++e) a[e] += xe[e];
            }
            out_vec(q, acc);
        }
        for (int i = nvec * N + lane; i < p.bin_cnt; i += 32) {
            T acc = __ldcg(p0 + i);
            for (int gg = gf + 1; gg <= gl; ++gg) acc += __ldcg(p.partials + (int64_t)(2 * gg) * p.bin_cnt + i);
            out(i, acc);
        }
        if (lane == 0) p.counters[v] = 0;
    }
    __syncwarp();
}

template <class T>
__device__ __forceinline__ T pick4(const T (&v)[4], uint32_t t) {
    const T lo = (t & 1u) ? v[1] : v[0];
    const T hi = (t & 1u) ? v[3] : v[2];
    return (t & 2u) ? hi : lo;
}

constexpr int XPF = 4;  // extra-round words a lane keeps in flight

// First XPF extra words of a non-SLOW tile (0 past its round count), loaded before the
// tile's main sub-rounds so that their latency hides behind them.
__device__ __forceinline__ void extra_prefetch(const uint32_t *extra, uint32_t flag, int lane, uint32_t (&pf)[XPF]) {
    const int R = (int)(flag & 0xffu);
    const uint32_t *xp = extra + (int64_t)(flag >> 8) * 32 + lane;
#pragma unroll
    for (int i = 0; i < XPF; ++i) pf[i] = (i < R) ? __ldg(xp + i * 32) : 0u;
}

// Extra rounds of a non-SLOW tile; word r + XPF is loaded while round r runs.
template <class T, bool WIN>
__device__ __forceinline__ void extra_rounds(const CompressContigParams<T> &p, T *bins, const T (&val)[4],
                                             uint32_t flag, int lane, uint32_t (&pf)[XPF]) {
    const int R = (int)(flag & 0xffu);
    const uint32_t *xp = p.extra + (int64_t)(flag >> 8) * 32 + lane;
    for (int r = 0; r < R; r += XPF) {
#pragma unroll
        for (int i = 0; i < XPF; ++i) {
            if (r + i < R) {
                const uint32_t w = pf[i];
                pf[i] = (r + i + XPF < R) ? __ldg(xp + (r + i + XPF) * 32) : 0u;
                rmw<T, WIN>(bins, pick4(val, (w >> 22) & 3u), w, (w & BIT_VALID) != 0u, p.bin_lo, p.bin_cnt);
                __syncwarp();
            }
        }
    }
}

// One 128-element tile kk of vector xv whose values are already in registers: lane holds
// elements 4*lane .. 4*lane+3; metadata of nonzero slot e is meta[(kk*nnz + e)*128 ...].
template <class T, bool WIN, bool CHECK>
__device__ __forceinline__ void tile_rounds(const CompressContigParams<T> &p, T *bins, const T (&val)[4], int64_t kk,
                                            int64_t j0, uint32_t flag, int lane) {
    if (flag & TILE_SLOW) {
        for (int e = 0; e < p.nnz; ++e)
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const bool valid = !CHECK || (j0 + t < p.L);
                const uint32_t w = valid ? __ldg(p.meta + (kk * p.nnz + e) * 128 + lane * 4 + t) : 0u;
                rmw_resolve<T, WIN>(bins, val[t], w, valid, p.bin_lo, p.bin_cnt, lane);
            }
        return;
    }
    uint32_t pf[XPF];
    extra_prefetch(p.extra, flag, lane, pf);
    for (int e = 0; e < p.nnz; ++e) {
        const uint32_t *mp = p.meta + (kk * p.nnz + e) * 128 + lane * 4;
        uint32_t mw[4];
        if (!CHECK || j0 + 3 < p.L) {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(mp));
            mw[0] = q.x; mw[1] = q.y; mw[2] = q.z; mw[3] = q.w;
        } else {
#pragma unroll
            for (int t = 0; t < 4; ++t) mw[t] = (j0 + t < p.L) ? __ldg(mp + t) : 0u;
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const bool valid = !CHECK || (j0 + t < p.L);
            rmw<T, WIN>(bins, val[t], mw[t], valid && !(mw[t] & BIT_DEFER), p.bin_lo, p.bin_cnt);
            __syncwarp();
        }
    }
    extra_rounds<T, WIN>(p, bins, val, flag, lane, pf);  // deferred items (warp-uniform count)
}

// U full CountSketch tiles held in registers.
template <class T, int U>
struct Batch {
    T val[U][4];
    uint32_t mw[U][4], fl[U];
    template <bool VEC>
    __device__ __forceinline__ void load_(const CompressContigParams<T> &p, const T *xv, int64_t k, int lane) {
#pragma unroll
        for (int b = 0; b < U; ++b) {
            const int64_t j0 = (k + b) * 128 + lane * 4;
            load4<T, VEC>(xv, j0, p.L, true, val[b]);
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p.meta + j0));
            mw[b][0] = q.x; mw[b][1] = q.y; mw[b][2] = q.z; mw[b][3] = q.w;
            fl[b] = __ldg(p.tile_flags + k + b);
        }
    }
    __device__ __forceinline__ void load(const CompressContigParams<T> &p, const T *xv, int64_t k, int lane) {
        // vector loads when the column start is 16-byte aligned
        if ((reinterpret_cast<uintptr_t>(xv) & 15u) == 0) load_<true>(p, xv, k, lane);
        else load_<false>(p, xv, k, lane);
    }
    template <bool WIN>
    __device__ __forceinline__ void run(const CompressContigParams<T> &p, T *bins, int64_t k, int lane) {
#pragma unroll
        for (int b = 0; b < U; ++b) {
            if (fl[b] & TILE_SLOW) {
                tile_rounds<T, WIN, false>(p, bins, val[b], k + b, (k + b) * 128 + lane * 4, fl[b], lane);
                continue;
            }
            uint32_t pf[XPF];
            extra_prefetch(p.extra, fl[b], lane, pf);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                rmw<T, WIN>(bins, val[b][t], mw[b][t], !(mw[b][t] & BIT_DEFER), p.bin_lo, p.bin_cnt);
                __syncwarp();
            }
            extra_rounds<T, WIN>(p, bins, val[b], fl[b], lane, pf);
        }
    }
};

template <class T, bool VEC, bool WIN, bool NNZ1>
__global__ void __launch_bounds__(384) compress_contig_kernel(CompressContigParams<T> p) {
    constexpr int U = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const int g = blockIdx.x * warps + wib;
    T *bins = reinterpret_cast<T *>(smem_raw) + (int64_t)wib * p.bin_cnt;
    for (int i = lane; i < p.bin_cnt; i += 32) bins[i] = T(0);
    __syncwarp();
    if (g >= p.split.W) return;
    const int64_t u0 = p.split.start(g), u1 = p.split.start(g + 1);
    if (u0 >= u1) return;
    const int64_t full_tiles = p.L / 128;  // tiles with all 128 elements inside the vector
    int64_t v = u0 / p.tpv;
    int64_t u = u0;
    while (u < u1) {
        const int64_t vbeg = v * p.tpv;
        const int64_t kend = min(u1, vbeg + p.tpv) - vbeg;
        const T *xv = p.X + v * p.x_ld;
        int64_t k = u - vbeg;
        const int64_t kfull = min(kend, full_tiles);
        if constexpr (NNZ1) {
            // CountSketch: batches of U tiles (data, metadata, flags); the next batch's loads
            // are issued before the current batch is processed (register double buffer).
            Batch<T, U> ba, bb;
            if (k + U <= kfull) ba.load(p, xv, k, lane);
            while (k + U <= kfull) {
                if (k + 2 * U <= kfull) bb.load(p, xv, k + U, lane);
                ba.template run<WIN>(p, bins, k, lane);
                k += U;
                if (k + U > kfull) break;
                if (k + 2 * U <= kfull) ba.load(p, xv, k + U, lane);
                bb.template run<WIN>(p, bins, k, lane);
                k += U;
            }
        }
        for (; k < kend; ++k) {
            const int64_t j0 = k * 128 + lane * 4;
            T val[4];
            const uint32_t fl = __ldg(p.tile_flags + k);
            if (k < kfull) {
                load4<T, VEC>(xv, j0, p.L, true, val);
                tile_rounds<T, WIN, false>(p, bins, val, k, j0, fl, lane);
            } else {
                load4<T, VEC>(xv, j0, p.L, true, val);
                tile_rounds<T, WIN, true>(p, bins, val, k, j0, fl, lane);
            }
        }
        const bool exclusive = (u0 <= vbeg) && (vbeg + p.tpv <= u1);
        flush_vector(p, bins, g, v, exclusive, lane);
        u = vbeg + kend;
        ++v;
    }
}

// ---- CountSketch, 512-element batches ------------------------------------------------
// One warp per CTA.  Shared memory: [bins (bin_cnt) | list (64) | dummy (32)] elements.
// Lane holds elements 4*lane + (i & 3) of tile (i >> 2) of the batch in val[i], and their
// words (byte offset of the target slot, sign in bit 31; see cs_sched_kernel) in mw[i].
// All targets of a batch's main words are distinct, so its 16 reads are issued before its
// 16 writes, with no predicates: a deferred element lands in its (cleared) list entry.  Up
// to two extra rounds then move list entry r*32 + lane into the bin at xb[r] and clear it.
// With WIN (bins cover [bin_lo, bin_lo + bin_cnt) of s) offsets are remapped at run time
// and targets outside the window go to the lane's dummy slot.
constexpr uint32_t CS_OFF_MASK = 0x00ffffffu;

template <class T>
__device__ __forceinline__ T &slot_at(unsigned char *base, uint32_t off) {
    return *reinterpret_cast<T *>(base + off);
}

template <class T, bool WIN>
__device__ __forceinline__ uint32_t cs_target(const CompressContigParams<T> &p, uint32_t off, uint32_t s_bytes,
                                              uint32_t dummy) {
    off &= CS_OFF_MASK;
    if constexpr (WIN) {
        const uint32_t lo = (uint32_t)p.bin_lo * sizeof(T), win = (uint32_t)p.bin_cnt * sizeof(T);
        if (off >= s_bytes) return off - s_bytes + win;  // list entry or dummy slot
        const uint32_t b = off - lo;                        // wraps when below the window
        return b < win ? b : dummy;
    }
    return off;
}

// Run-time resolution for a batch the scheduler could not place: lanes sharing a target
// slot are summed in lane order and the lowest lane adds the sum.
template <class T>
__device__ __noinline__ void cs_resolve(unsigned char *sm, T x, uint32_t o, int lane) {
    const unsigned grp = __match_any_sync(FULL, o);
    const int cnt = __popc(grp);
    const int maxc = (int)__reduce_max_sync(FULL, (unsigned)cnt);
    T sum = T(0);
    for (int q = 0; q < maxc; ++q) {
        const int src = q < cnt ? (int)__fns(grp, 0, q + 1) : lane;
        const T y = __shfl_sync(FULL, x, src);
        if (q < cnt) sum += y;
    }
    if ((grp & ((1u << lane) - 1u)) == 0u) slot_at<T>(sm, o) += sum;
    __syncwarp();
}

template <class T, bool CHECK>
struct CsBatch {
    T val[16];
    uint32_t mw[16];
    uint32_t fl, xb0, xb1;
    template <bool VEC>
    __device__ __forceinline__ void load(const CompressContigParams<T> &p, const T *xv, int64_t bt, int lane,
                                         uint32_t pad) {
        if constexpr (VEC && !CHECK) {
            // whole batch inside the vector: 16-byte loads at immediate offsets from one base
            const T *xb = xv + bt * 512 + lane * 4;
            const uint4 *mb = reinterpret_cast<const uint4 *>(p.meta + bt * 512 + lane * 4);
#pragma unroll
            for (int tb = 0; tb < 4; ++tb) {
                if constexpr (sizeof(T) == 4) {
                    const float4 q = __ldg(reinterpret_cast<const float4 *>(xb + tb * 128));
                    val[tb * 4] = q.x; val[tb * 4 + 1] = q.y; val[tb * 4 + 2] = q.z; val[tb * 4 + 3] = q.w;
                } else {
                    const double2 a = __ldg(reinterpret_cast<const double2 *>(xb + tb * 128));
                    const double2 b = __ldg(reinterpret_cast<const double2 *>(xb + tb * 128 + 2));
                    val[tb * 4] = a.x; val[tb * 4 + 1] = a.y; val[tb * 4 + 2] = b.x; val[tb * 4 + 3] = b.y;
                }
                const uint4 m = __ldg(mb + tb * 32);
                mw[tb * 4] = m.x; mw[tb * 4 + 1] = m.y; mw[tb * 4 + 2] = m.z; mw[tb * 4 + 3] = m.w;
            }
            const uint32_t *xp = p.extra + bt * 64 + lane;
            fl = __ldg(p.tile_flags + bt);
            xb0 = __ldg(xp);
            xb1 = __ldg(xp + 32);
            return;
        }
#pragma unroll
        for (int tb = 0; tb < 4; ++tb) {
            const int64_t j0 = bt * 512 + tb * 128 + lane * 4;
            T v4[4];
            load4<T, VEC>(xv, j0, p.L, true, v4);
#pragma unroll
            for (int t = 0; t < 4; ++t) val[tb * 4 + t] = v4[t];
            if (!CHECK || j0 + 3 < p.L) {
                const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p.meta + j0));
                mw[tb * 4] = q.x; mw[tb * 4 + 1] = q.y; mw[tb * 4 + 2] = q.z; mw[tb * 4 + 3] = q.w;
            } else {
#pragma unroll
                for (int t = 0; t < 4; ++t) mw[tb * 4 + t] = (j0 + t < p.L) ? __ldg(p.meta + j0 + t) : pad;
            }
        }
        fl = __ldg(p.tile_flags + bt);
        xb0 = __ldg(p.extra + bt * 64 + lane);
        xb1 = __ldg(p.extra + bt * 64 + 32 + lane);
    }
    template <bool WIN>
    __device__ __forceinline__ void run(const CompressContigParams<T> &p, unsigned char *sm, uint32_t s_bytes,
                                        uint32_t list_off, uint32_t dummy, int lane) {
        if (fl & TILE_SLOW) {
#pragma unroll
            for (int i = 0; i < 16; ++i)
                cs_resolve<T>(sm, apply_sign(val[i], mw[i]), cs_target<T, WIN>(p, mw[i], s_bytes, dummy), lane);
            return;
        }
        uint32_t o[16];
        T old[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            o[i] = cs_target<T, WIN>(p, mw[i], s_bytes, dummy);
            old[i] = slot_at<T>(sm, o[i]);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) slot_at<T>(sm, o[i]) = old[i] + apply_sign(val[i], mw[i]);
        __syncwarp();
        if (fl > 0u) {
            const uint32_t t0 = cs_target<T, WIN>(p, xb0, s_bytes, dummy);
            T &e0 = slot_at<T>(sm, list_off + lane * sizeof(T));
            slot_at<T>(sm, t0) += e0;
            e0 = T(0);
            __syncwarp();
            if (fl > 1u) {
                const uint32_t t1 = cs_target<T, WIN>(p, xb1, s_bytes, dummy);
                T &e1 = slot_at<T>(sm, list_off + (32 + lane) * sizeof(T));
                slot_at<T>(sm, t1) += e1;
                e1 = T(0);
                __syncwarp();
            }
        }
    }
};

template <class T, bool VEC, bool WIN>
__global__ void __launch_bounds__(32) cs_compress_kernel(CompressContigParams<T> p, int64_t s) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const int g = blockIdx.x;
    T *bins = reinterpret_cast<T *>(smem_raw);
    for (int i = lane; i < p.bin_cnt + 96; i += 32) bins[i] = T(0);
    __syncwarp();
    if (g >= p.split.W) return;
    const int64_t u0 = p.split.start(g), u1 = p.split.start(g + 1);
    if (u0 >= u1) return;
    const uint32_t s_bytes = (uint32_t)(s * (int64_t)sizeof(T));
    const uint32_t list_off = (uint32_t)p.bin_cnt * sizeof(T);
    const uint32_t dummy = list_off + (64 + lane) * sizeof(T);
    // a padding element's word: the lane's dummy slot, in the unwindowed encoding
    const uint32_t pad = (uint32_t)((s + 64 + lane) * (int64_t)sizeof(T));
    const int64_t full = p.L / 512;  // batches with all 512 elements inside the vector
    int64_t v = u0 / p.tpv;
    int64_t u = u0;
    while (u < u1) {
        const int64_t vbeg = v * p.tpv;
        const int64_t kend = min(u1, vbeg + p.tpv) - vbeg;
        const T *xv = p.X + v * p.x_ld;
        int64_t k = u - vbeg;
        const int64_t kfull = min(kend, full);
        CsBatch<T, false> ba, bb;
        if (k < kfull) ba.template load<VEC>(p, xv, k, lane, pad);
        while (k < kfull) {
            if (k + 1 < kfull) bb.template load<VEC>(p, xv, k + 1, lane, pad);
            ba.template run<WIN>(p, smem_raw, s_bytes, list_off, dummy, lane);
            if (++k >= kfull) break;
            if (k + 1 < kfull) ba.template load<VEC>(p, xv, k + 1, lane, pad);
            bb.template run<WIN>(p, smem_raw, s_bytes, list_off, dummy, lane);
            ++k;
        }
        for (; k < kend; ++k) {
            CsBatch<T, true> bc;
            bc.template load<false>(p, xv, k, lane, pad);
            bc.template run<WIN>(p, smem_raw, s_bytes, list_off, dummy, lane);
        }
        const bool exclusive = (u0 <= vbeg) && (vbeg + p.tpv <= u1);
        flush_vector(p, bins, g, v, exclusive, lane);
        u = vbeg + kend;
        ++v;
    }
}

// ---- strided-vector compress: element (k, v) at X[v + k*x_ld]; lane = vector ----------
template <class T>
struct CompressStridedParams {
    const T *X;
    int64_t x_ld;
    int64_t L, nv;
    const int32_t *bucket;
    const uint8_t *negative;
    int nnz;
    int64_t bin_lo;
    int bin_cnt;
    T *Y;
    int64_t y_es, y_vs;
    T alpha, beta;
    int beta_zero;
    T *partials;  // [group][split][bin_cnt][32] when P > 1
    int64_t klen;
    int P;
    int64_t ngroups;
};

template <class T>
__global__ void __launch_bounds__(256) compress_strided_kernel(CompressStridedParams<T> p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const int64_t unit = (int64_t)blockIdx.x * warps + wib;
    T *bins = reinterpret_cast<T *>(smem_raw) + (int64_t)wib * p.bin_cnt * 32;
    for (int i = lane; i < p.bin_cnt * 32; i += 32) bins[i] = T(0);
    __syncwarp();
    if (unit >= p.ngroups * p.P) return;
    const int64_t grp = unit / p.P;
    const int split = (int)(unit % p.P);
    const int64_t v = grp * 32 + lane;
    const bool vok = v < p.nv;
    const int64_t k0 = split * p.klen, k1 = min(p.L, k0 + p.klen);
    constexpr int UK = 8;
    for (int64_t k = k0; k < k1; k += UK) {
        T xs[UK];
#pragma unroll
        for (int b = 0; b < UK; ++b) xs[b] = (vok && k + b < k1) ? __ldg(p.X + v + (k + b) * p.x_ld) : T(0);
#pragma unroll
        for (int b = 0; b < UK; ++b) {
            if (k + b >= k1) break;
            for (int e = 0; e < p.nnz; ++e) {
                const int64_t idx = (k + b) * p.nnz + e;
                int bb = __ldg(p.bucket + idx) - (int)p.bin_lo;
                if ((unsigned)bb < (unsigned)p.bin_cnt) {
                    T x = __ldg(p.negative + idx) ? -xs[b] : xs[b];
                    bins[bb * 32 + lane] += x;
                }
            }
        }
    }
    __syncwarp();
    if (p.P == 1) {
        if (vok)
            for (int i = 0; i < p.bin_cnt; ++i) {
                T *yp = p.Y + (p.bin_lo + i) * p.y_es + v * p.y_vs;
                T r = p.alpha * bins[i * 32 + lane];
                if (!p.beta_zero) r += p.beta * *yp;
                *yp = r;
            }
    } else {
        T *part = p.partials + unit * (int64_t)p.bin_cnt * 32;
        for (int i = 0; i < p.bin_cnt; ++i) part[i * 32 + lane] = bins[i * 32 + lane];
    }
}

template <class T>
__global__ void compress_strided_reduce_kernel(CompressStridedParams<T> p) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t per = (int64_t)p.bin_cnt * 32;
    if (t >= p.ngroups * per) return;
    const int64_t grp = t / per;
    const int64_t rem = t % per;
    const int i = (int)(rem / 32), lane = (int)(rem % 32);
    const int64_t v = grp * 32 + lane;
    if (v >= p.nv) return;
    T acc = T(0);
    for (int sp = 0; sp < p.P; ++sp) acc += p.partials[(grp * p.P + sp) * per + rem];
    T *yp = p.Y + (p.bin_lo + i) * p.y_es + v * p.y_vs;
    T r = p.alpha * acc;
    if (!p.beta_zero) r += p.beta * *yp;
    *yp = r;
}

// ---- expand: Y(j, v) = alpha * sum_e sign(j,e) * X(bucket(j,e), v) + beta * Y(j, v) ------
template <class T>
__global__ void expand_kernel(const T *X, int64_t x_es, int64_t x_vs, int64_t L, int64_t nv,
                              const int32_t *bucket, const uint8_t *negative, int nnz, T *Y, int64_t y_es,
                              int64_t y_vs, int out_contig, T alpha, T beta, int beta_zero) {
    // fast thread index runs along the contiguous output dimension
    int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t b = blockIdx.y * (int64_t)blockDim.y + threadIdx.y;
    int64_t j = out_contig ? a : b;
    int64_t v = out_contig ? b : a;
    for (; (out_contig ? v : j) < (out_contig ? nv : L); ) {
        if (j < L && v < nv) {
            T acc = T(0);
            for (int e = 0; e < nnz; ++e) {
                const int64_t idx = j * nnz + e;
                T x = X[(int64_t)bucket[idx] * x_es + v * x_vs];
                acc += negative[idx] ? -x : x;
            }
            T *yp = Y + j * y_es + v * y_vs;
            T r = alpha * acc;
            if (!beta_zero) r += beta * *yp;
            *yp = r;
        }
        if (out_contig) v += (int64_t)gridDim.y * blockDim.y;
        else j += (int64_t)gridDim.y * blockDim.y;
    }
}

// ------------------------------------------------------------------------------------
// host-side launchers
// ------------------------------------------------------------------------------------
template <class T>
int sparse_compress(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv,
                    T *Y, int64_t y_es, int64_t y_vs, double alpha, double beta) {
    const int64_t L = sk->L, s = sk->s;
    const size_t es = sizeof(T);
    const int cap = ctx->smem_optin - 1024;
    const bool beta_zero = beta == 0.0;
    const T a = (T)(alpha * sk->scale);
    if (nv == 0) return RLA_OK;
    if (x_es == 1) {
        // contiguous vectors
        if (!sk->tile_flags)
            return set_error(ctx, RLA_E_UNSUPPORTED, "compression dimension above 2^22 on the contiguous-vector path");
        int warps = (int)std::min<int64_t>(12, cap / (int64_t)((s + 64) * es));
        int bin_cnt = (int)s;
        if (warps < 1) {
            warps = 4;
            bin_cnt = (int)(cap / (4 * es)) - 64;
        }
        const bool bm = sk->batch_mode != 0;          // CountSketch: 512-element batches
        const int64_t tpv = bm ? ceil_div(L, 512) : ceil_div(L, 128);
        const int64_t total = tpv * nv;
        const bool vec = (x_vs % (16 / es) == 0) && ((uintptr_t)X % 16 == 0);
        if (bm) {
            // one warp per CTA: bins + 64 list entries + 32 dummy slots
            int bins_cs = (int)s;
            if ((int64_t)(s + 96) * (int64_t)es > cap) bins_cs = (int)(cap / (4 * es)) - 96;
            const size_t smem = (size_t)(bins_cs + 96) * es;
            const bool win = bins_cs < s;
            auto kern = win ? (vec ? cs_compress_kernel<T, true, true> : cs_compress_kernel<T, false, true>)
                            : (vec ? cs_compress_kernel<T, true, false> : cs_compress_kernel<T, false, false>);
            RLA_CUDA_TRY(ctx, set_smem_max(kern));
            int per_sm = 1;
            RLA_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32, smem));
            const int64_t total_cs = tpv * nv;
            int64_t W = (int64_t)ctx->sm_count * std::max(per_sm, 1);
            W = std::max<int64_t>(1, std::min<int64_t>(W, ceil_div(total_cs, 32)));
            void *part = nullptr;
            int *cnt = nullptr;
            RLA_TRY(scratch_get(ctx, (size_t)(2 * W) * bins_cs * es, &part));
            RLA_TRY(counters_get(ctx, (size_t)nv, &cnt));
            CompressContigParams<T> p{X, x_vs, L, nv, sk->meta, sk->tile_flags, sk->extra, (int)sk->nnz, 0, bins_cs, Y, y_es,
                                      y_vs, a, (T)beta, beta_zero, (T *)part, cnt, tpv, Split::make(total_cs, (int)W)};
            for (int64_t lo = 0; lo < s; lo += bins_cs) {
                p.bin_lo = lo;
                p.bin_cnt = (int)std::min<int64_t>(bins_cs, s - lo);
                kern<<<(int)W, 32, smem, ctx->stream>>>(p, s);
                RLA_TRY(check_launch(ctx, "cs_compress"));
            }
            return RLA_OK;
        }
        const int blocks_per_sm = std::max(1, cap / (int)(warps * (bin_cnt + 64) * es + 1));
        int64_t W = (int64_t)ctx->sm_count * blocks_per_sm * warps;
        // fill the GPU even with few vectors (at least two tiles per warp), but split one
        // vector over at most 64 warps: its last warp adds all of their partial bin arrays
        W = std::min<int64_t>(W, std::min<int64_t>(ceil_div(total, 2), nv * 64));
        W = std::max<int64_t>(W, 1);
        const int blocks = ceil_div_i(W, warps);
        const size_t smem = (size_t)warps * (bin_cnt + 64) * es;
        void *part = nullptr;
        int *cnt = nullptr;
        RLA_TRY(scratch_get(ctx, (size_t)(2 * W) * bin_cnt * es, &part));
        RLA_TRY(counters_get(ctx, (size_t)nv, &cnt));
        CompressContigParams<T> p{X, x_vs, L, nv, sk->meta, sk->tile_flags, sk->extra, (int)sk->nnz, 0, bin_cnt, Y, y_es, y_vs, a, (T)beta,
                                  beta_zero, (T *)part, cnt, tpv, Split::make(total, (int)W)};
        for (int64_t lo = 0; lo < s; lo += bin_cnt) {
            p.bin_lo = lo;
            p.bin_cnt = (int)std::min<int64_t>(bin_cnt, s - lo);
            auto launch = [&](auto kern) {
                set_smem_max(kern);
                kern<<<blocks, warps * 32, smem, ctx->stream>>>(p);
            };
            const bool win = p.bin_cnt < s;
            const bool n1 = sk->nnz == 1;
#define RLA_CC(V, W, N) launch(compress_contig_kernel<T, V, W, N>)
            if (vec) {
                if (win) { if (n1) RLA_CC(true, true, true); else RLA_CC(true, true, false); }
                else { if (n1) RLA_CC(true, false, true); else RLA_CC(true, false, false); }
            } else {
                if (win) { if (n1) RLA_CC(false, true, true); else RLA_CC(false, true, false); }
                else { if (n1) RLA_CC(false, false, true); else RLA_CC(false, false, false); }
            }
#undef RLA_CC
            RLA_TRY(check_launch(ctx, "compress_contig"));
        }
        return RLA_OK;
    }
    // strided vectors (x_vs == 1): lane = vector
    int warps = 8;
    int bin_cnt = (int)std::min<int64_t>(s, cap / (int64_t)(warps * 32 * es));
    if (bin_cnt < 1) return set_error(ctx, RLA_E_UNSUPPORTED, "shared memory too small");
    if (bin_cnt < s && bin_cnt < 64) {
        warps = 2;
        bin_cnt = (int)std::min<int64_t>(s, cap / (int64_t)(warps * 32 * es));
    }
    const int64_t ngroups = ceil_div(nv, 32);
    const int64_t want = (int64_t)ctx->sm_count * 2 * warps;
    int P = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(want, ngroups), ceil_div(L, 256)));
    const int64_t klen = ceil_div(L, P);
    P = (int)ceil_div(L, klen);
    const size_t smem = (size_t)warps * bin_cnt * 32 * es;
    void *part = nullptr;
    if (P > 1) RLA_TRY(scratch_get(ctx, (size_t)ngroups * P * bin_cnt * 32 * es, &part));
    CompressStridedParams<T> p{X, x_es, L, nv, sk->bucket, sk->negative, (int)sk->nnz, 0, bin_cnt, Y, y_es, y_vs,
                               a, (T)beta, beta_zero, (T *)part, klen, P, ngroups};
    for (int64_t lo = 0; lo < s; lo += bin_cnt) {
        p.bin_lo = lo;
        p.bin_cnt = (int)std::min<int64_t>(bin_cnt, s - lo);
        const int64_t units = ngroups * P;
        set_smem_max(compress_strided_kernel<T>);
        compress_strided_kernel<T><<<ceil_div_i(units, warps), warps * 32, smem, ctx->stream>>>(p);
        RLA_TRY(check_launch(ctx, "compress_strided"));
        if (P > 1) {
            const int64_t n = ngroups * (int64_t)p.bin_cnt * 32;
            compress_strided_reduce_kernel<T><<<ceil_div_i(n, 256), 256, 0, ctx->stream>>>(p);
            RLA_TRY(check_launch(ctx, "compress_strided_reduce"));
        }
    }
    return RLA_OK;
}

template <class T>
int sparse_expand(rla_ctx *ctx, const rla_sketch *sk, const T *X, int64_t x_es, int64_t x_vs, int64_t nv, T *Y,
                  int64_t y_es, int64_t y_vs, double alpha, double beta) {
    if (nv == 0) return RLA_OK;
    const int64_t L = sk->L;
    const int out_contig = y_es == 1;
    const int64_t fast = out_contig ? L : nv, slow = out_contig ? nv : L;
    dim3 block(128, 2);
    dim3 grid(ceil_div_i(fast, 128), (unsigned)std::min<int64_t>(ceil_div(slow, 2), 65535));
    expand_kernel<T><<<grid, block, 0, ctx->stream>>>(X, x_es, x_vs, L, nv, sk->bucket, sk->negative, (int)sk->nnz, Y,
                                                      y_es, y_vs, out_contig, (T)(alpha * sk->scale), (T)beta,
                                                      beta == 0.0);
    return check_launch(ctx, "sparse_expand");
}

template int sparse_compress<float>(rla_ctx *, const rla_sketch *, const float *, int64_t, int64_t, int64_t, float *,
                                    int64_t, int64_t, double, double);
template int sparse_compress<double>(rla_ctx *, const rla_sketch *, const double *, int64_t, int64_t, int64_t,
                                     double *, int64_t, int64_t, double, double);
template int sparse_expand<float>(rla_ctx *, const rla_sketch *, const float *, int64_t, int64_t, int64_t, float *,
                                  int64_t, int64_t, double, double);
template int sparse_expand<double>(rla_ctx *, const rla_sketch *, const double *, int64_t, int64_t, int64_t, double *,
                                   int64_t, int64_t, double, double);

}  // namespace rla
