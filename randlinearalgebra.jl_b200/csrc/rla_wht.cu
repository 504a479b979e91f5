// rla_wht.cu -- Walsh-Hadamard based sketches (SRHT, FJLT).
//
// The reference applies SRHT block by block: zero a padding buffer, copy A, run the
// natural-order fwht! per column (log2 N passes over the column), gather the sampled
// rows (srht.jl:220-286, fwht.jl:21-70).  Here the left compress (S*A on column-major A)
// is one pass over A:
//
//   N = N1 * CH with CH = 2^14 (FP32) / 2^12 (FP64).  For a padded column x,
//   y[r] = sum_c (-1)^popc(r1 & c) * Z_c[r2],  r = r1*CH + r2,
//   where Z_c = H_CH (D x)[c*CH : (c+1)*CH] is the natural-order WHT of chunk c.
//
// A CTA of 2^TB threads holds one chunk in registers (2^TB values per thread): pass A
// covers the chunk bits held in registers after a 16-byte coalesced load (sign flip fused
// into the load), the chunk goes through a bank-conflict-free swizzled shared buffer,
// pass B covers the remaining bits, and each sampled row accumulates +-Z_c[r2] into a
// shared accumulator.  Columns are split over the persistent grid (stream-K); a column
// shared by several CTAs is finished by the last CTA to arrive, which adds the partial
// accumulators in CTA order, so results are reproducible bit for bit.
#include "rla_internal.cuh"

namespace rla {

struct SplitB {
    int64_t total;
    int W;
    __host__ __device__ int64_t start(int g) const { return (int64_t)((__int128)g * total / W); }
    __device__ int owner(int64_t u) const {
        int g = (int)((__int128)u * W / total);
        if (g >= W) g = W - 1;
        while (g + 1 < W && start(g + 1) <= u) ++g;
        while (g > 0 && start(g) > u) --g;
        return g;
    }
};

template <class T>
struct WhtCfg;
template <>
struct WhtCfg<float> {
    static constexpr int TB = 7, VB = 2;
};
template <>
struct WhtCfg<double> {
    static constexpr int TB = 6, VB = 1;
};

template <int TB, class T>
__device__ __forceinline__ void wht_regs(T (&r)[1 << TB]) {
#pragma unroll
    for (int h = 0; h < TB; ++h) {
#pragma unroll
        for (int q = 0; q < (1 << TB); ++q) {
            if (!(q & (1 << h))) {
                T a = r[q], b = r[q | (1 << h)];
                r[q] = a + b;
                r[q | (1 << h)] = a - b;
            }
        }
    }
}

template <class T>
struct SrhtParams {
    const T *X;
    int64_t x_ld;  // element (j, v) at X[j + v*x_ld]
    int64_t L, N;
    const uint32_t *signbits;
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
    SplitB split;
};

// Position of chunk element e in the swizzled shared buffer: the low 3 bits of the
// 16-byte vector index are XOR-ed with bits [VB+TB, VB+TB+3) of e.
template <int TB, int VB>
__device__ __forceinline__ int swz(int e) {
    int f = e >> VB;
    f ^= (e >> (VB + TB)) & 7;
    return (f << VB) | (e & ((1 << VB) - 1));
}

template <class T, bool VEC>
__global__ void __launch_bounds__(1 << WhtCfg<T>::TB) srht_fused_kernel(SrhtParams<T> p) {
    constexpr int TB = WhtCfg<T>::TB, VB = WhtCfg<T>::VB;
    constexpr int CH = 2 * TB, NT = 1 << TB, VW = 1 << VB, KV = 1 << (TB - VB);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Z = reinterpret_cast<T *>(smem_raw);
    T *acc = Z + (1 << CH);
    __shared__ int last_flag;
    const int t = threadIdx.x;
    const int g = blockIdx.x;
    for (int i = t; i < p.s_cnt; i += NT) acc[i] = T(0);
    __syncthreads();
    const int64_t u0 = p.split.start(g), u1 = p.split.start(g + 1);
    if (u0 >= u1) return;
    const int t_lo = t & (VW - 1), t_hi = t >> VB;
    int64_t v = u0 / p.cpv;
    int64_t u = u0;
    while (u < u1) {
        const int64_t vbeg = v * p.cpv;
        const int64_t vend = min(u1, vbeg + p.cpv);
        const T *xv = p.X + v * p.x_ld;
        for (int64_t c = u - vbeg; c < vend - vbeg; ++c) {
            T r[1 << TB];
            const int64_t cbase = c << CH;
            // ---- pass A: coalesced 16-byte loads, sign flip ----
#pragma unroll
            for (int k = 0; k < KV; ++k) {
                const int64_t e0 = cbase + ((int64_t)t << VB) + ((int64_t)k << (VB + TB));
                T vals[VW];
                if (VEC && e0 + VW <= p.L) {
                    if constexpr (sizeof(T) == 4) {
                        float4 q = __ldg(reinterpret_cast<const float4 *>(xv + e0));
                        vals[0] = q.x; vals[1] = q.y; vals[2] = q.z; vals[3] = q.w;
                    } else {
                        double2 q = __ldg(reinterpret_cast<const double2 *>(xv + e0));
                        vals[0] = q.x; vals[1] = q.y;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < VW; ++i) vals[i] = (e0 + i < p.L) ? __ldg(xv + e0 + i) : T(0);
                }
                const uint32_t bits = __ldg(p.signbits + (e0 >> 5)) >> (e0 & 31);
#pragma unroll
                for (int i = 0; i < VW; ++i) r[k * VW + i] = ((bits >> i) & 1u) ? vals[i] : -vals[i];
            }
            wht_regs<TB>(r);
#pragma unroll
            for (int k = 0; k < KV; ++k) {
                const int f = (t ^ (k & 7)) + (k << TB);
                if constexpr (sizeof(T) == 4) {
                    *reinterpret_cast<float4 *>(Z + (f << VB)) = make_float4(r[k * 4], r[k * 4 + 1], r[k * 4 + 2], r[k * 4 + 3]);
                } else {
                    *reinterpret_cast<double2 *>(Z + (f << VB)) = make_double2(r[k * 2], r[k * 2 + 1]);
                }
            }
            __syncthreads();
            // ---- pass B: remaining TB bits ----
#pragma unroll
            for (int q = 0; q < (1 << TB); ++q) {
                const int e = t_lo + (q << VB) + (t_hi << (VB + TB));
                r[q] = Z[swz<TB, VB>(e)];
            }
            wht_regs<TB>(r);
#pragma unroll
            for (int q = 0; q < (1 << TB); ++q) {
                const int e = t_lo + (q << VB) + (t_hi << (VB + TB));
                Z[swz<TB, VB>(e)] = r[q];
            }
            __syncthreads();
            // ---- sampled rows: acc[i] += (-1)^popc(r1 & c) * Z_c[r2] ----
            for (int i = t; i < p.s_cnt; i += NT) {
                const int32_t row = __ldg(p.rows + p.s_lo + i);
                const T z = Z[swz<TB, VB>(row & ((1 << CH) - 1))];
                const int par = __popcll((unsigned long long)(row >> CH) & (unsigned long long)c) & 1;
                acc[i] += par ? -z : z;
            }
            __syncthreads();
        }
        // ---- column finished in this CTA's range ----
        const bool first = (v == u0 / p.cpv);
        const bool exclusive = (u0 <= vbeg) && (vbeg + p.cpv <= u1);
        if (exclusive) {
            for (int i = t; i < p.s_cnt; i += NT) {
                T *yp = p.Y + (p.s_lo + i) * p.y_es + v * p.y_vs;
                T res = p.alpha * acc[i];
                if (!p.beta_zero) res += p.beta * *yp;
                *yp = res;
                acc[i] = T(0);
            }
        } else {
            T *part = p.partials + (int64_t)(2 * g + (first ? 0 : 1)) * p.s_cnt;
            for (int i = t; i < p.s_cnt; i += NT) {
                part[i] = acc[i];
                acc[i] = T(0);
            }
            __threadfence();
            __syncthreads();
            const int gf = p.split.owner(vbeg), gl = p.split.owner(vbeg + p.cpv - 1);
            if (t == 0) {
                int ncontrib = 0;
                for (int gg = gf; gg <= gl; ++gg) ncontrib += p.split.start(gg + 1) > p.split.start(gg);
                int old = atomicAdd(&p.counters[v], 1);
                last_flag = (old == ncontrib - 1);
            }
            __syncthreads();
            if (last_flag) {
                __threadfence();
                for (int i = t; i < p.s_cnt; i += NT) {
                    T a = T(0);
                    for (int gg = gf; gg <= gl; ++gg) {
                        const int64_t sg = p.split.start(gg);
                        if (p.split.start(gg + 1) <= sg) continue;
                        const int sl = 2 * gg + ((sg / p.cpv) == v ? 0 : 1);
                        a += __ldcg(p.partials + (int64_t)sl * p.s_cnt + i);
                    }
                    T *yp = p.Y + (p.s_lo + i) * p.y_es + v * p.y_vs;
                    T res = p.alpha * a;
                    if (!p.beta_zero) res += p.beta * *yp;
                    *yp = res;
                }
                if (t == 0) p.counters[v] = 0;
            }
        }
        __syncthreads();
        u = vend;
        ++v;
    }
}

// Small padded sizes (N <= 2^(2*TB)): one CTA per column, the whole padded column in
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
    constexpr int TB = WhtCfg<T>::TB, VB = WhtCfg<T>::VB, CH = 2 * TB;
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
    int s_win = (int)std::min<int64_t>(s, (cap / 2 - (int64_t)(es << CH)) / (int64_t)es);
    if (s_win < 256) s_win = (int)std::min<int64_t>(s, (cap - (int64_t)(es << CH)) / (int64_t)es);
    const int64_t total = cpv * nv;
    const int blocks_per_sm = std::max(1, cap / (int)((es << CH) + s_win * es + 64));
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
        cudaFuncSetAttribute(srht_small_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const int grid = (int)std::min<int64_t>(nv, (int64_t)ctx->sm_count * 8);
        srht_small_kernel<T><<<grid, 256, smem, ctx->stream>>>(Xc, ldx, L, N, nv, sk->signbits, sk->rows, s, Y, y_es,
                                                               y_vs, a, (T)beta, beta_zero);
        return check_launch(ctx, "srht_small");
    }
    int *cnt = nullptr;
    RLA_TRY(counters_get(ctx, (size_t)nv, &cnt));
    const bool vec = (ldx % (int64_t)(1 << VB) == 0) && ((uintptr_t)Xc % 16 == 0);
    SrhtParams<T> p{Xc, ldx, L, N, sk->signbits, sk->rows, 0, s_win, Y, y_es, y_vs, a, (T)beta, beta_zero,
                    (T *)(scratch + off_partials), cnt, cpv, SplitB{total, (int)W}};
    const size_t smem = (es << CH) + (size_t)s_win * es;
    for (int64_t lo = 0; lo < s; lo += s_win) {
        p.s_lo = lo;
        p.s_cnt = (int)std::min<int64_t>(s_win, s - lo);
        if (vec) {
            cudaFuncSetAttribute(srht_fused_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            srht_fused_kernel<T, true><<<(int)W, 1 << TB, smem, ctx->stream>>>(p);
        } else {
            cudaFuncSetAttribute(srht_fused_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            srht_fused_kernel<T, false><<<(int)W, 1 << TB, smem, ctx->stream>>>(p);
        }
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
