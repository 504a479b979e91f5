// rla_ctx.cu -- context, error reporting and workspace management.
#include <stdarg.h>

#include "rla_internal.cuh"

namespace rla {

int set_error(rla_ctx *ctx, int code, const char *fmt, ...) {
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return code;
}

int g_smem_optin = 227 * 1024;

int check_launch(rla_ctx *ctx, const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(ctx, RLA_E_CUDA, "%s launch failed: %s", what, cudaGetErrorString(e));
    return RLA_OK;
}

// Grows a context buffer in the order of ctx->stream, the only stream its users launch on:
// the old buffer goes back to the context's pool after the work already queued there, and the
// new one comes from the pool.  Nothing waits on the host: a synchronous cudaFree waits for
// every stream of every context on the device, which stalls the other workers of a server
// for as long as they keep the device busy.  Growth is refused while ctx->stream captures a
// graph (the captured launches would keep a buffer that the next growth releases).
static int grow_stream_ordered(rla_ctx *ctx, rla::Scratch *buf, size_t bytes, const char *what) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    RLA_CUDA_TRY(ctx, cudaStreamIsCapturing(ctx->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return set_error(ctx, RLA_E_ARG, "%s must be sized before graph capture (%zu bytes needed)", what, bytes);
    if (buf->ptr) RLA_CUDA_TRY(ctx, cudaFreeAsync(buf->ptr, ctx->stream));
    buf->ptr = nullptr;
    buf->bytes = 0;
    RLA_CUDA_TRY(ctx, pool_malloc_s(ctx, &buf->ptr, bytes, ctx->stream));
    buf->bytes = bytes;
    return RLA_OK;
}

int scratch_get(rla_ctx *ctx, size_t bytes, void **out) {
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    if (ctx->scratch.bytes < bytes) {
        RLA_TRY(grow_stream_ordered(ctx, &ctx->scratch, bytes, "scratch"));
        if ((int64_t)bytes > ctx->scratch_high_water) ctx->scratch_high_water = (int64_t)bytes;
    }
    *out = ctx->scratch.ptr;
    return RLA_OK;
}

int counters_get(rla_ctx *ctx, size_t n, int **out) {
    size_t bytes = ((n * sizeof(int)) + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    if (ctx->counters.bytes < bytes) {
        RLA_TRY(grow_stream_ordered(ctx, &ctx->counters, bytes, "counters"));
        RLA_CUDA_TRY(ctx, cudaMemsetAsync(ctx->counters.ptr, 0, bytes, ctx->stream));
    }
    *out = (int *)ctx->counters.ptr;
    return RLA_OK;
}

}  // namespace rla

using namespace rla;

extern "C" {

int rla_version(void) { return 1; }

const char *rla_status_string(int status) {
    switch (status) {
        case RLA_OK: return "ok";
        case RLA_E_DIM: return "DimensionMismatch";
        case RLA_E_ARG: return "ArgumentError";
        case RLA_E_DOMAIN: return "DomainError";
        case RLA_E_OOM: return "out of device memory";
        case RLA_E_CUDA: return "CUDA error";
        case RLA_E_TIMEOUT: return "device wait timed out";
        case RLA_E_NUMERIC: return "numerical breakdown";
        case RLA_E_UNSUPPORTED: return "unsupported";
        case RLA_E_CANCELLED: return "cancelled";
        default: return "unknown status";
    }
}

int rla_ctx_create(int device, void *stream, rla_ctx **out) {
    if (!out) return RLA_E_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return RLA_E_CUDA;
    if (device < 0 || device >= ndev) return RLA_E_ARG;
    rla_ctx *ctx = new rla_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return RLA_E_CUDA;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete ctx;
        return RLA_E_CUDA;
    }
    if (prop.major < 10) {
        delete ctx;
        return RLA_E_UNSUPPORTED;  // sm_100a kernels only
    }
    {
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        if (cudaMemPoolCreate(&ctx->pool, &pp) != cudaSuccess) {
            delete ctx;
            return RLA_E_CUDA;
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = (int)prop.sharedMemPerBlockOptin;
    g_smem_optin = ctx->smem_optin;
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->owns_stream = false;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return RLA_E_CUDA;
        }
        ctx->owns_stream = true;
    }
    *out = ctx;
    return RLA_OK;
}

int rla_ctx_destroy(rla_ctx *ctx) {
    if (!ctx) return RLA_OK;
    cudaSetDevice(ctx->device);
    if (ctx->scratch.ptr) cudaFreeAsync(ctx->scratch.ptr, ctx->stream);
    if (ctx->counters.ptr) cudaFreeAsync(ctx->counters.ptr, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->tc_status) cudaFree(ctx->tc_status);
    for (auto &v : ctx->timed)
        for (auto &e : v) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    if (ctx->owns_stream) cudaStreamDestroy(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return RLA_OK;
}

const char *rla_ctx_last_error(const rla_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int rla_ctx_synchronize(rla_ctx *ctx) {
    if (!ctx) return RLA_E_ARG;
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return RLA_OK;
}

int rla_ctx_set_stream(rla_ctx *ctx, void *stream) {
    if (!ctx) return RLA_E_ARG;
    if ((cudaStream_t)stream == ctx->stream) return RLA_OK;
    if (ctx->owns_stream) {
        RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        RLA_CUDA_TRY(ctx, cudaStreamDestroy(ctx->stream));
        ctx->owns_stream = false;
    }
    ctx->stream = (cudaStream_t)stream;  // NULL selects the legacy default stream
    return RLA_OK;
}

int rla_ctx_set_timing(rla_ctx *ctx, int enable) {
    if (!ctx) return RLA_E_ARG;
    ctx->timing = enable != 0;
    return RLA_OK;
}

int rla_ctx_set_wait_limit(rla_ctx *ctx, double seconds) {
    if (!ctx) return RLA_E_ARG;
    if (!(seconds >= 0.0) || seconds > 60.0)
        return set_error(ctx, RLA_E_ARG, "wait limit must lie in [0, 60] seconds");
    ctx->wait_ns = (uint64_t)(seconds * 1e9);
    return RLA_OK;
}

int rla_ctx_kernel_time(rla_ctx *ctx, int kernel_class, double *ms_total, int64_t *launches) {
    if (!ctx || !ms_total || !launches) return RLA_E_ARG;
    if (kernel_class < 0 || kernel_class > 3) return set_error(ctx, RLA_E_ARG, "unknown kernel class %d", kernel_class);
    RLA_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    double tot = 0.0;
    auto &v = ctx->timed[kernel_class];
    for (auto &e : v) {
        float ms = 0.f;
        RLA_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, e.first, e.second));
        tot += ms;
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    *ms_total = tot;
    *launches = (int64_t)v.size();
    v.clear();
    return RLA_OK;
}

int rla_ctx_scratch_bytes(const rla_ctx *ctx, int64_t *bytes) {
    if (!ctx || !bytes) return RLA_E_ARG;
    *bytes = ctx->scratch_high_water;
    return RLA_OK;
}

}  // extern "C"
