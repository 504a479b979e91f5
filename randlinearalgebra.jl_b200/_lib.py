"""ctypes binding of librla_b200.so (the C ABI declared in include/rla_b200.h).

The product path has no fallback: if the shared library is missing, or no B200 is
visible, every entry point raises.  Loading the library itself needs no GPU, so the
CPU-only tests can check that every declared symbol is exported.
"""
from __future__ import annotations

import ctypes
import os
import threading

from .errors import ArgumentError, DimensionMismatch, DomainError, RLAError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librla_b200.so")

RLA_OK, RLA_E_DIM, RLA_E_ARG, RLA_E_DOMAIN, RLA_E_OOM, RLA_E_CUDA, RLA_E_TIMEOUT, RLA_E_NUMERIC, RLA_E_UNSUPPORTED = range(9)
RLA_F32, RLA_F64 = 0, 1
RLA_LEFT, RLA_RIGHT = 0, 1
RLA_SPARSE_SIGN, RLA_COUNT_SKETCH, RLA_SRHT, RLA_FJLT, RLA_GAUSSIAN, RLA_SAMPLING = range(6)
RLA_DIST_UNIFORM, RLA_DIST_L2NORM, RLA_DIST_AGMON = range(3)
RLA_PROJ_KACZMARZ, RLA_PROJ_COLUMN = 0, 1
RLA_ERR_FULL_RESIDUAL, RLA_ERR_LS_GRADIENT, RLA_ERR_COMPRESSED_RESIDUAL = range(3)
RLA_SIDE_LEFT, RLA_SIDE_RIGHT = 0, 1
RLA_PREC_NATIVE, RLA_PREC_SPLIT_BF16 = 0, 1

i64 = ctypes.c_int64
vp = ctypes.c_void_p


class SketchParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("card", ctypes.c_int), ("dtype", ctypes.c_int),
                ("compression_dim", i64), ("long_dim", i64), ("nnz", i64), ("block_size", i64),
                ("sparsity", ctypes.c_double), ("seed", ctypes.c_uint64)]


class SketchInfo(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("card", ctypes.c_int), ("dtype", ctypes.c_int),
                ("n_rows", i64), ("n_cols", i64), ("compression_dim", i64), ("long_dim", i64),
                ("nnz", i64), ("block_size", i64), ("padded", i64), ("k_nnz", i64),
                ("sparsity", ctypes.c_double), ("scale", ctypes.c_double), ("draw_count", ctypes.c_uint64)]


class RangeParams(ctypes.Structure):
    _fields_ = [("power_its", i64), ("orthogonalize", ctypes.c_int), ("precision", ctypes.c_int)]


class SvdProblem(ctypes.Structure):
    _fields_ = [("m", i64), ("n", i64), ("k", i64), ("A", vp), ("lda", i64), ("U", vp), ("ldu", i64),
                ("S", vp), ("V", vp), ("ldv", i64), ("seed", ctypes.c_uint64)]


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("m", i64), ("n", i64), ("k", i64), ("A", vp), ("lda", i64), ("b", vp),
                ("x", vp), ("U", vp), ("ldu", i64), ("S", vp), ("V", vp), ("ldv", i64), ("seed", ctypes.c_uint64),
                ("tag", ctypes.c_uint64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int), ("max_group", ctypes.c_int), ("mode", ctypes.c_int),
                ("memory_budget", ctypes.c_uint64), ("sketch_cache_bytes", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_int64), ("running", ctypes.c_int64), ("workspace_bytes", ctypes.c_uint64),
                ("cache_bytes", ctypes.c_uint64), ("cache_entries", ctypes.c_int64), ("evictions", ctypes.c_int64)]


RLA_E_CANCELLED = 9
RLA_REQ_LS, RLA_REQ_SVD = 0, 1
RLA_SERVE_BATCHED, RLA_SERVE_PLAIN = 0, 1
RLA_BATCH_AUTOTUNE = 1
RLA_BATCH_EAGER = 2

# name -> (restype, argtypes); every function declared in include/rla_b200.h
SIGNATURES = {
    "rla_version": (ctypes.c_int, []),
    "rla_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rla_ctx_create": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(vp)]),
    "rla_ctx_destroy": (ctypes.c_int, [vp]),
    "rla_ctx_last_error": (ctypes.c_char_p, [vp]),
    "rla_ctx_synchronize": (ctypes.c_int, [vp]),
    "rla_ctx_set_stream": (ctypes.c_int, [vp, vp]),
    "rla_ctx_scratch_bytes": (ctypes.c_int, [vp, ctypes.POINTER(i64)]),
    "rla_sketch_create": (ctypes.c_int, [vp, ctypes.POINTER(SketchParams), ctypes.POINTER(vp)]),
    "rla_sketch_update": (ctypes.c_int, [vp, vp]),
    "rla_sketch_destroy": (ctypes.c_int, [vp]),
    "rla_sketch_get_info": (ctypes.c_int, [vp, ctypes.POINTER(SketchInfo)]),
    "rla_sketch_get_draws": (ctypes.c_int, [vp, vp, vp, vp, vp, vp]),
    "rla_sketch_set_draws": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, i64]),
    "rla_sketch_mul": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, i64, i64, vp, i64, ctypes.c_int,
                                      i64, i64, vp, i64, ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    "rla_sketch_mul_async": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, i64, i64, vp, i64, ctypes.c_int,
                                            i64, i64, vp, i64, ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    "rla_rangefinder": (ctypes.c_int, [vp, vp, ctypes.c_int, i64, i64, vp, i64, ctypes.POINTER(RangeParams), vp, i64]),
    "rla_randsvd": (ctypes.c_int, [vp, vp, ctypes.c_int, i64, i64, vp, i64, ctypes.POINTER(RangeParams), ctypes.c_int,
                                   vp, i64, vp, vp, i64]),
    "rla_lowrank_mul": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, i64, i64, i64,
                                       vp, i64, vp, vp, i64, i64, i64, vp, i64, ctypes.c_int, i64, i64, vp, i64,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    "rla_srht_mul_noalloc": (ctypes.c_int, [vp, vp, i64, i64, vp, i64, i64, i64, vp, i64, ctypes.c_double,
                                            ctypes.c_double]),
    "rla_randsvd_batch_create": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(SvdProblem), ctypes.POINTER(RangeParams),
                                                ctypes.c_int, ctypes.POINTER(vp)]),
    "rla_randsvd_batch_run": (ctypes.c_int, [vp, vp]),
    "rla_randsvd_batch_tiles": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(i64)]),
    "rla_randsvd_batch_destroy": (ctypes.c_int, [vp]),
    "rla_randsvd_grouped": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(SvdProblem), ctypes.POINTER(RangeParams)]),
    "rla_sketch_solve": (ctypes.c_int, [vp, vp, i64, i64, vp, i64, vp, vp]),
    "rla_sampling_create": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, i64, i64, ctypes.c_int, ctypes.c_int, i64,
                                           ctypes.c_uint64, ctypes.POINTER(vp)]),
    "rla_sampling_update": (ctypes.c_int, [vp, vp, i64, i64, vp, i64, vp, i64, vp, i64, vp]),
    "rla_proj_create": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, i64, i64, ctypes.c_double,
                                       ctypes.POINTER(vp)]),
    "rla_proj_start": (ctypes.c_int, [vp, vp, vp, i64, vp, vp, vp]),
    "rla_proj_step": (ctypes.c_int, [vp, vp, vp, i64, vp, vp, vp]),
    "rla_proj_error": (ctypes.c_int, [vp, vp, ctypes.c_int, vp, i64, vp, vp, vp, ctypes.POINTER(ctypes.c_double)]),
    "rla_proj_workspace": (ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]),
    "rla_proj_destroy": (ctypes.c_int, [vp]),
    "rla_ihs_create": (ctypes.c_int, [vp, vp, ctypes.c_int, i64, i64, ctypes.c_double, ctypes.POINTER(vp)]),
    "rla_ihs_start": (ctypes.c_int, [vp, vp, vp, i64, vp, vp, vp, vp]),
    "rla_ihs_step": (ctypes.c_int, [vp, vp, vp, i64, vp, vp, vp, vp]),
    "rla_ihs_errors": (ctypes.c_int, [vp, vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "rla_ihs_solve": (ctypes.c_int, [vp, vp, vp, i64, vp, vp, vp, vp, i64, i64, ctypes.c_double, ctypes.c_int,
                                     vp, i64, ctypes.POINTER(i64), ctypes.POINTER(ctypes.c_int)]),
    "rla_ihs_workspace": (ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                         ctypes.POINTER(vp)]),
    "rla_ihs_destroy": (ctypes.c_int, [vp]),
    "rla_server_start": (ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
    "rla_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(Request)]),
    "rla_server_poll": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "rla_server_wait_idle": (ctypes.c_int, [vp]),
    "rla_server_last_error": (ctypes.c_char_p, [vp]),
    "rla_server_stop": (ctypes.c_int, [vp]),
    "rla_server_cancel": (ctypes.c_int, [vp, ctypes.c_uint64]),
    "rla_server_inject_alloc_failure": (ctypes.c_int, [vp, ctypes.c_uint64]),
    "rla_server_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
    "rla_ctx_set_timing": (ctypes.c_int, [vp, ctypes.c_int]),
    "rla_ctx_set_wait_limit": (ctypes.c_int, [vp, ctypes.c_double]),
    "rla_sketch_mul_sparse_t": (ctypes.c_int, [vp, vp, i64, i64, vp, i64, i64, i64, i64, vp, vp, vp,
                                               ctypes.c_double, ctypes.c_double]),
    "rla_ctx_kernel_time": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i64)]),
    "rla_gemm_bf16x3": (ctypes.c_int, [vp, ctypes.c_int, i64, i64, i64, vp, i64, vp, i64, vp, i64,
                                       ctypes.c_double, ctypes.c_double]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """The loaded shared library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RLAError(f"librla_b200.so not found at {LIB_PATH}; build it with "
                               "`python randlinearalgebra.jl_b200/build.py` (no CPU fallback exists)")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def check(status: int, ctx=None) -> None:
    if status == RLA_OK:
        return
    msg = ""
    if ctx is not None:
        raw = lib().rla_ctx_last_error(ctx)
        msg = raw.decode() if raw else ""
    if not msg:
        msg = lib().rla_status_string(status).decode()
    if status == RLA_E_DIM:
        raise DimensionMismatch(msg)
    if status == RLA_E_ARG:
        raise ArgumentError(msg)
    if status == RLA_E_DOMAIN:
        raise DomainError(msg)
    raise RLAError(f"{lib().rla_status_string(status).decode()}: {msg}")


class Context:
    """One library context per CUDA device.  Each call re-points it at torch's current
    stream so work is ordered after the kernels that produced its inputs."""

    _per_device: dict = {}

    def __init__(self, device: int):
        self.device = device
        h = vp()
        check(lib().rla_ctx_create(device, None, ctypes.byref(h)))
        self.handle = h

    @classmethod
    def get(cls, device: int | None = None) -> "Context":
        import torch
        if not torch.cuda.is_available():
            raise RLAError("no CUDA device is visible; the B200 library has no CPU fallback")
        if device is None:
            device = torch.cuda.current_device()
        ctx = cls._per_device.get(device)
        if ctx is None:
            ctx = cls._per_device[device] = Context(device)
        stream = torch.cuda.current_stream(device).cuda_stream
        check(lib().rla_ctx_set_stream(ctx.handle, vp(stream)), ctx.handle)
        return ctx

    def __del__(self):
        try:
            if self.handle:
                lib().rla_ctx_destroy(self.handle)
        except Exception:
            pass
