"""Host mirror of the serving loop (rla_server_*) and of sketch-and-solve (rla_sketch_solve).

`Server` queues least-squares and RandSVD requests on Float32 device tensors; the library's
worker threads run them (continuous batching in RLA_SERVE_BATCHED mode) and `poll` returns
(tag, latency in seconds, status) for finished requests.  The caller keeps every tensor of a
request alive until the request is polled as done."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._arrays import Operand
from .errors import ArgumentError


def sketch_solve(S, A, b, x) -> None:
    """x = argmin ||S(Ax - b)|| (Float32 device tensors; S a completed Left compressor)."""
    Aop = Operand(A, "col")
    if Aop.trans:
        Aop = Operand(Aop.t.t().contiguous().t(), "col")
    ctx = L.Context.get(S._ctx.device)
    L.check(L.lib().rla_sketch_solve(ctx.handle, S.handle, Aop.rows, Aop.cols, Aop.ptr, Aop.ld, b.data_ptr(),
                                     x.data_ptr()), ctx.handle)


class Server:
    def __init__(self, device: int = 0, slots: int = 4, max_group: int = 64, plain: bool = False,
                 memory_budget: int = 0, sketch_cache_bytes: int = 0):
        cfg = L.ServerConfig(device, slots, max_group, L.RLA_SERVE_PLAIN if plain else L.RLA_SERVE_BATCHED,
                             memory_budget, sketch_cache_bytes)
        h = ctypes.c_void_p()
        st = L.lib().rla_server_start(ctypes.byref(cfg), ctypes.byref(h))
        if st != L.RLA_OK:
            raise ArgumentError(f"rla_server_start failed ({L.lib().rla_status_string(st).decode()})")
        self.handle = h
        self._keep = {}

    def submit_ls(self, A, b, x, seed: int, tag: int) -> None:
        """A (m x n), b (m), x (n): column-major Float32 device tensors."""
        m, n = A.shape
        r = L.Request(L.RLA_REQ_LS, m, n, 0, A.data_ptr(), A.stride(1), b.data_ptr(), x.data_ptr(), None, 0, None,
                      None, 0, seed, tag)
        self._submit(r, (A, b, x), tag)

    def submit_svd(self, A, k: int, U, S, V, seed: int, tag: int) -> None:
        m, n = A.shape
        r = L.Request(L.RLA_REQ_SVD, m, n, k, A.data_ptr(), A.stride(1), None, None, U.data_ptr(), U.stride(1),
                      S.data_ptr(), V.data_ptr(), V.stride(1), seed, tag)
        self._submit(r, (A, U, S, V), tag)

    def _submit(self, r, keep, tag):
        if L.lib().rla_server_submit(self.handle, ctypes.byref(r)) != L.RLA_OK:
            raise ArgumentError("request rejected (dimensions or buffers)")
        self._keep[tag] = keep

    def poll(self, max_n: int = 4096):
        tags = np.zeros(max_n, np.uint64)
        lat = np.zeros(max_n, np.float64)
        st = np.zeros(max_n, np.int32)
        cnt = ctypes.c_int()
        L.lib().rla_server_poll(self.handle, tags.ctypes.data, lat.ctypes.data, st.ctypes.data, max_n, ctypes.byref(cnt))
        out = []
        for i in range(cnt.value):
            out.append((int(tags[i]), float(lat[i]), int(st[i])))
            self._keep.pop(int(tags[i]), None)
        return out

    def last_error(self) -> str:
        raw = L.lib().rla_server_last_error(self.handle)
        return raw.decode() if raw else ""

    def wait_idle(self) -> None:
        L.lib().rla_server_wait_idle(self.handle)

    def cancel(self, tag: int) -> None:
        """Remove a queued request; poll then reports it with status RLA_E_CANCELLED."""
        if L.lib().rla_server_cancel(self.handle, tag) != L.RLA_OK:
            raise ArgumentError(f"no queued request with tag {tag}")

    def inject_alloc_failure(self, tag: int) -> None:
        """Fault injection: the request with this tag fails its workspace allocation."""
        L.check(L.lib().rla_server_inject_alloc_failure(self.handle, tag))

    def stats(self) -> dict:
        st = L.ServerStats()
        L.check(L.lib().rla_server_get_stats(self.handle, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in L.ServerStats._fields_}

    def stop(self) -> None:
        if self.handle:
            L.lib().rla_server_stop(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
