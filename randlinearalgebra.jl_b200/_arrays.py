"""Operand marshalling between Python arrays and the C ABI's (pointer, rows, cols, ld,
trans) column-major convention.

CUDA torch tensors are passed in place when their layout is column-major (the Julia
layout) or row-major (then they are the transpose of a column-major matrix, like Julia's
``transpose(X)`` wrapper).  Host arrays (numpy, CPU tensors) are copied to the device
and results copied back, which is the end-to-end path a host caller pays for.
"""
from __future__ import annotations

import numpy as np

from .errors import ArgumentError

_NP_OF = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}


def rla_dtype(dt) -> int:
    import torch
    if dt in (torch.float32, np.float32) or dt == np.dtype(np.float32) or dt == "Float32":
        return 0
    if dt in (torch.float64, np.float64) or dt == np.dtype(np.float64) or dt == "Float64":
        return 1
    raise ArgumentError(f"Element type {dt} is not supported by the B200 library (Float32 or Float64).")


class Operand:
    """A logical (rows x cols) matrix on the device.  1-D inputs are columns
    (orient='col') or rows (orient='row')."""

    def __init__(self, x, orient: str = "col", writable: bool = False):
        import torch
        self.orig = x
        self.writable = writable
        self.host = not (isinstance(x, torch.Tensor) and x.is_cuda)
        self.was_1d = x.ndim == 1
        if x.ndim not in (1, 2):
            raise ArgumentError("Only vectors and matrices are supported.")
        if self.host:
            if isinstance(x, torch.Tensor):
                if x.dtype not in (torch.float32, torch.float64):
                    raise ArgumentError(f"Element type {x.dtype} is not supported (Float32 or Float64).")
                # strides are preserved; pinned memory makes the copy asynchronous DMA
                self.t = x.to("cuda", non_blocking=x.is_pinned())
            else:
                arr = np.asarray(x)
                if arr.dtype not in _NP_OF:
                    raise ArgumentError(f"Element type {arr.dtype} is not supported (Float32 or Float64).")
                t = torch.from_numpy(np.asfortranarray(arr) if arr.ndim == 2 else np.ascontiguousarray(arr))
                self.t = t.to("cuda", non_blocking=False)
        else:
            self.t = x
        self.dtype = rla_dtype(self.t.dtype)
        self.copy_back = None
        t = self.t
        if t.ndim == 1:
            n = t.shape[0]
            st = t.stride(0) if n > 1 else 1
            if orient == "col":
                self.rows, self.cols = n, 1
                if st == 1:
                    self.trans, self.ld = 0, max(n, 1)
                else:
                    self.trans, self.ld = 1, st
            else:
                self.rows, self.cols = 1, n
                self.trans, self.ld = 0, max(st, 1)
        else:
            r, c = t.shape
            sr, sc = t.stride()
            self.rows, self.cols = r, c
            if (sr == 1 or r <= 1) and (c <= 1 or sc >= max(r, 1)):
                self.trans, self.ld = 0, (sc if c > 1 else max(r, 1))
            elif (sc == 1 or c <= 1) and (r <= 1 or sr >= max(c, 1)):
                self.trans, self.ld = 1, (sr if r > 1 else max(c, 1))
            else:
                tmp = t.t().contiguous().t()
                if writable:
                    self.copy_back = (t, tmp)
                self.t = tmp
                self.trans, self.ld = 0, max(r, 1)
        self.ptr = self.t.data_ptr()

    def finish(self) -> None:
        """Propagate results to the caller's array (only for outputs that needed a copy)."""
        if not self.writable:
            return
        if self.copy_back is not None:
            dst, tmp = self.copy_back
            dst.copy_(tmp)
        if self.host:
            import torch
            if isinstance(self.orig, torch.Tensor):
                self.orig.copy_(self.t)
            else:
                self.orig[...] = self.t.cpu().numpy()


def zeros_like_layout(ref, shape, dtype=None):
    """Zero array on the same side (device/host) as `ref`, column-major for matrices."""
    import torch
    if isinstance(ref, torch.Tensor) and ref.is_cuda:
        dt = ref.dtype if dtype is None else dtype
        if len(shape) == 1:
            return torch.zeros(shape[0], dtype=dt, device=ref.device)
        return torch.zeros(shape[1], shape[0], dtype=dt, device=ref.device).t()
    if isinstance(ref, torch.Tensor):
        dt = ref.dtype if dtype is None else dtype
        pin = ref.is_pinned()
        if len(shape) == 1:
            return torch.zeros(shape[0], dtype=dt, pin_memory=pin)
        return torch.zeros(shape[1], shape[0], dtype=dt, pin_memory=pin).t()
    arr = np.asarray(ref)
    return np.zeros(shape, dtype=arr.dtype if dtype is None else dtype, order="F")


def size2(x):
    """(size(x,1), size(x,2)) with Julia's convention for vectors."""
    return (x.shape[0], 1) if x.ndim == 1 else (x.shape[0], x.shape[1])
