"""Range approximators: host-side mirror of RangeFinder / RandSVD
(src/Approximators.jl, src/Approximators/RangeApproximators/*).

``rapproximate_`` runs the whole power-iteration / CholeskyQR2 / SVD pipeline in
librla_b200.so; the factors stay on the device.  As in the reference
(randsvd.jl:183-187), RandSVD's U, S and V are Float64 by default; ``factor_type`` keeps
them in the matrix's own type instead.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib as L
from ._arrays import Operand, rla_dtype, size2, zeros_like_layout
from .compressors import (Compressor, CompressorRecipe, Left, Right, SparseSign, complete_compressor)
from .errors import ArgumentError, DomainError
import warnings


class Approximator:
    """src/Approximators.jl:10."""


class RangeApproximator(Approximator):
    """src/Approximators.jl:44."""


class ApproximatorRecipe:
    """src/Approximators.jl:19."""


class RangeApproximatorRecipe(ApproximatorRecipe):
    """src/Approximators.jl:57."""


class RangeFinder(RangeApproximator):
    """rangefinder.jl:71-95."""

    def __init__(self, compressor: Optional[Compressor] = None, orthogonalize: bool = False, power_its: int = 0,
                 precision: int = L.RLA_PREC_NATIVE):
        if power_its < 0:
            raise ArgumentError("Field `power_its` must be non-negative.")
        self.compressor = SparseSign(cardinality=Right()) if compressor is None else compressor
        self.power_its, self.orthogonalize, self.precision = int(power_its), bool(orthogonalize), precision


class RandSVD(RangeApproximator):
    """randsvd.jl:337-361."""

    def __init__(self, compressor: Optional[Compressor] = None, orthogonalize: bool = False, power_its: int = 0,
                 block_size: int = 0, precision: int = L.RLA_PREC_NATIVE, factor_type=np.float64):
        if power_its < 0:
            raise ArgumentError("Field `power_its` must be non-negative.")
        if block_size < 0:
            raise ArgumentError("Field `block_size` must be non-negative.")
        self.compressor = SparseSign(cardinality=Right()) if compressor is None else compressor
        self.power_its, self.orthogonalize, self.block_size = int(power_its), bool(orthogonalize), int(block_size)
        self.precision, self.factor_type = precision, factor_type


class RangeFinderRecipe(RangeApproximatorRecipe):
    """rangefinder.jl:108-115: n_rows, n_cols, compressor, power_its, orthogonalize, range."""

    def __init__(self, approx: RangeFinder, A, seed=None):
        if isinstance(approx.compressor.cardinality, Left):
            warnings.warn("Compressor with cardinality `Left` being applied from `Right`.")
        self.compressor = complete_compressor(approx.compressor, A, seed=seed)
        self.n_rows = size2(A)[0]
        self.n_cols = self.compressor.n_cols
        self.power_its, self.orthogonalize, self.precision = approx.power_its, approx.orthogonalize, approx.precision
        self.range = None


class RandSVDRecipe(RangeApproximatorRecipe):
    """randsvd.jl:386-396: n_rows, n_cols, compressor, power_its, orthogonalize, U, S, V, buffer."""

    def __init__(self, approx: RandSVD, A, seed=None):
        if isinstance(approx.compressor.cardinality, Left):
            warnings.warn("Compressor with cardinality `Left` being applied from `Right`.")
        self.compressor = complete_compressor(approx.compressor, A, seed=seed)
        self.n_rows, self.n_cols = size2(A)
        self.power_its, self.orthogonalize, self.precision = approx.power_its, approx.orthogonalize, approx.precision
        self.factor_type = approx.factor_type
        self.block_size = self.n_cols if approx.block_size == 0 else approx.block_size
        self.U = self.S = self.V = None


class ApproximatorAdjoint:
    """src/Approximators.jl:122-132."""

    def __init__(self, parent):
        self.parent = parent

    @property
    def T(self):
        return self.parent


def _adjoint(R):
    return ApproximatorAdjoint(R)


RangeFinderRecipe.T = property(_adjoint)
RandSVDRecipe.T = property(_adjoint)


def is_approximator_operand(x) -> bool:
    return isinstance(x, (ApproximatorRecipe, ApproximatorAdjoint))


def complete_approximator(approx: Approximator, A, seed=None):
    """complete_approximator (rangefinder.jl:117-132, randsvd.jl:398-422)."""
    if isinstance(approx, RandSVD):
        return RandSVDRecipe(approx, A, seed)
    if isinstance(approx, RangeFinder):
        return RangeFinderRecipe(approx, A, seed)
    raise ArgumentError(f"No method `complete_approximator` exists for approximator of type"
                        f"{type(approx).__name__} and matrix of type {type(A).__name__}.")


def _range_params(R):
    p = L.RangeParams()
    p.power_its = R.power_its
    p.orthogonalize = 1 if R.orthogonalize else 0
    p.precision = R.precision
    return p


def rapproximate_(R, A) -> None:
    """rapproximate!(::RangeFinderRecipe | ::RandSVDRecipe, A)."""
    import torch
    if not isinstance(R, (RangeFinderRecipe, RandSVDRecipe)):
        raise ArgumentError(f"No `rapproximate` method exists for approximator of type"
                            f"{type(R).__name__} and matrix of type {type(A).__name__}.")
    Aop = Operand(A, "col")
    if Aop.trans:
        Aop = Operand(Aop.t.t().contiguous().t(), "col")
    S = R.compressor
    ctx = L.Context.get(S._ctx.device)
    m, n = Aop.rows, Aop.cols
    l = S.n_cols
    tdt = torch.float32 if Aop.dtype == 0 else torch.float64
    p = _range_params(R)
    dev = Aop.t.device
    if isinstance(R, RangeFinderRecipe):
        Q = torch.empty(l, m, dtype=tdt, device=dev).t()
        L.check(L.lib().rla_rangefinder(ctx.handle, S.handle, Aop.dtype, m, n, Aop.ptr, Aop.ld, ctypes.byref(p),
                                        Q.data_ptr(), m), ctx.handle)
        R.range = Q
        return
    fdt = rla_dtype(R.factor_type)
    ft = torch.float32 if fdt == 0 else torch.float64
    U = torch.empty(l, m, dtype=ft, device=dev).t()
    V = torch.empty(l, n, dtype=ft, device=dev).t()
    Sv = torch.empty(l, dtype=torch.float64, device=dev)
    L.check(L.lib().rla_randsvd(ctx.handle, S.handle, Aop.dtype, m, n, Aop.ptr, Aop.ld, ctypes.byref(p), fdt,
                                U.data_ptr(), m, Sv.data_ptr(), V.data_ptr(), n), ctx.handle)
    R.U, R.S, R.V = U, Sv, V


def rapproximate(approx: Approximator, A, seed=None):
    """rapproximate(approx, A) = complete_approximator then rapproximate! (src/Approximators.jl:222)."""
    R = complete_approximator(approx, A, seed)
    rapproximate_(R, A)
    return R


def size(R, dim=None):
    shp = (R.parent.n_cols, R.parent.n_rows) if isinstance(R, ApproximatorAdjoint) else (R.n_rows, R.n_cols)
    if dim is None:
        return shp
    if dim < 1 or dim > 2:
        raise DomainError("`dim` must be 1 or 2.")
    return shp[dim - 1]


def mul_(C, X, Y, alpha: float = 1.0, beta: float = 0.0) -> None:
    """mul! for approximator recipes (randsvd.jl:448-543, rangefinder.jl:151-191)."""
    if is_approximator_operand(X):
        side, R, A = L.RLA_SIDE_LEFT, X, Y
    else:
        side, R, A = L.RLA_SIDE_RIGHT, Y, X
    trans_r = 1 if isinstance(R, ApproximatorAdjoint) else 0
    Rp = R.parent if trans_r else R
    orient = "col" if side == L.RLA_SIDE_LEFT else "row"
    Aop = Operand(A, orient)
    Cop = Operand(C, orient, writable=True)
    if isinstance(Rp, RandSVDRecipe):
        if Rp.U is None:
            raise ArgumentError("rapproximate! has not been run on this recipe.")
        U, V, Sv = Rp.U, Rp.V, Rp.S
        m, n, k = U.shape[0], V.shape[0], U.shape[1]
        fdt = rla_dtype(U.dtype)
        args = (U.data_ptr(), U.stride(1), Sv.data_ptr(), V.data_ptr(), V.stride(1))
    else:
        if Rp.range is None:
            raise ArgumentError("rapproximate! has not been run on this recipe.")
        U = Rp.range
        m, k = U.shape
        n = k
        fdt = rla_dtype(U.dtype)
        args = (U.data_ptr(), U.stride(1), None, None, 1)
    ctx = L.Context.get(U.device.index)
    st = L.lib().rla_lowrank_mul(ctx.handle, fdt, Cop.dtype, side, trans_r, m, n, k, *args,
                                 Cop.rows, Cop.cols, Cop.ptr, Cop.ld, Cop.trans,
                                 Aop.rows, Aop.cols, Aop.ptr, Aop.ld, Aop.trans, float(alpha), float(beta))
    L.check(st, ctx.handle)
    Cop.finish()


def _times(X, Y):
    if is_approximator_operand(X):
        r_rows = size(X, 1)
        a_cols = size2(Y)[1]
        C = zeros_like_layout(Y, (r_rows,) if a_cols == 1 else (r_rows, a_cols))
    else:
        r_cols = size(Y, 2)
        a_rows = size2(X)[0] if X.ndim == 2 else 1
        C = zeros_like_layout(X, (r_cols,) if (a_rows == 1 and X.ndim == 1) else (a_rows, r_cols))
    mul_(C, X, Y)
    return C


for _cls in (RangeFinderRecipe, RandSVDRecipe, ApproximatorAdjoint):
    _cls.__matmul__ = lambda self, A: _times(self, A)
    _cls.__rmatmul__ = lambda self, A: _times(A, self)


class RandSVDBatch:
    """Many RandSVD instances at once (rla_randsvd_batch_*): instance i is
    rapproximate!(RandSVD(compressor=Gaussian(Right(), compression_dim=k_i), power_its,
    orthogonalize), A_i) with Float32 A_i; the factors U_i (m_i x k_i, Float32), S_i (k_i,
    Float64) and V_i (n_i x k_i, Float32) are allocated here.  Omega_i is the Gaussian
    sketch complete_compressor would draw with seed seeds[i].  The first run() captures the
    grouped launch sequence as a CUDA graph; later runs replay it.  With precision =
    RLA_PREC_SPLIT_BF16 the passes over A of the instances with k <= 64 run as grouped
    tensor-core products (split BF16, FP64 accumulation across k-chunks)."""

    def __init__(self, As, ks, seeds, power_its: int = 0, orthogonalize: bool = False, autotune: bool = True,
                 precision: int = 0):
        import torch
        if not (len(As) == len(ks) == len(seeds)):
            raise ArgumentError("As, ks and seeds must have the same length.")
        self.As, self.U, self.S, self.V = [], [], [], []
        probs = (L.SvdProblem * max(1, len(As)))()
        dev = None
        for i, (A, k, sd) in enumerate(zip(As, ks, seeds)):
            Aop = Operand(A, "col")
            if Aop.host or Aop.dtype != 0:
                raise ArgumentError("Batched RandSVD takes Float32 device matrices.")
            if Aop.trans:
                Aop = Operand(Aop.t.t().contiguous().t(), "col")
            dev = Aop.t.device
            m, n = Aop.rows, Aop.cols
            U = torch.empty(k, m, dtype=torch.float32, device=dev).t()
            S = torch.empty(k, dtype=torch.float64, device=dev)
            V = torch.empty(k, n, dtype=torch.float32, device=dev).t()
            self.As.append(Aop.t)
            self.U.append(U)
            self.S.append(S)
            self.V.append(V)
            probs[i] = L.SvdProblem(m, n, int(k), Aop.ptr, Aop.ld, U.data_ptr(), m, S.data_ptr(), V.data_ptr(), n,
                                    int(sd) & (2**64 - 1))
        self.ctx = L.Context.get(None if dev is None else dev.index)
        p = L.RangeParams()
        p.power_its = int(power_its)
        p.orthogonalize = 1 if orthogonalize else 0
        if precision not in (L.RLA_PREC_NATIVE, L.RLA_PREC_SPLIT_BF16):
            raise ArgumentError(f"Unknown precision mode {precision}.")
        p.precision = int(precision)
        h = ctypes.c_void_p()
        L.check(L.lib().rla_randsvd_batch_create(self.ctx.handle, len(As), probs, ctypes.byref(p),
                                                 L.RLA_BATCH_AUTOTUNE if autotune else 0, ctypes.byref(h)),
                self.ctx.handle)
        self.handle = h
        self._probs = probs

    def run(self) -> None:
        ctx = L.Context.get(self.ctx.device)
        L.check(L.lib().rla_randsvd_batch_run(ctx.handle, self.handle), ctx.handle)

    def tiles(self, c: int):
        a, b, ch = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        L.check(L.lib().rla_randsvd_batch_tiles(self.handle, c, ctypes.byref(a), ctypes.byref(b), ctypes.byref(ch)))
        return a.value, b.value, ch.value

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                L.lib().rla_randsvd_batch_destroy(self.handle)
                self.handle = None
        except Exception:
            pass
