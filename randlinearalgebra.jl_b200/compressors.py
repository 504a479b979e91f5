"""Compressors: the host-side mirror of RandLinearAlgebra.jl's Compressor API.

Same names, fields, defaults and error messages as the reference
(src/Compressors.jl, src/Compressors/{sparse_sign,count_sketch,srht,fjlt,gaussian}.jl);
Julia's bang functions end in ``_`` here (``update_compressor!`` -> ``update_compressor_``,
``mul!`` -> ``mul_``).  A recipe owns a device-side sketch in librla_b200.so; applying it
calls the C ABI with the operands' device pointers.  Draws are made on the device; the
reference-layout fields (``op``, ``signs``, ``mat`` ...) are downloaded on first access
so a recipe can be re-materialised and compared the way the reference tests do.
"""
from __future__ import annotations

import ctypes
import itertools
import math
import threading
from typing import Optional

import numpy as np

from . import _lib as L
from ._arrays import Operand, rla_dtype, size2, zeros_like_layout
from .errors import ArgumentError, DomainError


# ----------------------------------------------------------------------------------
# Cardinality (src/Compressors.jl:24-45)
# ----------------------------------------------------------------------------------
class Cardinality:
    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))

    def __repr__(self):
        return f"{type(self).__name__}()"


class Left(Cardinality):
    """Matrix multiplication from the left."""


class Right(Cardinality):
    """Matrix multiplication from the right."""


class Undef(Cardinality):
    """Matrix multiplication is undefined."""


# ----------------------------------------------------------------------------------
# Seeds: the reference draws from Julia's global RNG; here every completed compressor
# takes the next seed of a process-wide sequence (reset with `seed_`).
# ----------------------------------------------------------------------------------
_seed_lock = threading.Lock()
_seed_iter = itertools.count(0x5EED)


def seed_(seed: int) -> None:
    """Analogue of Random.seed!: restart the sequence of sketch seeds."""
    global _seed_iter
    with _seed_lock:
        _seed_iter = itertools.count(int(seed) * 0x9E3779B1 & 0xFFFFFFFFFFFF)


def _next_seed() -> int:
    with _seed_lock:
        return next(_seed_iter)


# ----------------------------------------------------------------------------------
# Compressors (user-facing parameter structs)
# ----------------------------------------------------------------------------------
class Compressor:
    """Abstract supertype of compression techniques (src/Compressors.jl:7)."""


class SparseSign(Compressor):
    """src/Compressors/sparse_sign.jl:65-127."""

    def __init__(self, cardinality: Cardinality = None, compression_dim: int = 2, nnz: Optional[int] = None,
                 type=np.float64):
        cardinality = Left() if cardinality is None else cardinality
        nnz = min(8, compression_dim) if nnz is None else nnz
        if compression_dim <= 0:
            raise ArgumentError("Field `compression_dim` must be positive.")
        if nnz > compression_dim:
            raise ArgumentError(f"Number of non-zero indices, {nnz}, must be less than or equal to compression "
                                f"dimension, {compression_dim}.")
        if nnz <= 0:
            raise ArgumentError("Field `nnz` must be positive.")
        object.__setattr__(self, "cardinality", cardinality)
        object.__setattr__(self, "compression_dim", int(compression_dim))
        object.__setattr__(self, "nnz", int(nnz))
        object.__setattr__(self, "type", type)

    def __setattr__(self, sym, val):
        # setproperty! (sparse_sign.jl:101-127)
        if sym == "compression_dim":
            if val <= 0:
                raise ArgumentError("Field `compression_dim` must be positive.")
            if self.nnz > val:
                raise ArgumentError(f"New `compression_dim`, {val}, must be greater than or equal to current "
                                    f"`nnz`, {self.nnz}.")
        elif sym == "nnz":
            if val <= 0:
                raise ArgumentError("Field `nnz` must be positive.")
            if val > self.compression_dim:
                raise ArgumentError(f"New `nnz`, {val}, must be less than or equal to current `compression_dim`, "
                                    f"{self.compression_dim}.")
        object.__setattr__(self, sym, val)


class CountSketch(Compressor):
    """src/Compressors/count_sketch.jl:60-90."""

    def __init__(self, cardinality: Cardinality = None, compression_dim: int = 2, type=np.float64):
        cardinality = Left() if cardinality is None else cardinality
        if compression_dim <= 0:
            raise ArgumentError("Field 'compression_dim' must be positive.")
        if cardinality == Undef():
            raise ArgumentError("`cardinality` must be specified as `Left()` or `Right()`."
                                "`Undef()` is not allowed in `CountSketch` structure.")
        self.cardinality, self.compression_dim, self.type = cardinality, int(compression_dim), type


class SRHT(Compressor):
    """src/Compressors/srht.jl:60-88."""

    def __init__(self, cardinality: Cardinality = None, compression_dim: int = 2, block_size: int = 10,
                 type=np.float64):
        cardinality = Left() if cardinality is None else cardinality
        if compression_dim <= 0:
            raise ArgumentError("Field `compression_dim` must be positive.")
        if block_size <= 0:
            raise ArgumentError("Field `block_size` must be positive.")
        if isinstance(cardinality, Undef):
            raise ArgumentError("Cardinality must be of type `Left` or `Right`.")
        self.cardinality, self.compression_dim, self.block_size, self.type = (
            cardinality, int(compression_dim), int(block_size), type)


class FJLT(Compressor):
    """src/Compressors/fjlt.jl (FJLT struct and keyword constructor)."""

    def __init__(self, cardinality: Cardinality = None, compression_dim: int = 2, block_size: int = 10,
                 sparsity: float = 0.0, type=np.float64):
        cardinality = Left() if cardinality is None else cardinality
        if compression_dim <= 0:
            raise ArgumentError("Field `compression_dim` must be positive.")
        if sparsity < 0 or sparsity > 1:
            raise ArgumentError("Field `sparsity` must be between 0 and 1.")
        if block_size <= 0:
            raise ArgumentError("Field `block_size` must be positive.")
        if isinstance(cardinality, Undef):
            raise ArgumentError("Cardinality must be of type `Left` or `Right`.")
        self.cardinality, self.compression_dim, self.block_size, self.sparsity, self.type = (
            cardinality, int(compression_dim), int(block_size), float(sparsity), type)


class Gaussian(Compressor):
    """src/Compressors/gaussian.jl:49-70."""

    def __init__(self, cardinality: Cardinality = None, compression_dim: int = 2, type=np.float64):
        cardinality = Left() if cardinality is None else cardinality
        if compression_dim <= 0:
            raise ArgumentError("Field 'compression_dim' must be positive.")
        self.cardinality, self.compression_dim, self.type = cardinality, int(compression_dim), type


_KIND = {SparseSign: L.RLA_SPARSE_SIGN, CountSketch: L.RLA_COUNT_SKETCH, SRHT: L.RLA_SRHT, FJLT: L.RLA_FJLT,
         Gaussian: L.RLA_GAUSSIAN}


# ----------------------------------------------------------------------------------
# Recipes
# ----------------------------------------------------------------------------------
class CompressorRecipe:
    """A completed compressor holding its device-side sketch (src/Compressors.jl:16).

    Common fields: ``cardinality``, ``n_rows``, ``n_cols``.  Reference-layout draws are
    available through the per-kind properties (downloaded once per draw)."""

    def __init__(self, compressor: Compressor, long_dim: int, seed: Optional[int], device: Optional[int]):
        kind = _KIND[type(compressor)]
        card = compressor.cardinality
        if not isinstance(card, (Left, Right)):
            raise ArgumentError("`cardinality` must be specified as `Left()` or `Right()`.")
        self.cardinality = card
        self.compressor = compressor
        self._dtype = rla_dtype(compressor.type)
        self._ctx = L.Context.get(device)
        p = L.SketchParams()
        p.kind = kind
        p.card = L.RLA_LEFT if isinstance(card, Left) else L.RLA_RIGHT
        p.dtype = self._dtype
        p.compression_dim = compressor.compression_dim
        p.long_dim = int(long_dim)
        p.nnz = getattr(compressor, "nnz", 1)
        p.block_size = getattr(compressor, "block_size", 10)
        p.sparsity = getattr(compressor, "sparsity", 0.0)
        p.seed = _next_seed() if seed is None else int(seed)
        h = ctypes.c_void_p()
        L.check(L.lib().rla_sketch_create(self._ctx.handle, ctypes.byref(p), ctypes.byref(h)), self._ctx.handle)
        self.handle = h
        self._cache = None
        self._refresh_info()

    def _refresh_info(self):
        info = L.SketchInfo()
        L.check(L.lib().rla_sketch_get_info(self.handle, ctypes.byref(info)))
        self.info = info
        self.n_rows = int(info.n_rows)
        self.n_cols = int(info.n_cols)

    @property
    def np_dtype(self):
        return np.float32 if self._dtype == 0 else np.float64

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                L.lib().rla_sketch_destroy(self.handle)
        except Exception:
            pass

    # ---- parity mode: draws in the reference's field layout -----------------------
    def draws(self) -> dict:
        """Download the current draws (0-based indices) in the reference's layout."""
        if self._cache is not None:
            return self._cache
        i = self.info
        kind = i.kind
        out = {}
        ctx = L.Context.get(self._ctx.device)
        if kind in (L.RLA_SPARSE_SIGN, L.RLA_COUNT_SKETCH):
            ne = i.long_dim * i.nnz
            idx = np.zeros(ne, np.int64)
            vals = np.zeros(ne, self.np_dtype)
            L.check(L.lib().rla_sketch_get_draws(ctx.handle, self.handle, idx.ctypes.data, vals.ctypes.data, None, None),
                    ctx.handle)
            out = {"rowval": idx, "nzval": vals}
        elif kind == L.RLA_SRHT:
            idx = np.zeros(i.compression_dim, np.int64)
            signs = np.zeros(i.padded, np.uint8)
            L.check(L.lib().rla_sketch_get_draws(ctx.handle, self.handle, idx.ctypes.data, None, signs.ctypes.data, None),
                    ctx.handle)
            out = {"op": idx, "signs": signs}
        elif kind == L.RLA_FJLT:
            ncol = i.padded if i.card == L.RLA_LEFT else i.compression_dim
            kptr = np.zeros(ncol + 1, np.int64)
            idx = np.zeros(max(i.k_nnz, 1), np.int64)
            vals = np.zeros(max(i.k_nnz, 1), self.np_dtype)
            signs = np.zeros(i.padded, np.uint8)
            L.check(L.lib().rla_sketch_get_draws(ctx.handle, self.handle, idx.ctypes.data, vals.ctypes.data,
                                                 signs.ctypes.data, kptr.ctypes.data), ctx.handle)
            out = {"colptr": kptr, "rowval": idx[: i.k_nnz], "nzval": vals[: i.k_nnz], "signs": signs}
        elif kind == L.RLA_SAMPLING:
            idx = np.zeros(i.compression_dim, np.int64)
            L.check(L.lib().rla_sketch_get_draws(ctx.handle, self.handle, idx.ctypes.data, None, None, None), ctx.handle)
            out = {"idx": idx}
        elif kind == L.RLA_GAUSSIAN:
            vals = np.zeros(i.n_rows * i.n_cols, self.np_dtype)
            L.check(L.lib().rla_sketch_get_draws(ctx.handle, self.handle, None, vals.ctypes.data, None, None), ctx.handle)
            out = {"op": vals.reshape(i.n_cols, i.n_rows).T}
        self._cache = out
        return out

    def load_draws(self, idx=None, vals=None, signs=None, kptr=None) -> None:
        """Replace the draws with externally supplied ones (0-based, reference layout)."""
        ctx = L.Context.get(self._ctx.device)
        def p(a, dt):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, dtype=dt)
            return a, a.ctypes.data
        a1, p1 = p(idx, np.int64)
        a2, p2 = p(None if vals is None else (np.asarray(vals).T.reshape(-1) if self.info.kind == L.RLA_GAUSSIAN else vals),
                   self.np_dtype)
        a3, p3 = p(signs, np.uint8)
        a4, p4 = p(kptr, np.int64)
        k_nnz = 0 if a1 is None else len(a1)
        L.check(L.lib().rla_sketch_set_draws(ctx.handle, self.handle, p1, p2, p3, p4, k_nnz), ctx.handle)
        self._cache = None
        self._refresh_info()

    # ---- operators -------------------------------------------------------------------
    @property
    def T(self):
        return CompressorAdjoint(self)

    def __matmul__(self, A):
        return _times(self, A)

    def __rmatmul__(self, A):
        return _times(A, self)

    __mul__ = __matmul__
    __rmul__ = __rmatmul__


class SparseSignRecipe(CompressorRecipe):
    """sparse_sign.jl:219-226: fields cardinality, n_rows, n_cols, nnz, scale, op."""

    @property
    def nnz(self):
        return int(self.info.nnz)

    @property
    def scale(self):
        sc = self.np_dtype(self.info.scale)
        return [-sc, sc]

    @property
    def op(self):
        """(colptr, rowval, nzval) of the CSC matrix (Left), or of op.parent (Right)."""
        d = self.draws()
        L_ = self.info.long_dim
        return (np.arange(0, L_ * self.nnz + 1, self.nnz, dtype=np.int64), d["rowval"], d["nzval"])


class CountSketchRecipe(CompressorRecipe):
    """count_sketch.jl:105-111: fields cardinality, compression_dim, n_rows, n_cols, mat."""

    @property
    def compression_dim(self):
        return int(self.info.compression_dim)

    @property
    def mat(self):
        d = self.draws()
        return (np.arange(self.info.long_dim + 1, dtype=np.int64), d["rowval"], d["nzval"])


class SRHTRecipe(CompressorRecipe):
    """srht.jl:125-133: fields cardinality, n_rows, n_cols, scale, op, signs, padding."""

    @property
    def scale(self) -> float:
        return float(self.info.scale)

    @property
    def op(self):
        return self.draws()["op"]

    @property
    def signs(self):
        return self.draws()["signs"].astype(bool)

    @property
    def padding_shape(self):
        N, b = int(self.info.padded), int(self.info.block_size)
        return (N, b) if self.info.card == L.RLA_LEFT else (b, N)


class FJLTRecipe(CompressorRecipe):
    """fjlt.jl:147-160: fields cardinality, n_rows, n_cols, sparsity, scale, op, signs, padding."""

    @property
    def sparsity(self) -> float:
        return float(self.info.sparsity)

    @property
    def scale(self) -> float:
        return float(self.info.scale)

    @property
    def op(self):
        d = self.draws()
        return (d["colptr"], d["rowval"], d["nzval"])

    @property
    def signs(self):
        return self.draws()["signs"].astype(bool)

    @property
    def padding_shape(self):
        N, b = int(self.info.padded), int(self.info.block_size)
        return (N, b) if self.info.card == L.RLA_LEFT else (b, N)


class GaussianRecipe(CompressorRecipe):
    """gaussian.jl:87-94: fields cardinality, compression_dim, n_rows, n_cols, scale, op."""

    @property
    def compression_dim(self):
        return int(self.info.compression_dim)

    @property
    def scale(self):
        return self.np_dtype(self.info.scale)

    @property
    def op(self):
        return self.draws()["op"]


_RECIPE = {SparseSign: SparseSignRecipe, CountSketch: CountSketchRecipe, SRHT: SRHTRecipe, FJLT: FJLTRecipe,
           Gaussian: GaussianRecipe}


class CompressorAdjoint:
    """src/Compressors.jl:94-104."""

    def __init__(self, parent: CompressorRecipe):
        self.parent = parent

    @property
    def T(self):
        return self.parent

    def __matmul__(self, A):
        return _times(self, A)

    def __rmatmul__(self, A):
        return _times(A, self)

    __mul__ = __matmul__
    __rmul__ = __rmatmul__


def adjoint(S):
    return S.parent if isinstance(S, CompressorAdjoint) else CompressorAdjoint(S)


transpose = adjoint


def size(S, dim: Optional[int] = None):
    """Base.size for recipes and their adjoints (src/Compressors.jl:310-323)."""
    shp = (S.parent.n_cols, S.parent.n_rows) if isinstance(S, CompressorAdjoint) else (S.n_rows, S.n_cols)
    if dim is None:
        return shp
    if dim < 1 or dim > 2:
        raise DomainError("`dim` must be 1 or 2.")
    return shp[dim - 1]


# ----------------------------------------------------------------------------------
# complete_compressor / update_compressor!  (src/Compressors.jl:126-305)
# ----------------------------------------------------------------------------------
def complete_compressor(compressor: Compressor, *args, seed: Optional[int] = None, device: Optional[int] = None):
    """complete_compressor(compressor, A), (compressor, A, b), (compressor, x, A, b), or
    (compressor, x) for a vector x (reshaped to a column)."""
    if len(args) == 3:
        A = args[1]
    elif len(args) in (1, 2):
        A = args[0]
    else:
        raise ArgumentError("complete_compressor takes (A), (A, b) or (x, A, b).")
    from . import sampling as _smp
    if isinstance(compressor, _smp.Sampling):
        return _smp.complete_sampling(compressor, args, seed, device)
    if type(compressor) not in _KIND:
        raise ArgumentError(f"No `complete_compressor` method exists for compressor of type "
                            f"{type(compressor).__name__} and matrix of type {type(A).__name__}.")
    rows, cols = size2(A)
    long_dim = rows if isinstance(compressor.cardinality, Left) else cols
    return _RECIPE[type(compressor)](compressor, long_dim, seed, device)


def update_compressor_(S, *args) -> None:
    """update_compressor!(S), (S, A), (S, A, b), (S, x, A, b): fresh draws in place."""
    if not isinstance(S, CompressorRecipe):
        raise ArgumentError(f"No method `update_compressor` exists for compressor recipe of type {type(S).__name__}.")
    from . import sampling as _smp
    if isinstance(S, _smp.SamplingRecipe):
        return _smp.update_sampling_(S, args)
    ctx = L.Context.get(S._ctx.device)
    L.check(L.lib().rla_sketch_update(ctx.handle, S.handle), ctx.handle)
    S._cache = None
    S._refresh_info()


# ----------------------------------------------------------------------------------
# mul! / *
# ----------------------------------------------------------------------------------
def _sketch_mul(C, S: CompressorRecipe, A, side: int, trans_s: int, alpha: float, beta: float) -> None:
    orient = "col" if side == L.RLA_SIDE_LEFT else "row"
    Aop = Operand(A, orient)
    Cop = Operand(C, orient, writable=True)
    if Aop.dtype != S._dtype or Cop.dtype != S._dtype:
        raise ArgumentError("The compressor, A and C must share one element type (Float32 or Float64).")
    ctx = L.Context.get(S._ctx.device)
    st = L.lib().rla_sketch_mul(ctx.handle, S.handle, side, trans_s, Cop.rows, Cop.cols, Cop.ptr, Cop.ld, Cop.trans,
                                Aop.rows, Aop.cols, Aop.ptr, Aop.ld, Aop.trans, float(alpha), float(beta))
    L.check(st, ctx.handle)
    Cop.finish()


def _is_sparse(x) -> bool:
    """A torch sparse-CSR tensor or a scipy.sparse matrix."""
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.layout == torch.sparse_csr
    except ImportError:
        pass
    return hasattr(x, "tocsr") and hasattr(x, "nnz")


def _sketch_mul_sparse(C, S: CompressorRecipe, A, alpha: float, beta: float) -> None:
    """mul!(C, S, transpose(B), alpha, beta) (sparse_sign.jl:364-442, count_sketch.jl:215-262).

    A sparse m x n matrix given by rows -- a torch sparse-CSR tensor or a scipy.sparse
    matrix -- is Julia's transpose(B) of the n x m SparseMatrixCSC B: the same three arrays.
    Host operands are copied to the device."""
    import torch
    if S.info.kind not in (L.RLA_SPARSE_SIGN, L.RLA_COUNT_SKETCH) or not isinstance(S.cardinality, Left):
        raise ArgumentError(f"No method `mul!` defined for ({type(C).__name__}, {type(S).__name__}, "
                            f"{type(A).__name__}, {type(alpha).__name__}, {type(beta).__name__}).")
    dev = torch.device("cuda", S._ctx.device)
    tdt = torch.float32 if S._dtype == 0 else torch.float64
    if isinstance(A, torch.Tensor):
        rows, cols = A.shape
        rowptr = A.crow_indices().to(dev, torch.int64).contiguous()
        colidx = A.col_indices().to(dev, torch.int64).contiguous()
        vals = A.values().to(dev).contiguous()
    else:
        csr = A.tocsr(copy=True)
        csr.sum_duplicates()
        rows, cols = csr.shape
        rowptr = torch.from_numpy(np.asarray(csr.indptr, np.int64)).to(dev)
        colidx = torch.from_numpy(np.asarray(csr.indices, np.int64)).to(dev)
        vals = torch.from_numpy(np.ascontiguousarray(csr.data)).to(dev)
    if vals.dtype != tdt:
        raise ArgumentError("The compressor, A and C must share one element type (Float32 or Float64).")
    Cop = Operand(C, "col", writable=True)
    if Cop.dtype != S._dtype:
        raise ArgumentError("The compressor, A and C must share one element type (Float32 or Float64).")
    if Cop.trans:
        raise ArgumentError("C must be stored column-major (a dense matrix, not a transpose).")
    ctx = L.Context.get(S._ctx.device)
    st = L.lib().rla_sketch_mul_sparse_t(ctx.handle, S.handle, Cop.rows, Cop.cols, Cop.ptr, Cop.ld, rows, cols,
                                         int(vals.numel()), rowptr.data_ptr(), colidx.data_ptr(), vals.data_ptr(),
                                         float(alpha), float(beta))
    L.check(st, ctx.handle)
    Cop.finish()


def mul_(C, X, Y, alpha: float = 1.0, beta: float = 0.0):
    """mul!(C, S, A, alpha, beta) / mul!(C, A, S, alpha, beta) and the adjoint forms;
    also dispatches to the approximator methods."""
    from . import approximators as _ap
    if _is_sparse(Y) and isinstance(X, CompressorRecipe):
        return _sketch_mul_sparse(C, X, Y, alpha, beta)
    if _is_sparse(X) or _is_sparse(Y):
        raise ArgumentError(f"No method `mul!` defined for ({type(C).__name__}, {type(X).__name__}, "
                            f"{type(Y).__name__}, {type(alpha).__name__}, {type(beta).__name__}).")
    if isinstance(X, CompressorRecipe):
        return _sketch_mul(C, X, Y, L.RLA_SIDE_LEFT, 0, alpha, beta)
    if isinstance(X, CompressorAdjoint):
        return _sketch_mul(C, X.parent, Y, L.RLA_SIDE_LEFT, 1, alpha, beta)
    if isinstance(Y, CompressorRecipe):
        return _sketch_mul(C, Y, X, L.RLA_SIDE_RIGHT, 0, alpha, beta)
    if isinstance(Y, CompressorAdjoint):
        return _sketch_mul(C, Y.parent, X, L.RLA_SIDE_RIGHT, 1, alpha, beta)
    if _ap.is_approximator_operand(X) or _ap.is_approximator_operand(Y):
        return _ap.mul_(C, X, Y, alpha, beta)
    raise ArgumentError(f"No method `mul!` defined for ({type(C).__name__}, {type(X).__name__}, "
                        f"{type(Y).__name__}, {type(alpha).__name__}, {type(beta).__name__}).")


def _times(X, Y):
    """Binary operators (src/Compressors.jl:416-449)."""
    if isinstance(X, (CompressorRecipe, CompressorAdjoint)):
        s_rows = size(X, 1)
        a_cols = size2(Y)[1]
        C = zeros_like_layout(Y, (s_rows,) if a_cols == 1 else (s_rows, a_cols))
        mul_(C, X, Y)
        return C
    s_cols = size(Y, 2)
    a_rows = size2(X)[0] if X.ndim == 2 else 1
    C = zeros_like_layout(X, (s_cols,) if (a_rows == 1 and X.ndim == 1) else (a_rows, s_cols))
    mul_(C, X, Y)
    return C
