"""CPU oracle for the RandLinearAlgebra.jl sketch / RandSVD path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` -- always as the checker or
as the timed CPU restatement of the reference, never as part of the B200 product path.

The reference (RandLinearAlgebra.jl v0.2.4) is pure Julia and Julia is not available on
these machines, so this module restates it:

* the element-wise loops (``fwht!``, the SRHT/FJLT block loops, the SparseArrays CSC
  kernels the sparse compressors call) are restated in C in ``rla_oracle.c`` and
  wrapped here with ctypes;
* the dense pieces (Gaussian apply, power iterations, RandSVD) are restated with numpy,
  whose ``qr``/``svd`` call the same LAPACK drivers (geqrf+orgqr, gesdd) that Julia's
  ``qr!``/``svd`` reach, so Householder sign conventions match.

Recipes are plain dataclasses whose fields carry the reference's recipe fields
(``op``, ``signs``, ``scale``, ``padding`` size ...) with 0-based indices.  They are
filled either from numpy draws (CPU-only tests) or from the draws the B200 library
produced (parity tests), which is how the reference's own tests load draws into
recipes (e.g. test/Compressors/sparse_sign.jl:104,396).

Parity pinning: tests/test_oracle_pins.py checks every routine against the reference
test formulas (explicit Sylvester Hadamard products, dense re-materialised operators)
and the fixtures in tests/golden/.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch."""


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    lib = ctypes.CDLL(_LIB_PATH)
    i64, dbl, vp = ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    for s in ("f", "d"):
        getattr(lib, f"orc_fwht_signed_{s}").argtypes = [vp, i64, i64, vp, i64, dbl]
        getattr(lib, f"orc_fwht_{s}").argtypes = [vp, i64, i64, dbl]
        getattr(lib, f"orc_csc_mul_{s}").argtypes = [vp, i64, i64, i64, i64, vp, vp, vp, vp, i64, i64, i64, dbl, dbl]
        getattr(lib, f"orc_csc_adj_mul_{s}").argtypes = [vp, i64, i64, i64, i64, vp, vp, vp, vp, i64, i64, i64, dbl, dbl]
        getattr(lib, f"orc_dense_mul_csc_{s}").argtypes = [vp, i64, i64, vp, i64, i64, i64, i64, i64, vp, vp, vp, dbl, dbl]
        getattr(lib, f"orc_dense_mul_csc_adj_{s}").argtypes = [vp, i64, i64, vp, i64, i64, i64, i64, i64, vp, vp, vp, dbl, dbl]
        for nm in ("srht_left_SA", "srht_left_AS", "srht_right_AS", "srht_right_SA"):
            getattr(lib, f"orc_{nm}_{s}").argtypes = [vp, i64, i64, vp, i64, i64, i64, i64, i64, i64, vp, vp, dbl, i64, dbl, dbl]
        for nm in ("fjlt_left_SA", "fjlt_left_AS", "fjlt_right_AS", "fjlt_right_SA"):
            getattr(lib, f"orc_{nm}_{s}").argtypes = [vp, i64, i64, vp, i64, i64, i64, i64, i64, i64, vp, vp, vp, vp, dbl, i64, dbl, dbl]
    _lib = lib
    return lib


def _sfx(x: np.ndarray) -> str:
    if x.dtype == np.float32:
        return "f"
    if x.dtype == np.float64:
        return "d"
    raise TypeError(f"oracle supports float32/float64, got {x.dtype}")


def _view(x: np.ndarray):
    """(pointer, row stride, col stride) in elements for a 1-D or 2-D numpy view."""
    es = x.itemsize
    if x.ndim == 1:
        return x.ctypes.data, x.strides[0] // es, 0
    return x.ctypes.data, x.strides[0] // es, x.strides[1] // es


def _as2d(x: np.ndarray) -> np.ndarray:
    return x.reshape(-1, 1) if x.ndim == 1 else x


def _ptr(a: np.ndarray):
    return a.ctypes.data


# ----------------------------------------------------------------------------------
# fwht!  (src/Compressors/helpers/fwht.jl:21-118)
# ----------------------------------------------------------------------------------
def fwht_(x: np.ndarray, signs: Optional[np.ndarray] = None, scaling: float = 1.0) -> None:
    """In-place natural-order Walsh-Hadamard transform of a strided 1-D view."""
    lib = _load()
    p, inc, _ = _view(x)
    if signs is None:
        rc = getattr(lib, f"orc_fwht_{_sfx(x)}")(p, x.shape[0], inc, float(scaling))
    else:
        sg = np.ascontiguousarray(signs, dtype=np.uint8)
        rc = getattr(lib, f"orc_fwht_signed_{_sfx(x)}")(p, x.shape[0], inc, _ptr(sg), sg.shape[0], float(scaling))
    if rc == 1:
        if signs is not None and len(signs) != x.shape[0]:
            raise DimensionMismatch("Vector `x` and vector `signs` must be same length.")
        raise DimensionMismatch("Size of vector must be power of 2.")


def hadamard(n: int) -> np.ndarray:
    """Natural-order (Sylvester) Hadamard matrix, the matrix the reference tests take
    from Hadamard.jl's ``hadamard(n)`` (test/Compressors/helpers/fwht.jl:38)."""
    H = np.ones((1, 1))
    while H.shape[0] < n:
        H = np.block([[H, H], [H, -H]])
    return H


def padded_size(n: int) -> int:
    """Smallest power of two >= n (srht.jl:147, fjlt.jl:174).  The reference computes
    ``Int64(2^(ceil(log(2, n))))`` in floating point, which overshoots for n = 2^29,
    2^31, 2^39 (glibc log); the exact value is used here and in the library."""
    return 1 << max(0, (int(n) - 1).bit_length())


# ----------------------------------------------------------------------------------
# Recipes (field layout of the reference's *Recipe structs, 0-based indices)
# ----------------------------------------------------------------------------------
@dataclass
class CSC:
    """SparseMatrixCSC{T,Int64} with 0-based colptr/rowval."""
    n_rows: int
    n_cols: int
    colptr: np.ndarray
    rowval: np.ndarray
    nzval: np.ndarray

    def dense(self) -> np.ndarray:
        D = np.zeros((self.n_rows, self.n_cols), dtype=np.float64)
        for j in range(self.n_cols):
            for k in range(self.colptr[j], self.colptr[j + 1]):
                D[self.rowval[k], j] += self.nzval[k]
        return D


@dataclass
class Recipe:
    """A completed compressor.  ``kind`` in {sparse_sign, count_sketch, srht, fjlt,
    gaussian}; ``card`` in {left, right}.  n_rows/n_cols follow the reference."""
    kind: str
    card: str
    n_rows: int
    n_cols: int
    dtype: type = np.float64
    nnz: int = 0
    csc: Optional[CSC] = None          # SparseSign op (parent of the adjoint for Right), CountSketch mat, FJLT op
    op: Optional[np.ndarray] = None    # SRHT sampled rows (0-based)
    signs: Optional[np.ndarray] = None  # SRHT/FJLT sign bits (1 = +1)
    scale: float = 1.0
    padded: int = 0
    block_size: int = 10
    dense_op: Optional[np.ndarray] = None  # Gaussian op
    idx: Optional[np.ndarray] = None       # Sampling: selected indices (0-based)

    @property
    def shape(self):
        return (self.n_rows, self.n_cols)

    def dense(self) -> np.ndarray:
        """Dense float64 re-materialisation of S, the way the reference tests compare."""
        if self.kind == "sampling":
            s = len(self.idx)
            L = self.n_cols if self.card == "left" else self.n_rows
            P = np.zeros((s, L))
            P[np.arange(s), self.idx] = 1.0
            return P if self.card == "left" else P.T
        if self.kind in ("sparse_sign",):
            D = self.csc.dense()
            return D if self.card == "left" else D.T
        if self.kind == "count_sketch":
            D = self.csc.dense()
            return D if self.card == "left" else D.T
        if self.kind == "gaussian":
            return self.dense_op.astype(np.float64)
        H = hadamard(self.padded)
        d = np.where(self.signs.astype(bool), 1.0, -1.0)
        if self.kind == "srht":
            K = np.zeros((len(self.op), self.padded))
            K[np.arange(len(self.op)), self.op] = 1.0
            full = self.scale * (K @ H @ np.diag(d))  # s x N
        else:
            Kd = self.csc.dense()  # Left: s x N ; Right: N x s
            full = self.scale * ((Kd if self.card == "left" else Kd.T) @ H @ np.diag(d))
        if self.card == "left":
            return full[:, : self.n_cols]
        return full[:, : self.n_rows].T


# ----------------------------------------------------------------------------------
# Draws for CPU-only tests (numpy).  Parity tests load the library's own draws instead.
# ----------------------------------------------------------------------------------
def draw_sampling(rng: np.random.Generator, card: str, s: int, long_dim: int, replace: bool = False,
                  weights: Optional[np.ndarray] = None, dtype=np.float64) -> Recipe:
    """SamplingRecipe (src/Compressors/sampling.jl:98-121) with wsample!(..., ordered = true)
    (Distributions/uniform.jl, strohmer_vershynin.jl): sorted 0-based indices."""
    p = None if weights is None else np.asarray(weights, np.float64) / np.sum(weights)
    idx = np.sort(rng.choice(long_dim, size=s, replace=replace, p=p))
    n_rows, n_cols = (s, long_dim) if card == "left" else (long_dim, s)
    return Recipe("sampling", card, n_rows, n_cols, dtype, idx=idx.astype(np.int64))


def l2norm_weights(A: np.ndarray, card: str) -> np.ndarray:
    """strohmer_vershynin.jl: squared row norms (Left) / column norms (Right)."""
    A = A.astype(np.float64)
    return np.sum(A * A, axis=1 if card == "left" else 0)


def agmon_select(A: np.ndarray, x: np.ndarray, b: np.ndarray, card: str, candidates: np.ndarray, k: int,
                 r: Optional[np.ndarray] = None) -> np.ndarray:
    """sample_distribution!(indices, ::AgmonRecipe) after the candidate draw (agmon.jl): the k
    candidates with the largest residual, ordered by (-residual, candidate)."""
    A = A.astype(np.float64)
    if card == "left":
        res = np.abs(r[candidates]) if r is not None else np.abs(A[candidates, :] @ x - b[candidates])
    else:
        rv = r if r is not None else A @ x - b
        res = np.abs(A[:, candidates].T @ rv)
    order = sorted(range(len(candidates)), key=lambda i: (-res[i], candidates[i]))
    return np.asarray([candidates[i] for i in order[:k]], np.int64)


def draw_sparse_sign(rng: np.random.Generator, card: str, s: int, long_dim: int, nnz: int, dtype=np.float64) -> Recipe:
    """SparseSignRecipe (src/Compressors/sparse_sign.jl:229-295): per long index, nnz
    distinct sorted rows of 0:s-1, values +-1/sqrt(nnz) (rounded to T)."""
    rows = np.stack([np.sort(rng.choice(s, size=nnz, replace=False)) for _ in range(long_dim)]).reshape(-1)
    sc = dtype(1.0 / math.sqrt(nnz))
    vals = np.where(rng.integers(0, 2, size=long_dim * nnz) == 1, sc, -sc).astype(dtype)
    colptr = np.arange(0, long_dim * nnz + 1, nnz, dtype=np.int64)
    csc = CSC(s, long_dim, colptr, rows.astype(np.int64), vals)
    if card == "left":
        return Recipe("sparse_sign", "left", s, long_dim, dtype, nnz=nnz, csc=csc)
    return Recipe("sparse_sign", "right", long_dim, s, dtype, nnz=nnz, csc=csc)


def draw_count_sketch(rng: np.random.Generator, card: str, s: int, long_dim: int, dtype=np.float64) -> Recipe:
    """CountSketchRecipe (src/Compressors/count_sketch.jl:113-147): one bucket in 0:s-1
    and one sign per long index; mat = sparse(groups, 1:L, signs, s, L)."""
    groups = rng.integers(0, s, size=long_dim).astype(np.int64)
    signs = np.where(rng.integers(0, 2, size=long_dim) == 1, 1.0, -1.0).astype(dtype)
    csc = CSC(s, long_dim, np.arange(long_dim + 1, dtype=np.int64), groups, signs)
    if card == "left":
        return Recipe("count_sketch", "left", s, long_dim, dtype, nnz=1, csc=csc)
    return Recipe("count_sketch", "right", long_dim, s, dtype, nnz=1, csc=csc)


def srht_scale(s: int, N: int, dtype) -> float:
    """scale = T(sqrt(s)/sqrt(N)) stored as Float64 (srht.jl:152,181)."""
    return float(dtype(math.sqrt(s) / math.sqrt(N)))


def draw_srht(rng: np.random.Generator, card: str, s: int, long_dim: int, block_size: int = 10, dtype=np.float64) -> Recipe:
    """SRHTRecipe (src/Compressors/srht.jl:135-191): N = next pow2, sign bits,
    s rows sampled without replacement (unordered)."""
    N = padded_size(long_dim)
    signs = rng.integers(0, 2, size=N).astype(np.uint8)
    op = rng.choice(N, size=s, replace=False).astype(np.int64)
    r = Recipe("srht", card, s if card == "left" else long_dim, long_dim if card == "left" else s, dtype,
               op=op, signs=signs, scale=srht_scale(s, N, dtype), padded=N, block_size=block_size)
    return r


def fjlt_default_sparsity(long_dim: int) -> float:
    """fjlt.jl:181 / :215: 0.25*log(L)^2/L (natural log) when sparsity == 0."""
    return 0.25 * math.log(long_dim) ** 2 / long_dim


def fjlt_scale(s: int, N: int, q: float, dtype) -> float:
    """scale = T(1/(sqrt(N)*sqrt(q)*sqrt(s))) (fjlt.jl:184,218)."""
    return float(dtype(1.0 / (math.sqrt(N) * math.sqrt(q) * math.sqrt(s))))


def draw_fjlt(rng: np.random.Generator, card: str, s: int, long_dim: int, sparsity: float = 0.0, block_size: int = 10, dtype=np.float64) -> Recipe:
    """FJLTRecipe (src/Compressors/fjlt.jl:162-225): K = sprandn(s, N, q) (Left) or
    sprandn(N, s, q) (Right), sign bits, scale 1/(sqrt(N q s))."""
    N = padded_size(long_dim)
    q = fjlt_default_sparsity(long_dim) if sparsity == 0.0 else sparsity
    kr, kc = (s, N) if card == "left" else (N, s)
    mask = rng.random((kr, kc)) < q
    vals = rng.standard_normal((kr, kc))
    colptr = np.zeros(kc + 1, dtype=np.int64)
    rows, nz = [], []
    for j in range(kc):
        idx = np.nonzero(mask[:, j])[0]
        rows.append(idx)
        nz.append(vals[idx, j])
        colptr[j + 1] = colptr[j] + len(idx)
    csc = CSC(kr, kc, colptr, np.concatenate(rows).astype(np.int64) if rows else np.zeros(0, np.int64),
              np.concatenate(nz).astype(dtype) if nz else np.zeros(0, dtype))
    signs = rng.integers(0, 2, size=N).astype(np.uint8)
    return Recipe("fjlt", card, s if card == "left" else long_dim, long_dim if card == "left" else s, dtype,
                  csc=csc, signs=signs, scale=fjlt_scale(s, N, q, dtype), padded=N, block_size=block_size)


def draw_gaussian(rng: np.random.Generator, card: str, s: int, long_dim: int, dtype=np.float64) -> Recipe:
    """GaussianRecipe (src/Compressors/gaussian.jl:96-124): op = T(1/sqrt(s)) * randn."""
    scale = dtype(1.0 / math.sqrt(s))
    shape = (s, long_dim) if card == "left" else (long_dim, s)
    op = (scale * rng.standard_normal(shape).astype(dtype)).astype(dtype)
    return Recipe("gaussian", card, shape[0], shape[1], dtype, dense_op=op, scale=float(scale))


# ----------------------------------------------------------------------------------
# mul!  (src/Compressors.jl:331-410 and the per-compressor methods)
# ----------------------------------------------------------------------------------
def left_mul_dimcheck(C, S, A):
    """src/helpers/mul_dim_checks.jl:41-64."""
    s_rows, s_cols = S.shape
    a_rows, a_cols = _as2d(A).shape
    c_rows, c_cols = _as2d(C).shape
    if a_rows != s_cols:
        raise DimensionMismatch(f"Matrix A has {a_rows} rows while S has {s_cols} columns.")
    if a_cols != c_cols:
        raise DimensionMismatch(f"Matrix A has {a_cols} columns while C has {c_cols} columns.")
    if c_rows != s_rows:
        raise DimensionMismatch(f"Matrix C has {c_rows} rows while S has {s_rows} rows.")


def right_mul_dimcheck(C, A, S):
    """src/helpers/mul_dim_checks.jl:110-133."""
    s_rows, s_cols = S.shape
    a_rows, a_cols = _as2d(A).shape
    c_rows, c_cols = _as2d(C).shape
    if a_cols != s_rows:
        raise DimensionMismatch(f"Matrix A has {a_cols} columns while S has {s_rows} rows.")
    if c_cols != s_cols:
        raise DimensionMismatch(f"Matrix C has {c_cols} columns while S has {s_cols} columns.")
    if c_rows != a_rows:
        raise DimensionMismatch(f"Matrix C has {c_rows} rows while A has {a_rows} rows.")


def _csc_args(csc: CSC, dtype):
    cp = np.ascontiguousarray(csc.colptr, dtype=np.int64)
    rv = np.ascontiguousarray(csc.rowval, dtype=np.int64)
    nz = np.ascontiguousarray(csc.nzval, dtype=dtype)
    return cp, rv, nz


def mul_SA(C: np.ndarray, S: Recipe, A: np.ndarray, alpha: float = 1.0, beta: float = 0.0) -> None:
    """mul!(C, S, A, alpha, beta): C = alpha*S*A + beta*C, C and A strided numpy views."""
    C2, A2 = _as2d(C), _as2d(A)
    left_mul_dimcheck(C2, S, A2)
    lib = _load()
    sfx = _sfx(C2)
    cp_, crs, ccs = _view(C2)
    ap_, ars, acs = _view(A2)
    if C2.ndim == 2 and C.ndim == 1:
        ccs = 0
    n = A2.shape[1]
    if S.kind == "sampling":
        A64 = A2.astype(np.float64)
        if S.card == "left":   # sampling.jl:145-157: C = alpha*A[idx, :] + beta*C
            C2[...] = (alpha * A64[S.idx, :] + (beta * C2.astype(np.float64) if beta != 0 else 0)).astype(C2.dtype)
        else:                  # sampling.jl:160-176: C .*= beta; C[idx, :] += alpha*A, in order
            acc = beta * C2.astype(np.float64) if beta != 0 else np.zeros(C2.shape)
            for i, t in enumerate(S.idx):
                acc[t, :] += alpha * A64[i, :]
            C2[...] = acc.astype(C2.dtype)
        return
    if S.kind == "gaussian":
        # gaussian.jl:145-156 -- BLAS gemm
        res = alpha * (S.dense_op.astype(np.float64) @ A2.astype(np.float64))
        C2[...] = (res + (beta * C2.astype(np.float64) if beta != 0 else 0)).astype(C2.dtype)
        return
    if S.kind in ("sparse_sign", "count_sketch"):
        cp, rv, nz = _csc_args(S.csc, C2.dtype)
        if S.card == "left":   # sparse_sign.jl:339-348 / count_sketch.jl:166-175
            getattr(lib, f"orc_csc_mul_{sfx}")(cp_, crs, ccs, S.csc.n_rows, S.csc.n_cols, _ptr(cp), _ptr(rv), _ptr(nz),
                                               ap_, ars, acs, n, float(alpha), float(beta))
        else:                  # op = adjoint(CSC) (sparse_sign.jl:290) / S.mat' (count_sketch.jl:191-200)
            getattr(lib, f"orc_csc_adj_mul_{sfx}")(cp_, crs, ccs, S.csc.n_rows, S.csc.n_cols, _ptr(cp), _ptr(rv), _ptr(nz),
                                                   ap_, ars, acs, n, float(alpha), float(beta))
        return
    op = np.ascontiguousarray(S.op if S.op is not None else np.zeros(0), dtype=np.int64)
    sg = np.ascontiguousarray(S.signs, dtype=np.uint8)
    if S.kind == "srht":
        if S.card == "left":   # srht.jl:220-286
            rc = getattr(lib, f"orc_srht_left_SA_{sfx}")(cp_, crs, ccs, ap_, ars, acs, S.n_cols, n, S.n_rows, S.padded,
                                                         _ptr(op), _ptr(sg), S.scale, S.block_size, float(alpha), float(beta))
        else:                  # srht.jl:432-504
            rc = getattr(lib, f"orc_srht_right_SA_{sfx}")(cp_, crs, ccs, ap_, ars, acs, S.n_rows, n, S.n_cols, S.padded,
                                                          _ptr(op), _ptr(sg), S.scale, S.block_size, float(alpha), float(beta))
    elif S.kind == "fjlt":
        cp, rv, nz = _csc_args(S.csc, C2.dtype)
        if S.card == "left":   # fjlt.jl:257-323
            rc = getattr(lib, f"orc_fjlt_left_SA_{sfx}")(cp_, crs, ccs, ap_, ars, acs, S.n_cols, n, S.n_rows, S.padded,
                                                         _ptr(cp), _ptr(rv), _ptr(nz), _ptr(sg), S.scale, S.block_size,
                                                         float(alpha), float(beta))
        else:                  # fjlt.jl:465-535
            rc = getattr(lib, f"orc_fjlt_right_SA_{sfx}")(cp_, crs, ccs, ap_, ars, acs, S.n_rows, n, S.n_cols, S.padded,
                                                          _ptr(cp), _ptr(rv), _ptr(nz), _ptr(sg), S.scale, S.block_size,
                                                          float(alpha), float(beta))
    else:
        raise ValueError(S.kind)
    if rc != 0:
        raise MemoryError("oracle allocation failed")


def mul_AS(C: np.ndarray, A: np.ndarray, S: Recipe, alpha: float = 1.0, beta: float = 0.0) -> None:
    """mul!(C, A, S, alpha, beta): C = alpha*A*S + beta*C."""
    C2 = C.reshape(1, -1) if C.ndim == 1 else C
    A2 = A.reshape(1, -1) if A.ndim == 1 else A
    right_mul_dimcheck(C2, A2, S)
    lib = _load()
    sfx = _sfx(C2)
    cp_, crs, ccs = _view(C2)
    ap_, ars, acs = _view(A2)
    ar = A2.shape[0]
    if S.kind == "sampling":
        A64 = A2.astype(np.float64)
        if S.card == "right":  # sampling.jl:178-188: C = alpha*A[:, idx] + beta*C
            C2[...] = (alpha * A64[:, S.idx] + (beta * C2.astype(np.float64) if beta != 0 else 0)).astype(C2.dtype)
        else:                  # sampling.jl:190-200: C .*= beta; C[:, idx] += alpha*A, in order
            acc = beta * C2.astype(np.float64) if beta != 0 else np.zeros(C2.shape)
            for i, t in enumerate(S.idx):
                acc[:, t] += alpha * A64[:, i]
            C2[...] = acc.astype(C2.dtype)
        return
    if S.kind == "gaussian":
        # gaussian.jl:159-170
        res = alpha * (A2.astype(np.float64) @ S.dense_op.astype(np.float64))
        C2[...] = (res + (beta * C2.astype(np.float64) if beta != 0 else 0)).astype(C2.dtype)
        return
    if S.kind in ("sparse_sign", "count_sketch"):
        cp, rv, nz = _csc_args(S.csc, C2.dtype)
        if S.card == "left":   # sparse_sign.jl:351-361 / count_sketch.jl:178-188
            getattr(lib, f"orc_dense_mul_csc_{sfx}")(cp_, crs, ccs, ap_, ars, acs, ar, S.csc.n_rows, S.csc.n_cols,
                                                     _ptr(cp), _ptr(rv), _ptr(nz), float(alpha), float(beta))
        else:                  # adjoint op (sparse_sign.jl:359, count_sketch.jl:203-213)
            getattr(lib, f"orc_dense_mul_csc_adj_{sfx}")(cp_, crs, ccs, ap_, ars, acs, ar, S.csc.n_rows, S.csc.n_cols,
                                                         _ptr(cp), _ptr(rv), _ptr(nz), float(alpha), float(beta))
        return
    op = np.ascontiguousarray(S.op if S.op is not None else np.zeros(0), dtype=np.int64)
    sg = np.ascontiguousarray(S.signs, dtype=np.uint8)
    if S.kind == "srht":
        if S.card == "left":   # srht.jl:289-363
            rc = getattr(lib, f"orc_srht_left_AS_{sfx}")(cp_, crs, ccs, ap_, ars, acs, ar, S.n_cols, S.n_rows, S.padded,
                                                         _ptr(op), _ptr(sg), S.scale, S.block_size, float(alpha), float(beta))
        else:                  # srht.jl:366-429
            rc = getattr(lib, f"orc_srht_right_AS_{sfx}")(cp_, crs, ccs, ap_, ars, acs, ar, S.n_rows, S.n_cols, S.padded,
                                                          _ptr(op), _ptr(sg), S.scale, S.block_size, float(alpha), float(beta))
    elif S.kind == "fjlt":
        cp, rv, nz = _csc_args(S.csc, C2.dtype)
        if S.card == "left":   # fjlt.jl:326-397
            rc = getattr(lib, f"orc_fjlt_left_AS_{sfx}")(cp_, crs, ccs, ap_, ars, acs, ar, S.n_cols, S.n_rows, S.padded,
                                                         _ptr(cp), _ptr(rv), _ptr(nz), _ptr(sg), S.scale, S.block_size,
                                                         float(alpha), float(beta))
        else:                  # fjlt.jl:400-463
            rc = getattr(lib, f"orc_fjlt_right_AS_{sfx}")(cp_, crs, ccs, ap_, ars, acs, ar, S.n_rows, S.n_cols, S.padded,
                                                          _ptr(cp), _ptr(rv), _ptr(nz), _ptr(sg), S.scale, S.block_size,
                                                          float(alpha), float(beta))
    else:
        raise ValueError(S.kind)
    if rc != 0:
        raise MemoryError("oracle allocation failed")


def mul_StA(C, S: Recipe, A, alpha=1.0, beta=0.0):
    """mul!(C, S', A, alpha, beta) -> mul!(transpose(C), transpose(A), S) (src/Compressors.jl:363-372)."""
    Ct = C.reshape(1, -1) if C.ndim == 1 else C.T
    At = A.reshape(1, -1) if A.ndim == 1 else A.T
    mul_AS(Ct, At, S, alpha, beta)


def mul_ASt(C, A, S: Recipe, alpha=1.0, beta=0.0):
    """mul!(C, A, S', alpha, beta) -> mul!(transpose(C), S, transpose(A)) (src/Compressors.jl:375-384)."""
    Ct = C.reshape(-1) if C.ndim == 1 else C.T
    At = A.reshape(-1) if A.ndim == 1 else A.T
    mul_SA(Ct, S, At, alpha, beta)


# ----------------------------------------------------------------------------------
# Range approximators (src/Approximators/RangeApproximators/*)
# ----------------------------------------------------------------------------------
def _qr_Q(Y: np.ndarray) -> np.ndarray:
    """Array(qr!(Y).Q): economy Householder Q (LAPACK geqrf/orgqr)."""
    return np.linalg.qr(Y, mode="reduced")[0]


def rand_power_it(A: np.ndarray, S: Recipe, q: int) -> np.ndarray:
    """helpers/power_its.jl:15-36 (Halko et al. Alg. 4.3), computed in float64."""
    A = A.astype(np.float64)
    Y = np.zeros((A.shape[0], S.n_cols))
    mul_AS(Y, A, _as_f64(S))
    for _ in range(q):
        Z = A.T @ Y
        Y = A @ Z
    return _qr_Q(Y)


def rand_ortho_it(A: np.ndarray, S: Recipe, q: int) -> np.ndarray:
    """helpers/power_its.jl:53-80 (Halko et al. Alg. 4.4), computed in float64."""
    A = A.astype(np.float64)
    Y = np.zeros((A.shape[0], S.n_cols))
    mul_AS(Y, A, _as_f64(S))
    Q = _qr_Q(Y)
    for _ in range(q):
        Q = _qr_Q(A.T @ Q)
        Q = _qr_Q(A @ Q)
    return Q


def _as_f64(S: Recipe) -> Recipe:
    """The same draws with float64 values, so oracle products accumulate in float64."""
    import copy
    R = copy.copy(S)
    R.dtype = np.float64
    if S.csc is not None:
        R.csc = CSC(S.csc.n_rows, S.csc.n_cols, S.csc.colptr, S.csc.rowval, S.csc.nzval.astype(np.float64))
    if S.dense_op is not None:
        R.dense_op = S.dense_op.astype(np.float64)
    return R


@dataclass
class RandSVDResult:
    U: np.ndarray
    S: np.ndarray
    V: np.ndarray


def rangefinder(A: np.ndarray, S: Recipe, q: int = 0, orthogonalize: bool = False) -> np.ndarray:
    """rapproximate!(::RangeFinderRecipe, A) (rangefinder.jl:134-143)."""
    return rand_ortho_it(A, S, q) if orthogonalize else rand_power_it(A, S, q)


def randsvd(A: np.ndarray, S: Recipe, q: int = 0, orthogonalize: bool = False) -> RandSVDResult:
    """rapproximate!(::RandSVDRecipe, A) (randsvd.jl:174-189): Q from the power
    iterations, QA = Q'A in Float64, svd(QA), U = Q*W."""
    Q = rangefinder(A, S, q, orthogonalize)
    QA = Q.T @ A.astype(np.float64)
    W, sig, Vt = np.linalg.svd(QA, full_matrices=False)
    return RandSVDResult(Q @ W, sig, Vt.T)


def randsvd_mul_left(C, R: RandSVDResult, A, alpha, beta, bs):
    """mul!(C, R::RandSVDRecipe, A, alpha, beta) blocked (randsvd.jl:198-243).  ``bs`` is
    size(R.buffer, 2): the recipe's block_size, or n_cols of the approximated A when 0
    (randsvd.jl:160)."""
    a_cols = A.shape[1]
    for c0 in range(0, a_cols, bs):
        c1 = min(a_cols, c0 + bs)
        buf = alpha * (R.V.T @ A[:, c0:c1])
        buf *= R.S[:, None]
        C[:, c0:c1] = R.U @ buf + beta * C[:, c0:c1]


def randsvd_mul_right(C, A, R: RandSVDResult, alpha, beta, bs):
    """mul!(C, A, R::RandSVDRecipe, alpha, beta) blocked (randsvd.jl:246-293)."""
    a_rows = A.shape[0]
    for r0 in range(0, a_rows, bs):
        r1 = min(a_rows, r0 + bs)
        buf = alpha * (A[r0:r1, :] @ R.U)
        buf *= R.S[None, :]
        C[r0:r1, :] = buf @ R.V.T + beta * C[r0:r1, :]


# ----------------------------------------------------------------------------------
# Solvers: IHS (src/Solvers/ihs.jl), BasicLogger (src/Solvers/Loggers/basic_logger.jl),
# FullResidual / LSGradient (src/Solvers/ErrorMethods/*.jl)
# ----------------------------------------------------------------------------------
@dataclass
class IHSResult:
    x: np.ndarray
    residual_vec: np.ndarray
    gradient_vec: np.ndarray
    hist: np.ndarray
    iteration: int
    converged: bool
    errors: list


def ihs_rsolve(A: np.ndarray, b: np.ndarray, x0: np.ndarray, sketches, alpha: float = 1.0, max_it: int = 0,
               threshold: float = 0.0, collection_rate: int = 1, error: str = "full") -> IHSResult:
    """rsolve!(::IHSRecipe, x, A, b) (ihs.jl:214-254) with a BasicLogger (threshold_stop,
    basic_logger.jl:84-130) in float64.  ``sketches(i)`` returns the Left compressor recipe
    drawn by update_compressor! in iteration i (1-based).  R comes from Householder QR of
    the sketched matrix (LAPACK geqrf, as qr!), the two solves are triangular solves.
    ``error``: "full" = FullResidual (||b - Ax||), "gradient" = ||A'r|| of the maintained
    residual (LSGradient)."""
    A = A.astype(np.float64)
    b = b.astype(np.float64)
    x = x0.astype(np.float64).copy()
    m, n = A.shape
    hist = np.zeros(int(math.ceil(max_it / collection_rate)) + 1 if max_it > 0 else 1)
    rec, it, conv = 0, 0, False
    errs = []
    r = b - A @ x                                   # :219-220
    g = np.zeros(n)
    for i in range(1, max_it + 1):
        g = A.T @ r                                 # :223
        err = float(np.linalg.norm(b - A @ x)) if error == "full" else float(np.linalg.norm(A.T @ r))
        errs.append(err)
        it = i                                      # update_logger! (basic_logger.jl:84-101)
        conv = (err < threshold) if i < max_it else True
        if conv:
            hist[rec] = err
        elif i % collection_rate == 0:
            hist[rec] = err
            rec += 1
        if conv:
            break
        S = _as_f64(sketches(i))                    # :231
        SA = np.zeros((S.n_rows, n))
        mul_SA(SA, S, A)                            # :236
        R = np.linalg.qr(SA, mode="r")              # :239
        y = _solve_tri(R.T, g, lower=True)          # :241
        u = _solve_tri(R, y, lower=False)           # :243
        x += alpha * u                              # :246
        r -= A @ u                                  # :249 (by A*u, not alpha*A*u)
    return IHSResult(x, r, g, hist, it, conv, errs)


def _solve_tri(T: np.ndarray, v: np.ndarray, lower: bool) -> np.ndarray:
    """ldiv! with a triangular matrix (plain substitution, float64)."""
    n = T.shape[0]
    out = np.zeros(n)
    rng = range(n) if lower else range(n - 1, -1, -1)
    for i in rng:
        if lower:
            out[i] = (v[i] - T[i, :i] @ out[:i]) / T[i, i]
        else:
            out[i] = (v[i] - T[i, i + 1:] @ out[i + 1:]) / T[i, i]
    return out


@dataclass
class ProjResult:
    x: np.ndarray
    residual_vec: Optional[np.ndarray]
    hist: np.ndarray
    iteration: int
    converged: bool
    errors: list


def _logger_update(state, err, i, max_it, threshold, collection_rate, hist):
    """update_logger! of BasicLogger (basic_logger.jl:84-101); state = [record_location]."""
    conv = (err < threshold) if i < max_it else True
    if conv:
        hist[state[0]] = err
    elif i % collection_rate == 0:
        hist[state[0]] = err
        state[0] += 1
    return conv


def kaczmarz_rsolve(A, b, x0, sketches, alpha=1.0, max_it=0, threshold=0.0, collection_rate=1,
                    error="full") -> ProjResult:
    """rsolve!(::KaczmarzRecipe, x, A, b) (kaczmarz.jl:323-368) in float64 with the LQ
    sub-solver (lq.jl: ldiv! through qr!(A')'); ``sketches(i)`` is the Left compressor drawn
    in iteration i.  error: "full" (FullResidual) or "compressed" (CompressedResidual on the
    last sketched rows, zero before the first)."""
    A = A.astype(np.float64)
    b = b.astype(np.float64)
    x = x0.astype(np.float64).copy()
    hist = np.zeros(int(math.ceil(max_it / collection_rate)) + 1 if max_it > 0 else 1)
    state, it, conv, errs = [0], 0, False, []
    SA, Sb = None, None
    for i in range(1, max_it + 1):
        if error == "full":
            err = float(np.linalg.norm(b - A @ x))
        else:
            err = 0.0 if SA is None else float(np.linalg.norm(Sb - SA @ x))
        errs.append(err)
        it = i
        conv = _logger_update(state, err, i, max_it, threshold, collection_rate, hist)
        if conv:
            break
        S = _as_f64(sketches(i))
        SA = np.zeros((S.n_rows, A.shape[1]))
        mul_SA(SA, S, A)
        Sb = np.zeros(S.n_rows)
        mul_SA(Sb, S, b)
        if not np.any(SA):
            continue
        if SA.shape[0] == 1:  # kaczmarz_update! (kaczmarz.jl:280-290)
            a = SA[0]
            scaling = alpha * (a @ x - Sb[0]) / (a @ a)
            x -= scaling * a
        else:                 # kaczmarz_update_block! with the LQ solve (kaczmarz.jl:292-305)
            r = Sb - SA @ x
            Q, R = np.linalg.qr(SA.T)  # SA' = QR, SA = R'Q'
            u = Q @ _solve_tri(R.T, r, lower=True)
            x += alpha * u
    return ProjResult(x, None, hist, it, conv, errs)


def colproj_rsolve(A, b, x0, sketches, alpha=1.0, max_it=0, threshold=0.0, collection_rate=1) -> ProjResult:
    """rsolve!(::ColumnProjectionRecipe, x, A, b) (col_projection.jl:328-372) in float64 with
    LSGradient and the QR sub-solver (qr.jl); ``sketches(i)`` is the Right compressor drawn in
    iteration i."""
    A = A.astype(np.float64)
    b = b.astype(np.float64)
    x = x0.astype(np.float64).copy()
    r = b - A @ x
    hist = np.zeros(int(math.ceil(max_it / collection_rate)) + 1 if max_it > 0 else 1)
    state, it, conv, errs = [0], 0, False, []
    for i in range(1, max_it + 1):
        err = float(np.linalg.norm(A.T @ r))
        errs.append(err)
        it = i - 1
        conv = _logger_update(state, err, i - 1, max_it, threshold, collection_rate, hist)
        if conv:
            return ProjResult(x, r, hist, it, conv, errs)
        S = _as_f64(sketches(i))
        AS = np.zeros((A.shape[0], S.n_cols))
        mul_AS(AS, A, S)
        if AS.shape[1] == 1:  # colproj_update! (col_projection.jl:300-307)
            u = np.array([AS[:, 0] @ r / (AS[:, 0] @ AS[:, 0])])
        else:                 # colproj_update_block! with qr!(AS) \ r
            Q, R = np.linalg.qr(AS)
            u = _solve_tri(R, Q.T @ r, lower=False)
        Su = np.zeros(A.shape[1])
        mul_SA(Su, S, u)
        x += alpha * Su
        r -= alpha * (AS @ u)
    err = float(np.linalg.norm(A.T @ r))
    errs.append(err)
    conv = _logger_update(state, err, max_it, max_it, threshold, collection_rate, hist)
    return ProjResult(x, r, hist, max_it, conv, errs)
