"""Solvers: the host-side mirror of RandLinearAlgebra.jl's Solver API for the Iterative
Hessian Sketch (src/Solvers.jl, src/Solvers/ihs.jl, src/Solvers/Loggers/basic_logger.jl,
src/Solvers/ErrorMethods/*.jl).

Same names, fields, defaults, warnings and error messages as the reference; Julia's bang
functions end in ``_`` here (``rsolve!`` -> ``rsolve_``).  The iteration runs on the device
through librla_b200.so (rla_ihs_*): one fused pass over A per iteration gives the residual
update, the error and the gradient, the second pass is the compressor apply, and the
sub-problem is solved with the FP64 Cholesky factor of the sketched Gram matrix.  Loggers
and error methods stay on the host so that user-defined ones plug in as in the reference:
a logger recipe with ``update_logger_(err, iteration)`` / ``reset_logger_()`` methods and a
``converged`` field, an error recipe with ``compute_error(solver, A, b)`` and a ``residual``
field.
"""
from __future__ import annotations

import copy
import ctypes
import math
import warnings

import numpy as np

from . import _lib as L
from ._arrays import Operand, rla_dtype
from .compressors import Compressor, CompressorRecipe, Left, SparseSign, complete_compressor
from .errors import ArgumentError, DimensionMismatch, RLAError


# ----------------------------------------------------------------------------------
# Abstract types (src/Solvers.jl:1-60)
# ----------------------------------------------------------------------------------
class Solver:
    """Abstract supertype of solvers."""


class SolverRecipe:
    """Abstract supertype of completed solvers."""


class Logger:
    """Abstract supertype of loggers (src/Solvers/Loggers.jl)."""


class LoggerRecipe:
    """Abstract supertype of completed loggers."""


class SolverError:
    """Abstract supertype of solver error methods (src/Solvers/ErrorMethods.jl)."""


class SolverErrorRecipe:
    """Abstract supertype of completed error methods."""


# ----------------------------------------------------------------------------------
# BasicLogger (src/Solvers/Loggers/basic_logger.jl)
# ----------------------------------------------------------------------------------
def threshold_stop(log) -> bool:
    """basic_logger.jl:120-130: stop once the latest error is below the threshold."""
    return log.error < log.threshold_info


class BasicLogger(Logger):
    """basic_logger.jl:15-42."""

    def __init__(self, max_it: int = 0, collection_rate: int = 1, threshold=0.0, stopping_criterion=threshold_stop):
        if max_it < 0:
            raise ArgumentError("Field `max_it` must be positive or 0.")
        elif collection_rate < 1:
            raise ArgumentError("Field `colection_rate` must be positive.")
        elif collection_rate > max_it and max_it > 0:
            raise ArgumentError("Field `colection_rate` must be smaller than `max_it`.")
        self.max_it = int(max_it)
        self.collection_rate = int(collection_rate)
        self.threshold_info = threshold
        self.stopping_criterion = stopping_criterion


class BasicLoggerRecipe(LoggerRecipe):
    """basic_logger.jl:44-67."""

    def __init__(self, max_it, error, threshold_info, iteration, record_location, collection_rate, converged,
                 stopping_criterion, hist):
        self.max_it = max_it
        self.error = error
        self.threshold_info = threshold_info
        self.iteration = iteration
        self.record_location = record_location
        self.collection_rate = collection_rate
        self.converged = converged
        self.stopping_criterion = stopping_criterion
        self.hist = hist

    def update_logger_(self, error: float, iteration: int) -> None:
        """basic_logger.jl:84-101 (record_location is 1-based like the reference's)."""
        self.iteration = iteration
        self.error = error
        self.converged = self.stopping_criterion(self) if iteration < self.max_it else True
        if self.converged:
            self.hist[self.record_location - 1] = error
        elif iteration % self.collection_rate == 0:
            self.hist[self.record_location - 1] = error
            self.record_location += 1

    def reset_logger_(self) -> None:
        """basic_logger.jl:103-110."""
        self.error = 0.0
        self.iteration = 1
        self.record_location = 1
        self.converged = False
        self.hist[:] = 0.0


def complete_logger(logger: Logger) -> LoggerRecipe:
    """basic_logger.jl:70-82 for BasicLogger; otherwise the logger's own complete_logger()."""
    if isinstance(logger, BasicLogger):
        max_collection = int(math.ceil(logger.max_it / logger.collection_rate))
        return BasicLoggerRecipe(logger.max_it, 0.0, logger.threshold_info, 1, 1, logger.collection_rate, False,
                                 logger.stopping_criterion, np.zeros(max_collection + 1))
    if hasattr(logger, "complete_logger"):
        return logger.complete_logger()
    raise ArgumentError(f"No method `complete_logger` exists for logger of type {type(logger).__name__}.")


def update_logger_(logger: LoggerRecipe, error: float, iteration: int) -> None:
    if not hasattr(logger, "update_logger_"):
        raise ArgumentError(f"No method `update_logger!` exists for logger of type {type(logger).__name__}.")
    logger.update_logger_(error, iteration)


def reset_logger_(logger: LoggerRecipe) -> None:
    if not hasattr(logger, "reset_logger_"):
        raise ArgumentError(f"No method `reset_logger!` exists for logger of type {type(logger).__name__}.")
    logger.reset_logger_()


# ----------------------------------------------------------------------------------
# Error methods (src/Solvers/ErrorMethods/{full_residual,ls_gradient,compressed_residual}.jl)
# ----------------------------------------------------------------------------------
class FullResidual(SolverError):
    """full_residual.jl: the norm of the full residual b - Ax."""


class FullResidualRecipe(SolverErrorRecipe):
    """full_residual.jl: field `residual` (b - Ax, refreshed at the end of rsolve_)."""

    def __init__(self, residual):
        self.residual = residual

    def compute_error(self, solver, A, b) -> float:
        if isinstance(solver, IHSRecipe) and solver._live:
            return solver._errors()[0]
        import torch
        x = solver.solution_vec
        return float(torch.linalg.vector_norm(b - A @ x))


class LSGradient(SolverError):
    """ls_gradient.jl: the norm of the least-squares gradient -A'(b - Ax)."""


class LSGradientRecipe(SolverErrorRecipe):
    """ls_gradient.jl: field `gradient` (-A'r of the solver's residual_vec)."""

    def __init__(self, gradient):
        self.gradient = gradient

    def compute_error(self, solver, A, b) -> float:
        if isinstance(solver, IHSRecipe) and solver._live:
            return solver._errors()[1]
        import torch
        return float(torch.linalg.vector_norm(A.T @ solver.residual_vec))


class CompressedResidual(SolverError):
    """compressed_residual.jl: the norm of the compressed residual Sb - SAx."""


class CompressedResidualRecipe(SolverErrorRecipe):
    def __init__(self, residual, residual_view):
        self.residual = residual
        self.residual_view = residual_view

    def compute_error(self, solver, A, b) -> float:
        if not hasattr(solver, "vec_view"):
            # the reference reads solver.vec_view, which an IHSRecipe does not have
            raise ArgumentError(f"type {type(solver).__name__} has no field vec_view")
        import torch
        return float(torch.linalg.vector_norm(solver.vec_view - solver.mat_view @ solver.solution_vec))


def complete_error(error: SolverError, solver: Solver, A, b) -> SolverErrorRecipe:
    import torch
    m, n = A.shape[0], A.shape[1]
    dev = A.device if isinstance(A, torch.Tensor) and A.is_cuda else "cuda"
    dt = A.dtype if isinstance(A, torch.Tensor) else getattr(torch, np.dtype(np.asarray(A).dtype).name)
    if isinstance(error, FullResidual):
        return FullResidualRecipe(torch.zeros(m, dtype=dt, device=dev))
    if isinstance(error, LSGradient):
        return LSGradientRecipe(torch.zeros(n, dtype=dt, device=dev))
    if isinstance(error, CompressedResidual):
        res = torch.zeros(m, dtype=dt, device=dev)
        return CompressedResidualRecipe(res, res[:1])
    if hasattr(error, "complete_error"):
        return error.complete_error(solver, A, b)
    raise ArgumentError(f"No method `complete_error` exists for error method of type {type(error).__name__}.")


def compute_error(error: SolverErrorRecipe, solver: SolverRecipe, A, b) -> float:
    if not hasattr(error, "compute_error"):
        raise ArgumentError(f"No method `compute_error` exists for error recipe of type {type(error).__name__}.")
    return float(error.compute_error(solver, A, b))


# ----------------------------------------------------------------------------------
# IHS (src/Solvers/ihs.jl)
# ----------------------------------------------------------------------------------
class IHS(Solver):
    """ihs.jl:40-80: fields alpha, log, compressor, error."""

    def __init__(self, compressor: Compressor = None, log: Logger = None, error: SolverError = None,
                 alpha: float = 1.0):
        compressor = SparseSign(cardinality=Left()) if compressor is None else compressor
        log = BasicLogger() if log is None else log
        error = FullResidual() if error is None else error
        if type(compressor.cardinality) is not Left:
            warnings.warn("Compressor has cardinality `Right` but IHS compresses from the `Left`.")
        if alpha < 0:
            warnings.warn("Negative step size could lead to divergent iterates.")
        self.alpha = float(alpha)
        self.log = log
        self.compressor = compressor
        self.error = error


class _DeviceView:
    """__cuda_array_interface__ over memory the solver owns (kept alive by `owner`)."""

    def __init__(self, ptr, shape, strides_bytes, typestr, owner):
        self.owner = owner
        self.__cuda_array_interface__ = {"data": (int(ptr), False), "shape": tuple(shape),
                                         "strides": tuple(strides_bytes), "typestr": typestr, "version": 3}


class IHSRecipe(SolverRecipe):
    """ihs.jl:82-125: fields log, compressor, error, alpha, compressed_mat, mat_view,
    residual_vec, gradient_vec, buffer_vec, solution_vec, R.  compressed_mat is the
    device solver's S*A workspace; R is the upper-triangular factor with R'R = (SA)'(SA)
    (positive diagonal, from the FP64 Cholesky factorisation), valid after a step."""

    def __init__(self, log, compressor, error, alpha, residual_vec, gradient_vec, buffer_vec, solution_vec, handle,
                 ctx, m, n, dtype):
        self.log = log
        self.compressor = compressor
        self.error = error
        self.alpha = alpha
        self.residual_vec = residual_vec
        self.gradient_vec = gradient_vec
        self.buffer_vec = buffer_vec
        self.solution_vec = solution_vec
        self._h = handle
        self._ctx = ctx
        self._m, self._n, self._dtype = m, n, dtype
        self._live = False

    def _workspace(self):
        sa, u, rq, d = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        L.check(L.lib().rla_ihs_workspace(self._h, ctypes.byref(sa), ctypes.byref(u), ctypes.byref(rq),
                                          ctypes.byref(d)))
        return sa.value, u.value, rq.value, d.value

    @property
    def compressed_mat(self):
        import torch
        s, n = self.compressor.n_rows, self._n
        es = 4 if self._dtype == L.RLA_F32 else 8
        v = _DeviceView(self._workspace()[0], (s, n), (es, es * s), "<f4" if es == 4 else "<f8", self)
        return torch.as_tensor(v, device=f"cuda:{self._ctx.device}")

    @property
    def mat_view(self):
        return self.compressed_mat[: self.compressor.n_rows, :]

    @property
    def R(self):
        import torch
        n = self._n
        _, _, rq, d = self._workspace()
        Rq = torch.as_tensor(_DeviceView(rq, (n, n), (8, 8 * n), "<f8", self), device=f"cuda:{self._ctx.device}")
        dv = torch.as_tensor(_DeviceView(d, (n,), (8,), "<f8", self), device=f"cuda:{self._ctx.device}")
        return torch.triu(Rq) / dv[None, :]

    def _errors(self):
        ef, eg = ctypes.c_double(), ctypes.c_double()
        L.check(L.lib().rla_ihs_errors(self._ctx.handle, self._h, ctypes.byref(ef), ctypes.byref(eg)),
                self._ctx.handle)
        return ef.value, eg.value

    def __del__(self):
        try:
            if self._h:
                L.lib().rla_ihs_destroy(self._h)
                self._h = None
        except Exception:
            pass


def _torch_dtype(A):
    import torch
    if isinstance(A, torch.Tensor):
        return A.dtype
    return torch.float32 if np.asarray(A).dtype == np.float32 else torch.float64


def complete_solver(ingredients: Solver, x, A, b, seed=None) -> SolverRecipe:
    """complete_solver(::IHS, x, A, b) (ihs.jl:127-206).  `seed` seeds the compressor's draws
    (default: the next seed of the process-wide sequence, see compressors.seed_)."""
    import torch
    if isinstance(ingredients, (Kaczmarz, ColumnProjection)):
        return _complete_proj(ingredients, x, A, b, seed)
    if not isinstance(ingredients, IHS):
        raise ArgumentError(f"No method `complete_solver` exists for solver of type {type(ingredients).__name__}.")
    dt = _torch_dtype(A)
    np_dt = np.float32 if dt == torch.float32 else np.float64
    comp = ingredients.compressor
    if getattr(comp, "type", np_dt) != np_dt:
        # the device sketch computes in A's element type
        comp = copy.copy(comp)
        object.__setattr__(comp, "type", np_dt)
    compressor = complete_compressor(comp, x, A, b, seed=seed)
    logger = complete_logger(ingredients.log)
    error = complete_error(ingredients.error, ingredients, A, b)
    sample_size = compressor.n_rows
    rows_a, cols_a = A.shape[0], A.shape[1]
    if not hasattr(error, "residual"):
        raise ArgumentError(f"ErrorRecipe {type(error).__name__} does not contain the field 'residual' and is "
                            "not valid for an IHS solver.")
    if not hasattr(logger, "converged"):
        raise ArgumentError(f"LoggerRecipe {type(logger).__name__} does not contain the field 'converged' and is "
                            "not valid for an IHS solver.")
    if cols_a > sample_size:
        raise ArgumentError("Compression dimension not larger than column dimension this will lead to singular QR "
                            "decompositions, which cannot be inverted.")
    if rows_a < sample_size:
        raise ArgumentError("Compression dimension larger row dimension.")
    if cols_a >= rows_a:
        raise ArgumentError("Matrix must have more rows than columns.")
    ctx = L.Context.get(compressor._ctx.device)
    h = ctypes.c_void_p()
    L.check(L.lib().rla_ihs_create(ctx.handle, compressor.handle, rla_dtype(dt), rows_a, cols_a,
                                   float(ingredients.alpha), ctypes.byref(h)), ctx.handle)
    dev = torch.device("cuda", ctx.device)
    res = torch.zeros(rows_a, dtype=dt, device=dev)
    grad = torch.zeros(cols_a, dtype=dt, device=dev)
    buf = torch.zeros(cols_a, dtype=dt, device=dev)
    return IHSRecipe(logger, compressor, error, ingredients.alpha, res, grad, buf, x, h, ctx, rows_a, cols_a,
                     rla_dtype(dt))


def _device_matrix(A, dt, dev):
    """Column-major device copy (or the tensor itself when it already is one)."""
    import torch
    if isinstance(A, torch.Tensor) and A.is_cuda and A.dtype == dt and A.stride(0) == 1 and (
            A.shape[1] <= 1 or A.stride(1) >= A.shape[0]):
        return A
    t = A if isinstance(A, torch.Tensor) else torch.from_numpy(np.asfortranarray(A))
    return t.to(device=dev, dtype=dt).t().contiguous().t()


def _device_vector(v, dt, dev):
    import torch
    if isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == dt and v.is_contiguous():
        return v, False
    t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v))
    return t.to(device=dev, dtype=dt).contiguous(), True


def rsolve_(solver: SolverRecipe, x, A, b) -> None:
    """rsolve!(::IHSRecipe, x, A, b) (ihs.jl:214-254)."""
    import torch
    if isinstance(solver, (KaczmarzRecipe, ColumnProjectionRecipe)):
        return _rsolve_proj(solver, x, A, b)
    if not isinstance(solver, IHSRecipe):
        raise ArgumentError(f"No method `rsolve!` exists for solver recipe of type {type(solver).__name__}.")
    if A.shape[0] != solver._m or A.shape[1] != solver._n:
        raise ArgumentError("Matrix dimensions differ from the ones the solver was completed with.")
    reset_logger_(solver.log)
    dt = solver.residual_vec.dtype
    dev = solver.residual_vec.device
    Ad = _device_matrix(A, dt, dev)
    bd, _ = _device_vector(b, dt, dev)
    xd, copied = _device_vector(x, dt, dev)
    solver.solution_vec = xd
    lib, ctx = L.lib(), L.Context.get(dev.index)
    lda = max(Ad.shape[0], 1) if Ad.shape[1] <= 1 else Ad.stride(1)
    args = (ctx.handle, solver._h, Ad.data_ptr(), lda, bd.data_ptr())
    vecs = (xd.data_ptr(), solver.residual_vec.data_ptr(), solver.gradient_vec.data_ptr())
    L.check(lib.rla_ihs_start(*args, *vecs), ctx.handle)
    solver._live = True
    try:
        for i in range(1, solver.log.max_it + 1):
            err = compute_error(solver.error, solver, Ad, bd)
            update_logger_(solver.log, err, i)
            if solver.log.converged:
                break
            L.check(lib.rla_ihs_step(*args, *vecs), ctx.handle)
            solver.compressor._cache = None  # update_compressor! drew new values
    finally:
        solver._live = False
        solver.compressor._refresh_info()
    if isinstance(solver.error, FullResidualRecipe) and solver.error.residual.shape[0] == solver._m:
        solver.error.residual.copy_(bd - Ad @ xd)
    if copied:
        if isinstance(x, torch.Tensor):
            x.copy_(xd)
        else:
            x[...] = xd.cpu().numpy()
        solver.solution_vec = x
    return None


# ----------------------------------------------------------------------------------
# Sub-solvers (src/Solvers/SubSolvers.jl, SubSolvers/{lq,qr}.jl)
# ----------------------------------------------------------------------------------
class SubSolver:
    """Abstract supertype of the solvers of a sketched block."""


class SubSolverRecipe:
    """Abstract supertype of completed sub-solvers."""


class LQSolver(SubSolver):
    """lq.jl: minimum-norm solution of a wide block (ldiv! through qr!(A')')."""


class QRSolver(SubSolver):
    """qr.jl: least-squares solution of a tall block (ldiv! through qr!(A))."""


class LQSolverRecipe(SubSolverRecipe):
    def __init__(self, A):
        self.A = A


class QRSolverRecipe(SubSolverRecipe):
    def __init__(self, A):
        self.A = A


def complete_sub_solver(solver: SubSolver, A, *args) -> SubSolverRecipe:
    if isinstance(solver, LQSolver):
        return LQSolverRecipe(A)
    if isinstance(solver, QRSolver):
        return QRSolverRecipe(A)
    raise ArgumentError(f"No method `complete_sub_solver` exists for sub-solver of type {type(solver).__name__}.")


def update_sub_solver_(solver: SubSolverRecipe, A) -> None:
    solver.A = A


def ldiv_(x, solver: SubSolverRecipe, b) -> None:
    """ldiv!(x, recipe, b): LQ -> minimum-norm solution, QR -> least-squares solution
    (a host convenience of the sub-solver API; the device solvers solve their blocks
    themselves)."""
    import torch
    A = solver.A if isinstance(solver.A, torch.Tensor) else torch.as_tensor(np.asarray(solver.A))
    bb = b if isinstance(b, torch.Tensor) else torch.as_tensor(np.asarray(b))
    A64, b64 = A.double().cpu(), bb.double().cpu()
    if isinstance(solver, LQSolverRecipe):
        sol = A64.T @ torch.linalg.solve(A64 @ A64.T, b64)
    elif isinstance(solver, QRSolverRecipe):
        sol = torch.linalg.lstsq(A64, b64.unsqueeze(1)).solution.squeeze(1)
    else:
        raise ArgumentError(f"No method `ldiv!` exists for sub-solver of type {type(solver).__name__}.")
    if isinstance(x, torch.Tensor):
        x.copy_(sol.to(x.dtype))
    else:
        x[...] = sol.numpy()


# ----------------------------------------------------------------------------------
# Kaczmarz (src/Solvers/kaczmarz.jl) and ColumnProjection (src/Solvers/col_projection.jl)
# ----------------------------------------------------------------------------------
class Kaczmarz(Solver):
    """kaczmarz.jl:63-107: fields alpha, compressor, log, error, sub_solver."""

    def __init__(self, compressor: Compressor = None, log: Logger = None, error: SolverError = None,
                 sub_solver: SubSolver = None, alpha: float = 1.0):
        compressor = SparseSign(cardinality=Left()) if compressor is None else compressor
        if type(compressor.cardinality) is not Left:
            warnings.warn("Compressor has cardinality `Right` but kaczmarzcompresses  from the  `Left`.")
        self.alpha = float(alpha)
        self.compressor = compressor
        self.log = BasicLogger() if log is None else log
        self.error = FullResidual() if error is None else error
        self.sub_solver = LQSolver() if sub_solver is None else sub_solver


class ColumnProjection(Solver):
    """col_projection.jl:89-121: fields alpha, compressor, error, log, sub_solver."""

    def __init__(self, alpha: float = 1.0, compressor: Compressor = None, error: SolverError = None,
                 log: Logger = None, sub_solver: SubSolver = None):
        from .compressors import Right
        compressor = SparseSign(cardinality=Right()) if compressor is None else compressor
        if type(compressor.cardinality) is not Right:
            warnings.warn("Compressor has cardinality `Left` but ColumnProjectioncompresses from the `Right`. This "
                          "may cause an inefficiency.")
        self.alpha = float(alpha)
        self.compressor = compressor
        self.error = LSGradient() if error is None else error
        self.log = BasicLogger() if log is None else log
        self.sub_solver = QRSolver() if sub_solver is None else sub_solver


class _ProjRecipe(SolverRecipe):
    """Shared device state of KaczmarzRecipe / ColumnProjectionRecipe (rla_proj_*)."""

    def _init_device(self, kind, A, dtype):
        ctx = L.Context.get(self.compressor._ctx.device)
        h = ctypes.c_void_p()
        m, n = A.shape[0], A.shape[1]
        L.check(L.lib().rla_proj_create(ctx.handle, self.compressor.handle, kind, rla_dtype(dtype), m, n,
                                        float(self.alpha), ctypes.byref(h)), ctx.handle)
        self._h, self._ctx, self._m, self._n, self._kind = h, ctx, m, n, kind
        self._live = False

    def _workspace(self):
        mat, vec = ctypes.c_void_p(), ctypes.c_void_p()
        L.check(L.lib().rla_proj_workspace(self._h, ctypes.byref(mat), ctypes.byref(vec)))
        return mat.value, vec.value

    def _view(self, ptr, shape, strides, dtype):
        import torch
        es = 4 if dtype == torch.float32 else 8
        v = _DeviceView(ptr, shape, tuple(es * s for s in strides), "<f4" if es == 4 else "<f8", self)
        return torch.as_tensor(v, device=f"cuda:{self._ctx.device}")

    def _error(self, kind, A, b, x, r) -> float:
        val = ctypes.c_double()
        lda = max(A.shape[0], 1) if A.shape[1] <= 1 else A.stride(1)
        L.check(L.lib().rla_proj_error(self._ctx.handle, self._h, kind, A.data_ptr(), lda,
                                       None if b is None else b.data_ptr(), None if x is None else x.data_ptr(),
                                       None if r is None else r.data_ptr(), ctypes.byref(val)), self._ctx.handle)
        return val.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                L.lib().rla_proj_destroy(self._h)
                self._h = None
        except Exception:
            pass


class KaczmarzRecipe(_ProjRecipe):
    """kaczmarz.jl:109-160: fields compressor, log, error, sub_solver, alpha, compressed_mat,
    compressed_vec, solution_vec, update_vec, mat_view, vec_view (views of the solver's last
    sketched block)."""

    @property
    def compressed_mat(self):
        s = self.compressor.n_rows
        return self._view(self._workspace()[0], (s, self._n), (self._n, 1), self._dtype)

    @property
    def compressed_vec(self):
        return self._view(self._workspace()[1], (self.compressor.n_rows,), (1,), self._dtype)

    @property
    def mat_view(self):
        return self.compressed_mat

    @property
    def vec_view(self):
        return self.compressed_vec


class ColumnProjectionRecipe(_ProjRecipe):
    """col_projection.jl:159-200: fields compressor, log, error, sub_solver, alpha,
    compressed_mat, solution_vec, update_vec, mat_view, residual_vec."""

    @property
    def compressed_mat(self):
        s = self.compressor.n_cols
        return self._view(self._workspace()[0], (self._m, s), (1, self._m), self._dtype)

    @property
    def mat_view(self):
        return self.compressed_mat


def _complete_proj(ingredients, x, A, b, seed):
    import torch
    kz = isinstance(ingredients, Kaczmarz)
    dt = _torch_dtype(A)
    np_dt = np.float32 if dt == torch.float32 else np.float64
    comp = ingredients.compressor
    if getattr(comp, "type", np_dt) != np_dt:
        comp = copy.copy(comp)
        object.__setattr__(comp, "type", np_dt)
    compressor = complete_compressor(comp, x, A, b, seed=seed) if kz else complete_compressor(comp, A, b, seed=seed)
    logger = complete_logger(ingredients.log)
    error = complete_error(ingredients.error, ingredients, A, b)
    name = "a kaczmarz solver" if kz else "a `ColumnProjection` solver"
    if kz:
        if not hasattr(error, "residual"):
            raise ArgumentError(f"ErrorRecipe {type(error).__name__} does not contain the field 'residual' and is "
                                f"not valid for {name}.")
        if not hasattr(logger, "converged"):
            raise ArgumentError(f"LoggerRecipe {type(logger).__name__} does not contain the field 'converged' and "
                                f"is not valid for {name}.")
        if not isinstance(ingredients.sub_solver, LQSolver):
            raise ArgumentError("The device Kaczmarz solver takes the LQSolver sub-solver.")
    else:
        if not hasattr(error, "gradient"):
            raise ArgumentError(f"ErrorRecipe {type(error).__name__} does not contain the field 'gradient' and is "
                                f"not valid for {name}.")
        if not hasattr(logger, "max_it"):
            raise ArgumentError(f"LoggerRecipe {type(logger).__name__} does not contain the field `max_it` and is "
                                f"not valid for {name}.")
        if not hasattr(logger, "converged"):
            raise ArgumentError(f"LoggerRecipe {type(logger).__name__} does not contain the field `converged` and "
                                f"is not valid for {name}.")
        if not isinstance(ingredients.sub_solver, QRSolver):
            raise ArgumentError("The device ColumnProjection solver takes the QRSolver sub-solver.")
    R = (KaczmarzRecipe if kz else ColumnProjectionRecipe)()
    R.compressor, R.log, R.error, R.alpha = compressor, logger, error, ingredients.alpha
    R.sub_solver = complete_sub_solver(ingredients.sub_solver, None)
    R.solution_vec = x
    R._dtype = dt
    R._init_device(L.RLA_PROJ_KACZMARZ if kz else L.RLA_PROJ_COLUMN, A, dt)
    dev = torch.device("cuda", R._ctx.device)
    R.update_vec = torch.zeros(A.shape[1] if kz else compressor.n_cols, dtype=dt, device=dev)
    if not kz:
        R.residual_vec = torch.zeros(A.shape[0], dtype=dt, device=dev)
    return R


def _proj_error(solver, A, b, x):
    """compute_error for the built-in error methods, on the device solver."""
    e = solver.error
    if isinstance(e, FullResidualRecipe):
        return solver._error(L.RLA_ERR_FULL_RESIDUAL, A, b, x, None)
    if isinstance(e, LSGradientRecipe):
        if not isinstance(solver, ColumnProjectionRecipe):
            raise ArgumentError(f"type {type(solver).__name__} has no field residual_vec")
        return solver._error(L.RLA_ERR_LS_GRADIENT, A, None, None, solver.residual_vec)
    if isinstance(e, CompressedResidualRecipe):
        if not isinstance(solver, KaczmarzRecipe):
            raise ArgumentError(f"type {type(solver).__name__} has no field vec_view")
        return solver._error(L.RLA_ERR_COMPRESSED_RESIDUAL, A, None, x, None)
    return compute_error(e, solver, A, b)


def _rsolve_proj(solver, x, A, b):
    import torch
    kz = isinstance(solver, KaczmarzRecipe)
    reset_logger_(solver.log)
    if kz:
        if x.shape[0] != A.shape[1]:
            raise DimensionMismatch(f"Dimension of `x`, {x.shape[0]} is different from number of columns in `A`,"
                                    f"{A.shape[1]}.")
        if b.shape[0] != A.shape[0]:
            raise DimensionMismatch(f"Dimension of `b`, {b.shape[0]} is different from number of rows in `A`,"
                                    f"{A.shape[0]}.")
    dt = solver._dtype
    dev = torch.device("cuda", solver._ctx.device)
    Ad = _device_matrix(A, dt, dev)
    bd, _ = _device_vector(b, dt, dev)
    xd, copied = _device_vector(x, dt, dev)
    solver.solution_vec = xd
    lib, ctx = L.lib(), solver._ctx
    lda = max(Ad.shape[0], 1) if Ad.shape[1] <= 1 else Ad.stride(1)
    rp = None if kz else solver.residual_vec.data_ptr()
    L.check(lib.rla_proj_start(ctx.handle, solver._h, Ad.data_ptr(), lda, bd.data_ptr(), xd.data_ptr(), rp),
            ctx.handle)
    off = 0 if kz else 1  # ColumnProjection logs iteration i-1 (col_projection.jl:334)
    for i in range(1, solver.log.max_it + 1):
        err = _proj_error(solver, Ad, bd, xd)
        update_logger_(solver.log, err, i - off)
        if solver.log.converged:
            break
        L.check(lib.rla_proj_step(ctx.handle, solver._h, Ad.data_ptr(), lda, bd.data_ptr(), xd.data_ptr(), rp),
                ctx.handle)
        solver.compressor._cache = None
    else:
        if not kz:  # col_projection.jl:368-369: the error after the last iteration
            update_logger_(solver.log, _proj_error(solver, Ad, bd, xd), solver.log.max_it)
    solver.compressor._refresh_info()
    if isinstance(solver.error, FullResidualRecipe) and solver.error.residual.shape[0] == Ad.shape[0]:
        solver.error.residual.copy_(bd - Ad @ xd)
    if isinstance(solver.error, LSGradientRecipe) and not kz:
        solver.error.gradient.copy_(-(Ad.T @ solver.residual_vec))
    if copied:
        if isinstance(x, torch.Tensor):
            x.copy_(xd)
        else:
            x[...] = xd.cpu().numpy()
        solver.solution_vec = x
    return None
