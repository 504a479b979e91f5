"""The Sampling compressor and its distributions: host mirror of
src/Compressors/sampling.jl and src/Compressors/Distributions{.jl,/uniform.jl,
/strohmer_vershynin.jl,/agmon.jl}.

Same names, fields, defaults and error messages as the reference, with 0-based indices.
A SamplingRecipe owns a device sketch of kind RLA_SAMPLING (rla_sampling_create): the draw
and the gather / scatter-add applies run on the device; ``idx`` downloads the current
indices.  The distribution recipes answer ``sample_distribution_`` with device draws as well
(one device sampler per requested sample size).

As in the reference, ``complete_compressor(Sampling(distribution=Agmon()), ...)`` raises: the
Sampling recipe completes its distribution from A alone, and Agmon has no such method
(agmon.jl defines complete_distribution for (x, A, b) only).  Agmon is reached through
``complete_distribution(Agmon(...), x, A, b)`` and ``sample_distribution_``.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib as L
from ._arrays import rla_dtype
from .compressors import Cardinality, Compressor, CompressorRecipe, Left, Right, Undef, _next_seed
from .errors import ArgumentError, DimensionMismatch


# ----------------------------------------------------------------------------------
# Distributions (src/Compressors/Distributions.jl and Distributions/*.jl)
# ----------------------------------------------------------------------------------
class Distribution:
    """Abstract supertype of index distributions for sampling."""


class DistributionRecipe:
    """Abstract supertype of completed distributions."""


class Uniform(Distribution):
    """uniform.jl: equal weights over the rows (Left) or columns (Right)."""

    def __init__(self, cardinality: Cardinality = None, replace: bool = False):
        self.cardinality = Undef() if cardinality is None else cardinality
        self.replace = bool(replace)


class L2Norm(Distribution):
    """strohmer_vershynin.jl: weights = squared row (Left) or column (Right) norms of A."""

    def __init__(self, cardinality: Cardinality = None, replace: bool = False):
        self.cardinality = Undef() if cardinality is None else cardinality
        self.replace = bool(replace)


class Agmon(Distribution):
    """agmon.jl: the indices of largest residual among beta random candidates."""

    def __init__(self, cardinality: Cardinality = None, replace: bool = False, beta: int = 1):
        if beta < 1:
            raise ArgumentError(f"`Agmon` beta must be >= 1, got beta={beta}")
        self.cardinality = Undef() if cardinality is None else cardinality
        self.replace = bool(replace)
        self.beta = int(beta)


_DIST = {Uniform: L.RLA_DIST_UNIFORM, L2Norm: L.RLA_DIST_L2NORM, Agmon: L.RLA_DIST_AGMON}


def _device_matrix(A):
    import torch
    if isinstance(A, torch.Tensor) and A.is_cuda and A.stride(0) == 1 and (A.shape[1] <= 1 or
                                                                          A.stride(1) >= max(A.shape[0], 1)):
        return A
    t = A if isinstance(A, torch.Tensor) else torch.from_numpy(np.asfortranarray(A))
    return t.to("cuda").t().contiguous().t()


def _lda(Ad) -> int:
    """Leading dimension of a column-major device matrix (a single column may report any stride)."""
    return max(Ad.shape[0], 1) if Ad.shape[1] <= 1 else Ad.stride(1)


def _device_vector(v, dtype):
    import torch
    if v is None:
        return None
    t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v))
    return t.to(device="cuda", dtype=dtype).contiguous().reshape(-1)


def _card_code(card) -> int:
    return L.RLA_LEFT if isinstance(card, Left) else L.RLA_RIGHT


def _undef_error(name: str, fn: str):
    return ArgumentError(f"`{name}` cardinality must be specified as `Left()` or `Right()`."
                         f"`Undef()` is not allowed in `{fn}`.")


class _DeviceSampler:
    """One device sampling sketch per sample size (rla_sampling_create)."""

    def __init__(self, card, dtype, dim, dist, replace, beta, seed):
        self.args = (card, dtype, dim, dist, replace, beta)
        self.seed = seed
        self.by_k = {}

    def sketch(self, k: int):
        h = self.by_k.get(k)
        if h is None:
            ctx = L.Context.get()
            h = ctypes.c_void_p()
            card, dtype, dim, dist, replace, beta = self.args
            L.check(L.lib().rla_sampling_create(ctx.handle, card, dtype, k, dim, dist, int(replace), beta,
                                                self.seed + k, ctypes.byref(h)), ctx.handle)
            self.by_k[k] = h
        return h

    def __del__(self):
        try:
            for h in self.by_k.values():
                L.lib().rla_sketch_destroy(h)
        except Exception:
            pass


class _RecipeBase(DistributionRecipe):
    def _sample(self, k: int) -> np.ndarray:
        ctx = L.Context.get()
        h = self._sampler.sketch(k)
        A, x, b, r = self._data
        if self._dist == L.RLA_DIST_UNIFORM:
            L.check(L.lib().rla_sketch_update(ctx.handle, h), ctx.handle)
        else:
            L.check(L.lib().rla_sampling_update(ctx.handle, h, A.shape[0], A.shape[1], A.data_ptr(), _lda(A),
                                                None if x is None else x.data_ptr(), 0 if x is None else x.numel(),
                                                None if b is None else b.data_ptr(), 0 if b is None else b.numel(),
                                                None if r is None else r.data_ptr()), ctx.handle)
        out = np.zeros(k, np.int64)
        L.check(L.lib().rla_sketch_get_draws(ctx.handle, h, out.ctypes.data, None, None, None), ctx.handle)
        return out


class UniformRecipe(_RecipeBase):
    """uniform.jl: fields cardinality, replace, state_space, weights."""

    def __init__(self, cardinality, replace, A, seed):
        self.cardinality, self.replace = cardinality, replace
        self._set(A, seed)

    @property
    def state_space(self):
        return np.arange(self._dim)

    @property
    def weights(self):
        return np.ones(self._dim)

    def _set(self, A, seed=None):
        Ad = _device_matrix(A)
        dim = Ad.shape[0] if isinstance(self.cardinality, Left) else Ad.shape[1]
        self._dim = dim
        self._dist = L.RLA_DIST_UNIFORM
        if seed is not None or not hasattr(self, "_sampler") or self._sampler.args[2] != dim:
            self._sampler = _DeviceSampler(_card_code(self.cardinality), rla_dtype(Ad.dtype), dim, self._dist,
                                           self.replace, 1, _next_seed() if seed is None else seed)
        self._data = (Ad, None, None, None)


class L2NormRecipe(_RecipeBase):
    """strohmer_vershynin.jl: fields cardinality, replace, state_space, weights."""

    def __init__(self, cardinality, replace, A, seed):
        self.cardinality, self.replace = cardinality, replace
        self._sampler = None
        self._set(A, seed)

    @property
    def state_space(self):
        return np.arange(self._dim)

    @property
    def weights(self):
        """Squared row (Left) / column (Right) norms of the A of the last update (computed on access)."""
        import torch
        Ad = self._data[0]
        left = isinstance(self.cardinality, Left)
        return torch.linalg.vector_norm(Ad.double(), dim=1 if left else 0).pow(2).cpu().numpy()

    def _set(self, A, seed=None):
        Ad = _device_matrix(A)
        left = isinstance(self.cardinality, Left)
        dim = Ad.shape[0] if left else Ad.shape[1]
        self._dim = dim
        self._dist = L.RLA_DIST_L2NORM
        if self._sampler is None or self._sampler.args[2] != dim:
            self._sampler = _DeviceSampler(_card_code(self.cardinality), rla_dtype(Ad.dtype), dim, self._dist,
                                           self.replace, 1, _next_seed() if seed is None else seed)
        self._data = (Ad, None, None, None)


class AgmonRecipe(_RecipeBase):
    """agmon.jl: fields cardinality, replace, beta, state_space, sample_buffer, A, b, x, r."""

    def __init__(self, cardinality, replace, beta, x, A, b, seed):
        self.cardinality, self.replace, self.beta = cardinality, replace, beta
        self._sampler = None
        self._seed = seed
        self._set(x, A, b, None)

    def _set(self, x, A, b, r):
        Ad = _device_matrix(A)
        left = isinstance(self.cardinality, Left)
        m, n = Ad.shape
        dim, exp_x, exp_b = (m, n, m) if left else (n, n, m)
        if len(b) != exp_b:
            raise DimensionMismatch(f"Vector b has length {len(b)}, expected {exp_b} to match rows of A")
        if len(x) != exp_x:
            raise DimensionMismatch(f"Vector x has length {len(x)}, expected {exp_x} to match columns of A")
        if self.beta > dim:
            raise ArgumentError(f"`Agmon` beta must be <= number of {'rows' if left else 'columns'} ({dim}), "
                                f"got beta={self.beta}")
        self._dim = dim
        self.sample_buffer = np.zeros(self.beta, np.int64)
        self.A, self.b, self.x, self.r = A, b, x, r
        self._dist = L.RLA_DIST_AGMON
        if self._sampler is None or self._sampler.args[2] != dim:
            self._sampler = _DeviceSampler(_card_code(self.cardinality), rla_dtype(Ad.dtype), dim, self._dist,
                                           self.replace, self.beta,
                                           _next_seed() if self._seed is None else self._seed)
        self._data = (Ad, _device_vector(x, Ad.dtype), _device_vector(b, Ad.dtype), _device_vector(r, Ad.dtype))

    @property
    def state_space(self):
        return np.arange(self._dim)

    def _sample(self, k: int) -> np.ndarray:
        if k > self.beta:
            raise ArgumentError(f"`Agmon` cannot output {k} indices when beta={self.beta}.")
        return super()._sample(k)


def complete_distribution(distribution: Distribution, *args, seed: Optional[int] = None) -> DistributionRecipe:
    """complete_distribution(distribution, A), (…, A, b) and (…, x, A, b) (Distributions.jl);
    Agmon completes from (x, A, b) only."""
    if isinstance(distribution, Agmon):
        if len(args) != 3:
            A = args[-1] if len(args) == 1 else args[0]
            raise ArgumentError(f"No `complete_distribution` method defined for a distribution of type Agmon and "
                                f"{type(A).__name__}.")
        x, A, b = args
        if isinstance(distribution.cardinality, Undef):
            raise _undef_error("Agmon", "complete_distribution")
        return AgmonRecipe(distribution.cardinality, distribution.replace, distribution.beta, x, A, b, seed)
    A = args[1] if len(args) == 3 else args[0]
    if isinstance(distribution, (Uniform, L2Norm)):
        name = type(distribution).__name__
        if isinstance(distribution.cardinality, Undef):
            raise _undef_error(name, "complete_distribution")
        cls = UniformRecipe if isinstance(distribution, Uniform) else L2NormRecipe
        return cls(distribution.cardinality, distribution.replace, A, seed)
    raise ArgumentError(f"No `complete_distribution` method defined for a distribution of type "
                        f"{type(distribution).__name__} and {type(A).__name__}.")


def update_distribution_(recipe: DistributionRecipe, *args, r=None) -> None:
    """update_distribution!(recipe, A), (…, A, b), (…, x, A, b); Agmon takes (x, A, b; r)."""
    if isinstance(recipe, AgmonRecipe):
        if len(args) != 3:
            raise ArgumentError("No `update_distribution!` method defined for a distribution of type AgmonRecipe.")
        x, A, b = args
        recipe._set(x, A, b, r)
        return
    if isinstance(recipe, (UniformRecipe, L2NormRecipe)):
        recipe._set(args[1] if len(args) == 3 else args[0])
        return
    raise ArgumentError(f"No `update_distribution!` method defined for a distribution of type {type(recipe).__name__}.")


def sample_distribution_(indices, recipe: DistributionRecipe) -> None:
    """sample_distribution!(indices, recipe): fills `indices` (numpy or torch, 0-based)."""
    if not isinstance(recipe, _RecipeBase):
        raise ArgumentError(f"No `sample_distribution!` method defined for a distribution of type "
                            f"{type(recipe).__name__}.")
    out = recipe._sample(len(indices))
    if isinstance(indices, np.ndarray):
        indices[...] = out
    else:
        indices.copy_(__import__("torch").from_numpy(out))


# ----------------------------------------------------------------------------------
# Sampling (src/Compressors/sampling.jl)
# ----------------------------------------------------------------------------------
class Sampling(Compressor):
    """sampling.jl:42-70: fields cardinality, compression_dim, distribution."""

    def __init__(self, cardinality: Cardinality = None, compression_dim: int = 2, distribution: Distribution = None):
        cardinality = Left() if cardinality is None else cardinality
        distribution = Uniform() if distribution is None else distribution
        if compression_dim <= 0:
            raise ArgumentError("Field `compression_dim` must be positive.")
        if isinstance(cardinality, Undef):
            raise ArgumentError("`cardinality` must be specified as `Left()` or `Right()`.`Undef()` is not allowed "
                                "in `Sampling` structure.")
        self.cardinality = cardinality
        self.compression_dim = int(compression_dim)
        self.distribution = distribution


class SamplingRecipe(CompressorRecipe):
    """sampling.jl:72-96: fields cardinality, compression_dim, n_rows, n_cols,
    distribution_recipe, idx, idx_v (idx 0-based, downloaded from the device)."""

    def __init__(self, compressor: Sampling, A, seed: Optional[int], device: Optional[int]):
        card = compressor.cardinality
        dist = compressor.distribution
        dist.cardinality = card  # sampling.jl:119
        if type(dist) not in _DIST:
            raise ArgumentError(f"No `complete_distribution` method defined for a distribution of type "
                                f"{type(dist).__name__} and {type(A).__name__}.")
        if isinstance(dist, Agmon):
            raise ArgumentError(f"No `complete_distribution` method defined for a distribution of type Agmon and "
                                f"{type(A).__name__}.")
        Ad = _device_matrix(A)
        self.cardinality = card
        self.compressor = compressor
        self.compression_dim = compressor.compression_dim
        self._dtype = rla_dtype(Ad.dtype)
        self._ctx = L.Context.get(device)
        long_dim = Ad.shape[0] if isinstance(card, Left) else Ad.shape[1]
        h = ctypes.c_void_p()
        L.check(L.lib().rla_sampling_create(self._ctx.handle, _card_code(card), self._dtype,
                                            compressor.compression_dim, long_dim, _DIST[type(dist)],
                                            int(dist.replace), 1, _next_seed() if seed is None else int(seed),
                                            ctypes.byref(h)), self._ctx.handle)
        self.handle = h
        self._cache = None
        self.distribution_recipe = (UniformRecipe if isinstance(dist, Uniform) else L2NormRecipe)(
            card, dist.replace, Ad, 0 if seed is None else int(seed))
        if isinstance(dist, L2Norm):
            self._update(Ad, None, None)
        self._refresh_info()

    def _update(self, Ad, x, b) -> None:
        ctx = L.Context.get(self._ctx.device)
        L.check(L.lib().rla_sampling_update(ctx.handle, self.handle, Ad.shape[0], Ad.shape[1], Ad.data_ptr(),
                                            _lda(Ad), None, 0, None, 0, None), ctx.handle)
        self._cache = None

    @property
    def idx(self) -> np.ndarray:
        return self.draws()["idx"]

    @property
    def idx_v(self) -> np.ndarray:
        return self.idx

    @property
    def np_dtype(self):
        return np.float32 if self._dtype == 0 else np.float64


def complete_sampling(compressor: Sampling, args, seed=None, device=None) -> SamplingRecipe:
    A = args[1] if len(args) == 3 else args[0]
    return SamplingRecipe(compressor, A, seed, device)


def update_sampling_(S: SamplingRecipe, args) -> None:
    """update_compressor!(S, x, A, b) (sampling.jl:137-141); the shorter forms reach the
    generic update_compressor!(S), which has no method for a SamplingRecipe."""
    if len(args) != 3:
        raise ArgumentError(f"No method `update_compressor` exists for compressor recipe of type "
                            f"{type(S).__name__}.")
    x, A, b = args
    Ad = _device_matrix(A)
    update_distribution_(S.distribution_recipe, x, Ad, b)
    S._update(Ad, x, b)
    S._refresh_info()
