"""The Sampling compressor and its distributions on the B200 (src/Compressors/sampling.jl,
src/Compressors/Distributions/*.jl).

mul! of every orientation is compared with the oracle's restatement of sampling.jl on the
library's own indices (gather for S*A / A*S, in-order scatter-add for the transposed forms);
the draws are checked for what the reference's wsample!(..., ordered = true) promises (sorted,
distinct without replacement, zero-weight indices never drawn, frequencies proportional to
the weights) and Agmon against the oracle's selection when every index is a candidate.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_recipe, rel_err, to_dev
from test_gpu_sketch import run_orient

pytestmark = pytest.mark.gpu


def sampler(rla, dev, card, s, L, dtype, replace=False, dist="uniform", seed=5, k_other=7):
    rng = np.random.default_rng(seed)
    shape = (L, k_other) if card == "left" else (k_other, L)
    A = rng.standard_normal(shape).astype(dtype)
    if dist == "l2":
        A[::3] = 0.0 if card == "left" else A[::3]
    cardo = rla.Left() if card == "left" else rla.Right()
    D = (rla.Uniform if dist == "uniform" else rla.L2Norm)(replace=replace)
    return rla.complete_compressor(rla.Sampling(cardinality=cardo, compression_dim=s, distribution=D),
                                   to_dev(A, dev), seed=seed), A


@pytest.mark.parametrize("card", ["left", "right"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("orient", ["SA", "AS", "StA", "ASt"])
@pytest.mark.parametrize("replace", [False, True])
def test_orientations(rla, orc, dev, card, dtype, orient, replace):
    rng = np.random.default_rng(11)
    for L, s, k in [(10, 3, 6), (64, 17, 5), (1000, 64, 33), (50, 120, 4)]:
        if s > L and not replace:
            continue
        S, _ = sampler(rla, dev, card, s, L, dtype, replace)
        err = run_orient(rla, orc, S, orient, k, dtype, dev, rng, alpha=2.0, beta=0.5)
        assert err < TOL[dtype], (card, orient, L, s, k, err)


def test_row_major_and_vectors(rla, orc, dev):
    rng = np.random.default_rng(3)
    S, _ = sampler(rla, dev, "left", 9, 40, np.float64, replace=True)
    assert run_orient(rla, orc, S, "SA", 6, np.float64, dev, rng, transpose_a=True) < 1e-12
    x = rng.standard_normal(40)
    y = rla.mul_(np.zeros(9), S, x) if False else (S @ to_dev(x, dev)).cpu().numpy()
    assert np.array_equal(y, x[S.idx])


@pytest.mark.parametrize("card", ["left", "right"])
def test_uniform_draws(rla, dev, card):
    for replace in (False, True):
        S, _ = sampler(rla, dev, card, 500, 2000, np.float64, replace)
        idx = S.idx
        assert idx.min() >= 0 and idx.max() < 2000
        d = np.diff(idx)
        assert (d > 0).all() if not replace else (d >= 0).all()
        old = idx.copy()
        rng = np.random.default_rng(0)
        shape = (2000, 7) if card == "left" else (7, 2000)
        A = to_dev(rng.standard_normal(shape), dev)
        rla.update_compressor_(S, np.zeros(shape[1]), A, np.zeros(shape[0]))
        assert S.info.draw_count == 2 and not np.array_equal(S.idx, old)


def test_uniform_without_replacement_takes_all(rla, dev):
    # 300 samples go through the key selection, 200 through Floyd's algorithm (s <= 256)
    for s in (300, 200):
        S, _ = sampler(rla, dev, "left", s, s, np.float32, False)
        assert np.array_equal(S.idx, np.arange(s))


def test_uniform_without_replacement_inclusion_law(rla, dev):
    """Small s (Floyd's algorithm): distinct increasing indices, each index drawn with
    probability s/L (1500 draws of 8 from 32: standard deviation 0.011 around 0.25)."""
    S, A = sampler(rla, dev, "left", 8, 32, np.float64, False, seed=11)
    A_d = to_dev(A, dev)
    x0, b0 = np.zeros(A.shape[1]), np.zeros(A.shape[0])
    counts = np.zeros(32)
    for _ in range(1500):
        rla.update_compressor_(S, x0, A_d, b0)
        idx = np.asarray(S.idx)
        assert len(idx) == 8 and (np.diff(idx) > 0).all() and idx[0] >= 0 and idx[-1] < 32
        counts[idx] += 1
    freq = counts / 1500
    assert np.abs(freq - 0.25).max() < 0.06, freq


def test_l2norm_weights_and_frequencies(rla, dev):
    """Zero rows are never drawn; with replacement the counts follow the squared norms."""
    L, s = 12, 60000
    norms = np.array([0, 1, 2, 3, 0, 1, 4, 2, 0, 1, 1, 5], np.float64)
    A = np.zeros((L, 2))
    A[:, 0] = norms
    S = rla.complete_compressor(rla.Sampling(compression_dim=s, distribution=rla.L2Norm(replace=True)),
                                to_dev(A, dev), seed=2)
    idx = S.idx
    assert (np.diff(idx) >= 0).all()
    cnt = np.bincount(idx, minlength=L)
    w = norms ** 2
    p = w / w.sum()
    assert (cnt[w == 0] == 0).all()
    sd = np.sqrt(s * p * (1 - p))
    assert (np.abs(cnt - s * p) <= 6 * sd + 1).all(), (cnt, s * p)
    # without replacement: all 9 positive-weight rows, in order
    S2 = rla.complete_compressor(rla.Sampling(compression_dim=9, distribution=rla.L2Norm()), to_dev(A, dev), seed=3)
    assert np.array_equal(S2.idx, np.nonzero(w)[0])
    with pytest.raises(rla.ArgumentError):
        rla.complete_compressor(rla.Sampling(compression_dim=10, distribution=rla.L2Norm()), to_dev(A, dev))


def test_l2norm_without_replacement_first_draw_law(rla, dev):
    """Successive sampling: the heaviest of two indices is drawn alone ~ w1 / (w1 + w2)."""
    A = np.array([[1.0], [2.0]])  # weights 1 and 4
    hits = 0
    trials = 400
    for t in range(trials):
        S = rla.complete_compressor(rla.Sampling(compression_dim=1, distribution=rla.L2Norm()), to_dev(A, dev),
                                    seed=100 + t)
        hits += int(S.idx[0] == 1)
    p = 4 / 5
    assert abs(hits / trials - p) < 5 * np.sqrt(p * (1 - p) / trials)


@pytest.mark.parametrize("card", ["left", "right"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_agmon_all_candidates_matches_oracle(rla, orc, dev, card, dtype):
    rng = np.random.default_rng(8)
    m, n, k = 300, 40, 7
    A = rng.standard_normal((m, n)).astype(dtype)
    x = rng.standard_normal(n).astype(dtype)
    b = rng.standard_normal(m).astype(dtype)
    dim = m if card == "left" else n
    cardo = rla.Left() if card == "left" else rla.Right()
    R = rla.complete_distribution(rla.Agmon(cardinality=cardo, beta=dim), to_dev(x, dev), to_dev(A, dev),
                                  to_dev(b, dev), seed=4)
    idx = np.zeros(k, np.int64)
    rla.sample_distribution_(idx, R)
    ref = orc.agmon_select(A, x.astype(np.float64), b.astype(np.float64), card, np.arange(dim), k)
    assert np.array_equal(idx, ref), (idx, ref)


def test_agmon_candidates_and_errors(rla, dev):
    rng = np.random.default_rng(9)
    m, n = 500, 10
    A, x, b = rng.standard_normal((m, n)), rng.standard_normal(n), rng.standard_normal(m)
    Ad, xd, bd = to_dev(A, dev), to_dev(x, dev), to_dev(b, dev)
    R = rla.complete_distribution(rla.Agmon(cardinality=rla.Left(), beta=50), xd, Ad, bd, seed=1)
    idx = np.zeros(5, np.int64)
    rla.sample_distribution_(idx, R)
    res = np.abs(A @ x - b)[idx]
    assert len(set(idx.tolist())) == 5 and (np.diff(res) <= 0).all()
    one = np.zeros(1, np.int64)
    rla.sample_distribution_(one, rla.complete_distribution(rla.Agmon(cardinality=rla.Left()), xd, Ad, bd))
    assert 0 <= one[0] < m
    with pytest.raises(rla.ArgumentError, match=r"^`Agmon` cannot output 6 indices when beta=5\.$"):
        rla.sample_distribution_(np.zeros(6, np.int64),
                                 rla.complete_distribution(rla.Agmon(cardinality=rla.Left(), beta=5), xd, Ad, bd))
    with pytest.raises(rla.ArgumentError, match=r"^`Agmon` beta must be <= number of rows \(500\), got beta=501$"):
        rla.complete_distribution(rla.Agmon(cardinality=rla.Left(), beta=501), xd, Ad, bd)
    with pytest.raises(rla.DimensionMismatch, match=r"^Vector b has length 499, expected 500 to match rows of A$"):
        rla.complete_distribution(rla.Agmon(cardinality=rla.Left(), beta=5), xd, Ad, bd[:499])
    with pytest.raises(rla.ArgumentError, match="`Agmon` cardinality must be specified"):
        rla.complete_distribution(rla.Agmon(beta=5), xd, Ad, bd)
    # the Sampling recipe completes its distribution from A alone, which Agmon does not offer
    with pytest.raises(rla.ArgumentError, match="No `complete_distribution` method defined for a distribution "
                                                "of type Agmon"):
        rla.complete_compressor(rla.Sampling(compression_dim=2, distribution=rla.Agmon()), Ad)


def test_sampling_constructor_and_update_errors(rla, dev):
    with pytest.raises(rla.ArgumentError, match=r"^Field `compression_dim` must be positive\.$"):
        rla.Sampling(compression_dim=0)
    with pytest.raises(rla.ArgumentError, match="`Undef\\(\\)` is not allowed in `Sampling` structure."):
        rla.Sampling(cardinality=rla.Undef())
    with pytest.raises(rla.ArgumentError, match=r"^`Agmon` beta must be >= 1, got beta=0$"):
        rla.Agmon(beta=0)
    S, _ = sampler(rla, dev, "left", 4, 30, np.float64)
    with pytest.raises(rla.ArgumentError, match="No method `update_compressor` exists for compressor recipe of type "
                                                "SamplingRecipe."):
        rla.update_compressor_(S)
    with pytest.raises(rla.ArgumentError, match="`Uniform` cardinality must be specified"):
        rla.complete_distribution(rla.Uniform(), to_dev(np.zeros((3, 2)), dev))
    # fields (sampling.jl:72-96)
    assert (S.n_rows, S.n_cols, S.compression_dim) == (4, 30, 4)
    assert isinstance(S.distribution_recipe, rla.UniformRecipe) and len(S.idx_v) == 4


def test_load_indices_parity_mode(rla, orc, dev):
    """Externally supplied (unsorted, repeated) indices drive the same applies."""
    S, _ = sampler(rla, dev, "right", 6, 20, np.float64)
    S.load_draws(idx=np.array([5, 1, 5, 19, 0, 5]))
    assert np.array_equal(S.idx, [5, 1, 5, 19, 0, 5])
    rng = np.random.default_rng(1)
    for orient in ("SA", "AS", "StA", "ASt"):
        assert run_orient(rla, orc, S, orient, 3, np.float64, dev, rng, alpha=1.5, beta=0.25) < 1e-12
