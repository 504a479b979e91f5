"""Host-side Solver API (no GPU): BasicLogger (port of test/Solvers/Loggers/basic_logger.jl),
the IHS constructor (test/Solvers/ihs.jl:150-210) and the IHS oracle
(src/Solvers/ihs.jl:214-254 restated in oracle/)."""
import math
import warnings

import numpy as np
import pytest


def test_basic_logger_constructor_checks(rla):
    with pytest.raises(rla.ArgumentError, match=r"^Field `max_it` must be positive or 0\.$"):
        rla.BasicLogger(-1, 1, 1e-2)
    with pytest.raises(rla.ArgumentError, match=r"^Field `colection_rate` must be positive\.$"):
        rla.BasicLogger(0, 0, 1e-2)
    with pytest.raises(rla.ArgumentError, match=r"^Field `colection_rate` must be smaller than `max_it`\.$"):
        rla.BasicLogger(1, 2, 1e-2)
    L1 = rla.BasicLogger()
    assert isinstance(L1, rla.Logger)
    assert (L1.max_it, L1.collection_rate, L1.threshold_info) == (0, 1, 0)
    assert L1.stopping_criterion is rla.threshold_stop


def test_basic_logger_complete(rla):
    n_rows = 4
    Lm = rla.complete_logger(rla.BasicLogger(max_it=3 * n_rows))
    assert isinstance(Lm, rla.LoggerRecipe)
    assert Lm.max_it == 3 * n_rows and Lm.hist.shape[0] == 3 * n_rows + 1
    assert Lm.threshold_info == 0 and not Lm.converged and Lm.iteration == 1 and Lm.record_location == 1
    Lm = rla.complete_logger(rla.BasicLogger(max_it=1000, collection_rate=2, threshold=1e-6))
    assert Lm.hist.shape[0] == int(math.ceil(1000 / 2)) + 1 and Lm.threshold_info == 1e-6


def test_basic_logger_update(rla):
    mk = lambda: rla.complete_logger(rla.BasicLogger(collection_rate=2, threshold=1e-5, max_it=12))
    Lm = mk()
    rla.update_logger_(Lm, 1e-2, 1)  # nothing recorded at iteration 1
    assert Lm.hist[0] == 0.0 and Lm.record_location == 1 and Lm.iteration == 1 and not Lm.converged
    rla.update_logger_(Lm, 1e-6, 1)  # threshold met: recorded
    assert Lm.hist[0] == 1e-6 and Lm.record_location == 1 and Lm.converged
    Lm = mk()
    rla.update_logger_(Lm, 1e-2, 2)
    assert Lm.hist[0] == 1e-2 and Lm.record_location == 2 and Lm.iteration == 2 and not Lm.converged
    Lm = mk()
    rla.update_logger_(Lm, 1e-1, 13)  # past max_it: converged
    assert Lm.hist[0] == 1e-1 and Lm.record_location == 1 and Lm.iteration == 13 and Lm.converged


def test_basic_logger_reset_and_threshold_stop(rla):
    Lm = rla.complete_logger(rla.BasicLogger(collection_rate=2, threshold=1e-5, max_it=12))
    Lm.hist[1] = 23.0
    Lm.iteration, Lm.converged, Lm.error = 2, True, 23.0
    rla.reset_logger_(Lm)
    assert Lm.error == 0.0 and Lm.iteration == 1 and Lm.record_location == 1 and not Lm.converged
    assert np.count_nonzero(Lm.hist) == 0
    Lm.error = 1.01e-5
    assert not rla.threshold_stop(Lm)
    Lm.error = 9.99e-6
    assert rla.threshold_stop(Lm)


def test_ihs_constructor(rla):
    s = rla.IHS()
    assert s.alpha == 1.0
    assert type(s.compressor) is rla.SparseSign and type(s.compressor.cardinality) is rla.Left
    assert type(s.log) is rla.BasicLogger and type(s.error) is rla.FullResidual
    s = rla.IHS(alpha=2.0, compressor=rla.CountSketch(compression_dim=5), log=rla.BasicLogger(max_it=5),
                error=rla.LSGradient())
    assert s.alpha == 2.0 and type(s.compressor) is rla.CountSketch
    with pytest.warns(UserWarning, match="Compressor has cardinality `Right` but IHS compresses from the `Left`."):
        rla.IHS(compressor=rla.SparseSign(cardinality=rla.Right(), compression_dim=5))
    with pytest.warns(UserWarning, match="Negative step size could lead to divergent iterates."):
        rla.IHS(alpha=-2.0)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        rla.IHS(alpha=0.0)


def test_ihs_oracle_converges(orc):
    """A consistent system: the oracle's IHS reaches the solution (geometric rate)."""
    rng = np.random.default_rng(12312)
    m, n, s = 400, 20, 160
    A = rng.standard_normal((m, n))
    xs = rng.standard_normal(n)
    b = A @ xs
    sk = [orc.draw_sparse_sign(rng, "left", s, m, 8) for _ in range(40)]
    res = orc.ihs_rsolve(A, b, np.zeros(n), lambda i: sk[i - 1], max_it=40, threshold=1e-9 * np.linalg.norm(b))
    assert res.converged and res.iteration < 40
    assert np.linalg.norm(res.x - xs) < 1e-8 * np.linalg.norm(xs)
    assert all(e2 < e1 for e1, e2 in zip(res.errors, res.errors[1:]))


def test_ihs_oracle_residual_quirk(orc):
    """With alpha != 1 the reference updates the maintained residual by A*u, not alpha*A*u
    (ihs.jl:246-249), so residual_vec drifts from b - Ax; the oracle keeps that."""
    rng = np.random.default_rng(5)
    m, n, s = 300, 10, 60
    A = rng.standard_normal((m, n))
    b = rng.standard_normal(m)
    sk = [orc.draw_sparse_sign(rng, "left", s, m, 8) for _ in range(4)]
    res = orc.ihs_rsolve(A, b, np.zeros(n), lambda i: sk[i - 1], alpha=0.5, max_it=4)
    assert res.iteration == 4
    assert np.linalg.norm(res.residual_vec - (b - A @ res.x)) > 1e-3 * np.linalg.norm(b)
    res1 = orc.ihs_rsolve(A, b, np.zeros(n), lambda i: sk[i - 1], alpha=1.0, max_it=4)
    assert np.linalg.norm(res1.residual_vec - (b - A @ res1.x)) < 1e-10 * np.linalg.norm(b)


def test_ihs_oracle_max_it_zero(orc):
    """BasicLogger's default max_it = 0: rsolve! runs no iteration."""
    rng = np.random.default_rng(1)
    A = rng.standard_normal((50, 4))
    b = rng.standard_normal(50)
    res = orc.ihs_rsolve(A, b, np.ones(4), lambda i: None, max_it=0)
    assert res.iteration == 0 and np.array_equal(res.x, np.ones(4))
    assert np.allclose(res.residual_vec, b - A @ np.ones(4))


# ---- Sampling (src/Compressors/sampling.jl) -------------------------------------------
@pytest.mark.parametrize("card", ["left", "right"])
@pytest.mark.parametrize("replace", [False, True])
def test_oracle_sampling_matches_dense(orc, card, replace):
    """The oracle's gather / in-order scatter-add equals the dense selection matrix
    (P(i, idx(i)) = 1; S = P for Left, P' for Right) in all four orientations."""
    rng = np.random.default_rng(4)
    S = orc.draw_sampling(rng, card, 9, 25, replace=replace)
    D = S.dense()
    nr, nc = S.n_rows, S.n_cols
    A = rng.standard_normal((nc, 3)); C = rng.standard_normal((nr, 3)); C0 = C.copy()
    orc.mul_SA(C, S, A, 2.0, 0.5)
    assert np.allclose(C, 2 * D @ A + 0.5 * C0)
    A = rng.standard_normal((4, nr)); C = rng.standard_normal((4, nc)); C0 = C.copy()
    orc.mul_AS(C, A, S, 2.0, 0.5)
    assert np.allclose(C, 2 * A @ D + 0.5 * C0)
    A = rng.standard_normal((nr, 2)); C = rng.standard_normal((nc, 2)); C0 = C.copy()
    orc.mul_StA(C, S, A, 1.5, 0.0)
    assert np.allclose(C, 1.5 * D.T @ A)
    A = rng.standard_normal((2, nc)); C = rng.standard_normal((2, nr)); C0 = C.copy()
    orc.mul_ASt(C, A, S, 1.5, 0.25)
    assert np.allclose(C, 1.5 * A @ D.T + 0.25 * C0)


def test_oracle_agmon_order(orc):
    """agmon.jl: the k largest residuals, ties by candidate index."""
    A = np.eye(5)
    x = np.array([3.0, 1.0, 3.0, 2.0, 0.0])
    b = np.zeros(5)
    assert orc.agmon_select(A, x, b, "left", np.arange(5), 3).tolist() == [0, 2, 3]
    assert orc.agmon_select(A, x, b, "left", np.array([4, 2, 0]), 2).tolist() == [0, 2]


def test_sampling_constructors(rla):
    s = rla.Sampling()
    assert type(s.cardinality) is rla.Left and s.compression_dim == 2 and type(s.distribution) is rla.Uniform
    with pytest.raises(rla.ArgumentError, match=r"^Field `compression_dim` must be positive\.$"):
        rla.Sampling(compression_dim=-1)
    with pytest.raises(rla.ArgumentError, match="`Undef\\(\\)` is not allowed in `Sampling` structure."):
        rla.Sampling(cardinality=rla.Undef())
    d = rla.Agmon()
    assert type(d.cardinality) is rla.Undef and d.replace is False and d.beta == 1
    with pytest.raises(rla.ArgumentError, match=r"^`Agmon` beta must be >= 1, got beta=0$"):
        rla.Agmon(beta=0)
    assert type(rla.L2Norm().cardinality) is rla.Undef and rla.Uniform(replace=True).replace
