"""Kaczmarz and ColumnProjection on the B200 against the oracle (src/Solvers/kaczmarz.jl,
src/Solvers/col_projection.jl restated in oracle/).

Parity is per iteration: after each device step the draws that step used are downloaded
and replayed by the oracle (float64, LAPACK QR for the LQ / QR sub-solvers).  Also ports
test/Solvers/kaczmarz.jl's constructor warning, field checks and dimension errors, and the
residual-decrease / threshold-stop behaviour of both solvers.
"""
import numpy as np
import pytest

from helpers import oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-9, np.float32: 2e-4}


def _steps(rla, orc, solver, A_d, b_d, x_d, iters, kz):
    from randlinearalgebra_b200 import _lib as L
    ctx = solver._ctx
    lib = L.lib()
    lda = A_d.stride(1)
    rp = None if kz else solver.residual_vec.data_ptr()
    L.check(lib.rla_proj_start(ctx.handle, solver._h, A_d.data_ptr(), lda, b_d.data_ptr(), x_d.data_ptr(), rp),
            ctx.handle)
    draws = []
    for _ in range(iters):
        L.check(lib.rla_proj_step(ctx.handle, solver._h, A_d.data_ptr(), lda, b_d.data_ptr(), x_d.data_ptr(), rp),
                ctx.handle)
        solver.compressor._cache = None
        draws.append(oracle_recipe(orc, solver.compressor))
    return draws


@pytest.mark.parametrize("dtype,s,kind", [(np.float64, 1, "sparse_sign"), (np.float64, 8, "sparse_sign"),
                                          (np.float32, 8, "sparse_sign"), (np.float64, 6, "sampling"),
                                          (np.float64, 1, "sampling"), (np.float64, 12, "gaussian")])
def test_kaczmarz_matches_oracle(rla, orc, dev, dtype, s, kind):
    rng = np.random.default_rng(s + 7)
    m, n = 300, 40
    A = rng.standard_normal((m, n)).astype(dtype)
    b = (A.astype(np.float64) @ rng.standard_normal(n)).astype(dtype)
    x0 = np.zeros(n, dtype)
    comp = {"sparse_sign": lambda: rla.SparseSign(compression_dim=s, nnz=min(4, s), type=dtype),
            "sampling": lambda: rla.Sampling(compression_dim=s, distribution=rla.Uniform(replace=False)),
            "gaussian": lambda: rla.Gaussian(compression_dim=s, type=dtype)}[kind]()
    A_d, b_d, x_d = to_dev(A, dev), to_dev(b, dev), to_dev(x0, dev)
    solver = rla.complete_solver(rla.Kaczmarz(compressor=comp, alpha=0.9, log=rla.BasicLogger(max_it=30)), x_d,
                                 A_d, b_d, seed=5)
    iters = 12
    draws = _steps(rla, orc, solver, A_d, b_d, x_d, iters, True)
    ref = orc.kaczmarz_rsolve(A, b, x0, lambda i: draws[i - 1], alpha=0.9, max_it=iters + 1, threshold=-1.0)
    assert rel_err(x_d.cpu().numpy(), ref.x) < TOL[dtype]


@pytest.mark.parametrize("dtype,s", [(np.float64, 1), (np.float64, 5), (np.float32, 5)])
def test_colproj_matches_oracle(rla, orc, dev, dtype, s):
    rng = np.random.default_rng(s + 3)
    m, n = 200, 30
    A = rng.standard_normal((m, n)).astype(dtype)
    b = (A.astype(np.float64) @ rng.standard_normal(n) + 0.01 * rng.standard_normal(m)).astype(dtype)
    x0 = (0.1 * rng.standard_normal(n)).astype(dtype)
    A_d, b_d, x_d = to_dev(A, dev), to_dev(b, dev), to_dev(x0, dev)
    comp = rla.SparseSign(cardinality=rla.Right(), compression_dim=s, nnz=min(3, s), type=dtype)
    solver = rla.complete_solver(rla.ColumnProjection(compressor=comp, alpha=1.0, log=rla.BasicLogger(max_it=30)),
                                 x_d, A_d, b_d, seed=9)
    iters = 10
    draws = _steps(rla, orc, solver, A_d, b_d, x_d, iters, False)
    ref = orc.colproj_rsolve(A, b, x0, lambda i: draws[i - 1], max_it=iters, threshold=-1.0)
    assert rel_err(x_d.cpu().numpy(), ref.x) < TOL[dtype]
    assert rel_err(solver.residual_vec.cpu().numpy(), ref.residual_vec) < 10 * TOL[dtype]


def test_kaczmarz_rsolve_converges_and_errors(rla, orc, dev):
    """Consistent system: FullResidual threshold stop; CompressedResidual is zero before the
    first step, so a positive threshold stops at once (compressed_residual.jl)."""
    import torch
    rng = np.random.default_rng(1)
    m, n = 400, 25
    A = rng.standard_normal((m, n))
    xs = rng.standard_normal(n)
    b = A @ xs
    A_d, b_d = to_dev(A, dev), to_dev(b, dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    thr = 1e-9 * np.linalg.norm(b)
    solver = rla.complete_solver(rla.Kaczmarz(compressor=rla.SparseSign(compression_dim=10, nnz=4),
                                              log=rla.BasicLogger(max_it=500, threshold=thr)), x, A_d, b_d)
    rla.rsolve_(solver, x, A_d, b_d)
    assert solver.log.converged and solver.log.iteration < 500 and solver.log.error < thr
    assert rel_err(x.cpu().numpy(), xs) < 1e-8
    x2 = torch.zeros(n, dtype=torch.float64, device=dev)
    s2 = rla.complete_solver(rla.Kaczmarz(compressor=rla.SparseSign(compression_dim=10, nnz=4),
                                          error=rla.CompressedResidual(),
                                          log=rla.BasicLogger(max_it=50, threshold=1e-3)), x2, A_d, b_d)
    rla.rsolve_(s2, x2, A_d, b_d)
    assert s2.log.converged and s2.log.iteration == 1 and not x2.any()
    assert s2.compressed_mat.shape == (10, n) and s2.vec_view.shape == (10,)


def test_colproj_rsolve_converges(rla, dev):
    import torch
    rng = np.random.default_rng(2)
    m, n = 300, 20
    A = rng.standard_normal((m, n))
    b = A @ rng.standard_normal(n) + 0.05 * rng.standard_normal(m)
    A_d, b_d = to_dev(A, dev), to_dev(b, dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    xls = np.linalg.lstsq(A, b, rcond=None)[0]
    solver = rla.complete_solver(rla.ColumnProjection(compressor=rla.SparseSign(cardinality=rla.Right(),
                                                                                 compression_dim=5, nnz=3),
                                                      log=rla.BasicLogger(max_it=3000, threshold=1e-8)), x, A_d, b_d)
    rla.rsolve_(solver, x, A_d, b_d)
    assert solver.log.converged and rel_err(x.cpu().numpy(), xls) < 1e-7
    assert np.allclose(solver.residual_vec.cpu().numpy(), b - A @ x.cpu().numpy(), atol=1e-10)
    assert np.allclose(solver.error.gradient.cpu().numpy(), -(A.T @ (b - A @ x.cpu().numpy())), atol=1e-9)


def test_kaczmarz_zero_block_is_skipped(rla, dev):
    """kaczmarz_update! does nothing when the sketched rows are zero."""
    import torch
    A = np.zeros((6, 3))
    A[1] = [1.0, 2.0, 3.0]
    b = np.ones(6)
    A_d, b_d = to_dev(A, dev), to_dev(b, dev)
    x = torch.zeros(3, dtype=torch.float64, device=dev)
    solver = rla.complete_solver(rla.Kaczmarz(compressor=rla.Sampling(compression_dim=1),
                                              log=rla.BasicLogger(max_it=3)), x, A_d, b_d, seed=2)
    solver.compressor.load_draws(idx=np.array([4]))  # a zero row
    from randlinearalgebra_b200 import _lib as L
    ctx = solver._ctx
    L.check(L.lib().rla_proj_start(ctx.handle, solver._h, A_d.data_ptr(), 6, b_d.data_ptr(), x.data_ptr(), None),
            ctx.handle)
    # steps redraw; run until a zero row is drawn and check x is unchanged by it
    for _ in range(6):
        before = x.clone()
        L.check(L.lib().rla_proj_step(ctx.handle, solver._h, A_d.data_ptr(), 6, b_d.data_ptr(), x.data_ptr(), None),
                ctx.handle)
        solver.compressor._cache = None
        if solver.compressor.idx[0] != 1:
            assert torch.equal(x, before)


def test_constructors_and_field_checks(rla, dev):
    import torch
    with pytest.warns(UserWarning, match="Compressor has cardinality `Right` but kaczmarzcompresses  from the  "
                                         "`Left`."):
        rla.Kaczmarz(compressor=rla.SparseSign(cardinality=rla.Right(), compression_dim=3))
    with pytest.warns(UserWarning, match="Compressor has cardinality `Left` but ColumnProjectioncompresses"):
        rla.ColumnProjection(compressor=rla.SparseSign(compression_dim=3))
    k = rla.Kaczmarz()
    assert k.alpha == 1.0 and type(k.sub_solver) is rla.LQSolver and type(k.error) is rla.FullResidual
    c = rla.ColumnProjection()
    assert type(c.sub_solver) is rla.QRSolver and type(c.error) is rla.LSGradient
    rng = np.random.default_rng(0)
    A_d, b_d = to_dev(rng.random((20, 4)), dev), to_dev(rng.random(20), dev)
    x = torch.zeros(4, dtype=torch.float64, device=dev)
    with pytest.raises(rla.ArgumentError, match="does not contain the field 'residual' and is not valid for a "
                                                "kaczmarz solver."):
        rla.complete_solver(rla.Kaczmarz(compressor=rla.SparseSign(compression_dim=3), error=rla.LSGradient()),
                            x, A_d, b_d)
    with pytest.raises(rla.ArgumentError, match="does not contain the field 'gradient' and is not valid for a "
                                                "`ColumnProjection` solver."):
        rla.complete_solver(rla.ColumnProjection(compressor=rla.SparseSign(cardinality=rla.Right(),
                                                                           compression_dim=2),
                                                 error=rla.FullResidual()), x, A_d, b_d)
    s = rla.complete_solver(rla.Kaczmarz(compressor=rla.SparseSign(compression_dim=3),
                                         log=rla.BasicLogger(max_it=2)), x, A_d, b_d)
    with pytest.raises(rla.DimensionMismatch, match=r"^Dimension of `x`, 5 is different from number of columns"):
        rla.rsolve_(s, torch.zeros(5, dtype=torch.float64, device=dev), A_d, b_d)
    with pytest.raises(rla.DimensionMismatch, match=r"^Dimension of `b`, 19 is different from number of rows"):
        rla.rsolve_(s, x, A_d, b_d[:19])
