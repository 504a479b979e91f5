"""IHS on the B200 against the oracle (src/Solvers/ihs.jl:214-254 restated in oracle/).

Parity is checked iteration by iteration: after each device step the compressor's draws
(update_compressor! in that step) are downloaded and handed to the oracle, which replays
rsolve! in float64 with Householder QR.  Also ports test/Solvers/ihs.jl:215-470
(complete_solver's ArgumentErrors, the residual decreasing under max_it and threshold stops).
"""
import ctypes

import numpy as np
import pytest

from helpers import oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu

# relative tolerances against the float64 oracle on the same draws
TOL = {np.float64: 1e-9, np.float32: 2e-4}


def _steps(rla, orc, solver, A_d, b_d, x_d, iters):
    """start + `iters` steps through the C ABI; returns per-iteration (full residual,
    gradient norm) and the oracle recipes of the draws each step used."""
    from randlinearalgebra_b200 import _lib as L
    ctx = L.Context.get(0)
    lib = L.lib()
    args = (ctx.handle, solver._h, A_d.data_ptr(), A_d.stride(1), b_d.data_ptr())
    vecs = (x_d.data_ptr(), solver.residual_vec.data_ptr(), solver.gradient_vec.data_ptr())
    L.check(lib.rla_ihs_start(*args, *vecs), ctx.handle)
    errs, draws = [solver._errors()], []
    for _ in range(iters):
        L.check(lib.rla_ihs_step(*args, *vecs), ctx.handle)
        solver.compressor._cache = None
        draws.append(oracle_recipe(orc, solver.compressor))
        errs.append(solver._errors())
    return errs, draws


@pytest.mark.parametrize("dtype,m,n,s,alpha,kind", [
    (np.float64, 3000, 48, 192, 1.0, "sparse_sign"),    # fused pass (n <= 256 in FP64)
    (np.float64, 4000, 300, 1200, 1.0, "sparse_sign"),  # any-n kernels
    (np.float64, 2500, 40, 160, 0.6, "sparse_sign"),    # alpha != 1: residual_vec quirk
    (np.float32, 5000, 100, 400, 1.0, "sparse_sign"),   # fused pass (n <= 512 in FP32)
    (np.float32, 6000, 600, 2400, 1.0, "sparse_sign"),  # any-n kernels
    (np.float64, 3000, 30, 240, 1.0, "count_sketch"),
    (np.float64, 2000, 30, 120, 1.0, "gaussian"),
    (np.float32, 4096, 64, 512, 1.0, "srht"),
])
def test_ihs_matches_oracle(rla, orc, dev, dtype, m, n, s, alpha, kind):
    import torch
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((m, n)).astype(dtype)
    b = (A.astype(np.float64) @ rng.standard_normal(n) + 0.1 * rng.standard_normal(m)).astype(dtype)
    x0 = (0.1 * rng.standard_normal(n)).astype(dtype)
    comp = {"sparse_sign": lambda: rla.SparseSign(compression_dim=s, type=dtype),
            "count_sketch": lambda: rla.CountSketch(compression_dim=s, type=dtype),
            "gaussian": lambda: rla.Gaussian(compression_dim=s, type=dtype),
            "srht": lambda: rla.SRHT(compression_dim=s, type=dtype)}[kind]()
    A_d, b_d, x_d = to_dev(A, dev), to_dev(b, dev), to_dev(x0, dev)
    solver = rla.complete_solver(rla.IHS(compressor=comp, alpha=alpha, log=rla.BasicLogger(max_it=10)), x_d, A_d,
                                 b_d, seed=77)
    iters = 5
    errs, draws = _steps(rla, orc, solver, A_d, b_d, x_d, iters)
    ref = orc.ihs_rsolve(A, b, x0, lambda i: draws[i - 1], alpha=alpha, max_it=iters + 1, threshold=-1.0)
    tol = TOL[dtype]
    assert rel_err(x_d.cpu().numpy(), ref.x) < tol
    assert rel_err(solver.residual_vec.cpu().numpy(), ref.residual_vec) < tol
    assert rel_err(solver.gradient_vec.cpu().numpy(), ref.gradient_vec) < 50 * tol
    assert np.allclose([e[0] for e in errs], ref.errors, rtol=tol, atol=0)
    if alpha != 1.0:
        # the maintained residual is not b - Ax (ihs.jl:246-249)
        true_r = b.astype(np.float64) - A.astype(np.float64) @ x_d.cpu().numpy()
        assert rel_err(solver.residual_vec.cpu().numpy(), true_r) > 1e-3


def test_ihs_rsolve_threshold_stop(rla, dev):
    """test/Solvers/ihs.jl 'using threshold stop': a 1 % improvement is reached before
    max_it and the residual decreases; a consistent system converges to its solution."""
    import torch
    rng = np.random.default_rng(12312)
    m, n = 2000, 20
    A = np.linalg.qr(rng.random((m, n)))[0]
    xsol = np.ones(n)
    b = A @ xsol
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    A_d, b_d = to_dev(A, dev), to_dev(b, dev)
    log = rla.BasicLogger(max_it=40, threshold=np.linalg.norm(b) * 0.99)
    solver = rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=9 * n), log=log), x, A_d, b_d)
    rla.rsolve_(solver, x, A_d, b_d)
    assert solver.log.converged and solver.log.iteration < 40
    assert np.linalg.norm(A @ x.cpu().numpy() - b) < np.linalg.norm(b)
    x2 = torch.zeros(n, dtype=torch.float64, device=dev)
    log = rla.BasicLogger(max_it=60, threshold=1e-10 * np.linalg.norm(b))
    solver = rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=9 * n), log=log), x2, A_d, b_d)
    rla.rsolve_(solver, x2, A_d, b_d)
    assert solver.log.converged and solver.log.error < 1e-10 * np.linalg.norm(b)
    assert rel_err(x2.cpu().numpy(), xsol) < 1e-9
    # the error field holds b - Ax at the end (full_residual.jl)
    assert np.allclose(solver.error.residual.cpu().numpy(), b - A @ x2.cpu().numpy(), atol=1e-12)


def test_ihs_rsolve_max_it_float32_host_inputs(rla, dev):
    """test/Solvers/ihs.jl 'test maxit stop' with Float32 host arrays (copied in and out);
    the default Float64 SparseSign is completed in A's element type."""
    rng = np.random.default_rng(3)
    m, n = 1500, 12
    A = np.asfortranarray(np.linalg.qr(rng.random((m, n)))[0].astype(np.float32))
    b = (A @ np.ones(n, np.float32)).astype(np.float32)
    x = np.zeros(n, np.float32)
    solver = rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=9 * n),
                                         log=rla.BasicLogger(max_it=10)), x, A, b)
    rla.rsolve_(solver, x, A, b)
    assert solver.log.iteration == 10 and solver.log.converged
    assert np.linalg.norm(A @ x - b) < np.linalg.norm(b)
    assert solver.compressed_mat.shape == (9 * n, n) and solver.R.shape == (n, n)
    # R'R = (SA)'(SA) for the last step's compressed matrix
    SA = solver.compressed_mat.double().cpu().numpy()
    R = solver.R.cpu().numpy()
    assert rel_err(R.T @ R, SA.T @ SA) < 1e-6


def test_ihs_c_loop_matches_python_loop(rla, dev):
    """rla_ihs_solve (the BasicLogger loop in C) and rsolve_ give the same iterates."""
    import torch
    from randlinearalgebra_b200 import _lib as L
    rng = np.random.default_rng(9)
    m, n = 3000, 40
    A_d = to_dev(rng.standard_normal((m, n)), dev)
    b_d = to_dev(rng.standard_normal(m), dev)
    mk = lambda x: rla.complete_solver(
        rla.IHS(compressor=rla.SparseSign(compression_dim=4 * n), log=rla.BasicLogger(max_it=8, collection_rate=2,
                                                                                      threshold=1e-3)),
        x, A_d, b_d, seed=123)
    x1 = torch.zeros(n, dtype=torch.float64, device=dev)
    s1 = mk(x1)
    rla.rsolve_(s1, x1, A_d, b_d)
    x2 = torch.zeros(n, dtype=torch.float64, device=dev)
    s2 = mk(x2)
    ctx = L.Context.get(0)
    hist = np.zeros(5)
    it, conv = ctypes.c_int64(), ctypes.c_int()
    L.check(L.lib().rla_ihs_solve(ctx.handle, s2._h, A_d.data_ptr(), A_d.stride(1), b_d.data_ptr(), x2.data_ptr(),
                                  s2.residual_vec.data_ptr(), s2.gradient_vec.data_ptr(), 8, 2, 1e-3, 0,
                                  hist.ctypes.data, 5, ctypes.byref(it), ctypes.byref(conv)), ctx.handle)
    assert torch.equal(x1, x2)
    assert it.value == s1.log.iteration and bool(conv.value) == s1.log.converged
    assert np.array_equal(hist, s1.log.hist)


def test_ihs_complete_solver_errors(rla, dev):
    """test/Solvers/ihs.jl:215-330: the checks of complete_solver, same wording."""
    import torch
    rng = np.random.default_rng(2)
    A_d = to_dev(rng.random((20, 2)), dev)
    b_d = to_dev(rng.random(20), dev)
    x = torch.zeros(2, dtype=torch.float64, device=dev)
    with pytest.raises(rla.ArgumentError, match=r"^ErrorRecipe LSGradientRecipe does not contain the field "
                                                r"'residual' and is not valid for an IHS solver\.$"):
        rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=4), error=rla.LSGradient()), x, A_d, b_d)

    class NoConvLog(rla.Logger):
        def complete_logger(self):
            return rla.LoggerRecipe()

    with pytest.raises(rla.ArgumentError, match=r"^LoggerRecipe LoggerRecipe does not contain the field "
                                                r"'converged' and is not valid for an IHS solver\.$"):
        rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=4), log=NoConvLog()), x, A_d, b_d)
    with pytest.raises(rla.ArgumentError, match=r"^Compression dimension not larger than column dimension this "
                                                r"will lead to singular QR decompositions, which cannot be "
                                                r"inverted\.$"):
        rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=1)), x, A_d, b_d)
    with pytest.raises(rla.ArgumentError, match=r"^Compression dimension larger row dimension\.$"):
        rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=21)), x, A_d, b_d)
    A10 = torch.zeros(10, 10, dtype=torch.float64, device=dev)
    with pytest.raises(rla.ArgumentError, match=r"^Matrix must have more rows than columns\.$"):
        rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=10)),
                            torch.zeros(10, dtype=torch.float64, device=dev), A10, b_d[:10])
    s = rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=16)), x, A_d, b_d)
    assert s.compressed_mat.shape == (16, 2) and s.residual_vec.shape == (20,) and s.gradient_vec.shape == (2,)
    assert s.buffer_vec.shape == (2,) and s.solution_vec is x and s.alpha == 1.0
