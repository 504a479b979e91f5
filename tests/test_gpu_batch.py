"""Batched RandSVD (grouped launches captured in a CUDA graph) against the single-instance
path and the FP64 oracle.

Each instance is rapproximate!(RandSVD(Gaussian(Right(), k), power_its, orthogonalize), A)
(randsvd.jl:174-189) on Float32 data.  The batch draws the same Omega as
complete_compressor with the same seed, so its factors agree with the single-instance run
to FP32 accumulation level; against the FP64 oracle run on the same draws the singular
values and the projection error ||A - UU'A|| / ||A|| agree within 1e-4."""
import numpy as np
import pytest

from helpers import oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu


def low_rank(rng, m, n, decay=0.9, noise=1e-6):
    r = min(m, n)
    U = np.linalg.qr(rng.standard_normal((m, r)))[0]
    V = np.linalg.qr(rng.standard_normal((n, r)))[0]
    s = decay ** np.arange(r)
    return ((U * s) @ V.T + noise * rng.standard_normal((m, n))).astype(np.float32)


def make_batch(rng, count, kset=(4, 16, 20, 32, 48, 64, 100)):
    As, ks, seeds = [], [], []
    for i in range(count):
        m = int(rng.integers(300, 5000))
        n = int(rng.integers(110, 420))
        k = int(kset[i % len(kset)])
        As.append(low_rank(rng, m, n))
        ks.append(min(k, n))
        seeds.append(1000 + 7 * i)
    return As, ks, seeds


@pytest.mark.parametrize("q,ortho,kset", [(0, False, (4, 16, 20, 32, 48, 64, 100)),
                                          (1, True, (4, 16, 20, 32, 48, 64, 100)),
                                          (2, True, (16, 32, 64)),
                                          (1, False, (4, 8, 16))])
def test_batch_matches_single_and_oracle(rla, orc, dev, q, ortho, kset):
    """Unorthogonalised power iterations are checked only where cond(Y) ~ (s1/sk)^(2q+1)
    stays within what FP32 storage of Y resolves (the reference's Float32 BLAS path has the
    same limit); beyond it the trailing triplets of any FP32 run are noise."""
    rng = np.random.default_rng(40 + q + (0 if ortho else 10))
    As, ks, seeds = make_batch(rng, 14, kset=kset)
    Ad = [to_dev(A, dev) for A in As]
    B = rla.RandSVDBatch(Ad, ks, seeds, power_its=q, orthogonalize=ortho, autotune=False)
    B.run()
    for i, (A, k, sd) in enumerate(zip(As, ks, seeds)):
        comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
        rec = rla.rapproximate(rla.RandSVD(compressor=comp, power_its=q, orthogonalize=ortho, factor_type=np.float32),
                               Ad[i], seed=sd)
        S_b = B.S[i].cpu().numpy()
        assert rel_err(S_b, rec.S.cpu().numpy()) < 1e-5, (i, k)
        ref = orc.randsvd(A.astype(np.float64), oracle_recipe(orc, rec.compressor), q=q, orthogonalize=ortho)
        assert rel_err(S_b, ref.S) < 1e-4, (i, k)
        U = B.U[i].cpu().numpy().astype(np.float64)
        V = B.V[i].cpu().numpy().astype(np.float64)
        A64 = A.astype(np.float64)
        nA = np.linalg.norm(A64)
        e_b = np.linalg.norm(A64 - U @ (U.T @ A64)) / nA
        e_r = np.linalg.norm(A64 - ref.U @ (ref.U.T @ A64)) / nA
        assert abs(e_b - e_r) < 1e-4, (i, k, e_b, e_r)
        assert np.allclose(U.T @ U, np.eye(k), atol=1e-5) and np.allclose(V.T @ V, np.eye(k), atol=1e-5)
        assert rel_err((U * S_b) @ V.T, (ref.U * ref.S) @ ref.V.T) < 1e-4


def test_batch_graph_replay_and_autotune(rla, dev):
    rng = np.random.default_rng(5)
    As, ks, seeds = make_batch(rng, 10, kset=(16, 32, 64, 128))
    ks = [min(k, A.shape[1], A.shape[0]) for A, k in zip(As, ks)]
    Ad = [to_dev(A, dev) for A in As]
    B = rla.RandSVDBatch(Ad, ks, seeds, autotune=True)
    B.run()
    first = [s.cpu().numpy().copy() for s in B.S]
    B.run()  # graph replay
    for a, s in zip(first, B.S):
        assert np.array_equal(a, s.cpu().numpy())
    for c in range(4):
        bm, br, ch = B.tiles(c)
        assert bm in (64, 128, 256) and br in (64, 128, 256) and ch in (2048, 8192, 32768)


def test_batch_rank_deficient_falls_back(rla, dev):
    """k above rank(A): the grouped Cholesky breaks down and the instance is recomputed by
    the single-instance path (shifted CholeskyQR / Householder)."""
    rng = np.random.default_rng(6)
    U0 = np.linalg.qr(rng.standard_normal((400, 5)))[0]
    V0 = np.linalg.qr(rng.standard_normal((150, 5)))[0]
    A = ((U0 * (2.0 ** -np.arange(5))) @ V0.T).astype(np.float32)
    Ad = to_dev(A, dev)
    B = rla.RandSVDBatch([Ad, to_dev(low_rank(rng, 300, 120), dev)], [12, 8], [3, 4], autotune=False)
    B.run()
    U, S, V = B.U[0].cpu().numpy(), B.S[0].cpu().numpy(), B.V[0].cpu().numpy()
    assert rel_err((U * S) @ V.T, A) < 1e-5


def test_batch_argument_errors(rla, dev):
    A = to_dev(np.zeros((50, 20), np.float32), dev)
    with pytest.raises(rla.ArgumentError):
        rla.RandSVDBatch([A], [30], [1])
    with pytest.raises(rla.ArgumentError):
        rla.RandSVDBatch([to_dev(np.zeros((50, 20)), dev)], [4], [1])


@pytest.mark.parametrize("q,ortho", [(0, False), (1, True)])
def test_batch_tensor_core_passes_vs_oracle(rla, orc, dev, q, ortho):
    """RLA_PREC_SPLIT_BF16: the passes over A (A*Omega, A'Q, and A'Q / A*Z of the power
    iterations) of the instances with k <= 64 run as grouped tcgen05 products of split-BF16
    operands with FP64 accumulation across k-chunks; the rest of the algorithm is unchanged.
    Against the FP64 oracle on the same draws: singular values, the projection error and the
    factor product within 1e-4; the batch graph replays bit for bit."""
    rng = np.random.default_rng(70 + q)
    As, ks, seeds = make_batch(rng, 12, kset=(4, 16, 20, 32, 48, 64, 100))
    As[0] = low_rank(rng, 20000, 700)  # long K for A'Q
    ks[0] = 64
    Ad = [to_dev(A, dev) for A in As]
    B = rla.RandSVDBatch(Ad, ks, seeds, power_its=q, orthogonalize=ortho, autotune=False,
                         precision=rla.RLA_PREC_SPLIT_BF16)
    B.run()
    first = [s.cpu().numpy().copy() for s in B.S]
    B.run()
    for i, (A, k, sd) in enumerate(zip(As, ks, seeds)):
        assert np.array_equal(first[i], B.S[i].cpu().numpy()), i
        comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
        rec = rla.complete_compressor(comp, Ad[i], seed=sd)
        ref = orc.randsvd(A.astype(np.float64), oracle_recipe(orc, rec), q=q, orthogonalize=ortho)
        S_b = B.S[i].cpu().numpy()
        assert rel_err(S_b, ref.S) < 1e-4, (i, k, rel_err(S_b, ref.S))
        U = B.U[i].cpu().numpy().astype(np.float64)
        V = B.V[i].cpu().numpy().astype(np.float64)
        A64 = A.astype(np.float64)
        nA = np.linalg.norm(A64)
        e_b = np.linalg.norm(A64 - U @ (U.T @ A64)) / nA
        e_r = np.linalg.norm(A64 - ref.U @ (ref.U.T @ A64)) / nA
        assert abs(e_b - e_r) < 1e-4, (i, k, e_b, e_r)
        assert rel_err((U * S_b) @ V.T, (ref.U * ref.S) @ ref.V.T) < 1e-4, i
