"""RangeFinder / RandSVD on the B200 against the oracle.

Ports test/Approximators/RangeApproximator/range_finder_helpers.jl:36-134 (Q of the
power iterations equals the Householder Q of the explicit product chain, sign
convention included), randsvd.jl:204-273 (orthogonality, exact recovery when the
compression dimension equals n) and randsvd.jl:495-605 (mul! of the factors), and the
RandSVD example of docs/src/manual/introduction.md:24-40.
"""
import numpy as np
import pytest

from helpers import oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu


def gaussian_right(rla, n, l, dtype=np.float64, seed=1):
    return rla.Gaussian(cardinality=rla.Right(), compression_dim=l, type=dtype), seed


def qr_Q(Y):
    return np.linalg.qr(Y, mode="reduced")[0]


@pytest.mark.parametrize("power_its", [0, 3])
@pytest.mark.parametrize("ortho", [False, True])
def test_power_iterations_match_householder_chain(rla, orc, dev, power_its, ortho):
    rng = np.random.default_rng(31)
    m, n, l = 40, 25, 2
    A = rng.random((m, n))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=l)
    R = rla.complete_approximator(rla.RangeFinder(compressor=comp, power_its=power_its, orthogonalize=ortho),
                                  to_dev(A, dev), seed=4)
    rla.rapproximate_(R, to_dev(A, dev))
    Om = R.compressor.op
    if not ortho:
        Y = A @ Om
        for _ in range(power_its):
            Y = A @ (A.T @ Y)
        Qt = qr_Q(Y)
    else:
        Q1 = qr_Q(A @ Om)
        for _ in range(power_its):
            Q2 = qr_Q(A.T @ Q1)
            Q1 = qr_Q(A @ Q2)
        Qt = Q1
    Q = R.range.cpu().numpy()
    assert rel_err(Q, Qt) < 1e-8
    G = Q.T @ Q
    assert abs(np.linalg.norm(G, 2) - 1) < 1e-10 and np.allclose(np.diag(G), 1, atol=1e-10)


@pytest.mark.parametrize("kind", ["sparse_sign", "srht", "count_sketch"])
def test_rangefinder_oracle_sketches(rla, orc, dev, kind):
    """Default compressor family: sketch applied from the right on the B200."""
    rng = np.random.default_rng(8)
    m, n, l = 300, 90, 12
    A = rng.standard_normal((m, n))
    cd = rla.Right()
    comp = {"sparse_sign": rla.SparseSign(cardinality=cd, compression_dim=l),
            "srht": rla.SRHT(cardinality=cd, compression_dim=l),
            "count_sketch": rla.CountSketch(cardinality=cd, compression_dim=l)}[kind]
    R = rla.rapproximate(rla.RangeFinder(compressor=comp, power_its=1, orthogonalize=True), to_dev(A, dev), seed=5)
    Qref = orc.rangefinder(A, oracle_recipe(orc, R.compressor), q=1, orthogonalize=True)
    assert rel_err(R.range.cpu().numpy(), Qref) < 1e-10


def test_randsvd_exact_recovery(rla, dev):
    """randsvd.jl:242-273: compression_dim == n spans the range exactly."""
    rng = np.random.default_rng(2)
    A = rng.random((10, 10))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=10)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp, power_its=2), to_dev(A, dev), seed=6)
    U, V = rec.U.cpu().numpy(), rec.V.cpu().numpy()
    G = U.T @ U
    assert np.allclose(np.diag(G), 1, atol=1e-10) and abs(np.linalg.norm(G, 2) - 1) < 1e-10
    assert np.linalg.norm(A - U @ (U.T @ A)) < 1e-10
    assert np.linalg.norm(A - A @ V @ V.T) < 1e-10
    assert rec.U.dtype.is_floating_point and str(rec.S.dtype) == "torch.float64"


@pytest.mark.parametrize("ortho", [False, True])
def test_randsvd_matches_oracle(rla, orc, dev, ortho):
    rng = np.random.default_rng(12)
    m, n, k = 400, 150, 20
    Uo = qr_Q(rng.standard_normal((m, n)))
    Vo = qr_Q(rng.standard_normal((n, n)))
    sig = np.arange(1, n + 1, dtype=float) ** -1.5
    A = (Uo * sig) @ Vo.T
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp, power_its=2, orthogonalize=ortho), to_dev(A, dev), seed=9)
    ref = orc.randsvd(A, oracle_recipe(orc, rec.compressor), q=2, orthogonalize=ortho)
    S = rec.S.cpu().numpy()
    # Without orthogonalisation Y = (AA')^2 A Omega has cond(Y) ~ (s1/s20)^5 ~ 5e9 here, which
    # amplifies rounding in both the Householder oracle and CholeskyQR2 alike.
    tol = 1e-12 if ortho else 1e-8
    assert rel_err(S, ref.S) < tol
    U, V = rec.U.cpu().numpy(), rec.V.cpu().numpy()
    sgn = np.sign(np.sum(U * ref.U, axis=0))
    assert rel_err(U * sgn, ref.U) < 1e3 * tol and rel_err(V * sgn, ref.V) < 1e3 * tol


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rank_deficient_sketch(rla, dev, dtype):
    """Compression dimension above rank(A): CholeskyQR breaks down and the Householder path
    takes over; the factorization is still exact and orthonormal."""
    rng = np.random.default_rng(22)
    U0 = qr_Q(rng.standard_normal((300, 8)))
    V0 = qr_Q(rng.standard_normal((120, 8)))
    M = ((U0 * (2.0 ** -np.arange(8))) @ V0.T).astype(dtype)
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=10, type=dtype)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp), to_dev(M, dev), seed=23)
    U, S, V = rec.U.cpu().numpy(), rec.S.cpu().numpy(), rec.V.cpu().numpy()
    tol = 1e-10 if dtype == np.float64 else 1e-5
    assert rel_err((U * S) @ V.T, M) < tol
    assert np.allclose(U.T @ U, np.eye(10), atol=tol) and np.allclose(V.T @ V, np.eye(10), atol=tol)


def test_randsvd_float32_vs_fp64_oracle(rla, orc, dev):
    """Float32 input, factors in Float64: within 1e-4 of the FP64 oracle on the same draws."""
    rng = np.random.default_rng(13)
    m, n, k = 2000, 500, 40
    Uo = qr_Q(rng.standard_normal((m, 200)))
    Vo = qr_Q(rng.standard_normal((n, 200)))
    sig = np.arange(1, 201, dtype=float) ** -1.5
    A = ((Uo * sig) @ Vo.T + 1e-6 * rng.standard_normal((m, n))).astype(np.float32)
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp, power_its=2, orthogonalize=True), to_dev(A, dev), seed=10)
    ref = orc.randsvd(A.astype(np.float64), oracle_recipe(orc, rec.compressor), q=2, orthogonalize=True)
    assert rel_err(rec.S.cpu().numpy(), ref.S) < 1e-4
    U = rec.U.cpu().numpy()
    A64 = A.astype(np.float64)
    e_gpu = np.linalg.norm(A64 - U @ (U.T @ A64)) / np.linalg.norm(A64)
    e_ref = np.linalg.norm(A64 - ref.U @ (ref.U.T @ A64)) / np.linalg.norm(A64)
    assert abs(e_gpu - e_ref) < 1e-4


@pytest.mark.parametrize("side", ["left", "right"])
@pytest.mark.parametrize("adj", [False, True])
def test_randsvd_mul(rla, orc, dev, side, adj):
    """randsvd.jl:495-605: mul! with the factors equals U*(S.*V') products."""
    rng = np.random.default_rng(14)
    A = rng.standard_normal((60, 30))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=6)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp, block_size=3), to_dev(A, dev), seed=15)
    U, S, V = rec.U.cpu().numpy(), rec.S.cpu().numpy(), rec.V.cpu().numpy()
    Rm = (U * S) @ V.T
    op = Rm.T if adj else Rm
    Rx = rec.T if adj else rec
    if side == "left":
        X = rng.standard_normal((op.shape[1], 7))
        C = rng.standard_normal((op.shape[0], 7))
        Cd = to_dev(C, dev)
        rla.mul_(Cd, Rx, to_dev(X, dev), 2.0, 1.5)
        ref = 2.0 * op @ X + 1.5 * C
    else:
        X = rng.standard_normal((7, op.shape[0]))
        C = rng.standard_normal((7, op.shape[1]))
        Cd = to_dev(C, dev)
        rla.mul_(Cd, to_dev(X, dev), Rx, 2.0, 1.5)
        ref = 2.0 * X @ op + 1.5 * C
    assert rel_err(Cd.cpu().numpy(), ref) < 1e-12


def test_rangefinder_mul(rla, dev):
    rng = np.random.default_rng(16)
    A = rng.standard_normal((50, 20))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=5)
    R = rla.rapproximate(rla.RangeFinder(compressor=comp), to_dev(A, dev), seed=17)
    Q = R.range.cpu().numpy()
    X = rng.standard_normal((5, 4))
    C = R @ to_dev(X, dev)
    assert rel_err(C.cpu().numpy(), Q @ X) < 1e-12
    Y = rng.standard_normal((50, 3))
    C2 = R.T @ to_dev(Y, dev)
    assert rel_err(C2.cpu().numpy(), Q.T @ Y) < 1e-12


def test_doc_example_rank20(rla, dev):
    """docs/src/manual/introduction.md:24-40: 3000x3000 rank-20 Float64 matrix, Gaussian
    compression_dim 22; the published distance to the truncated SVD is 6.9e-11."""
    rng = np.random.default_rng(20)
    n = 3000
    A = rng.standard_normal((n, 20)) @ rng.standard_normal((20, n))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=22)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp), to_dev(A, dev), seed=21)
    U, S, V = rec.U.cpu().numpy(), rec.S.cpu().numpy(), rec.V.cpu().numpy()
    Ut, St, Vt = np.linalg.svd(A, full_matrices=False)
    trunc = (Ut[:, :22] * St[:22]) @ Vt[:22]
    err = np.linalg.norm((U * S) @ V.T - trunc)
    assert err < 1e-9, err


def _low_rank_plus_noise(rng, m, n, r, noise=1e-6):
    Uo = qr_Q(rng.standard_normal((m, r)))
    Vo = qr_Q(rng.standard_normal((n, r)))
    sig = np.arange(1, r + 1, dtype=float) ** -1.5
    return ((Uo * sig) @ Vo.T + noise * rng.standard_normal((m, n))).astype(np.float32)


@pytest.mark.parametrize("m,n,k,q", [(2000, 500, 40, 2), (8192, 2048, 272, 2), (3001, 777, 33, 1)])
def test_randsvd_split_bf16_vs_fp64_oracle(rla, orc, dev, m, n, k, q):
    """RLA_PREC_SPLIT_BF16 (products with A on the tensor cores as hi*hi + hi*lo + lo*hi BF16
    with FP32 accumulation; Gram, Cholesky, triangular inverse and the SVD of B in FP64):
    singular values and the projection error ||A - UU'A|| / ||A|| within 1e-4 of the FP64
    oracle run of the same algorithm on the same Gaussian draws."""
    rng = np.random.default_rng(m + k)
    A = _low_rank_plus_noise(rng, m, n, min(n, 512))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp, power_its=q, orthogonalize=True,
                                       precision=rla.RLA_PREC_SPLIT_BF16), to_dev(A, dev), seed=10)
    A64 = A.astype(np.float64)
    ref = orc.randsvd(A64, oracle_recipe(orc, rec.compressor), q=q, orthogonalize=True)
    assert rel_err(rec.S.cpu().numpy(), ref.S) < 1e-4
    U = rec.U.cpu().numpy().astype(np.float64)
    nA = np.linalg.norm(A64)
    e_gpu = np.linalg.norm(A64 - U @ (U.T @ A64)) / nA
    e_ref = np.linalg.norm(A64 - ref.U @ (ref.U.T @ A64)) / nA
    assert abs(e_gpu - e_ref) < 1e-4, (e_gpu, e_ref)
    assert np.allclose(U.T @ U, np.eye(k), atol=1e-5)


@pytest.mark.parametrize("q,ortho", [(1, True), (0, False)])
def test_rangefinder_split_bf16(rla, orc, dev, q, ortho):
    """Power iterations without re-orthogonalisation are left out: Y = (AA')^q A Omega has
    cond(Y) ~ (s1/sk)^(2q+1) (1.6e6 for q = 1 here), which turns the 2^-16 product error
    into subspace error above 1e-4 -- the reason the split path is run orthogonalised."""
    rng = np.random.default_rng(77)
    m, n, k = 1500, 640, 24
    A = _low_rank_plus_noise(rng, m, n, 300)
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
    R = rla.rapproximate(rla.RangeFinder(compressor=comp, power_its=q, orthogonalize=ortho,
                                         precision=rla.RLA_PREC_SPLIT_BF16), to_dev(A, dev), seed=3)
    A64 = A.astype(np.float64)
    Qref = orc.rangefinder(A64, oracle_recipe(orc, R.compressor), q=q, orthogonalize=ortho)
    Q = R.range.cpu().numpy().astype(np.float64)
    nA = np.linalg.norm(A64)
    e_gpu = np.linalg.norm(A64 - Q @ (Q.T @ A64)) / nA
    e_ref = np.linalg.norm(A64 - Qref @ (Qref.T @ A64)) / nA
    assert abs(e_gpu - e_ref) < 1e-4, (e_gpu, e_ref)


def test_split_bf16_rejects_float64(rla, dev):
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=4)
    A = np.random.default_rng(1).standard_normal((20, 10))
    with pytest.raises(rla.ArgumentError, match="Split-BF16 products take Float32 data."):
        rla.rapproximate(rla.RandSVD(compressor=comp, precision=rla.RLA_PREC_SPLIT_BF16), to_dev(A, dev), seed=1)


def test_randsvd_split_bf16_full_size_vs_oracle(rla, orc, dev):
    """The mixed-precision RandSVD workload at its full size: A 65536x8192 Float32 =
    U diag(i^-1.5) V' (rank 512, U and V orthonormal) + 1e-6 N(0,1), k = 256, p = 16 (l = 272),
    q = 2, orthogonalized, split-BF16 products (randsvd.jl:174-189, power_its.jl:53-80).

    The oracle runs the same algorithm in numpy FP64 on the host with the library's Gaussian
    draws.  Singular values and the projection error ||A - UU'A|| / ||A|| of the library's
    factors agree with the oracle's within 1e-4; both projection errors are evaluated by
    the same FP64 products."""
    import torch
    m, n, k, p, q, r = 65536, 8192, 256, 16, 2, 512
    l = k + p
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    Uo = torch.linalg.qr(torch.randn(m, r, device=dev, generator=g))[0]
    Vo = torch.linalg.qr(torch.randn(n, r, device=dev, generator=g))[0]
    sig = torch.arange(1, r + 1, device=dev, dtype=torch.float32) ** -1.5
    At = (Vo * sig) @ Uo.t()
    At.add_(torch.randn(n, m, device=dev, generator=g), alpha=1e-6)
    del Uo, Vo
    A = At.t()  # column-major m x n
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=l, type=np.float32)
    rec = rla.rapproximate(rla.RandSVD(compressor=comp, power_its=q, orthogonalize=True,
                                       precision=rla.RLA_PREC_SPLIT_BF16), A, seed=3000)
    U = rec.U.double()
    S = rec.S.cpu().numpy().astype(np.float64)
    A64h = np.asfortranarray(At.t().double().cpu().numpy())
    ref = orc.randsvd(A64h, oracle_recipe(orc, rec.compressor), q=q, orthogonalize=True)
    assert rel_err(S, ref.S) < 1e-4, rel_err(S, ref.S)
    del A64h
    A64 = A.double()
    nA = torch.linalg.norm(A64)

    def proj_err(Q):
        return float(torch.linalg.norm(A64 - Q @ (Q.t() @ A64)) / nA)

    e_gpu = proj_err(U)
    e_ref = proj_err(torch.from_numpy(np.ascontiguousarray(ref.U)).to(dev))
    assert abs(e_gpu - e_ref) < 1e-4, (e_gpu, e_ref)
    I = torch.eye(l, device=dev, dtype=torch.float64)
    assert float(torch.max(torch.abs(U.t() @ U - I))) < 1e-5


@pytest.mark.parametrize("l", [1, 16, 17, 100, 272, 383, 384, 385, 520])
def test_cholesky_qr_orders(rla, dev, l):
    """The orthogonalisation at orders around the blocked Cholesky/inverse kernels' limits
    (blocks of 16, l <= 384) and past them (the panel kernels): Q of a rangefinder without power
    iterations equals the Householder Q of A*Omega, sign convention included, and is
    orthonormal."""
    rng = np.random.default_rng(100 + l)
    m, n = 2 * l + 64, l + 40
    A = rng.standard_normal((m, n))
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=l)
    R = rla.complete_approximator(rla.RangeFinder(compressor=comp, power_its=0, orthogonalize=True),
                                  to_dev(A, dev), seed=7)
    rla.rapproximate_(R, to_dev(A, dev))
    Q = R.range.cpu().numpy()
    Qt = qr_Q(A @ R.compressor.op)
    assert rel_err(Q, Qt) < 1e-9, l
    assert np.abs(Q.T @ Q - np.eye(l)).max() < 1e-12, l
