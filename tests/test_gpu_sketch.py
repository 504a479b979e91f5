"""Parity of the B200 compressor kernels with the oracle, on the library's own draws.

Ports the reference's multiplication tests (test/Compressors/sparse_sign.jl:299-459,
count_sketch.jl:207-330, srht.jl:270-527, fjlt.jl:321-560, gaussian.jl:200-280): every
orientation (S*A, A*S, S'*A, A*S'), vectors, 5-argument mul! with alpha = beta = 2 / 1,
padded (non power of two) sizes.  Tolerance: relative Frobenius error against the FP64
oracle on the same draws, 1e-6 for Float32 and 1e-12 for Float64.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu

KINDS = ["sparse_sign", "count_sketch", "srht", "fjlt", "gaussian"]


def make(rla, kind, card, s, L, dtype, seed=3):
    cd = rla.Left() if card == "left" else rla.Right()
    if kind == "sparse_sign":
        comp = rla.SparseSign(cardinality=cd, compression_dim=s, nnz=min(8, s), type=dtype)
    elif kind == "count_sketch":
        comp = rla.CountSketch(cardinality=cd, compression_dim=s, type=dtype)
    elif kind == "srht":
        comp = rla.SRHT(cardinality=cd, compression_dim=s, block_size=3, type=dtype)
    elif kind == "fjlt":
        comp = rla.FJLT(cardinality=cd, compression_dim=s, block_size=3, sparsity=0.3, type=dtype)
    else:
        comp = rla.Gaussian(cardinality=cd, compression_dim=s, type=dtype)
    shape = (L, 1) if card == "left" else (1, L)
    return rla.complete_compressor(comp, np.zeros(shape, dtype=dtype), seed=seed)


def run_orient(rla, orc, S, orient, k, dtype, dev, rng, alpha=2.0, beta=1.0, transpose_a=False):
    nr, nc = S.n_rows, S.n_cols
    R = oracle_recipe(orc, S)
    if orient == "SA":
        A, C = rng.standard_normal((nc, k)), rng.standard_normal((nr, k))
    elif orient == "AS":
        A, C = rng.standard_normal((k, nr)), rng.standard_normal((k, nc))
    elif orient == "StA":
        A, C = rng.standard_normal((nr, k)), rng.standard_normal((nc, k))
    else:
        A, C = rng.standard_normal((k, nc)), rng.standard_normal((k, nr))
    A, C = A.astype(dtype), C.astype(dtype)
    Ad = to_dev(A, dev) if not transpose_a else to_dev(np.ascontiguousarray(A), dev, fortran=False)
    Cd = to_dev(C, dev)
    ref = C.astype(np.float64).copy(order="F")
    A64 = A.astype(np.float64)
    if orient == "SA":
        rla.mul_(Cd, S, Ad, alpha, beta)
        orc.mul_SA(ref, R, A64, alpha, beta)
    elif orient == "AS":
        rla.mul_(Cd, Ad, S, alpha, beta)
        orc.mul_AS(ref, A64, R, alpha, beta)
    elif orient == "StA":
        rla.mul_(Cd, S.T, Ad, alpha, beta)
        orc.mul_StA(ref, R, A64, alpha, beta)
    else:
        rla.mul_(Cd, Ad, S.T, alpha, beta)
        orc.mul_ASt(ref, A64, R, alpha, beta)
    return rel_err(Cd.cpu().numpy(), ref)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("card", ["left", "right"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("orient", ["SA", "AS", "StA", "ASt"])
def test_orientations_small(rla, orc, dev, kind, card, dtype, orient):
    rng = np.random.default_rng(hash((kind, card, orient)) % 2**32)
    for L, s, k in [(10, 3, 6), (64, 17, 5), (1000, 64, 33)]:
        S = make(rla, kind, card, s, L, dtype)
        err = run_orient(rla, orc, S, orient, k, dtype, dev, rng)
        assert err < TOL[dtype], (kind, card, orient, L, s, k, err)


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch", "srht"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_left_compress_fused_path(rla, orc, dev, kind, dtype):
    """Sizes that take the fused / stream-K kernels: padded N >= 2^14, many columns."""
    rng = np.random.default_rng(5)
    for L, s, k in [(20000, 300, 7), (40000, 64, 130), (16384, 4096, 3)]:
        S = make(rla, kind, "left", s, L, dtype, seed=L + s)
        err = run_orient(rla, orc, S, "SA", k, dtype, dev, rng, alpha=1.5, beta=0.0)
        assert err < TOL[dtype], (kind, L, s, k, err)


@pytest.mark.parametrize("s", [24, 40, 96, 128, 256, 2048])
def test_sparse_sign_deferral_regimes(rla, orc, dev, s):
    """nnz = 8 over compression dimensions from ones whose tiles overflow the deferral
    schedule (run-time resolution) through many extra rounds per tile to almost none."""
    rng = np.random.default_rng(s)
    for dtype in (np.float32, np.float64):
        S = make(rla, "sparse_sign", "left", s, 30011, dtype, seed=3 * s)
        err = run_orient(rla, orc, S, "SA", 9, dtype, dev, rng, alpha=1.0, beta=0.0)
        assert err < TOL[dtype], (s, dtype, err)


@pytest.mark.parametrize("dtype,L,s,k", [(np.float64, 70001, 40000, 3), (np.float32, 100003, 60000, 2)])
def test_count_sketch_windowed_bins(rla, orc, dev, dtype, L, s, k):
    """Compression dimensions whose bins exceed one CTA's shared memory (several bin windows)."""
    rng = np.random.default_rng(13)
    S = make(rla, "count_sketch", "left", s, L, dtype, seed=s)
    err = run_orient(rla, orc, S, "SA", k, dtype, dev, rng, alpha=0.5, beta=2.0)
    assert err < TOL[dtype], (L, s, k, err)


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch", "srht", "gaussian"])
def test_row_major_operand(rla, orc, dev, kind):
    """A given as Julia's transpose(X) view (row-major storage)."""
    rng = np.random.default_rng(9)
    S = make(rla, kind, "left", 40, 3000, np.float32)
    err = run_orient(rla, orc, S, "SA", 9, np.float32, dev, rng, transpose_a=True)
    assert err < 1e-6, err


@pytest.mark.parametrize("kind", KINDS)
def test_vectors(rla, orc, dev, kind):
    """S*x, x'*S (test/Compressors/sparse_sign.jl:338-348)."""
    rng = np.random.default_rng(11)
    S = make(rla, kind, "left", 16, 300, np.float64)
    R = oracle_recipe(orc, S)
    x = rng.standard_normal(300)
    y = rng.standard_normal(16)
    yd, xd = to_dev(y, dev), to_dev(x, dev)
    rla.mul_(yd, S, xd, 2.0, 1.0)
    ref = y.copy()
    orc.mul_SA(ref, R, x, 2.0, 1.0)
    assert rel_err(yd.cpu().numpy(), ref) < 1e-12
    z = rng.standard_normal(300)
    zd = to_dev(z, dev)
    w = rng.standard_normal(16)
    rla.mul_(zd, to_dev(w, dev), S, 2.0, 1.0)
    refz = z.copy()
    orc.mul_AS(refz, w, R, 2.0, 1.0)
    assert rel_err(zd.cpu().numpy(), refz) < 1e-12


def test_times_operator_allocates(rla, orc, dev):
    rng = np.random.default_rng(2)
    S = make(rla, "srht", "left", 8, 100, np.float64)
    A = rng.standard_normal((100, 4))
    C = S @ to_dev(A, dev)
    assert tuple(C.shape) == (8, 4)
    ref = np.zeros((8, 4))
    orc.mul_SA(ref, oracle_recipe(orc, S), A)
    assert rel_err(C.cpu().numpy(), ref) < 1e-12
    # host arrays go through the end-to-end path (copy in, compute, copy out)
    Ch = S @ A
    assert isinstance(Ch, np.ndarray) and rel_err(Ch, ref) < 1e-12


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch", "srht"])
def test_deterministic(rla, dev, kind):
    """No atomics: two applies give bitwise-identical results."""
    rng = np.random.default_rng(4)
    S = make(rla, kind, "left", 512, 50000, np.float32)
    Ad = to_dev(rng.standard_normal((50000, 40)).astype(np.float32), dev)
    c1 = (S @ Ad).cpu().numpy()
    c2 = (S @ Ad).cpu().numpy()
    assert np.array_equal(c1, c2)


def test_dimension_errors(rla, dev):
    S = make(rla, "srht", "left", 4, 10, np.float64)
    A = to_dev(np.zeros((9, 3)), dev)
    C = to_dev(np.zeros((4, 3)), dev)
    with pytest.raises(rla.DimensionMismatch, match="Matrix A has 9 rows while S has 10 columns."):
        rla.mul_(C, S, A)
    A = to_dev(np.zeros((10, 3)), dev)
    C = to_dev(np.zeros((4, 2)), dev)
    with pytest.raises(rla.DimensionMismatch, match="Matrix A has 3 columns while C has 2 columns."):
        rla.mul_(C, S, A)
    C = to_dev(np.zeros((5, 3)), dev)
    with pytest.raises(rla.DimensionMismatch, match="Matrix C has 5 rows while S has 4 rows."):
        rla.mul_(C, S, A)
    # adjoint route: right_mul_dimcheck on the transposes (src/Compressors.jl:363-372)
    with pytest.raises(rla.DimensionMismatch, match="Matrix A has 10 columns while S has 4 rows."):
        rla.mul_(to_dev(np.zeros((10, 3)), dev), S.T, to_dev(np.zeros((10, 3)), dev))


def test_size_and_domain(rla):
    pytest.importorskip("torch")
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    S = make(rla, "count_sketch", "right", 7, 20, np.float64)
    assert rla.size(S) == (20, 7) and rla.size(S.T) == (7, 20)
    with pytest.raises(rla.DomainError, match="`dim` must be 1 or 2."):
        rla.size(S, 3)


@pytest.mark.parametrize("kind", KINDS)
def test_update_changes_draws(rla, kind):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    S = make(rla, kind, "left", 16, 256, np.float64)
    before = {k: np.array(v, copy=True) for k, v in S.draws().items()}
    rla.update_compressor_(S)
    after = S.draws()
    changed = any(not np.array_equal(before[k], after[k]) for k in before if before[k].shape == after[k].shape)
    assert changed and S.info.draw_count == 2


def test_draw_properties(rla):
    """Distributional invariants pinned by the reference tests
    (test/Compressors/sparse_sign.jl:153-155, count_sketch.jl:200-202, srht.jl:82-88)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    S = make(rla, "sparse_sign", "left", 50, 2000, np.float32)
    colptr, rowval, nzval = S.op
    assert np.array_equal(colptr, np.arange(0, 2000 * 8 + 1, 8))
    rv = rowval.reshape(2000, 8)
    assert np.all(np.diff(rv, axis=1) > 0) and rv.min() >= 0 and rv.max() < 50
    sc = np.float32(1 / np.sqrt(8))
    assert set(np.unique(nzval)) <= {sc, -sc}
    assert abs(np.mean(nzval > 0) - 0.5) < 0.05
    C = make(rla, "count_sketch", "left", 30, 5000, np.float64)
    _, rv, nz = C.mat
    assert rv.min() >= 0 and rv.max() < 30 and set(np.unique(nz)) <= {1.0, -1.0}
    H = make(rla, "srht", "left", 100, 1000, np.float32)
    assert H.info.padded == 1024 and len(np.unique(H.op)) == 100 and H.op.max() < 1024
    assert H.scale == float(np.float32(np.sqrt(100) / np.sqrt(1024)))


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch", "srht", "fjlt", "gaussian"])
def test_load_draws_parity_mode(rla, orc, dev, kind):
    """Externally supplied draws (oracle-side numpy draws) give the oracle's answer."""
    rng = np.random.default_rng(21)
    L, s = 700, 24
    S = make(rla, kind, "left", s, L, np.float64)
    if kind == "sparse_sign":
        R = orc.draw_sparse_sign(rng, "left", s, L, 8)
        S.load_draws(idx=R.csc.rowval, vals=R.csc.nzval)
    elif kind == "count_sketch":
        R = orc.draw_count_sketch(rng, "left", s, L)
        S.load_draws(idx=R.csc.rowval, vals=R.csc.nzval)
    elif kind == "srht":
        R = orc.draw_srht(rng, "left", s, L, block_size=3)
        S.load_draws(idx=R.op, signs=R.signs)
    elif kind == "fjlt":
        R = orc.draw_fjlt(rng, "left", s, L, sparsity=0.3, block_size=3)
        S.load_draws(idx=R.csc.rowval, vals=R.csc.nzval, signs=R.signs, kptr=R.csc.colptr)
        R.scale = S.scale
    else:
        R = orc.draw_gaussian(rng, "left", s, L)
        S.load_draws(vals=R.dense_op)
    A = rng.standard_normal((L, 5))
    Cd = to_dev(np.zeros((s, 5)), dev)
    rla.mul_(Cd, S, to_dev(A, dev))
    ref = np.zeros((s, 5))
    orc.mul_SA(ref, R, A)
    assert rel_err(Cd.cpu().numpy(), ref) < 1e-12


def test_sparse_sign_left_fp64_4096x256(rla, orc, dev):
    """The plain SparseSign workload exactly: A 4096x256 Float64 ~ N(0,1), compression
    dimension 512, 8 nonzeros per column, Left (test/Compressors/sparse_sign.jl:299-459).

    The draws exported into the oracle recipe satisfy the reference's invariants (8 sorted,
    distinct rows per column; values +-1/sqrt(8) exactly), S*I materialises exactly the
    dense operator built from those draws (every entry is one signed term), and S*A agrees
    with the oracle's CSC loop to 1e-12 relative, alone and in 5-argument form."""
    m, n, s, nnz = 4096, 256, 512, 8
    rng = np.random.default_rng(1)
    S = rla.complete_compressor(rla.SparseSign(cardinality=rla.Left(), compression_dim=s, nnz=nnz, type=np.float64),
                                np.zeros((m, 1)), seed=1)
    colptr, rowval, nzval = S.op
    assert np.array_equal(colptr, np.arange(0, m * nnz + 1, nnz))
    rv = rowval.reshape(m, nnz)
    assert np.all(np.diff(rv, axis=1) > 0) and rv.min() >= 0 and rv.max() < s
    sc = 1 / np.sqrt(np.float64(nnz))
    assert set(np.unique(nzval)) <= {sc, -sc}
    dense = np.zeros((s, m))
    dense[rowval, np.repeat(np.arange(m), nnz)] = nzval
    mat = to_dev(np.zeros((s, m)), dev)
    rla.mul_(mat, S, to_dev(np.eye(m), dev))
    assert np.array_equal(mat.cpu().numpy(), dense)
    R = oracle_recipe(orc, S)
    A = rng.standard_normal((m, n))
    Cd = to_dev(np.zeros((s, n)), dev)
    rla.mul_(Cd, S, to_dev(A, dev))
    ref = np.zeros((s, n))
    orc.mul_SA(ref, R, A)
    assert rel_err(Cd.cpu().numpy(), ref) < 1e-12
    assert rel_err(Cd.cpu().numpy(), dense @ A) < 1e-12
    C0 = rng.standard_normal((s, n))
    Cd = to_dev(C0, dev)
    rla.mul_(Cd, S, to_dev(A, dev), 2.0, 2.0)
    ref = C0.copy(order="F")
    orc.mul_SA(ref, R, A, 2.0, 2.0)
    assert rel_err(Cd.cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("orient", ["SA", "AS", "StA", "ASt"])
@pytest.mark.parametrize("card", ["left", "right"])
def test_gaussian_float32_tensor_core_sizes(rla, orc, dev, card, orient):
    """Float32 Gaussian applies run on the tensor cores: three BF16 terms per operand, six
    MMAs per k-step, FP32 accumulation in tensor memory for four k-blocks at a time and FP64
    accumulation across those chunks.  At long dimension 20000 (long accumulation chains,
    split-K, ragged tiles) every orientation stays within the Float32 tolerance of the FP64
    oracle (gaussian.jl:154,168)."""
    rng = np.random.default_rng(hash((card, orient)) % 2**32)
    S = make(rla, "gaussian", card, 300, 20000, np.float32, seed=5)
    err = run_orient(rla, orc, S, orient, 70, np.float32, dev, rng, alpha=1.5, beta=0.5)
    assert err < TOL[np.float32], (card, orient, err)
