"""Pins the CPU oracle to the reference's own known-answer tests (CPU only).

The reference has no stored vectors; its tests compare against explicit formulas
(Hadamard.jl's natural-order hadamard(n), dense re-materialised operators).  These
tests port those assertions onto the oracle and check it against the fixtures in
tests/golden/ (made by tests/golden/make_golden.py from the same formulas).
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


# ---- fwht!  (test/Compressors/helpers/fwht.jl:8-72) ---------------------------------
def test_fwht_errors(orc):
    with pytest.raises(orc.DimensionMismatch, match="same length"):
        orc.fwht_(np.random.rand(4), np.ones(5, np.uint8))
    with pytest.raises(orc.DimensionMismatch, match="power of 2"):
        orc.fwht_(np.random.rand(3), np.ones(3, np.uint8))
    with pytest.raises(orc.DimensionMismatch, match="power of 2"):
        orc.fwht_(np.random.rand(3))


@pytest.mark.parametrize("ln", [8, 16])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fwht_hadamard_and_inverse(orc, ln, dtype):
    rng = np.random.default_rng(ln)
    H = orc.hadamard(ln)
    x = rng.random(ln).astype(dtype)
    y = x.copy()
    orc.fwht_(y)
    assert np.allclose(y, H @ x, rtol=np.sqrt(np.finfo(dtype).eps))
    orc.fwht_(y, scaling=dtype(1 / ln))
    assert np.allclose(y, x, rtol=np.sqrt(np.finfo(dtype).eps))
    signs = rng.integers(0, 2, ln).astype(np.uint8)
    z = x.copy()
    orc.fwht_(z, signs)
    assert np.allclose(z, H @ (np.where(signs, 1, -1) * x), rtol=np.sqrt(np.finfo(dtype).eps))
    ones = np.ones(ln, np.uint8)
    w = x.copy()
    orc.fwht_(w, ones)
    orc.fwht_(w, ones, scaling=dtype(1 / ln))
    assert np.allclose(w, x, rtol=np.sqrt(np.finfo(dtype).eps))


def test_fwht_golden(orc):
    g = np.load(os.path.join(GOLD, "fwht.npz"))
    for ln in (8, 16):
        x, sg = g[f"fwht_{ln}_x"], g[f"fwht_{ln}_signs"]
        y = x.copy(); orc.fwht_(y)
        assert np.allclose(y, g[f"fwht_{ln}_plain"], rtol=1e-14, atol=1e-14)
        y = x.copy(); orc.fwht_(y, sg)
        assert np.allclose(y, g[f"fwht_{ln}_signed"], rtol=1e-14, atol=1e-14)
        y = x.copy(); orc.fwht_(y, sg, scaling=1 / ln)
        assert np.allclose(y, g[f"fwht_{ln}_signed_scaled"], rtol=1e-14, atol=1e-14)


# ---- SRHT  (test/Compressors/srht.jl:65-169, :270-527) ------------------------------
def test_srht_constructor_pins(orc):
    rng = np.random.default_rng(0)
    for L, N in [(8, 8), (6, 8), (10, 16), (1, 1), (2**14 + 1, 2**15)]:
        R = orc.draw_srht(rng, "left", 1, L, dtype=np.float32)
        assert R.padded == N
        assert R.scale == float(np.float32(np.sqrt(1) / np.sqrt(N)))
    assert orc.padded_size(2**29) == 2**29


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "srht_*.npz"))))
def test_srht_golden(orc, path):
    g = np.load(path)
    card = "left" if "_left_" in path else "right"
    L = int(path.rsplit("_", 1)[1].split(".")[0])
    s = len(g["op"])
    R = orc.Recipe("srht", card, s if card == "left" else L, L if card == "left" else s, np.float64,
                   op=g["op"], signs=g["signs"], scale=float(g["scale"]), padded=int(g["N"]), block_size=2)
    C = g["SA_C"].copy(order="F")
    orc.mul_SA(C, R, g["SA_A"], 2.0, 1.0)
    assert np.allclose(C, g["SA_out"], rtol=1e-12, atol=1e-12)
    C = g["AS_C"].copy(order="F")
    orc.mul_AS(C, g["AS_A"], R, 2.0, 1.0)
    assert np.allclose(C, g["AS_out"], rtol=1e-12, atol=1e-12)


# ---- SparseSign / CountSketch (sparse_sign.jl:299-459, count_sketch.jl:207-330) ------
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "sparse_sign_*.npz")) +
                                        glob.glob(os.path.join(GOLD, "count_sketch_*.npz"))))
def test_sparse_golden(orc, path):
    g = np.load(path)
    kind = "sparse_sign" if "sparse_sign" in path else "count_sketch"
    card = "left" if path.endswith("_left.npz") else "right"
    nnz = int(g["nnz"])
    L = len(g["rowval"]) // nnz
    s = 12  # compression dimension used by make_golden.sparse_case
    csc = orc.CSC(s, L, np.arange(0, L * nnz + 1, nnz), g["rowval"], g["nzval"])
    R = orc.Recipe(kind, card, s if card == "left" else L, L if card == "left" else s, np.float64, nnz=nnz, csc=csc)
    C = g["SA_C"].copy(order="F")
    orc.mul_SA(C, R, g["SA_A"], 2.0, 1.0)
    assert np.allclose(C, g["SA_out"], rtol=1e-12, atol=1e-12)
    C = g["AS_C"].copy(order="F")
    orc.mul_AS(C, g["AS_A"], R, 2.0, 1.0)
    assert np.allclose(C, g["AS_out"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch", "srht", "fjlt", "gaussian"])
@pytest.mark.parametrize("card", ["left", "right"])
def test_all_orientations_vs_dense(orc, kind, card):
    """S*A, A*S, S'*A, A*S' (and vectors) against the dense operator."""
    rng = np.random.default_rng(hash((kind, card)) % 2**32)
    L, s = 13, 5
    draw = {"sparse_sign": lambda: orc.draw_sparse_sign(rng, card, s, L, 3),
            "count_sketch": lambda: orc.draw_count_sketch(rng, card, s, L),
            "srht": lambda: orc.draw_srht(rng, card, s, L, block_size=2),
            "fjlt": lambda: orc.draw_fjlt(rng, card, s, L, sparsity=0.5, block_size=2),
            "gaussian": lambda: orc.draw_gaussian(rng, card, s, L)}[kind]
    R = draw()
    D = R.dense()
    nr, nc = D.shape
    k = 4
    for orient in ("SA", "AS", "StA", "ASt"):
        if orient == "SA":
            A, C = rng.random((nc, k)), rng.random((nr, k)); want = C + 2 * D @ A
            Cx = C.copy(order="F"); orc.mul_SA(Cx, R, A, 2.0, 1.0)
        elif orient == "AS":
            A, C = rng.random((k, nr)), rng.random((k, nc)); want = C + 2 * A @ D
            Cx = C.copy(order="F"); orc.mul_AS(Cx, A, R, 2.0, 1.0)
        elif orient == "StA":
            A, C = rng.random((nr, k)), rng.random((nc, k)); want = C + 2 * D.T @ A
            Cx = C.copy(order="F"); orc.mul_StA(Cx, R, A, 2.0, 1.0)
        else:
            A, C = rng.random((k, nc)), rng.random((k, nr)); want = C + 2 * A @ D.T
            Cx = C.copy(order="F"); orc.mul_ASt(Cx, A, R, 2.0, 1.0)
        assert np.allclose(Cx, want, rtol=1e-12, atol=1e-12), orient
    x = rng.random(nc); y = rng.random(nr)
    yy = y.copy(); orc.mul_SA(yy, R, x, 2.0, 1.0)
    assert np.allclose(yy, y + 2 * D @ x, rtol=1e-12, atol=1e-12)


def test_dimension_messages(orc):
    rng = np.random.default_rng(1)
    R = orc.draw_srht(rng, "left", 4, 10)
    with pytest.raises(orc.DimensionMismatch, match="Matrix A has 9 rows while S has 10 columns."):
        orc.mul_SA(np.zeros((4, 3)), R, np.zeros((9, 3)))
    with pytest.raises(orc.DimensionMismatch, match="Matrix A has 3 columns while C has 2 columns."):
        orc.mul_SA(np.zeros((4, 2)), R, np.zeros((10, 3)))
    with pytest.raises(orc.DimensionMismatch, match="Matrix C has 5 rows while S has 4 rows."):
        orc.mul_SA(np.zeros((5, 3)), R, np.zeros((10, 3)))


# ---- power iterations / RandSVD ------------------------------------------------------
def test_power_iteration_chain(orc):
    """range_finder_helpers.jl:59-78 / :104-132 on the oracle."""
    rng = np.random.default_rng(3)
    A = rng.random((30, 20))
    R = orc.draw_gaussian(rng, "right", 2, 20)
    Om = R.dense_op
    Q = orc.rand_power_it(A, R, 3)
    want = np.linalg.qr(A @ A.T @ A @ A.T @ A @ A.T @ A @ Om)[0]
    assert np.allclose(Q, want, rtol=1e-8, atol=1e-8)
    Q = orc.rand_ortho_it(A, R, 3)
    Q1 = np.linalg.qr(A @ Om)[0]
    for _ in range(3):
        Q1 = np.linalg.qr(A @ np.linalg.qr(A.T @ Q1)[0])[0]
    assert np.allclose(Q, Q1, rtol=1e-10, atol=1e-10)


def test_randsvd_exact_recovery(orc):
    """randsvd.jl:242-273 on the oracle."""
    rng = np.random.default_rng(4)
    A = rng.random((10, 10))
    R = orc.draw_gaussian(rng, "right", 10, 10)
    res = orc.randsvd(A, R, q=2)
    assert np.linalg.norm(A - res.U @ (res.U.T @ A)) < 1e-10
    assert np.linalg.norm(A - A @ res.V @ res.V.T) < 1e-10


def test_doc_example_rank20(orc):
    """docs/src/manual/introduction.md:24-40 (smaller n for the CPU suite)."""
    rng = np.random.default_rng(5)
    n = 800
    A = rng.standard_normal((n, 20)) @ rng.standard_normal((20, n))
    R = orc.draw_gaussian(rng, "right", 22, n)
    res = orc.randsvd(A, R)
    Ut, St, Vt = np.linalg.svd(A, full_matrices=False)
    trunc = (Ut[:, :22] * St[:22]) @ Vt[:22]
    assert np.linalg.norm((res.U * res.S) @ res.V.T - trunc) < 1e-9
