"""S * transpose(B) for a sparse B (sparse_sign.jl:364-442, count_sketch.jl:215-262).

Ports the reference's "Left Multiplication Sparse Transpose" testsets
(test/Compressors/sparse_sign.jl:353-380, count_sketch.jl:256-281): C = alpha*S*A +
beta*C against the dense product, with beta = 0 and beta != 0, plus larger cases (several
column tiles, empty rows and columns, Float32) against the oracle's CSC loop on the
densified operand.  Tolerance: relative Frobenius error 1e-12 (Float64) / 1e-6 (Float32).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import TOL, oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu


def _make(rla, kind, s, m, dtype, seed):
    if kind == "sparse_sign":
        comp = rla.SparseSign(compression_dim=s, nnz=min(8, s), type=dtype)
    else:
        comp = rla.CountSketch(compression_dim=s, type=dtype)
    return rla.complete_compressor(comp, np.zeros((m, 1), dtype), seed=seed)


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch"])
def test_reference_small_cases(rla, orc, dev, kind):
    rng = np.random.default_rng(3)
    n_rows, n_cols, c_dim = (6, 4, 5) if kind == "sparse_sign" else (7, 5, 4)
    alpha, beta = (1.25, 0.4) if kind == "sparse_sign" else (1.4, 0.5)
    B = sp.random(n_cols, n_rows, density=0.6, random_state=1, format="csc")
    A = B.T.tocsr()  # transpose(B): n_rows x n_cols
    S = _make(rla, kind, c_dim, n_rows, np.float64, 11)
    dense_S = np.zeros((c_dim, n_rows))
    R = oracle_recipe(orc, S)
    orc.mul_SA(dense_S, R, np.eye(n_rows))
    C0 = rng.random((c_dim, n_cols))
    Cd = to_dev(C0, dev)
    rla.mul_(Cd, S, A, alpha, beta)
    assert rel_err(Cd.cpu().numpy(), alpha * dense_S @ A.toarray() + beta * C0) < 1e-12
    Cd = to_dev(rng.random((c_dim, n_cols)), dev)
    rla.mul_(Cd, S, A, alpha, 0.0)
    assert rel_err(Cd.cpu().numpy(), alpha * dense_S @ A.toarray()) < 1e-12


@pytest.mark.parametrize("kind", ["sparse_sign", "count_sketch"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_large_against_oracle(rla, orc, dev, kind, dtype):
    """m = 3000 rows, n = 2500 columns (three column tiles), 1 % density with a block of
    empty rows and columns; the result equals the oracle's apply to the dense operand."""
    import torch
    m, n, s = 3000, 2500, 96
    B = sp.random(n, m, density=0.01, random_state=7, format="csc", dtype=np.float64)
    B = B.tolil()
    B[:, 100:140] = 0.0
    B[200:260, :] = 0.0
    A = B.tocsc().T.tocsr().astype(dtype)
    S = _make(rla, kind, s, m, dtype, 21)
    R = oracle_recipe(orc, S)
    rng = np.random.default_rng(9)
    C0 = rng.standard_normal((s, n)).astype(dtype)
    ref = C0.astype(np.float64).copy(order="F")
    orc.mul_SA(ref, R, A.toarray().astype(np.float64), 2.0, 1.0)
    Cd = to_dev(C0, dev)
    rla.mul_(Cd, S, A, 2.0, 1.0)
    assert rel_err(Cd.cpu().numpy(), ref) < TOL[dtype]
    # the same operand as a torch sparse-CSR tensor on the device; repeated calls agree bitwise
    At = torch.sparse_csr_tensor(torch.from_numpy(A.indptr.astype(np.int64)),
                                 torch.from_numpy(A.indices.astype(np.int64)),
                                 torch.from_numpy(A.data), size=A.shape).to(dev)
    C1 = to_dev(C0, dev)
    rla.mul_(C1, S, At, 2.0, 1.0)
    assert torch.equal(C1, Cd)
    # after a redraw the plan is rebuilt
    rla.update_compressor_(S)
    R2 = oracle_recipe(orc, S)
    ref2 = np.zeros((s, n))
    orc.mul_SA(ref2, R2, A.toarray().astype(np.float64))
    C2 = to_dev(np.zeros((s, n), dtype), dev)
    rla.mul_(C2, S, At)
    assert rel_err(C2.cpu().numpy(), ref2) < TOL[dtype]


def test_sparse_operand_errors(rla, dev):
    A = sp.random(20, 6, density=0.3, random_state=2, format="csr")
    Sr = rla.complete_compressor(rla.SparseSign(cardinality=rla.Right(), compression_dim=4), np.zeros((1, 20)), seed=1)
    with pytest.raises(rla.ArgumentError, match="No method `mul!`"):
        rla.mul_(to_dev(np.zeros((4, 6)), dev), Sr, A)
    Sg = rla.complete_compressor(rla.Gaussian(compression_dim=4), np.zeros((20, 1)), seed=1)
    with pytest.raises(rla.ArgumentError, match="No method `mul!`"):
        rla.mul_(to_dev(np.zeros((4, 6)), dev), Sg, A)
    S = rla.complete_compressor(rla.CountSketch(compression_dim=4), np.zeros((20, 1)), seed=1)
    with pytest.raises(rla.DimensionMismatch, match="Matrix C has 5 rows while S has 4 rows."):
        rla.mul_(to_dev(np.zeros((5, 6)), dev), S, A)
    with pytest.raises(rla.DimensionMismatch, match="Matrix A has 6 columns while C has 7 columns."):
        rla.mul_(to_dev(np.zeros((4, 7)), dev), S, A)
