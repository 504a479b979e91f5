"""Checks at the benchmark sizes, on the library's own draws.

Covers the sketch-apply configurations (A 2^20x512 and 2^22x128 FP32, compression dimension
4096, SRHT / CountSketch / SparseSign from the left) and the least-squares SparseSign shape
(2^18x512, s = 2048, nnz = 8).  The FP64 oracle is too slow for every column at these sizes,
so each case checks:

* a few columns of S*A (first, second, middle, last) against the oracle's ``mul!``
  (test/Compressors/srht.jl:270-527, count_sketch.jl:207-330, sparse_sign.jl:299-459), with
  the apply run over all columns so the full-size work split is the one exercised;
* linearity over every column, S*(A1 + A2) = S*A1 + S*A2, which any wrong bin, sign or
  sample in any column breaks.

Tolerances: 1e-6 relative (Frobenius, FP32 against FP64) for the oracle columns; 1e-5 for
linearity, whose two sides differ by the FP32 rounding of A1 + A2 as well.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_recipe, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    ("srht", 2**20, 512, 4096),
    ("count_sketch", 2**20, 512, 4096),
    ("srht", 2**22, 128, 4096),
    ("count_sketch", 2**22, 128, 4096),
    ("sparse_sign", 2**18, 512, 2048),
]


def _compressor(rla, kind, s, dtype):
    if kind == "srht":
        return rla.SRHT(compression_dim=s, type=dtype)
    if kind == "count_sketch":
        return rla.CountSketch(compression_dim=s, type=dtype)
    return rla.SparseSign(compression_dim=s, nnz=8, type=dtype)


def _randn(torch, L, ncol, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.randn(ncol, L, device="cuda", generator=g).t()  # column-major L x ncol


@pytest.mark.parametrize("kind,L,ncol,s", CASES)
def test_fullsize_columns_match_oracle(rla, orc, dev, kind, L, ncol, s):
    import torch
    A = _randn(torch, L, ncol, seed=L + ncol)
    S = rla.complete_compressor(_compressor(rla, kind, s, np.float32), np.zeros((L, 1), np.float32), seed=s + ncol)
    C = torch.empty(ncol, s, device="cuda").t()
    rla.mul_(C, S, A)
    cols = [0, 1, ncol // 2, ncol - 1]
    A64 = A[:, cols].cpu().numpy().astype(np.float64)
    ref = np.zeros((s, len(cols)), order="F")
    orc.mul_SA(ref, oracle_recipe(orc, S), np.asfortranarray(A64), 1.0, 0.0)
    got = C[:, cols].cpu().numpy()
    err = rel_err(got, ref)
    assert err < TOL[np.float32], (kind, L, ncol, err)
    del A, C
    torch.cuda.empty_cache()


@pytest.mark.parametrize("kind,L,ncol,s", CASES)
def test_fullsize_linearity(rla, dev, kind, L, ncol, s):
    import torch
    A1 = _randn(torch, L, ncol, seed=1)
    A2 = _randn(torch, L, ncol, seed=2)
    S = rla.complete_compressor(_compressor(rla, kind, s, np.float32), np.zeros((L, 1), np.float32), seed=7)
    C1 = torch.empty(ncol, s, device="cuda").t()
    C2 = torch.empty(ncol, s, device="cuda").t()
    rla.mul_(C1, S, A1)
    rla.mul_(C2, S, A2)
    A1.add_(A2)  # A1 <- A1 + A2, in place to stay within a few GB
    del A2
    C12 = torch.empty(ncol, s, device="cuda").t()
    rla.mul_(C12, S, A1)
    diff = (C12.double() - C1.double() - C2.double()).norm().item()
    den = C12.double().norm().item()
    assert diff / den < 1e-5, (kind, L, ncol, diff / den)
    # the same holds column by column: no column may be off while the total looks fine
    col_err = ((C12.double() - C1.double() - C2.double()).norm(dim=0) / C12.double().norm(dim=0)).max().item()
    assert col_err < 1e-5, (kind, L, ncol, col_err)
    del A1, C1, C2, C12
    torch.cuda.empty_cache()
