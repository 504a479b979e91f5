"""Generates the golden fixtures in this directory.

The reference (RandLinearAlgebra.jl) ships no stored vectors: its tests compare each
compressor against an explicit formula -- the natural-order Hadamard matrix of
Hadamard.jl for fwht!/SRHT/FJLT (test/Compressors/helpers/fwht.jl:34-70,
test/Compressors/srht.jl:270-527, test/Compressors/fjlt.jl:321-560) and the dense
re-materialised operator for the sparse and Gaussian compressors
(test/Compressors/sparse_sign.jl:299-459, count_sketch.jl:207-330, gaussian.jl:200-280).
This script evaluates exactly those formulas in float64 with numpy on seeded inputs and
draws and stores inputs, draws and expected outputs, so the oracle and the B200 library
are both checked against values computed without their own loops.

Run: python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def hadamard(n):
    H = np.ones((1, 1))
    while H.shape[0] < n:
        H = np.block([[H, H], [H, -H]])
    return H


def pad_pow2(n):
    return 1 << max(0, (n - 1).bit_length())


def fwht_cases(rng):
    out = {}
    for ln in (8, 16):
        x = rng.random(ln)
        signs = rng.integers(0, 2, ln).astype(np.uint8)
        H = hadamard(ln)
        out[f"fwht_{ln}_x"] = x
        out[f"fwht_{ln}_signs"] = signs
        out[f"fwht_{ln}_plain"] = H @ x                                  # fwht.jl:39
        out[f"fwht_{ln}_signed"] = H @ (np.where(signs, 1.0, -1.0) * x)  # fwht.jl:59
        out[f"fwht_{ln}_signed_scaled"] = out[f"fwht_{ln}_signed"] / ln  # fwht.jl:62
    return out


def srht_case(rng, card, m_long, s, k):
    """srht.jl test formulas with alpha = 2, beta = 1."""
    N = pad_pow2(m_long)
    H = hadamard(N)
    signs = rng.integers(0, 2, N).astype(np.uint8)
    d = np.where(signs, 1.0, -1.0)
    op = rng.choice(N, s, replace=False)
    scale = np.sqrt(s) / np.sqrt(N)
    sI = np.zeros((N, s))
    sI[op, np.arange(s)] = 1.0
    res = {"signs": signs, "op": op, "scale": np.float64(scale), "N": np.int64(N)}
    if card == "left":  # S is s x m
        A = rng.random((m_long, k)); C = rng.random((s, k))
        pad = np.zeros((N, k)); pad[:m_long] = A
        res.update(SA_A=A, SA_C=C, SA_out=C + (H @ (d[:, None] * pad) * 2 * scale)[op, :])
        A2 = rng.random((k, s)); C2 = rng.random((k, m_long))
        res.update(AS_A=A2, AS_C=C2, AS_out=C2 + 2 * (A2 @ sI.T @ H @ np.diag(d) * scale)[:, :m_long])
    else:  # S is n x s
        A = rng.random((s, k)); C = rng.random((m_long, k))
        res.update(SA_A=A, SA_C=C, SA_out=C + (np.diag(d) @ H @ sI @ A * 2 * scale)[:m_long, :])
        A2 = rng.random((k, m_long)); C2 = rng.random((k, s))
        pad = np.zeros((k, N)); pad[:, :m_long] = A2
        res.update(AS_A=A2, AS_C=C2, AS_out=C2 + 2 * (pad @ np.diag(d) @ H * scale)[:, op])
    return res


def sparse_case(rng, kind, card, long_dim, s, k, nnz):
    """sparse_sign.jl / count_sketch.jl tests: compare with the dense operator."""
    if kind == "sparse_sign":
        rows = np.stack([np.sort(rng.choice(s, nnz, replace=False)) for _ in range(long_dim)]).reshape(-1)
        vals = np.where(rng.integers(0, 2, long_dim * nnz) == 1, 1.0, -1.0) / np.sqrt(nnz)
    else:
        nnz = 1
        rows = rng.integers(0, s, long_dim)
        vals = np.where(rng.integers(0, 2, long_dim) == 1, 1.0, -1.0)
    P = np.zeros((s, long_dim))
    for j in range(long_dim):
        for e in range(nnz):
            P[rows[j * nnz + e], j] += vals[j * nnz + e]
    S = P if card == "left" else P.T
    nr, nc = S.shape
    A = rng.random((nc, k)); C = rng.random((nr, k))
    A2 = rng.random((k, nr)); C2 = rng.random((k, nc))
    return {"rowval": rows.astype(np.int64), "nzval": vals, "nnz": np.int64(nnz),
            "SA_A": A, "SA_C": C, "SA_out": C + 2 * S @ A,
            "AS_A": A2, "AS_C": C2, "AS_out": C2 + 2 * A2 @ S}


def main():
    rng = np.random.default_rng(20260101)
    np.savez(os.path.join(HERE, "fwht.npz"), **fwht_cases(rng))
    for card in ("left", "right"):
        for long_dim in (8, 10):
            np.savez(os.path.join(HERE, f"srht_{card}_{long_dim}.npz"), **srht_case(rng, card, long_dim, 3, 6))
        for kind in ("sparse_sign", "count_sketch"):
            np.savez(os.path.join(HERE, f"{kind}_{card}.npz"), **sparse_case(rng, kind, card, 40, 12, 5, 4))


if __name__ == "__main__":
    main()
