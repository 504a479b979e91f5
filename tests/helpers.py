"""Shared test helpers: load the library's own draws into oracle recipes (the way the
reference's tests load draws into recipe fields, test/Compressors/sparse_sign.jl:104,396)
and compare results."""
import numpy as np


def oracle_recipe(orc, S, dtype=np.float64):
    """Oracle recipe holding exactly the draws of the library recipe S (values in `dtype`)."""
    i = S.info
    d = S.draws()
    card = "left" if i.card == 0 else "right"
    if i.kind == 5:  # Sampling
        return orc.Recipe("sampling", card, int(i.n_rows), int(i.n_cols), dtype, idx=d["idx"].astype(np.int64))
    if i.kind in (0, 1):
        kind = "sparse_sign" if i.kind == 0 else "count_sketch"
        nnz = int(i.nnz)
        L = int(i.long_dim)
        csc = orc.CSC(int(i.compression_dim), L, np.arange(0, L * nnz + 1, nnz, dtype=np.int64),
                      d["rowval"].astype(np.int64), d["nzval"].astype(dtype))
        return orc.Recipe(kind, card, int(i.n_rows), int(i.n_cols), dtype, nnz=nnz, csc=csc)
    if i.kind == 2:
        return orc.Recipe("srht", card, int(i.n_rows), int(i.n_cols), dtype, op=d["op"], signs=d["signs"],
                          scale=float(i.scale), padded=int(i.padded), block_size=int(i.block_size))
    if i.kind == 3:
        N, s = int(i.padded), int(i.compression_dim)
        shape = (s, N) if card == "left" else (N, s)
        csc = orc.CSC(shape[0], shape[1], d["colptr"], d["rowval"], d["nzval"].astype(dtype))
        return orc.Recipe("fjlt", card, int(i.n_rows), int(i.n_cols), dtype, csc=csc, signs=d["signs"],
                          scale=float(i.scale), padded=N, block_size=int(i.block_size))
    return orc.Recipe("gaussian", card, int(i.n_rows), int(i.n_cols), dtype, dense_op=d["op"].astype(dtype),
                      scale=float(i.scale))


def rel_err(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref)
    return np.linalg.norm(x - ref) / (den if den > 0 else 1.0)


def to_dev(x, dev, fortran=True):
    import torch
    a = np.asfortranarray(x) if (fortran and x.ndim == 2) else np.ascontiguousarray(x)
    return torch.from_numpy(a).to(dev)


# Tolerances (relative Frobenius error against the FP64 oracle on the same draws):
TOL = {np.float32: 1e-6, np.float64: 1e-12}
