"""The allocation-free SRHT entry point (rla_srht_mul_noalloc).

It exists for callers that cannot call cudaMalloc -- code that hands out a fixed device
memory budget itself, code whose memory belongs to another runtime's pool, paths that
must not touch the allocator -- and keeps its partial sums in library-owned fixed device
arrays.  Its results must match the regular entry point (rla_sketch_mul) within the
Float32 tolerance of the other tests, on two calls in a row (the second call reuses the
arrays the first one left behind).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_err, to_dev

pytestmark = pytest.mark.gpu


def _noalloc(rla, S, C, A, alpha, beta):
    import torch
    from randlinearalgebra_b200 import _lib
    ctx = _lib.Context.get(C.device.index)
    torch.cuda.synchronize()
    st = _lib.lib().rla_srht_mul_noalloc(ctx.handle, S.handle, C.shape[0], C.shape[1], C.data_ptr(), C.stride(1),
                                         A.shape[0], A.shape[1], A.data_ptr(), A.stride(1), alpha, beta)
    _lib.check(st, ctx.handle)
    _lib.check(_lib.lib().rla_ctx_synchronize(ctx.handle), ctx.handle)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("m,n,s", [(40000, 37, 300), (1000, 5, 24)])
def test_noalloc_matches_regular_entry(rla, dev, dtype, m, n, s):
    rng = np.random.default_rng(m + s)
    S = rla.complete_compressor(rla.SRHT(compression_dim=s, type=dtype), np.zeros((m, 1), dtype), seed=77)
    tol = 1e-6 if dtype == np.float32 else 1e-12
    for call in range(2):  # two calls in a row share the fixed scratch
        A = rng.standard_normal((m, n)).astype(dtype)
        C0 = rng.standard_normal((s, n)).astype(dtype)
        Ad = to_dev(A, dev)
        ref = to_dev(C0, dev)
        rla.mul_(ref, S, Ad, 1.5, 0.5)
        out = to_dev(C0, dev)
        _noalloc(rla, S, out, Ad, 1.5, 0.5)
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < tol, (call, m, n, s)


def test_noalloc_rejects_too_many_columns(rla, dev):
    S = rla.complete_compressor(rla.SRHT(compression_dim=4, type=np.float32), np.zeros((8, 1), np.float32), seed=1)
    ncols = 65537  # one above RLA_NOALLOC_MAX_COLS
    A = to_dev(np.zeros((8, ncols), np.float32), dev)
    C = to_dev(np.zeros((4, ncols), np.float32), dev)
    with pytest.raises(rla.ArgumentError, match="allocation-free limit"):
        _noalloc(rla, S, C, A, 1.0, 0.0)
