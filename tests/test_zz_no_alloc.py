"""The allocation-free SRHT entry point (rla_srht_mul_noalloc).

It exists for callers that cannot call cudaMalloc -- code that hands out a fixed device
memory budget itself, code whose memory belongs to another runtime's pool, paths that
must not touch the allocator -- and keeps its partial sums in library-owned fixed device
arrays.  Its results must match the regular entry point (rla_sketch_mul) within the
tolerance of the other tests, on two calls in a row (the second call reuses the arrays
the first one left behind).  The larger cases also go through the oracle: a compression
dimension above one sample window (several launches share the arrays within one call),
a Float64 window whose partial sums cap the number of CTAs, and a padded leading
dimension that takes the scalar load path.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from helpers import TOL, oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu


def _noalloc(rla, S, C, A, alpha, beta, dims=None):
    import torch
    from randlinearalgebra_b200 import _lib
    ctx = _lib.Context.get(C.device.index)
    torch.cuda.synchronize()
    c_rows, c_cols, a_rows, a_cols = dims if dims else (C.shape[0], C.shape[1], A.shape[0], A.shape[1])
    st = _lib.lib().rla_srht_mul_noalloc(ctx.handle, S.handle, c_rows, c_cols, C.data_ptr(), C.stride(1),
                                         a_rows, a_cols, A.data_ptr(), A.stride(1), alpha, beta)
    _lib.check(st, ctx.handle)
    _lib.check(_lib.lib().rla_ctx_synchronize(ctx.handle), ctx.handle)


def _padded_dev(A, dev, pad):
    """A on the device as the leading m rows of an (m + pad) x n column-major buffer."""
    m, n = A.shape
    buf = np.zeros((m + pad, n), A.dtype)
    buf[:m] = A
    return to_dev(buf, dev)[:m]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("m,n,s", [(40000, 37, 300), (1000, 5, 24)])
def test_noalloc_matches_regular_entry(rla, dev, dtype, m, n, s):
    rng = np.random.default_rng(m + s)
    S = rla.complete_compressor(rla.SRHT(compression_dim=s, type=dtype), np.zeros((m, 1), dtype), seed=77)
    tol = TOL[dtype]
    for call in range(2):  # two calls in a row share the fixed scratch
        A = rng.standard_normal((m, n)).astype(dtype)
        C0 = rng.standard_normal((s, n)).astype(dtype)
        Ad = to_dev(A, dev)
        ref = to_dev(C0, dev)
        rla.mul_(ref, S, Ad, 1.5, 0.5)
        out = to_dev(C0, dev)
        _noalloc(rla, S, out, Ad, 1.5, 0.5)
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < tol, (call, m, n, s)


# (dtype, m, n, s, lda padding): s = 5000 spans two sample windows (4096 + 904); Float64
# s = 4096 leaves room for 8 MiB / (2 * 4096 * 8 B) = 128 CTAs, fewer than two per SM; a
# padding of one row makes lda odd, so the kernel takes its scalar load path.
_AWKWARD = [
    (np.float32, 40000, 9, 5000, 0),
    (np.float64, 40000, 7, 5000, 0),
    (np.float64, 70000, 6, 4096, 0),
    (np.float32, 40000, 11, 300, 1),
    (np.float64, 20000, 5, 5000, 1),
]


@pytest.mark.parametrize("dtype,m,n,s,pad", _AWKWARD)
def test_noalloc_windows_clamp_and_padding(rla, orc, dev, dtype, m, n, s, pad):
    rng = np.random.default_rng(m + s + pad)
    S = rla.complete_compressor(rla.SRHT(compression_dim=s, type=dtype), np.zeros((m, 1), dtype), seed=91)
    R = oracle_recipe(orc, S)
    tol = TOL[dtype]
    for call in range(2):
        A = rng.standard_normal((m, n)).astype(dtype)
        C0 = rng.standard_normal((s, n)).astype(dtype)
        Ad = _padded_dev(A, dev, pad)
        assert Ad.stride(1) == m + pad
        ref = to_dev(C0, dev)
        rla.mul_(ref, S, to_dev(A, dev), 2.0, -1.0)
        out = to_dev(C0, dev)
        _noalloc(rla, S, out, Ad, 2.0, -1.0)
        got = out.cpu().numpy()
        assert rel_err(got, ref.cpu().numpy()) < tol, ("regular", call)
        exp = C0.astype(np.float64).copy()
        orc.mul_SA(exp, R, A.astype(np.float64), 2.0, -1.0)
        assert rel_err(got, exp) < tol, ("oracle", call)


def test_noalloc_rejects_too_many_columns(rla, dev):
    S = rla.complete_compressor(rla.SRHT(compression_dim=4, type=np.float32), np.zeros((8, 1), np.float32), seed=1)
    ncols = 65537  # one above RLA_NOALLOC_MAX_COLS
    A = to_dev(np.zeros((8, ncols), np.float32), dev)
    C = to_dev(np.zeros((4, ncols), np.float32), dev)
    with pytest.raises(rla.ArgumentError, match="allocation-free limit"):
        _noalloc(rla, S, C, A, 1.0, 0.0)


def test_noalloc_rejects_negative_dimensions(rla, dev):
    S = rla.complete_compressor(rla.SRHT(compression_dim=4, type=np.float32), np.zeros((8, 1), np.float32), seed=1)
    A = to_dev(np.zeros((8, 3), np.float32), dev)
    C = to_dev(np.zeros((4, 3), np.float32), dev)
    with pytest.raises(rla.ArgumentError, match="Negative dimension"):
        _noalloc(rla, S, C, A, 1.0, 0.0, dims=(4, -3, 8, -3))


def test_noalloc_keeps_callers_device(rla, dev):
    """A call on a context of device 0 leaves another current device in place; the next call
    still runs on device 0.  Needs two GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    rng = np.random.default_rng(5)
    m, n, s = 30000, 4, 64
    S = rla.complete_compressor(rla.SRHT(compression_dim=s, type=np.float32), np.zeros((m, 1), np.float32), seed=3)
    A = rng.standard_normal((m, n)).astype(np.float32)
    Ad = to_dev(A, dev)
    ref = torch.zeros((s, n), dtype=torch.float32, device=dev).t().contiguous().t()
    rla.mul_(ref, S, Ad, 1.0, 0.0)
    for call in range(2):
        torch.cuda.set_device(1)
        out = torch.zeros((s, n), dtype=torch.float32, device=dev).t().contiguous().t()
        _noalloc(rla, S, out, Ad, 1.0, 0.0)
        assert torch.cuda.current_device() == 1, call
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < TOL[np.float32], call
    torch.cuda.set_device(0)
