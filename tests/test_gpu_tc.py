"""Split-BF16 tensor-core GEMM (rla_gemm_bf16x3, the product kernel of the
RLA_PREC_SPLIT_BF16 RandSVD path) against an FP64 product of the same FP32 data.

Each FP32 operand is split into bf16 hi + lo and the kernel forms hi*hi + hi*lo + lo*hi
with FP32 accumulation, so the relative Frobenius error is a few 2^-17 (tolerance 3e-5).
Shapes cover both operand layouts (A*B and A'*B), ragged M/N/K tiles, the two-chunk
288-column tile, and split-K."""
import ctypes

import numpy as np
import pytest

TOL = 3e-5


def colmajor(torch, rows, cols, dev, gen, ld=None):
    ld = ld or rows
    buf = torch.randn((cols, ld), generator=gen, device=dev, dtype=torch.float32)
    return buf.t()[:rows, :]  # column-major view, leading dimension ld


def run_gemm(rla, torch, dev, trans_a, m, n, k, alpha=1.0, beta=0.0, lda_pad=0):
    gen = torch.Generator(device=dev).manual_seed(m * 7 + n * 3 + k)
    a_rows, a_cols = (k, m) if trans_a else (m, k)
    A = colmajor(torch, a_rows, a_cols, dev, gen, a_rows + lda_pad)
    B = colmajor(torch, k, n, dev, gen)
    C = colmajor(torch, m, n, dev, gen)
    C0 = C.clone()
    L = rla._lib.lib()
    ctx = rla._lib.Context.get(dev.index or 0)
    st = L.rla_gemm_bf16x3(ctx.handle, trans_a, m, n, k, ctypes.c_void_p(A.data_ptr()), A.stride(1),
                           ctypes.c_void_p(B.data_ptr()), B.stride(1), ctypes.c_void_p(C.data_ptr()), C.stride(1),
                           alpha, beta)
    rla._lib.check(st, ctx.handle)
    opA = A.double().t() if trans_a else A.double()
    ref = alpha * (opA @ B.double()) + beta * C0.double()
    err = (C.double() - ref).norm() / ref.norm()
    return float(err)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(256, 64, 128), (300, 272, 200), (128, 288, 64), (1000, 16, 5000),
                                   (70, 33, 31), (4096, 256, 2048)])
def test_gemm_mn_major(rla, dev, m, n, k):
    import torch
    err = run_gemm(rla, torch, dev, 0, m, n, k)
    assert err < TOL, (m, n, k, err)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(200, 272, 3000), (64, 40, 100000), (128, 16, 32), (513, 100, 777)])
def test_gemm_k_major(rla, dev, m, n, k):
    import torch
    err = run_gemm(rla, torch, dev, 1, m, n, k)
    assert err < TOL, (m, n, k, err)


@pytest.mark.gpu
def test_gemm_alpha_beta_and_wide_n(rla, dev):
    import torch
    # N above one 288-column tile, padded leading dimension, alpha/beta epilogue
    err = run_gemm(rla, torch, dev, 0, 384, 600, 256, alpha=1.5, beta=0.5, lda_pad=8)
    assert err < TOL, err
    err = run_gemm(rla, torch, dev, 1, 96, 300, 1024, alpha=-2.0, beta=1.0)
    assert err < TOL, err


@pytest.mark.gpu
def test_gemm_deterministic(rla, dev):
    import torch
    gen = torch.Generator(device=dev).manual_seed(1)
    A = colmajor(torch, 65536, 512, dev, gen)
    B = colmajor(torch, 65536, 64, dev, gen)
    L = rla._lib.lib()
    ctx = rla._lib.Context.get(dev.index or 0)
    outs = []
    for _ in range(2):
        C = torch.zeros((64, 512), device=dev).t()
        rla._lib.check(L.rla_gemm_bf16x3(ctx.handle, 1, 512, 64, 65536, ctypes.c_void_p(A.data_ptr()), A.stride(1),
                                          ctypes.c_void_p(B.data_ptr()), B.stride(1), ctypes.c_void_p(C.data_ptr()),
                                          C.stride(1), 1.0, 0.0), ctx.handle)
        outs.append(C.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_wait_limit_runs_out_and_context_recovers(rla, dev):
    """Failure detection without a GPU fault.  With a wait limit of zero every mbarrier wait
    of the GEMM kernel that is not already satisfied runs out: the kernel records the
    failure in its status word, stops issuing copies and MMAs, waits (bounded) for the ones
    already issued, releases its tensor memory and exits, and the call reports
    RLA_E_TIMEOUT.  The same context then computes the product correctly."""
    import torch
    L = rla._lib.lib()
    ctx = rla._lib.Context.get(dev.index or 0)
    rla._lib.check(L.rla_ctx_set_wait_limit(ctx.handle, 0.0), ctx.handle)
    try:
        with pytest.raises(rla.RLAError, match="timed out"):
            run_gemm(rla, torch, dev, 0, 4096, 256, 2048)
    finally:
        rla._lib.check(L.rla_ctx_set_wait_limit(ctx.handle, 2.0), ctx.handle)
    for trans_a in (0, 1):
        err = run_gemm(rla, torch, dev, trans_a, 4096, 256, 2048)
        assert err < TOL, (trans_a, err)
    with pytest.raises(rla.ArgumentError, match="wait limit"):
        rla._lib.check(L.rla_ctx_set_wait_limit(ctx.handle, -1.0), ctx.handle)
