"""Serving loop (rla_server_*): mixed sketch-and-solve and RandSVD requests.

A request's result is the same alone and in the mix (bitwise: grouped kernels map each tile
to one instance and add partials in a fixed order), the least-squares solve matches the
oracle's solve of the same sketched problem, and RandSVD matches the FP64 oracle on the same
draws within 1e-4."""
import numpy as np
import pytest

from helpers import oracle_recipe, rel_err, to_dev

pytestmark = pytest.mark.gpu


def lowrank(rng, m, n, decay=0.9):
    r = min(m, n, 120)
    U = np.linalg.qr(rng.standard_normal((m, r)))[0]
    V = np.linalg.qr(rng.standard_normal((n, r)))[0]
    return ((U * decay ** np.arange(r)) @ V.T + 1e-6 * rng.standard_normal((m, n))).astype(np.float32)


def make_pool(rng, dev):
    ls, svd = [], []
    for i in range(5):
        m, n = int(rng.integers(2000, 20000)), int(rng.integers(16, 96))
        A = rng.standard_normal((m, n)).astype(np.float32)
        x0 = rng.standard_normal(n)
        b = (A @ x0 + 1e-3 * rng.standard_normal(m)).astype(np.float32)
        ls.append((A, b, to_dev(A, dev), to_dev(b, dev), 500 + i))
    for i, k in enumerate([8, 32, 64, 100, 150]):
        m, n = int(rng.integers(800, 6000)), int(rng.integers(180, 500))
        A = lowrank(rng, m, n)
        svd.append((A, to_dev(A, dev), k, 700 + i))
    return ls, svd


def submit_all(torch, srv, reqs, dev):
    outs = {}
    for tag, (kind, item) in enumerate(reqs):
        if kind == "ls":
            A, b, Ad, bd, seed = item
            x = torch.zeros(A.shape[1], dtype=torch.float32, device=dev)
            srv.submit_ls(Ad, bd, x, seed, tag)
            outs[tag] = (x,)
        else:
            A, Ad, k, seed = item
            m, n = A.shape
            U = torch.zeros(k, m, dtype=torch.float32, device=dev).t()
            S = torch.zeros(k, dtype=torch.float64, device=dev)
            V = torch.zeros(k, n, dtype=torch.float32, device=dev).t()
            srv.submit_svd(Ad, k, U, S, V, seed, tag)
            outs[tag] = (U, S, V)
    return outs


def test_sketch_solve_matches_oracle(rla, orc, dev):
    import torch
    rng = np.random.default_rng(3)
    m, n = 6000, 40
    A = rng.standard_normal((m, n)).astype(np.float32)
    b = (A @ rng.standard_normal(n) + 1e-3 * rng.standard_normal(m)).astype(np.float32)
    Ad = to_dev(A, dev)
    S = rla.complete_compressor(rla.SparseSign(cardinality=rla.Left(), compression_dim=4 * n, nnz=8, type=np.float32),
                                Ad, seed=11)
    x = torch.zeros(n, dtype=torch.float32, device=dev)
    rla.sketch_solve(S, Ad, to_dev(b, dev), x)
    R = oracle_recipe(orc, S)
    SA = np.zeros((4 * n, n), order="F")
    Sb = np.zeros((4 * n, 1), order="F")
    orc.mul_SA(SA, R, A.astype(np.float64))
    orc.mul_SA(Sb, R, b.astype(np.float64).reshape(-1, 1))
    xr = np.linalg.lstsq(SA, Sb[:, 0], rcond=None)[0]
    assert rel_err(x.cpu().numpy(), xr) < 1e-4


def test_mix_equals_alone_and_oracle(rla, orc, dev):
    import torch
    rng = np.random.default_rng(9)
    ls, svd = make_pool(rng, dev)
    reqs = [("ls", ls[i % 5]) if i % 5 < 3 else ("svd", svd[i % 5]) for i in range(30)]
    reqs += [("svd", s) for s in svd]
    srv = rla.Server(slots=3, max_group=8)
    mix = submit_all(torch, srv, reqs, dev)
    srv.wait_idle()
    done = srv.poll()
    assert len(done) == len(reqs) and all(st == 0 for _, _, st in done)
    assert all(lat > 0 for _, lat, _ in done)
    for tag, req in enumerate(reqs):
        alone = submit_all(torch, srv, [req], dev)[0]
        srv.wait_idle()
        assert srv.poll()[0][2] == 0
        for a, b in zip(mix[tag], alone):
            assert torch.equal(a, b), (tag, req[0])
    srv.stop()
    # accuracy against the oracle on the same draws
    for (A, Ad, k, seed), tag in zip(svd, range(30, 30 + len(svd))):
        comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
        rec = rla.complete_compressor(comp, Ad, seed=seed)
        ref = orc.randsvd(A.astype(np.float64), oracle_recipe(orc, rec))
        assert rel_err(mix[tag][1].cpu().numpy(), ref.S) < 1e-4, (k, seed)


def test_plain_mode_and_tiny_budget(rla, dev):
    import torch
    rng = np.random.default_rng(12)
    ls, svd = make_pool(rng, dev)
    reqs = [("ls", ls[0]), ("svd", svd[1]), ("ls", ls[1]), ("svd", svd[2])]
    plain = rla.Server(plain=True)
    o1 = submit_all(torch, plain, reqs, dev)
    plain.wait_idle()
    assert all(st == 0 for _, _, st in plain.poll())
    plain.stop()
    tiny = rla.Server(slots=2, max_group=4, memory_budget=1)  # every request runs alone
    o2 = submit_all(torch, tiny, reqs, dev)
    tiny.wait_idle()
    assert all(st == 0 for _, _, st in tiny.poll())
    tiny.stop()
    for t in (0, 2):  # least squares: same kernels in both modes
        assert torch.equal(o1[t][0], o2[t][0])
    for t in (1, 3):  # RandSVD: single-instance path (FP64 accumulation) vs grouped (FP32)
        assert rel_err(o1[t][1].cpu().numpy(), o2[t][1].cpu().numpy()) < 1e-5


def test_sketch_cache_is_bounded_and_counted(rla, dev):
    """Per-request seeds: every least-squares request of a new seed makes a new resident
    sketch.  The cache stays within its cap (least recently used sketches not held by a
    running request are destroyed), its bytes are reported, and results are unchanged: a
    request whose sketch was evicted and made again gives the same solution bit for bit."""
    import torch
    rng = np.random.default_rng(17)
    m, n = 65536, 64  # SparseSign s = 256, nnz = 8: about 6 MB of draws per seed
    A = rng.standard_normal((m, n)).astype(np.float32)
    b = (A @ rng.standard_normal(n)).astype(np.float32)
    Ad, bd = to_dev(A, dev), to_dev(b, dev)
    cap = 20 << 20
    srv = rla.Server(slots=2, max_group=4, sketch_cache_bytes=cap)
    xs = []
    for tag in range(24):
        x = torch.zeros(n, dtype=torch.float32, device=dev)
        srv.submit_ls(Ad, bd, x, 1000 + tag, tag)
        xs.append(x)
    srv.wait_idle()
    assert all(st == 0 for _, _, st in srv.poll())
    st = srv.stats()
    assert st["cache_bytes"] <= cap and st["cache_entries"] <= 4 and st["evictions"] >= 20, st
    again = torch.zeros(n, dtype=torch.float32, device=dev)
    srv.submit_ls(Ad, bd, again, 1000, 99)  # seed 1000 was evicted long ago
    srv.wait_idle()
    assert srv.poll()[0][2] == 0
    assert torch.equal(again, xs[0])
    srv.stop()


def test_injected_allocation_failure_fails_only_that_request(rla, dev):
    """Host-side fault injection: the tagged requests' workspace allocations fail (one
    least-squares request, one RandSVD request inside a grouped batch).  They complete with
    RLA_E_OOM; every other request completes and equals its result alone."""
    import torch
    rng = np.random.default_rng(21)
    ls, svd = make_pool(rng, dev)
    reqs = [("ls", ls[i % 5]) if i % 2 == 0 else ("svd", svd[i % 3]) for i in range(12)]
    srv = rla.Server(slots=1, max_group=8)
    srv.inject_alloc_failure(2)   # least squares
    srv.inject_alloc_failure(5)   # RandSVD
    outs = submit_all(torch, srv, reqs, dev)
    srv.wait_idle()
    status = {tag: st for tag, _, st in srv.poll()}
    assert len(status) == len(reqs)
    assert status[2] == rla._lib.RLA_E_OOM and status[5] == rla._lib.RLA_E_OOM
    assert all(st == 0 for tag, st in status.items() if tag not in (2, 5)), status
    assert "injected" in srv.last_error()
    for tag in (0, 3, 7):
        alone = submit_all(torch, srv, [reqs[tag]], dev)[0]
        srv.wait_idle()
        assert srv.poll()[0][2] == 0
        for a, b in zip(outs[tag], alone):
            assert torch.equal(a, b), tag
    srv.stop()


def test_cancel_queued_and_reject_malformed(rla, dev):
    import torch
    rng = np.random.default_rng(23)
    ls, svd = make_pool(rng, dev)
    srv = rla.Server(plain=True)  # one request at a time: the later ones wait in the queue
    reqs = [("svd", svd[4])] + [("ls", ls[i]) for i in range(5)]
    submit_all(torch, srv, reqs, dev)
    srv.cancel(5)
    srv.wait_idle()
    status = {tag: st for tag, _, st in srv.poll()}
    assert status[5] == rla._lib.RLA_E_CANCELLED
    assert all(status[t] == 0 for t in range(5))
    with pytest.raises(rla.ArgumentError, match="no queued request"):
        srv.cancel(0)  # already done
    # malformed requests are refused at submit; the server keeps serving
    A, Ad, k, seed = svd[0]
    m, n = A.shape
    U = torch.zeros(k, m, dtype=torch.float32, device=dev).t()
    S = torch.zeros(k, dtype=torch.float64, device=dev)
    V = torch.zeros(k, n, dtype=torch.float32, device=dev).t()
    with pytest.raises(rla.ArgumentError, match="rejected"):
        srv.submit_svd(Ad, min(m, n) + 1, U, S, V, seed, 50)  # k above min(m, n)
    x = torch.zeros(n, dtype=torch.float32, device=dev)
    with pytest.raises(rla.ArgumentError, match="rejected"):
        srv.submit_ls(Ad[:n - 1, :], to_dev(np.zeros(n - 1, np.float32), dev), x, 1, 51)  # n > m
    submit_all(torch, srv, [("ls", ls[0])], dev)
    srv.wait_idle()
    assert [st for _, _, st in srv.poll()] == [0]
    srv.stop()
