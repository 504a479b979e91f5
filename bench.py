#!/usr/bin/env python
"""Sketch-apply benchmark: SRHT and CountSketch applied from the left, Float32.

Workload: A is 2^20 x 512 (column-major, i.i.d. N(0,1), synthetic, generated on the
device), compressed to 4096 x 512 by an SRHT (length-2^20 Walsh-Hadamard transform,
Rademacher signs, 4096 rows sampled without replacement) and by a CountSketch (one
bucket and one sign per row).  One step = both applies over A.  The metric is HBM
throughput in GB/s of algorithmic bytes, 4*(m*n + s*n) per apply.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs one replica per GPU under torchrun (weak scaling: each rank sketches its own
2^20 x 512 block; no data-path collective), timed on the device as the max over ranks.
`--impl reference` times the CPU restatement of the reference (oracle/) on the host cores
on a bounded sample of the same workload.

`--workload randsvd` measures the mixed-precision RandSVD instead: A = U diag(s) V' +
1e-6 N(0,1), 65536 x 8192 Float32, s_i = i^-1.5 for i <= 512 (U, V orthonormal from QR of
Gaussians, seed 3), Gaussian sketch, k = 256, p = 16 (l = 272), q = 2, orthogonalised; the
products with A on the tensor cores in split BF16, Gram/Cholesky/triangular inverse and the
SVD of B in FP64.  One step = one rapproximate!.  The metric is GFLOP/s of 2*m*n*l*(2q+2);
the line also carries the error against the FP64 run of the same algorithm on the same draws.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M, NCOL, S = 2**20, 512, 4096


def bytes_per_apply(ncol: int = NCOL) -> int:
    """Algorithmic bytes of one apply: read A once, write C once."""
    return 4 * (M * ncol + S * ncol)


BYTES_PER_APPLY = bytes_per_apply()
WORKLOAD = "srht+countsketch left apply, fp32, A 2^20x512 -> 4096x512"
METRIC = "sketch apply throughput (SRHT + CountSketch, HBM GB/s of algorithmic bytes)"
# DRAM bytes (read + write) per full-size launch: ncu capture of each kernel on the
# 2^20x128 case, scaled by 512/128 columns; the work splits evenly by column.
TRAFFIC_PER_LAUNCH = {"srht_fused_kernel": 2186983424, "cs_compress_kernel": 2250834944}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (clocks, throttle reasons) while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(gpus):
    """One rank per GPU over NCCL (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the
    launcher).  Without a GPU the same plumbing runs over gloo, which is how the host-side
    logic of the N > 1 path is tested."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cuda = torch.cuda.is_available()
    if world > 1:
        import datetime
        import torch.distributed as dist
        if cuda:
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    elif cuda:
        torch.cuda.set_device(0)
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    """Max over ranks (the step time every rank reports is the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, bytes_per_rank: float, seconds: float) -> float:
    """Whole-job GB/s: every rank processed `bytes_per_rank`; `seconds` is the max over ranks."""
    return world * bytes_per_rank / seconds / 1e9


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------------------
# CPU restatement of the reference (oracle/), timed on the host
# --------------------------------------------------------------------------------------
def cpu_sample(threads: int, budget_s: float, srht_draws=None, cs_draws=None):
    """Times the oracle's SRHT and CountSketch left applies on column samples of the
    workload, `threads` column blocks in parallel (ctypes releases the GIL).  Returns
    (GB/s, sample description)."""
    import concurrent.futures as cf

    import numpy as np

    from __graft_entry__ import load_oracle
    orc = load_oracle()
    rng = np.random.default_rng(2)
    if srht_draws is None:
        R1 = orc.draw_srht(rng, "left", S, M, block_size=10, dtype=np.float32)
    else:
        R1 = orc.Recipe("srht", "left", S, M, np.float32, op=srht_draws["op"], signs=srht_draws["signs"],
                        scale=srht_draws["scale"], padded=M, block_size=10)
    if cs_draws is None:
        R2 = orc.draw_count_sketch(rng, "left", S, M, dtype=np.float32)
    else:
        R2 = orc.Recipe("count_sketch", "left", S, M, np.float32, nnz=1,
                        csc=orc.CSC(S, M, np.arange(M + 1), cs_draws["rowval"], cs_draws["nzval"]))
    A = np.asfortranarray(rng.standard_normal((M, 10 * threads), dtype=np.float32))

    def run(kind, ncols):
        C = np.zeros((S, ncols), np.float32, order="F")
        cols = [(c0, min(ncols, c0 + 10)) for c0 in range(0, ncols, 10)]

        def one(c):
            c0, c1 = c
            src = A[:, (c0 % A.shape[1]):(c0 % A.shape[1]) + (c1 - c0)]
            dst = C[:, c0:c1]
            orc.mul_SA(dst, R1 if kind == "srht" else R2, src)
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(one, cols))
        return time.perf_counter() - t0

    # calibrate on one block, then size each kernel's sample to ~budget/2 seconds
    t_s = run("srht", 10) / 10
    t_c = run("count_sketch", 10) / 10
    n_s = int(max(10, min(NCOL, round(budget_s / 2 / t_s * threads / 10) * 10)))
    n_c = int(max(10, min(NCOL, round(budget_s / 2 / t_c * threads / 10) * 10)))
    ts = run("srht", n_s)
    tc = run("count_sketch", n_c)
    gbs = 4 * (M + S) * (n_s + n_c) / (ts + tc) / 1e9
    desc = (f"SRHT on {n_s} and CountSketch on {n_c} columns of a {M}-row A "
            f"({threads} thread(s), column blocks of 10 as srht.jl:240 walks them)")
    return gbs, desc, ts + tc


def sketch_config(m: int, ncol: int, world: int) -> dict:
    """The `config` of a sketch-apply line; both arms print the same one."""
    wl = WORKLOAD if (ncol, m) == (512, 2**20) else \
        WORKLOAD.replace("2^20x512", f"{m}x{ncol}").replace("512 ->", f"{ncol} ->").replace("4096x512", f"4096x{ncol}")
    return {"workload": wl, "m": m, "n": ncol, "s": S, "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 ({4 * m * ncol / 1e9:.2f} GB per A), no flush needed"}


def reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(threads, budget_s=1.0)
    vals, tot = [], 0.0
    for _ in range(args.steps):
        g, desc, dt = cpu_sample(threads, budget_s=3.0)
        vals.append(g)
        tot += dt
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * tot / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic N(0,1), seed 2",
            "config": sketch_config(M, args.cols, args.gpus),
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                             "sample": desc + "; CPU restatement in oracle/ (Julia is not installed)"},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------
# B200 arm
# --------------------------------------------------------------------------------------
def b200_arm(args):
    import ctypes

    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    from randlinearalgebra_b200 import _lib as L
    dev = torch.device("cuda", local if world > 1 else 0)
    g = torch.Generator(device=dev)
    g.manual_seed(2 + rank)
    NCOL = args.cols
    BYTES_PER_APPLY = bytes_per_apply(NCOL)
    A = torch.randn(NCOL, M, device=dev, generator=g, dtype=torch.float32).t()  # column-major 2^20 x NCOL
    srht = rla.complete_compressor(rla.SRHT(compression_dim=S, type=np.float32), A, seed=1000 + rank)
    cs = rla.complete_compressor(rla.CountSketch(compression_dim=S, type=np.float32), A, seed=2000 + rank)
    C1 = torch.zeros(NCOL, S, device=dev).t()
    C2 = torch.zeros(NCOL, S, device=dev).t()
    stream = torch.cuda.current_stream(dev)
    ctx = L.Context.get(dev.index)
    lib = L.lib()

    def apply(sk, C):
        st = lib.rla_sketch_mul_async(ctx.handle, sk.handle, 0, 0, S, NCOL, C.data_ptr(), S, 0, M, NCOL,
                                      A.data_ptr(), M, 0, 1.0, 0.0)
        L.check(st, ctx.handle)

    for _ in range(args.warmup):
        apply(srht, C1)
        apply(cs, C2)
    torch.cuda.synchronize()
    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0.record(stream)
    for k in range(K):
        ev[k][0].record(stream)
        apply(srht, C1)
        ev[k][1].record(stream)
        ev[k][2].record(stream)
        apply(cs, C2)
        ev[k][3].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms_local = t0.elapsed_time(t1)
    ms = allreduce_max(ms_local, world)
    srht_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    cs_ms = statistics.mean(e[2].elapsed_time(e[3]) for e in ev)
    value = job_throughput(world, 2 * BYTES_PER_APPLY * K, ms / 1e3)

    # correctness guard on a few columns (no oracle: S*A for a column subset must agree)
    sub = A[:, :8]
    chk = srht @ sub
    assert torch.allclose(chk, C1[:, :8], rtol=1e-5, atol=1e-4), "SRHT result changed across calls"

    # ---- end to end through the public API with pinned host buffers -------------------
    A_h = torch.empty(NCOL, M, dtype=torch.float32, pin_memory=True).t()
    A_h.copy_(A)
    Ch1 = torch.zeros(NCOL, S, dtype=torch.float32, pin_memory=True).t()
    Ch2 = torch.zeros(NCOL, S, dtype=torch.float32, pin_memory=True).t()
    e2e_steps = max(1, min(K, 3))
    rla.mul_(Ch1, srht, A_h)  # warm
    torch.cuda.synchronize()
    barrier(world)
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        rla.mul_(Ch1, srht, A_h)
        rla.mul_(Ch2, cs, A_h)
    torch.cuda.synchronize()
    e2e_s = allreduce_max((time.perf_counter() - w0) / e2e_steps, world)
    e2e = {"value": round(job_throughput(world, 2 * BYTES_PER_APPLY, e2e_s), 3), "unit": "GB/s",
           "h2d_bytes_per_step": 2 * (4 * M * NCOL + 4 * S * NCOL), "d2h_bytes_per_step": 2 * 4 * S * NCOL,
           "ms_per_step": round(e2e_s * 1e3, 3)}
    del A_h

    # ---- the metric's second half on the same GPU: config-3 RandSVD and the served mix ----
    extras = {}
    if world == 1 and not args.no_extras and (M, NCOL) == (2**20, 512):
        del A, C1, C2
        torch.cuda.empty_cache()
        r = rs_measure(rla, torch, dev, RS_M, RS_N, 3, 3, with_e2e=False)
        extras["randsvd"] = {"workload": RS_WORKLOAD, "ms_per_rapproximate": round(r["ms"], 3),
                             "tflops": round(r["flops"] / (r["ms"] / 1e3) / 1e12, 2),
                             "roofline": rs_roofline(RS_M, RS_N, r), "error": r["error"], "clocks": r["clocks"]}
        ls, svd, servers = serve_setup(rla, torch, dev, 4)
        # median of SV_REPS runs per rate and mode, as in the serving workload's own line
        curve = sv_curve(rla, torch, dev, ls, svd, servers, SV_SLO_RATES, 200, SV_REPS, seed0=20)
        for srv in servers.values():
            srv.stop()
        del ls, svd
        torch.cuda.empty_cache()
        extras["serve"] = {"workload": SV_WORKLOAD + f"; offered rates below saturation, 200 requests per rate, median of {SV_REPS} runs",
                           "curve": curve, "at_slo": sv_at_slo(curve, SV_SLO_RATES)}

    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    peak, peak_kind = peaks()
    dom_name, dom_ms = ("srht_fused_kernel", srht_ms) if srht_ms >= cs_ms else ("cs_compress_kernel", cs_ms)
    achieved = BYTES_PER_APPLY / (dom_ms / 1e3) / 1e9
    traffic = TRAFFIC_PER_LAUNCH.get(dom_name) if (M, NCOL) == (2**20, 512) else None
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 2), "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "algorithmic_bytes_per_launch": BYTES_PER_APPLY}
    kernels = {"srht": {"ms": round(srht_ms, 4), "gbs": round(BYTES_PER_APPLY / srht_ms / 1e6, 2),
                        "frac": round(BYTES_PER_APPLY / srht_ms / 1e6 / peak, 4)},
               "countsketch": {"ms": round(cs_ms, 4), "gbs": round(BYTES_PER_APPLY / cs_ms / 1e6, 2),
                               "frac": round(BYTES_PER_APPLY / cs_ms / 1e6 / peak, 4)}}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        d1 = srht.draws()
        d2 = cs.draws()
        gbs, desc, _ = cpu_sample(1, budget_s=12.0,
                                  srht_draws={"op": d1["op"], "signs": d1["signs"], "scale": srht.scale},
                                  cs_draws={"rowval": d2["rowval"], "nzval": d2["nzval"]})
        cpu = {"value": round(gbs, 4), "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": desc + "; C restatement of the reference's Julia loops (oracle/), single thread "
                                "like the reference's fwht!/SparseArrays loops"}
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic N(0,1) generated on device (torch.randn, seed 2+rank)",
            "config": sketch_config(M, NCOL, world),
            "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": 2 * K, **extras}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------------------
# RandSVD workload (mixed precision)
# --------------------------------------------------------------------------------------
RS_M, RS_N, RS_K, RS_P, RS_Q, RS_R = 65536, 8192, 256, 16, 2, 512
RS_METRIC = "RandSVD throughput (GFLOP/s of 2*m*n*l*(2q+2), split-BF16 tensor-core products)"
RS_WORKLOAD = "randsvd 65536x8192 fp32, k=256 p=16 q=2 orthogonalize, gaussian sketch"


def rs_flops(m=RS_M, n=RS_N, l=RS_K + RS_P, q=RS_Q):
    return 2.0 * m * n * l * (2 * q + 2)


def rs_problem(torch, dev, m, n, r, seed):
    """Column-major m x n Float32: U diag(i^-1.5) V' + 1e-6 N(0,1)."""
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    U = torch.linalg.qr(torch.randn(m, r, device=dev, generator=g))[0]
    V = torch.linalg.qr(torch.randn(n, r, device=dev, generator=g))[0]
    sig = torch.arange(1, r + 1, device=dev, dtype=torch.float32) ** -1.5
    At = (V * sig) @ U.t()  # n x m row-major storage = A column-major
    At.add_(torch.randn(n, m, device=dev, generator=g), alpha=1e-6)
    del U, V
    return At.t()


def rs_cpu_sample(threads_note: str, budget_s: float = 20.0):
    """FP64 RandSVD of the oracle (numpy/LAPACK, all BLAS threads) on a scaled-down instance
    of the same problem family; returns (GFLOP/s, description, seconds)."""
    import numpy as np

    from __graft_entry__ import load_oracle
    orc = load_oracle()
    rng = np.random.default_rng(3)
    m, n, l = 8192, 2048, RS_K + RS_P
    U = np.linalg.qr(rng.standard_normal((m, RS_R)))[0]
    V = np.linalg.qr(rng.standard_normal((n, RS_R)))[0]
    A = np.asfortranarray((U * np.arange(1, RS_R + 1) ** -1.5) @ V.T + 1e-6 * rng.standard_normal((m, n)))
    R = orc.draw_gaussian(rng, "right", l, n)
    t0 = time.perf_counter()
    reps = 0
    while True:
        orc.randsvd(A, R, q=RS_Q, orthogonalize=True)
        reps += 1
        if time.perf_counter() - t0 > budget_s / 2 or reps >= 5:
            break
    dt = (time.perf_counter() - t0) / reps
    fl = rs_flops(m, n, l, RS_Q)
    return fl / dt / 1e9, (f"FP64 RandSVD of the oracle (numpy/LAPACK) on an {m}x{n} instance of the same family, "
                           f"l={l}, q={RS_Q}, orthogonalized, {reps} run(s); {threads_note}"), dt


def randsvd_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    rs_cpu_sample(f"{threads} host threads", budget_s=4.0)
    vals, tot = [], 0.0
    for _ in range(max(1, min(args.steps, 3))):
        g, desc, dt = rs_cpu_sample(f"{threads} host threads")
        vals.append(g)
        tot += dt
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": RS_METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": args.gpus,
            "steps": len(vals), "warmup": 1, "ms_per_step": round(1000 * tot / len(vals), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic low-rank + noise, seed 3", "config": {"workload": RS_WORKLOAD},
            "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": round(v, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def rs_measure(rla, torch, dev, m, n, steps, warmup, rank=0, world=1, with_e2e=True):
    """Config-3 RandSVD on this GPU: timed rapproximate! calls, tensor-core GEMM kernel time,
    error against the FP64 run of the same algorithm on the same draws, and (optionally) the
    end-to-end rate with A in pinned host memory."""
    import ctypes

    import numpy as np
    from randlinearalgebra_b200 import _lib as L
    l, q = RS_K + RS_P, RS_Q
    A = rs_problem(torch, dev, m, n, min(RS_R, n), 3 + rank)
    comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=l, type=np.float32)
    rec = rla.complete_approximator(rla.RandSVD(compressor=comp, power_its=q, orthogonalize=True,
                                                precision=rla.RLA_PREC_SPLIT_BF16, factor_type=np.float32),
                                    A, seed=3000 + rank)
    ctx = L.Context.get(dev.index)
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        rla.rapproximate_(rec, A)
    lib.rla_ctx_set_timing(ctx.handle, 1)
    ms_tc, n_tc = ctypes.c_double(), ctypes.c_int64()
    L.check(lib.rla_ctx_kernel_time(ctx.handle, 0, ctypes.byref(ms_tc), ctypes.byref(n_tc)), ctx.handle)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0.record(stream)
    for _ in range(steps):
        rla.rapproximate_(rec, A)
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = allreduce_max(t0.elapsed_time(t1), world)
    L.check(lib.rla_ctx_kernel_time(ctx.handle, 0, ctypes.byref(ms_tc), ctypes.byref(n_tc)), ctx.handle)
    lib.rla_ctx_set_timing(ctx.handle, 0)
    fl = rs_flops(m, n, l, q)

    # ---- error against the FP64 run of the same algorithm on the same draws --------------
    U32, S32 = rec.U.double(), rec.S.double()
    A64 = A.t().double().t()  # column-major FP64 copy
    comp64 = rla.Gaussian(cardinality=rla.Right(), compression_dim=l, type=np.float64)
    rec64 = rla.complete_approximator(rla.RandSVD(compressor=comp64, power_its=q, orthogonalize=True), A64, seed=1)
    rec64.compressor.load_draws(vals=rec.compressor.draws()["op"].astype(np.float64))
    rla.rapproximate_(rec64, A64)
    nA = torch.linalg.norm(A64)

    def proj_err(U):
        return float(torch.linalg.norm(A64 - U @ (U.t() @ A64)) / nA)

    e32, e64 = proj_err(U32), proj_err(rec64.U)
    s_err = float(torch.linalg.norm(S32 - rec64.S) / torch.linalg.norm(rec64.S))
    del A64, rec64
    torch.cuda.empty_cache()
    out = {"ms": ms / steps, "flops": fl, "tc_ms": ms_tc.value, "tc_launches": n_tc.value, "clocks": clk,
           "error": {"proj_err_split": e32, "proj_err_fp64": e64, "proj_err_diff": abs(e32 - e64),
                     "sigma_rel_err": s_err, "tolerance": 1e-4}}
    if with_e2e:
        # ---- end to end: host A (pinned) in, factors out, through the public API ----------
        A_h = torch.empty(n, m, dtype=torch.float32, pin_memory=True).t()
        A_h.copy_(A)
        e2e_steps = 2
        rla.rapproximate_(rec, A_h)
        torch.cuda.synchronize()
        barrier(world)
        w0 = time.perf_counter()
        for _ in range(e2e_steps):
            rla.rapproximate_(rec, A_h)
            rec.U.cpu(), rec.S.cpu(), rec.V.cpu()
        e2e_s = allreduce_max((time.perf_counter() - w0) / e2e_steps, world)
        out["e2e"] = {"value": round(world * fl / e2e_s / 1e9, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 4 * m * n,
                      "d2h_bytes_per_step": 4 * (m + n) * l + 8 * l, "ms_per_step": round(e2e_s * 1e3, 3)}
        del A_h
    del A, rec
    torch.cuda.empty_cache()
    return out


def rs_roofline(m, n, r):
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        peak_bf16, peak_kind = float(pk["bf16_tflops"]), "measured"
    except Exception:
        peak_bf16, peak_kind = 1590.0, "fallback"
    l = RS_K + RS_P
    tc_avg_ms = r["tc_ms"] / max(r["tc_launches"], 1)
    tc_flops = 2.0 * m * n * l  # each of the 2q+2 products with A
    achieved = tc_flops / (tc_avg_ms / 1e3) / 1e12
    return {"bound": "tensor", "kernel": "tc_gemm_kernel", "achieved": round(achieved, 2),
            "peak": round(peak_bf16 / 3, 2), "peak_source": f"{peak_kind} bf16 dense / 3 (three BF16 products per split product)",
            "unit": "TFLOP/s", "frac": round(achieved / (peak_bf16 / 3), 4), "traffic": None,
            "launches_timed": r["tc_launches"], "avg_launch_ms": round(tc_avg_ms, 4),
            "tensor_flops_per_launch": 3 * tc_flops}


def randsvd_arm(args):
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    dev = torch.device("cuda", local if world > 1 else 0)
    m, n, l, q = args.rs_m, args.rs_n, RS_K + RS_P, RS_Q
    K = args.steps
    r = rs_measure(rla, torch, dev, m, n, K, args.warmup, rank, world)
    value = world * r["flops"] / (r["ms"] / 1e3) / 1e9
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        g, desc, _ = rs_cpu_sample(f"{os.cpu_count()} host threads")
        cpu = {"value": round(g, 3), "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": "port", "sample": desc}
    line = {"metric": RS_METRIC, "value": round(value, 2), "unit": "GFLOP/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(r["ms"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 data, bf16x3 products, f64 small factorizations",
            "data": "synthetic U diag(i^-1.5) V' + 1e-6 N(0,1) generated on device (seed 3+rank)",
            "config": {"workload": RS_WORKLOAD if (m, n) == (RS_M, RS_N) else
                       RS_WORKLOAD.replace("65536x8192", f"{m}x{n}"), "m": m, "n": n, "k": RS_K, "p": RS_P, "q": q,
                       "parallelism": f"replicas x{world}", "l2": "A is 2.15 GB (larger than L2), no flush needed"},
            "roofline": rs_roofline(m, n, r), "error": r["error"],
            "cpu_baseline": cpu, "e2e": r["e2e"], "clocks": r["clocks"], "gpu_launches_tensor_core": r["tc_launches"]}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------------------
# Plain SparseSign workload (left apply, Float64)
# --------------------------------------------------------------------------------------
SS_M, SS_N, SS_S, SS_NNZ = 4096, 256, 512, 8
SS_WORKLOAD = "sparse_sign left apply, fp64, A 4096x256 -> 512x256, nnz=8"


def sparse_sign_arm(args):
    """SparseSign Left, Float64, A 4096x256 ~ N(0,1) compressed to 512x256 with 8 nonzeros
    per column.  One step = one S*A through the C ABI on device-resident A.  A and C (9.4 MB)
    stay in L2 between steps, so the rate is an L2 rate; the line says so."""
    import ctypes

    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    from randlinearalgebra_b200 import _lib as L
    dev = torch.device("cuda", local if world > 1 else 0)
    g = torch.Generator(device=dev)
    g.manual_seed(1 + rank)
    A = torch.randn(SS_N, SS_M, device=dev, generator=g, dtype=torch.float64).t()
    S = rla.complete_compressor(rla.SparseSign(cardinality=rla.Left(), compression_dim=SS_S, nnz=SS_NNZ,
                                               type=np.float64), A, seed=1 + rank)
    C = torch.zeros(SS_N, SS_S, device=dev, dtype=torch.float64).t()
    ctx = L.Context.get(dev.index)
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)

    def apply():
        L.check(lib.rla_sketch_mul_async(ctx.handle, S.handle, 0, 0, SS_S, SS_N, C.data_ptr(), SS_S, 0, SS_M, SS_N,
                                         A.data_ptr(), SS_M, 0, 1.0, 0.0), ctx.handle)

    for _ in range(args.warmup):
        apply()
    K = args.steps
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0.record(stream)
    for _ in range(K):
        apply()
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = allreduce_max(t0.elapsed_time(t1), world) / K
    nbytes = 8 * (SS_M * SS_N + SS_S * SS_N)
    value = world * nbytes / (ms / 1e3) / 1e9
    # end to end: host A in, host C out
    A_h = torch.empty(SS_N, SS_M, dtype=torch.float64, pin_memory=True).t()
    A_h.copy_(A)
    C_h = torch.zeros(SS_N, SS_S, dtype=torch.float64, pin_memory=True).t()
    rla.mul_(C_h, S, A_h)
    w0 = time.perf_counter()
    for _ in range(10):
        rla.mul_(C_h, S, A_h)
    e2e_s = allreduce_max((time.perf_counter() - w0) / 10, world)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from __graft_entry__ import load_oracle
        orc = load_oracle()
        d = S.draws()
        R = orc.Recipe("sparse_sign", "left", SS_S, SS_M, np.float64, nnz=SS_NNZ,
                       csc=orc.CSC(SS_S, SS_M, np.arange(0, SS_M * SS_NNZ + 1, SS_NNZ), d["rowval"], d["nzval"]))
        Ah = A.cpu().numpy()
        Ch = np.zeros((SS_S, SS_N), order="F")
        reps, w0 = 0, time.perf_counter()
        while time.perf_counter() - w0 < 3.0:
            orc.mul_SA(Ch, R, Ah)
            reps += 1
        dt = (time.perf_counter() - w0) / reps
        cpu = {"value": round(nbytes / dt / 1e9, 4), "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": f"the whole workload, {reps} applies; C restatement of SparseArrays' CSC loop (oracle/)"}
    line = {"metric": "SparseSign apply throughput (GB/s of algorithmic bytes 8*(m*n + s*n))", "value": round(value, 2),
            "unit": "GB/s", "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": round(ms, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic N(0,1) generated on device (seed 1+rank)",
            "config": {"workload": SS_WORKLOAD, "m": SS_M, "n": SS_N, "s": SS_S, "nnz": SS_NNZ,
                       "parallelism": f"replicas x{world}",
                       "l2": "A and C (9.4 MB) stay in L2 between steps: an L2 rate, not an HBM rate"},
            "roofline": {"bound": "hbm", "kernel": "compress_contig_kernel", "achieved": round(value / world, 2),
                         "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                         "frac": round(value / world / peak, 4), "traffic": None,
                         "note": "L2-resident workload; the fraction is of HBM peak for scale only"},
            "cpu_baseline": cpu,
            "e2e": {"value": round(world * nbytes / e2e_s / 1e9, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": 8 * SS_M * SS_N, "d2h_bytes_per_step": 8 * SS_S * SS_N,
                    "ms_per_step": round(e2e_s * 1e3, 4)},
            "clocks": clk, "gpu_launches": K}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------------------
# IHS workload
# --------------------------------------------------------------------------------------
IHS_M, IHS_N = 2**18, 512
IHS_METRIC = "IHS iterations/s (sketch, sketched Cholesky solve, fused residual/gradient pass)"
# kernel launches of one IHS step at the default shape (ncu launch list, profiles/)
IHS_LAUNCHES_PER_STEP = 29


def ihs_arm(args):
    """rsolve!(IHS) on A 2^18 x 512 Float32 ~ N(0,1), b = A x* + 1e-3 N(0,1), SparseSign Left
    s = 4n = 2048, nnz = 8 (the largest least-squares request shape of the serving workload).
    One step = one IHS iteration: update_compressor!, S*A, the sketched Cholesky solve, x += u,
    and the fused pass r -= A u, ||b - Ax||, g = A'r."""
    import ctypes

    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    from randlinearalgebra_b200 import _lib as L
    dev = torch.device("cuda", local if world > 1 else 0)
    m, n = args.ihs_m, args.ihs_n
    s = 4 * n
    g = torch.Generator(device=dev)
    g.manual_seed(6 + rank)
    A = torch.randn(n, m, device=dev, generator=g, dtype=torch.float32).t()
    xs = torch.randn(n, device=dev, generator=g, dtype=torch.float32)
    b = A @ xs + 1e-3 * torch.randn(m, device=dev, generator=g, dtype=torch.float32)
    x = torch.zeros(n, device=dev, dtype=torch.float32)
    solver = rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=s, nnz=8, type=np.float32),
                                         log=rla.BasicLogger(max_it=args.steps + args.warmup + 1)),
                                 x, A, b, seed=6000 + rank)
    ctx = L.Context.get(dev.index)
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)
    cargs = (ctx.handle, solver._h, A.data_ptr(), A.stride(1), b.data_ptr())
    vecs = (x.data_ptr(), solver.residual_vec.data_ptr(), solver.gradient_vec.data_ptr())
    L.check(lib.rla_ihs_start(*cargs, *vecs), ctx.handle)
    for _ in range(args.warmup):
        L.check(lib.rla_ihs_step(*cargs, *vecs), ctx.handle)
    torch.cuda.synchronize()
    lib.rla_ctx_set_timing(ctx.handle, 1)
    for c in (1, 2):
        lib.rla_ctx_kernel_time(ctx.handle, c, ctypes.byref(ctypes.c_double()), ctypes.byref(ctypes.c_int64()))
    K = args.steps
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0.record(stream)
    for _ in range(K):
        L.check(lib.rla_ihs_step(*cargs, *vecs), ctx.handle)
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = allreduce_max(t0.elapsed_time(t1), world)
    kt = {}
    for c in (1, 2):
        tot, cnt = ctypes.c_double(), ctypes.c_int64()
        L.check(lib.rla_ctx_kernel_time(ctx.handle, c, ctypes.byref(tot), ctypes.byref(cnt)), ctx.handle)
        kt[c] = (tot.value / max(cnt.value, 1), cnt.value)
    lib.rla_ctx_set_timing(ctx.handle, 0)
    ef, eg = solver._errors()
    value = world * K / (ms / 1e3)
    # least-squares optimality of the final iterate: ||A'(b - Ax)|| relative to ||A'b||
    grad_rel = float(torch.linalg.vector_norm(A.t() @ (b - A @ x)) / torch.linalg.vector_norm(A.t() @ b))

    # ---- end to end: host A, b in (pinned), x out, through rsolve_ ------------------------
    A_h = torch.empty(n, m, dtype=torch.float32, pin_memory=True).t()
    A_h.copy_(A)
    b_h = b.cpu().pin_memory()
    e2e_it = max(3, min(K, 10))
    x_h = torch.zeros(n, dtype=torch.float32, pin_memory=True)
    sol_h = rla.complete_solver(rla.IHS(compressor=rla.SparseSign(compression_dim=s, nnz=8, type=np.float32),
                                        log=rla.BasicLogger(max_it=e2e_it)), x_h, A_h, b_h, seed=7000 + rank)
    torch.cuda.synchronize()
    barrier(world)
    w0 = time.perf_counter()
    rla.rsolve_(sol_h, x_h, A_h, b_h)
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - w0, world)
    e2e = {"value": round(world * e2e_it / e2e_s, 3), "unit": "iterations/s",
           "h2d_bytes_per_step": round(4 * (m * n + m + n) / e2e_it), "d2h_bytes_per_step": round(4 * n / e2e_it + 24),
           "ms_per_step": round(e2e_s * 1e3 / e2e_it, 3),
           "note": f"one rsolve_ of {e2e_it} iterations from pinned host A, b, x (A copied once per solve)"}
    del A_h
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    pass_ms, pass_n = kt[1]
    pass_bytes = 4 * (m * n + 3 * m + 2 * n)
    achieved = pass_bytes / (pass_ms / 1e3) / 1e9
    sk_ms, sk_n = kt[2]
    sk_bytes = 4 * (m * n + s * n)
    roofline = {"bound": "hbm", "kernel": "ihs_pass_kernel", "achieved": round(achieved, 2), "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                "algorithmic_bytes_per_launch": pass_bytes, "avg_launch_ms": round(pass_ms, 4),
                "launches_timed": pass_n}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = ihs_cpu_sample(m, n, s)
    line = {"metric": IHS_METRIC, "value": round(value, 3), "unit": "iterations/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (Gram, Cholesky and triangular solves f64)",
            "data": "synthetic A ~ N(0,1), b = A x* + 1e-3 N(0,1), generated on device (seed 6+rank)",
            "config": {"workload": f"ihs: A {m}x{n} f32, sparse_sign left s={s} nnz=8", "m": m, "n": n, "s": s,
                       "parallelism": f"replicas x{world}", "l2": f"A is {4 * m * n / 1e9:.2f} GB (larger than L2)"},
            "roofline": roofline,
            "kernels": {"ihs_pass": {"ms": round(pass_ms, 4), "gbs": round(achieved, 1),
                                     "frac": round(achieved / peak, 4)},
                        "sketch_apply": {"ms": round(sk_ms, 4), "gbs": round(sk_bytes / (sk_ms / 1e3) / 1e9, 1),
                                         "frac": round(sk_bytes / (sk_ms / 1e3) / 1e9 / peak, 4)}},
            "solution": {"full_residual": ef, "ls_gradient": eg, "rel_normal_eq_residual": grad_rel},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": IHS_LAUNCHES_PER_STEP * K}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def ihs_cpu_sample(m, n, s, iters=2):
    """The oracle's rsolve! (float64 numpy + the C SparseSign loop, 1 thread for the sparse
    product, all cores for numpy BLAS/LAPACK) for `iters` iterations of the same shape."""
    import numpy as np

    from __graft_entry__ import load_oracle
    orc = load_oracle()
    rng = np.random.default_rng(6)
    A = np.asfortranarray(rng.standard_normal((m, n), dtype=np.float32))
    b = (A @ rng.standard_normal(n).astype(np.float32)).astype(np.float32)
    sk = [orc.draw_sparse_sign(rng, "left", s, m, 8, dtype=np.float32) for _ in range(iters)]
    t0 = time.perf_counter()
    orc.ihs_rsolve(A, b, np.zeros(n, np.float32), lambda i: sk[i - 1], max_it=iters + 1, threshold=-1.0)
    dt = time.perf_counter() - t0
    return {"value": round(iters / dt, 4), "unit": "iterations/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{iters} iterations of the oracle's rsolve! on the same {m}x{n} shape (float64 numpy "
                      "BLAS/LAPACK on all cores, single-threaded C SparseSign product)"}


# --------------------------------------------------------------------------------------
# Sampling workload
# --------------------------------------------------------------------------------------
SMP_METRIC = "sampling compressor step (update_compressor! with L2Norm weights + draw, then S*A), GB/s"


def sampling_arm(args):
    """Sampling(Left, compression_dim = 4096, L2Norm(replace = false)) on A 2^20 x 512 FP32 ~ N(0,1).
    One step = update_compressor!(S, x, A, b) (squared row norms of A, Efraimidis-Spirakis keys,
    radix select of the 4096 smallest, expand plan) followed by mul!(C, S, A) (row gather).
    Algorithmic bytes per step: 4*m*n (A read by the weights pass) + 2*4*s*n (gather)."""
    import ctypes

    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    from randlinearalgebra_b200 import _lib as L
    dev = torch.device("cuda", local if world > 1 else 0)
    m, n, s = M, args.cols, S
    g = torch.Generator(device=dev)
    g.manual_seed(7 + rank)
    A = torch.randn(n, m, device=dev, generator=g, dtype=torch.float32).t()
    x = torch.zeros(n, device=dev)
    b = torch.zeros(m, device=dev)
    Sm = rla.complete_compressor(rla.Sampling(compression_dim=s, distribution=rla.L2Norm()), A, seed=8000 + rank)
    C = torch.zeros(n, s, device=dev).t()
    ctx = L.Context.get(dev.index)
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)

    def step():
        rla.update_compressor_(Sm, x, A, b)
        rla.mul_(C, Sm, A)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lib.rla_ctx_set_timing(ctx.handle, 1)
    lib.rla_ctx_kernel_time(ctx.handle, 3, ctypes.byref(ctypes.c_double()), ctypes.byref(ctypes.c_int64()))
    K = args.steps
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0.record(stream)
    for _ in range(K):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = allreduce_max(t0.elapsed_time(t1), world)
    tot, cnt = ctypes.c_double(), ctypes.c_int64()
    L.check(lib.rla_ctx_kernel_time(ctx.handle, 3, ctypes.byref(tot), ctypes.byref(cnt)), ctx.handle)
    lib.rla_ctx_set_timing(ctx.handle, 0)
    bytes_step = 4 * m * n + 2 * 4 * s * n
    value = job_throughput(world, bytes_step * K, ms / 1e3)
    # correctness guard: the gathered rows are the sampled rows of A
    idx = torch.from_numpy(Sm.idx).to(dev)
    assert torch.equal(C, A[idx, :]), "gather differs from A[idx, :]"

    # ---- end to end: pinned host A in, C out, one step through the public API ------------
    A_h = torch.empty(n, m, dtype=torch.float32, pin_memory=True).t()
    A_h.copy_(A)
    C_h = torch.zeros(n, s, dtype=torch.float32, pin_memory=True).t()
    torch.cuda.synchronize()
    barrier(world)
    w0 = time.perf_counter()
    Ad = A_h.to(dev, non_blocking=True)
    rla.update_compressor_(Sm, x, Ad, b)
    rla.mul_(C_h, Sm, Ad)
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - w0, world)
    e2e = {"value": round(job_throughput(world, bytes_step, e2e_s), 3), "unit": "GB/s",
           "h2d_bytes_per_step": 4 * m * n, "d2h_bytes_per_step": 4 * s * n, "ms_per_step": round(e2e_s * 1e3, 3)}
    del A_h, Ad
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    w_ms = tot.value / max(cnt.value, 1)
    w_gbs = 4 * m * n / (w_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "sq_norms_rows_kernel", "achieved": round(w_gbs, 2), "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(w_gbs / peak, 4), "traffic": None,
                "algorithmic_bytes_per_launch": 4 * m * n, "avg_launch_ms": round(w_ms, 4),
                "launches_timed": cnt.value}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = sampling_cpu_sample(m, s)
    line = {"metric": SMP_METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (weights f64)",
            "data": "synthetic N(0,1) generated on device (seed 7+rank)",
            "config": {"workload": f"sampling left L2Norm without replacement, A {m}x{n} f32 -> {s}x{n}",
                       "m": m, "n": n, "s": s, "parallelism": f"replicas x{world}",
                       "l2": "A is 2.15 GB (larger than L2), no flush needed"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def sampling_cpu_sample(m, s, ncol=64):
    """The oracle's restatement on the host: squared row norms (numpy, all cores), weighted
    sampling without replacement (numpy Generator.choice), the row gather, on `ncol` columns."""
    import numpy as np

    from __graft_entry__ import load_oracle
    orc = load_oracle()
    rng = np.random.default_rng(7)
    A = np.asfortranarray(rng.standard_normal((m, ncol), dtype=np.float32))
    t0 = time.perf_counter()
    w = orc.l2norm_weights(A, "left")
    R = orc.draw_sampling(rng, "left", s, m, replace=False, weights=w, dtype=np.float32)
    C = np.zeros((s, ncol), np.float32, order="F")
    orc.mul_SA(C, R, A)
    dt = time.perf_counter() - t0
    return {"value": round((4 * m * ncol + 8 * s * ncol) / dt / 1e9, 4), "unit": "GB/s", "cores": os.cpu_count(),
            "kind": "port", "sample": f"one update + apply on {ncol} of the columns of the {m}-row A (numpy)"}


# --------------------------------------------------------------------------------------
# Kaczmarz workload
# --------------------------------------------------------------------------------------
KZ_METRIC = "block Kaczmarz iterations/s (sampled rows, LQ block solve)"
# kernel launches of one step: redraw (Sampling: keys, 8 radix hist/pick pairs, count, scan,
# write, plan), S*A and S*b gathers, residual (2), Gram (2), zero check, equilibration (2),
# Cholesky (1 CTA for s < 128), triangular solve, mask, update
KZ_LAUNCHES_PER_STEP = 15


def kaczmarz_arm(args):
    """rsolve!(Kaczmarz) on A 2^18 x 512 FP32 ~ N(0,1), b = A x*, with a Sampling(Left,
    compression_dim = 64, Uniform(replace = false)) compressor: one step = one iteration
    (update_compressor!, the 64 sampled rows and entries of b, the LQ block solve through the
    FP64 Cholesky factor of their Gram matrix, x += u)."""
    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    from randlinearalgebra_b200 import _lib as L
    dev = torch.device("cuda", local if world > 1 else 0)
    m, n, s = args.ihs_m, args.ihs_n, 64
    g = torch.Generator(device=dev)
    g.manual_seed(9 + rank)
    A = torch.randn(n, m, device=dev, generator=g, dtype=torch.float32).t()
    b = A @ torch.randn(n, device=dev, generator=g, dtype=torch.float32)
    x = torch.zeros(n, device=dev, dtype=torch.float32)
    solver = rla.complete_solver(rla.Kaczmarz(compressor=rla.Sampling(compression_dim=s,
                                                                      distribution=rla.Uniform()),
                                              log=rla.BasicLogger(max_it=10)), x, A, b, seed=9000 + rank)
    ctx = solver._ctx
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)
    cargs = (ctx.handle, solver._h, A.data_ptr(), A.stride(1), b.data_ptr(), x.data_ptr(), None)
    L.check(lib.rla_proj_start(*cargs), ctx.handle)
    for _ in range(args.warmup):
        L.check(lib.rla_proj_step(*cargs), ctx.handle)
    K = args.steps
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    h0 = time.perf_counter()
    t0.record(stream)
    for _ in range(K):
        L.check(lib.rla_proj_step(*cargs), ctx.handle)
    t1.record(stream)
    torch.cuda.synchronize()
    host_s = time.perf_counter() - h0
    clk = clocks.stop()
    barrier(world)
    ms = allreduce_max(t0.elapsed_time(t1), world)
    value = world * K / (ms / 1e3)
    res = float(torch.linalg.vector_norm(b - A @ x) / torch.linalg.vector_norm(b))
    # end to end: rsolve_ with pinned host A, b, x (A copied once per solve)
    A_h = torch.empty(n, m, dtype=torch.float32, pin_memory=True).t()
    A_h.copy_(A)
    b_h = b.cpu().pin_memory()
    x_h = torch.zeros(n, dtype=torch.float32, pin_memory=True)
    e2e_it = 50
    sol_h = rla.complete_solver(rla.Kaczmarz(compressor=rla.Sampling(compression_dim=s, distribution=rla.Uniform()),
                                             log=rla.BasicLogger(max_it=e2e_it)), x_h, A_h, b_h, seed=9500 + rank)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    rla.rsolve_(sol_h, x_h, A_h, b_h)
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - w0, world)
    e2e = {"value": round(world * e2e_it / e2e_s, 3), "unit": "iterations/s",
           "h2d_bytes_per_step": round(4 * (m * n + m + n) / e2e_it), "d2h_bytes_per_step": round(4 * n / e2e_it + 8),
           "ms_per_step": round(e2e_s * 1e3 / e2e_it, 3),
           "note": f"one rsolve_ of {e2e_it} iterations (FullResidual checked every iteration: a pass over A)"}
    del A_h
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = kaczmarz_cpu_sample(m, n, s)
    line = {"metric": KZ_METRIC, "value": round(value, 2), "unit": "iterations/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (Gram, Cholesky and solves f64)",
            "data": "synthetic A ~ N(0,1), b = A x* generated on device (seed 9+rank)",
            "config": {"workload": f"kaczmarz: A {m}x{n} f32, sampling left s={s} uniform without replacement",
                       "m": m, "n": n, "s": s, "parallelism": f"replicas x{world}",
                       "host_ms_per_step": round(host_s * 1e3 / K, 4)},
            "roofline": {"bound": "latency", "note": "each step moves ~4*s*n bytes; the step is a chain of 15 "
                         "small launches", "achieved": None, "peak": None, "frac": None, "traffic": None},
            "solution": {"rel_residual_after_warmup_and_steps": res},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": KZ_LAUNCHES_PER_STEP * K}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def kaczmarz_cpu_sample(m, n, s, iters=200):
    """The oracle's rsolve! (numpy float64, LAPACK QR for the LQ block) on the same shape."""
    import numpy as np

    from __graft_entry__ import load_oracle
    orc = load_oracle()
    rng = np.random.default_rng(9)
    A = np.asfortranarray(rng.standard_normal((m, n), dtype=np.float32))
    b = A @ rng.standard_normal(n).astype(np.float32)
    sk = [orc.draw_sampling(rng, "left", s, m, replace=False, dtype=np.float32) for _ in range(iters)]
    t0 = time.perf_counter()
    orc.kaczmarz_rsolve(A, b, np.zeros(n, np.float32), lambda i: sk[i - 1], max_it=iters + 1, threshold=-1.0,
                        error="compressed")
    dt = time.perf_counter() - t0
    return {"value": round(iters / dt, 3), "unit": "iterations/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{iters} iterations of the oracle's Kaczmarz rsolve! (CompressedResidual, so no full pass "
                      f"over A per iteration) on the same {m}x{n} shape"}


# --------------------------------------------------------------------------------------
# Batched RandSVD workload
# --------------------------------------------------------------------------------------
BT_COUNT = 512
BT_METRIC = "batched RandSVD throughput (instances/s; grouped launches in a CUDA graph)"
BT_WORKLOAD = ("batched randsvd: 512 fp32 instances, m~U[2^12,2^16], n~U[64,1024], k in {16,32,64}, "
               "s_i = 0.9^i + 1e-6 N(0,1), gaussian sketch, p=0, q=0")


def bt_shapes(count, seed=4):
    import numpy as np
    rng = np.random.default_rng(seed)
    ms = rng.integers(2**12, 2**16 + 1, size=count)
    ns = rng.integers(64, 1025, size=count)
    ks = rng.choice([16, 32, 64], size=count)
    return [(int(m), int(n), int(min(k, n))) for m, n, k in zip(ms, ns, ks)]


def bt_matrix(torch, dev, m, n, g):
    """m x n Float32 column-major: U diag(0.9^i) V' + 1e-6 N(0,1), U and V orthonormal with
    min(n, 160) columns (0.9^160 < 1e-7, below the noise)."""
    r = min(n, 160)
    U = torch.linalg.qr(torch.randn(m, r, device=dev, generator=g))[0]
    V = torch.linalg.qr(torch.randn(n, r, device=dev, generator=g))[0]
    s = 0.9 ** torch.arange(r, device=dev, dtype=torch.float32)
    At = (V * s) @ U.t()
    At.add_(torch.randn(n, m, device=dev, generator=g), alpha=1e-6)
    return At.t()


def batched_arm(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    dev = torch.device("cuda", local if world > 1 else 0)
    shapes = bt_shapes(args.batch_count)
    g = torch.Generator(device=dev)
    g.manual_seed(4 + rank)
    As = [bt_matrix(torch, dev, m, n, g) for (m, n, k) in shapes]
    ks = [k for (_, _, k) in shapes]
    seeds = [4000 + 7 * i + 100000 * rank for i in range(len(shapes))]
    bytes_alg = sum(4 * 2 * m * n for (m, n, _) in shapes)   # A read twice (A*Omega, A'Q)
    flops = sum(4.0 * m * n * k for (m, n, k) in shapes)
    t_plan = time.perf_counter()
    prec = rla.RLA_PREC_SPLIT_BF16 if args.batch_precision == "split" else rla.RLA_PREC_NATIVE
    B = rla.RandSVDBatch(As, ks, seeds, autotune=not args.no_autotune, precision=prec)
    t_plan = time.perf_counter() - t_plan
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        B.run()
    torch.cuda.synchronize()
    K = args.steps
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    barrier(world)
    clocks.start()
    t0.record(stream)
    for _ in range(K):
        B.run()
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = allreduce_max(t0.elapsed_time(t1) / K, world)
    n_inst = len(shapes)
    value = world * n_inst / (ms / 1e3)

    # ---- plain path: one rapproximate! (its own launch sequence) per instance ---------------
    def plain_once():
        out = []
        for A, k, sd in zip(As, ks, seeds):
            comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=k, type=np.float32)
            out.append(rla.rapproximate(rla.RandSVD(compressor=comp, factor_type=np.float32, precision=prec), A,
                                        seed=sd))
        return out
    plain_once()
    torch.cuda.synchronize()
    p0 = time.perf_counter()
    recs = plain_once()
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - p0

    # ---- error on a sample against the FP64 run of the same algorithm on the same draws --------
    errs = []
    for i in range(0, n_inst, max(1, n_inst // 12)):
        A64 = As[i].t().double().t()
        comp = rla.Gaussian(cardinality=rla.Right(), compression_dim=ks[i])
        r64 = rla.complete_approximator(rla.RandSVD(compressor=comp), A64, seed=1)
        r64.compressor.load_draws(vals=recs[i].compressor.draws()["op"].astype(np.float64))
        rla.rapproximate_(r64, A64)
        U = B.U[i].double()
        nA = torch.linalg.norm(A64)
        e_b = float(torch.linalg.norm(A64 - U @ (U.t() @ A64)) / nA)
        e_r = float(torch.linalg.norm(A64 - r64.U @ (r64.U.t() @ A64)) / nA)
        s_err = float(torch.linalg.norm(B.S[i] - r64.S) / torch.linalg.norm(r64.S))
        errs.append((abs(e_b - e_r), s_err))
        del A64, r64
    del recs

    # ---- end to end: host inputs in, factors out -----------------------------------------
    e2e = None
    try:
        Ah = [torch.empty(n, m, dtype=torch.float32, pin_memory=True).t() for (m, n, _) in shapes]
        for a, h in zip(As, Ah):
            h.copy_(a)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for a, h in zip(As, Ah):
            a.copy_(h, non_blocking=True)
        B.run()
        outs = [(u.cpu(), s_.cpu(), v.cpu()) for u, s_, v in zip(B.U, B.S, B.V)]
        e2e_s = time.perf_counter() - w0
        e2e = {"value": round(world * n_inst / e2e_s, 3), "unit": "instances/s",
               "h2d_bytes_per_step": sum(4 * m * n for (m, n, _) in shapes),
               "d2h_bytes_per_step": sum(4 * (m + n) * k + 8 * k for (m, n, k) in shapes),
               "ms_per_step": round(e2e_s * 1e3, 3)}
        del Ah, outs
    except RuntimeError as ex:  # host memory for pinned copies of every A
        e2e = {"unavailable": f"pinned host copies of all inputs: {ex}"[:200]}
    barrier(world)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    gbs = bytes_alg / (ms / 1e3) / 1e9
    tiles = {c: dict(zip(("rows_a_omega", "cols_at_q", "chunk_at_q"), B.tiles(c))) for c in range(3)}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from __graft_entry__ import load_oracle
        orc = load_oracle()
        idx = list(range(0, n_inst, max(1, n_inst // 8)))
        c0 = time.perf_counter()
        for i in idx:
            A = As[i].cpu().numpy().astype(np.float64)
            R = orc.Recipe("gaussian", "right", A.shape[1], ks[i], np.float64,
                           dense_op=np.random.default_rng(i).standard_normal((A.shape[1], ks[i])) / np.sqrt(ks[i]),
                           scale=1.0 / np.sqrt(ks[i]))
            orc.randsvd(A, R)
        cdt = (time.perf_counter() - c0) / len(idx)
        cpu = {"value": round(1.0 / cdt, 3), "unit": "instances/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"FP64 RandSVD of the oracle (numpy/LAPACK, all BLAS threads) on {len(idx)} of the instances"}
    line = {"metric": BT_METRIC, "value": round(value, 2), "unit": "instances/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("f32 data, split-bf16 tensor-core passes over A (k <= 64), f64 small factorizations"
                      if args.batch_precision == "split" else "f32 data, f32 products, f64 small factorizations"),
            "data": "synthetic low-rank + noise generated on device (seed 4+rank)",
            "config": {"workload": BT_WORKLOAD if n_inst == BT_COUNT else BT_WORKLOAD.replace("512", str(n_inst)),
                       "instances": n_inst, "parallelism": f"replicas x{world}",
                       "l2": f"{bytes_alg / 2 / 1e9:.1f} GB of A per pass, larger than L2"},
            "roofline": {"bound": "hbm", "kernel": "whole batch (grouped launches)", "achieved": round(gbs, 2),
                         "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": round(gbs / peak, 4),
                         "traffic": None, "algorithmic_bytes_per_step": bytes_alg, "gflops": round(flops / ms / 1e6, 1)},
            "plain": {"instances_per_s": round(n_inst / plain_s, 2), "ms": round(plain_s * 1e3, 2),
                      "speedup_batched": round(plain_s * 1e3 / ms, 2)},
            "error": {"max_proj_err_diff": max(e[0] for e in errs), "max_sigma_rel_err": max(e[1] for e in errs),
                      "instances_checked": len(errs), "tolerance": 1e-4},
            "autotuned_tiles": tiles, "plan_s": round(t_plan, 3),
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------------------
# Serving workload
# --------------------------------------------------------------------------------------
SV_METRIC = "served requests/s (60% sketch-and-solve LS, 40% RandSVD; continuous batching)"
SV_REPS = 3  # runs per arrival rate and mode; the median is reported
SV_WORKLOAD = ("serving: Poisson arrivals, 60% LS m~U[2^14,2^18] n~U[32,512] s=4n SparseSign nnz=8, "
               "40% RandSVD m<=32768 n<=4096 k in {32,64,128}; device-resident inputs (H2D excluded)")


def sv_pool(torch, dev, n_ls, n_svd, seed=5):
    import numpy as np
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    ls, svd = [], []
    for i in range(n_ls):
        m, n = int(rng.integers(2**14, 2**18 + 1)), int(rng.integers(32, 513))
        A = torch.randn(n, m, device=dev, generator=g).t()
        x0 = torch.randn(n, device=dev, generator=g)
        b = A @ x0 + 1e-3 * torch.randn(m, device=dev, generator=g)
        ls.append((A, b, 50000 + i))
    for i in range(n_svd):
        m, n = int(rng.integers(4096, 32769)), int(rng.integers(256, 4097))
        k = int(rng.choice([32, 64, 128]))
        svd.append((bt_matrix(torch, dev, m, n, g), min(k, n), 60000 + i))
    return ls, svd


def sv_warm(torch, dev, ls, svd, srv):
    """Submit every pool problem once and wait: builds the server's sketch cache for all of them."""
    outs, n = [], 0
    for i, (A, b, sd) in enumerate(ls):
        x = torch.empty(A.shape[1], dtype=torch.float32, device=dev)
        outs.append(x)
        srv.submit_ls(A, b, x, sd, n)
        n += 1
    for A, k, sd in svd:
        m, nn = A.shape
        U = torch.empty(k, m, dtype=torch.float32, device=dev).t()
        S = torch.empty(k, dtype=torch.float64, device=dev)
        V = torch.empty(k, nn, dtype=torch.float32, device=dev).t()
        outs.append((U, S, V))
        srv.submit_svd(A, k, U, S, V, sd, n)
        n += 1
    done = 0
    while done < n:
        for tag, _, st in srv.poll():
            if st != 0:
                raise RuntimeError(f"warm-up request {tag} failed with status {st}: {srv.last_error()}")
            done += 1
        time.sleep(2e-4)


def sv_run(rla, torch, dev, ls, svd, lam, nreq, srv, seed, ls_frac=0.6):
    """Submit nreq requests with Poisson(lam) arrivals to the running server srv; returns
    (throughput, p50, p99)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    kinds = rng.random(nreq) < ls_frac
    picks = [int(rng.integers(0, len(ls) if k else len(svd))) for k in kinds]
    arrivals = np.cumsum(rng.exponential(1.0 / lam, size=nreq))
    outs, sched, lat = {}, {}, {}
    t0 = time.perf_counter()
    i = 0
    while len(lat) < nreq:
        now = time.perf_counter() - t0
        while i < nreq and arrivals[i] <= now:
            if kinds[i]:
                A, b, sd = ls[picks[i]]
                x = torch.empty(A.shape[1], dtype=torch.float32, device=dev)
                outs[i] = (x,)
                srv.submit_ls(A, b, x, sd, i)
            else:
                A, k, sd = svd[picks[i]]
                m, n = A.shape
                U = torch.empty(k, m, dtype=torch.float32, device=dev).t()
                S = torch.empty(k, dtype=torch.float64, device=dev)
                V = torch.empty(k, n, dtype=torch.float32, device=dev).t()
                outs[i] = (U, S, V)
                srv.submit_svd(A, k, U, S, V, sd, i)
            sched[i] = now - arrivals[i]  # submission lag behind the scheduled arrival
            i += 1
        for tag, l, st in srv.poll():
            if st != 0:
                raise RuntimeError(f"request {tag} failed with status {st}: {srv.last_error()}")
            lat[tag] = l + sched[tag]
            outs.pop(tag, None)
        if i < nreq:
            time.sleep(min(2e-4, max(0.0, arrivals[i] - (time.perf_counter() - t0))))
        else:
            time.sleep(2e-4)
    t_end = time.perf_counter() - t0
    ls_lat = sorted(lat.values())
    thr = nreq / (t_end - arrivals[0])
    return thr, float(np.percentile(ls_lat, 50)), float(np.percentile(ls_lat, 99))


SV_SLO_RATES = [100, 200, 400, 700, 1000, 1500]  # offered rates of the latency-throughput curve


def sv_curve(rla, torch, dev, ls, svd, servers, rates, nreq, reps, seed0=10):
    """Latency-throughput curve of both modes: per offered rate, `reps` runs of nreq requests
    and, field by field, the median over the runs of the throughput, p50 and p99 latency.
    Returns {"batched": {rate: ...}, "plain": {rate: ...}}."""
    import numpy as np
    res = {"batched": {}, "plain": {}}
    for lam in rates:
        for mode, plain in (("batched", False), ("plain", True)):
            runs = [sv_run(rla, torch, dev, ls, svd, lam, nreq, servers[plain], seed0 + lam + 1000 * r)
                    for r in range(reps)]
            thr, p50, p99 = (float(np.median([x[i] for x in runs])) for i in range(3))
            res[mode][lam] = {"req_per_s": round(thr, 1), "p50_ms": round(1e3 * p50, 3), "p99_ms": round(1e3 * p99, 3),
                              "runs_req_per_s": [round(x[0], 1) for x in runs],
                              "runs_p99_ms": [round(1e3 * x[2], 3) for x in runs]}
    return res


def sv_at_slo(curve, rates):
    """Throughput at a fixed p99 SLO.  The SLO is twice the plain path's p99 at the lowest
    offered rate (its service latency when nothing queues); each mode's figure is the highest
    measured throughput among the rates whose p99 stays within the SLO."""
    slo = 2.0 * curve["plain"][rates[0]]["p99_ms"]
    out = {"p99_slo_ms": round(slo, 3)}
    for mode in ("batched", "plain"):
        ok = [curve[mode][r]["req_per_s"] for r in rates if curve[mode][r]["p99_ms"] <= slo]
        out[f"{mode}_req_per_s"] = max(ok) if ok else None
    b, pl = out["batched_req_per_s"], out["plain_req_per_s"]
    out["ratio"] = None if (b is None or not pl) else round(b / pl, 2)
    return out


def serve_setup(rla, torch, dev, slots, rank=0):
    """Pool of device-resident problems and one warmed, long-running server per mode."""
    ls, svd = sv_pool(torch, dev, 24, 16, seed=5 + rank)
    torch.cuda.synchronize()
    servers = {False: rla.Server(slots=slots, max_group=32, plain=False),
               True: rla.Server(slots=1, max_group=32, plain=True)}
    for srv in servers.values():
        sv_warm(torch, dev, ls, svd, srv)
    sv_run(rla, torch, dev, ls, svd, 5000, 60, servers[False], 1)
    sv_run(rla, torch, dev, ls, svd, 5000, 30, servers[True], 2)
    return ls, svd, servers


def serve_arm(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from __graft_entry__ import load_package
    rla = load_package()
    dev = torch.device("cuda", local if world > 1 else 0)
    lams = [int(x) for x in args.serve_rates.split(",")]
    # one long-running server per mode, as a deployment keeps it: its contexts, sketch cache
    # and memory pools are built once, during the warm-up
    ls, svd, servers = serve_setup(rla, torch, dev, args.slots, rank)
    if args.serve_mix is not None:  # capacity of one request type (diagnostics)
        for plain in (False, True):
            thr, p50, p99 = sv_run(rla, torch, dev, ls, svd, max(lams), args.serve_requests, servers[plain], 3,
                                   ls_frac=args.serve_mix)
            print(json.dumps({"ls_fraction": args.serve_mix, "plain": plain, "req_per_s": round(thr, 1),
                              "p50_ms": round(1e3 * p50, 2), "p99_ms": round(1e3 * p99, 2)}), flush=True)
        for srv in servers.values():
            srv.stop()
        return
    props = torch.cuda.get_device_properties(dev)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else dev.index)
    clocks.start()
    # SV_REPS runs per rate and mode; per-field medians over the runs are reported, so one run
    # disturbed by other work on the shared host does not decide the line
    res = sv_curve(rla, torch, dev, ls, svd, servers, lams, args.serve_requests, SV_REPS)
    # below saturation: the latency-throughput curve and the throughput at a fixed p99 SLO
    slo_curve = sv_curve(rla, torch, dev, ls, svd, servers, SV_SLO_RATES, args.serve_requests // 2, SV_REPS, seed0=20)
    clk = clocks.stop()
    for srv in servers.values():
        srv.stop()
    barrier(world)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    top = max(lams)
    value = world * res["batched"][top]["req_per_s"]
    # throughput at equal p99: the plain path's best rate against the batched rate whose p99
    # is not above the plain path's p99 at that rate
    pl_best = max(lams, key=lambda L: res["plain"][L]["req_per_s"])
    p99_budget = res["plain"][pl_best]["p99_ms"]
    ok = [L for L in lams if res["batched"][L]["p99_ms"] <= p99_budget]
    b_at = max((res["batched"][L]["req_per_s"] for L in ok), default=None)
    line = {"metric": SV_METRIC, "value": round(value, 1), "unit": "req/s", "n_gpus": world,
            "steps": args.serve_requests, "warmup": 2, "ms_per_step": round(1e3 / max(value, 1e-9), 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 data, f32/f64 as in the request kernels",
            "data": "synthetic device-resident pool (24 LS, 16 RandSVD problems, seed 5+rank)",
            "config": {"workload": SV_WORKLOAD, "arrival_rates": lams, "requests_per_rate": args.serve_requests,
                       "runs_per_rate": SV_REPS, "server": "one per mode, warmed before timing",
                       "slots": args.slots, "max_group": 32, "memory_budget_gb": 150,
                       "parallelism": f"replicas x{world}"},
            "serving": res,
            "below_saturation": {"curve": slo_curve, "at_slo": sv_at_slo(slo_curve, SV_SLO_RATES)},
            "equal_p99": {"plain_req_per_s": res["plain"][pl_best]["req_per_s"], "p99_budget_ms": p99_budget,
                          "batched_req_per_s": b_at,
                          "ratio": None if b_at is None else round(b_at / res["plain"][pl_best]["req_per_s"], 2)},
            "e2e": {"value": round(value, 1), "unit": "req/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "note": "inputs come from a device-resident pool by the workload's definition"},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    global M, BYTES_PER_APPLY
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="sketch workload: skip the RandSVD and serving keys of the line (profiling runs)")
    ap.add_argument("--rows", type=int, default=M,
                    help="rows of A (default 2^20; 4194304 with --cols 128 is the tall-skinny variant)")
    ap.add_argument("--cols", type=int, default=NCOL,
                    help="columns of A (default 512, the benchmark workload; smaller values make small "
                         "cases of the same kernels for profiler captures)")
    ap.add_argument("--workload", choices=["sketch", "randsvd", "batched", "serve", "ihs", "sampling", "kaczmarz",
                                           "sparse_sign"],
                    default="sketch",
                    help="sketch: SRHT + CountSketch apply (default); randsvd: mixed-precision RandSVD; "
                         "batched: 512 uneven RandSVD instances")
    ap.add_argument("--batch-count", type=int, default=BT_COUNT, help="instances of the batched workload")
    ap.add_argument("--no-autotune", action="store_true", help="batched workload: default tile shapes")
    ap.add_argument("--batch-precision", choices=["split", "native"], default="split",
                    help="batched workload: split-BF16 tensor-core passes over A (default) or FP32 CUDA-core passes; "
                         "the plain path uses the same precision")
    ap.add_argument("--serve-requests", type=int, default=600, help="serving workload: requests per arrival rate")
    ap.add_argument("--slots", type=int, default=4, help="serving workload: concurrent workers")
    ap.add_argument("--serve-rates", default="2000,5000,10000,20000", help="serving workload: arrival rates (req/s)")
    ap.add_argument("--serve-mix", type=float, default=None,
                    help="serving diagnostics: fraction of LS requests (prints per-type capacity only)")
    ap.add_argument("--ihs-m", type=int, default=IHS_M, help="IHS rows (default 2^18)")
    ap.add_argument("--ihs-n", type=int, default=IHS_N, help="IHS columns (default 512; s = 4n)")
    ap.add_argument("--rs-m", type=int, default=RS_M, help="RandSVD rows (default 65536; smaller for profiler cases)")
    ap.add_argument("--rs-n", type=int, default=RS_N, help="RandSVD columns (default 8192)")
    args = ap.parse_args()
    if args.rows != M:
        M = args.rows
        BYTES_PER_APPLY = bytes_per_apply()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference" and int(os.environ.get("RANK", "0")) != 0:
        return  # the reference arm runs on rank 0 alone; other ranks exit without work
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "serving workload: the reference arm is timed "
                              "for the sketch and randsvd workloads only"}), flush=True)
        else:
            serve_arm(args)
    elif args.workload == "batched":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "batched workload: the reference arm is timed "
                              "for the sketch and randsvd workloads only"}), flush=True)
        else:
            batched_arm(args)
    elif args.workload == "kaczmarz":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "kaczmarz workload: the reference arm is timed "
                              "for the sketch and randsvd workloads only (the CPU restatement is in cpu_baseline)"}),
                  flush=True)
        else:
            kaczmarz_arm(args)
    elif args.workload == "sampling":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "sampling workload: the reference arm is timed "
                              "for the sketch and randsvd workloads only (the CPU restatement is in cpu_baseline)"}),
                  flush=True)
        else:
            sampling_arm(args)
    elif args.workload == "ihs":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "ihs workload: the reference arm is timed "
                              "for the sketch and randsvd workloads only (the CPU restatement is in cpu_baseline)"}),
                  flush=True)
        else:
            ihs_arm(args)
    elif args.workload == "sparse_sign":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "sparse_sign workload: the reference arm is timed "
                              "for the sketch and randsvd workloads only (the CPU restatement is in cpu_baseline)"}),
                  flush=True)
        else:
            sparse_sign_arm(args)
    elif args.workload == "randsvd":
        if args.impl == "reference":
            randsvd_reference_arm(args)
        else:
            randsvd_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
