"""Source check: the serving loop's request paths allocate and free device memory only in
stream order.

A synchronous cudaFree (and cudaDeviceSynchronize) waits for every stream of every context
on the device, so one worker of a multi-worker server that calls it stalls all the others for
as long as they keep the device busy (measured: 30-680 ms p99 spikes at 100-400 req/s before
the context scratch and the grouped plans moved to the contexts' stream-ordered pools).  The
request paths are sketch-and-solve least squares (rla_ls.cu ls_sketch_solve, rla_sparse.cu),
single-instance RandSVD (rla_range.cu, rla_tc.cu, rla_dgemm.cu, rla_linalg.cu,
rla_cholinv.cu, rla_gemm.cu) and grouped RandSVD (rla_batch.cu); the context's grow-only
buffers live in rla_ctx.cu.  Allowed: the one-time status word of the tensor-core kernels
(allocated once per context) and its release when the context is destroyed.
"""
import pathlib
import re

CSRC = pathlib.Path(__file__).resolve().parents[1] / "randlinearalgebra.jl_b200" / "csrc"
SYNC = re.compile(r"\b(cudaFree|cudaMalloc|cudaMallocHost|cudaFreeHost|cudaDeviceSynchronize)\s*\(")
WHOLE_FILES = ["rla_range.cu", "rla_dgemm.cu", "rla_linalg.cu", "rla_cholinv.cu", "rla_batch.cu",
               "rla_server.cu", "rla_sparse.cu", "rla_gemm.cu", "rla_tc.cu", "rla_ctx.cu"]
# (file, line fragment) pairs that may keep a synchronous call
ALLOWED = {("rla_tc.cu", "ctx->tc_status, 256"), ("rla_ctx.cu", "cudaFree(ctx->tc_status)")}


def strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def function_body(src: str, signature: str) -> str:
    start = src.index(signature)
    end = src.index("\n}\n", start)
    return src[start:end]


def offending_lines(name: str, text: str):
    out = []
    for i, line in enumerate(text.splitlines(), 1):
        if SYNC.search(line) and not any(f == name and frag in line for f, frag in ALLOWED):
            out.append(f"{name}:{i}: {line.strip()}")
    return out


def test_request_paths_have_no_synchronous_allocation():
    bad = []
    for name in WHOLE_FILES:
        bad += offending_lines(name, strip_comments((CSRC / name).read_text()))
    ls = strip_comments((CSRC / "rla_ls.cu").read_text())
    bad += offending_lines("rla_ls.cu", function_body(ls, "int ls_sketch_solve("))
    assert not bad, "synchronous device allocation on a request path:\n" + "\n".join(bad)


def test_scan_sees_a_planted_call():
    # the check itself: a synchronous free in a scanned text is reported, an allowed one is not
    planted = "void f(void *p) {\n    cudaFree(p);\n}\n"
    assert offending_lines("rla_range.cu", strip_comments(planted)) == ["rla_range.cu:2: cudaFree(p);"]
    assert offending_lines("rla_range.cu", strip_comments("// cudaFree(p);\n")) == []
    assert offending_lines("rla_tc.cu", "RLA_CUDA_TRY(ctx, cudaMalloc((void **)&ctx->tc_status, 256));") == []
