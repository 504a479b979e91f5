"""The C ABI: the shared library loads without a GPU and exports every function that
include/rla_b200.h declares; the ctypes binding covers each of them (CPU only)."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "rla_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rla_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("rla_ctx_create", "rla_sketch_create", "rla_sketch_update", "rla_sketch_mul",
                 "rla_rangefinder", "rla_randsvd", "rla_lowrank_mul", "rla_sketch_get_draws",
                 "rla_sketch_set_draws"):
        assert must in names


def test_library_exports_every_declared_symbol(rla):
    lib = rla.lib()  # loads librla_b200.so; no device is touched
    for name in declared_functions():
        assert hasattr(lib, name), name
    from importlib import import_module
    sigs = import_module("randlinearalgebra_b200._lib").SIGNATURES
    assert set(declared_functions()) <= set(sigs), set(declared_functions()) - set(sigs)


def test_symbols_are_extern_c():
    so = os.path.join(ROOT, "randlinearalgebra.jl_b200", "librla_b200.so")
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    for name in declared_functions():
        assert name in exported, name


def test_status_strings(rla):
    lib = rla.lib()
    assert lib.rla_status_string(0) == b"ok"
    assert lib.rla_status_string(1) == b"DimensionMismatch"
    assert lib.rla_version() >= 1
