"""The C-ABI library loads and exports every entry point include/nec2c_cuda.h
declares (CPU; no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nec2c_cuda.h")
LIB = os.path.join(ROOT, "nec2c_b200", "lib", "libnec2c_cuda.so")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(nec2c_cuda_[a-z0-9_]+)\s*\(", text))
    names -= {"nec2c_cuda_near_tensor_fn"}
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    for want in ("nec2c_cuda_vie_fft_create", "nec2c_cuda_gmres_plan",
                 "nec2c_cuda_dense_factor_classic", "nec2c_cuda_dense_solve_row_major",
                 "nec2c_cuda_hybrid_apply"):
        assert want in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "run __graft_entry__.build() first"
    lib = C.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_only():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", LIB],
                         capture_output=True, text=True).stdout
    arches = set(re.findall(r"sm_(\d+a?)", out))
    assert arches == {"100a"}, arches


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=gnu11", "-fsyntax-only", "-x", "c", HEADER],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_backend_names():
    import nec2c_b200 as nb
    lib = nb.load()
    assert lib.nec2c_cuda_vie_fft_backend_set(b"cuda")
    assert lib.nec2c_cuda_vie_fft_backend_name() == b"cuda"
    assert lib.nec2c_cuda_vie_fft_backend_set(b"cuda-mixed")
    assert lib.nec2c_cuda_vie_fft_backend_name() == b"cuda-mixed"
    assert not lib.nec2c_cuda_vie_fft_backend_set(b"fftw")
    assert lib.nec2c_cuda_vie_fft_backend_set(b"cuda")
    assert lib.nec2c_cuda_dense_backend_set(b"cuda")
    assert not lib.nec2c_cuda_dense_backend_set(b"lapack")


def test_product_never_loads_the_oracle():
    """The product library links no oracle code."""
    out = subprocess.run(["nm", "-D", LIB], capture_output=True, text=True).stdout
    assert "oracle_" not in out and "ref_" not in out
