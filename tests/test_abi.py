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


def test_new_entry_points_refuse_bad_arguments_without_a_device():
    """The batch, schedule and far-field entry points check their arguments
    before any device call."""
    import nec2c_b200 as nb
    lib = nb.load()
    vp = C.c_void_p
    h = vp()
    assert not lib.nec2c_cuda_vie_batch_create(None, None, 1)
    assert not lib.nec2c_cuda_vie_batch_create(C.byref(h), None, 1)
    assert not lib.nec2c_cuda_vie_batch_create(C.byref(h), (vp * 1)(None), 0)
    assert not lib.nec2c_cuda_vie_batch_create(C.byref(h), (vp * 1)(None), 1) and not h.value
    assert not lib.nec2c_cuda_hybrid_batch_create(C.byref(h), (vp * 1)(None), 1) and not h.value
    reps = (nb.GmresReport * 1)()
    assert not lib.nec2c_cuda_gmres_batch_device(None, vp(16), vp(32), None, reps)
    assert not lib.nec2c_cuda_vie_fft_tune(None, 1)
    tiles, r1 = (C.c_int * 5)(), (C.c_int * 5)()
    assert lib.nec2c_cuda_vie_fft_schedule(None, 1, tiles, r1) == -1
    assert not lib.nec2c_cuda_vie_fft_set_schedule(None, 1, tiles, r1)
    assert not lib.nec2c_cuda_vie_batch_schedule(None, tiles, r1)
    assert not lib.nec2c_cuda_vie_batch_set_schedule(None, tiles, r1)
    origin = (C.c_double * 3)(0, 0, 0)
    assert not lib.nec2c_cuda_vie_fft_radiation_device(None, origin, vp(16), 1, vp(16), vp(16))
    assert "radiation" in nb.last_error()


def test_bad_arguments_say_why_without_a_device():
    """Entry points refuse null handles and bad values before any device call,
    with the reason in nec2c_cuda_last_error (no crash on a null handle)."""
    import nec2c_b200 as nb
    lib = nb.load()
    vp = C.c_void_p
    buf = (C.c_double * 8)()
    cases = [
        (lambda: lib.nec2c_cuda_vie_fft_backend_set(b"bogus"), "unknown FFT backend"),
        (lambda: lib.nec2c_cuda_vie_fft_apply(None, buf, buf), "null plan"),
        (lambda: lib.nec2c_cuda_vie_fft_precondition(None, buf, buf), "null plan"),
        (lambda: lib.nec2c_cuda_vie_fft_apply_device(None, vp(16), vp(32)), "null plan"),
        (lambda: lib.nec2c_cuda_hybrid_apply(None, buf, buf), "null hybrid"),
        (lambda: lib.nec2c_cuda_hybrid_precondition(None, buf, buf), "null hybrid"),
        (lambda: lib.nec2c_cuda_hybrid_set_blocks(None, buf), "set_blocks"),
        (lambda: lib.nec2c_cuda_vie_fft_spectrum(None, buf), "spectrum"),
        (lambda: lib.nec2c_cuda_gmres_batch_device(None, vp(16), vp(32), None, (nb.GmresReport * 1)()),
         "batch solve"),
        (lambda: lib.nec2c_cuda_gmres_batch(None, None, None, None, None), "batch solve"),
        (lambda: lib.nec2c_cuda_vie_batch_apply_device(None, vp(16), vp(32)), "batch apply"),
        (lambda: lib.nec2c_cuda_vie_batch_schedule(None, None, None), "batch schedule"),
    ]
    for call, why in cases:
        assert not call()
        assert why in nb.last_error(), (why, nb.last_error())
    assert lib.nec2c_cuda_vie_fft_backend_set(b"cuda")


def test_autotune_switch():
    import nec2c_b200 as nb
    before = nb.fft_autotune_enabled()
    nb.set_fft_autotune(False)
    assert not nb.fft_autotune_enabled()
    nb.set_fft_autotune(True)
    assert nb.fft_autotune_enabled()
    nb.set_fft_autotune(before)
