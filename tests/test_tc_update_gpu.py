"""Tensor-core trailing update of the split-precision LU, both forms
(n2d_gemm_tf32x3: operands staged by the threads, one tile per CTA;
n2d_gemm_tf32x3_persistent: TMA-fed, one CTA per SM over a band's tiles):
C -= A B for complex FP32 blocks through tcgen05 3xTF32, against a float64
numpy product.  The 3xTF32 split keeps the result at FP32 accuracy: the
tolerance is 2e-6 relative to the largest |A||B| term."""
import ctypes as C

import numpy as np
import pytest

import nec2c_b200 as nb

pytestmark = pytest.mark.gpu


def pack_bt(u):
    """Packed real expansion of the 32 x N complex block u: 2N rows of 64
    floats (row 2n: Re, -Im per k; row 2n+1: Im, Re), split hi + lo."""
    k, n = u.shape
    bt = np.empty((2 * n, 2 * k), dtype=np.float32)
    ur = u.real.astype(np.float32).T
    ui = u.imag.astype(np.float32).T
    bt[0::2, 0::2] = ur
    bt[0::2, 1::2] = -ui
    bt[1::2, 0::2] = ui
    bt[1::2, 1::2] = ur
    hi = (bt.view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)
    lo = (bt - hi).astype(np.float32)
    return np.ascontiguousarray(hi), np.ascontiguousarray(lo)


@pytest.mark.parametrize("form", ["n2d_gemm_tf32x3", "n2d_gemm_tf32x3_persistent"])
@pytest.mark.parametrize("m,n,ld", [(128, 128, 256), (300, 517, 600), (1, 3, 64), (1000, 1000, 1040),
                                    (1100, 1300, 1340), (2047, 1024, 1090)])
def test_tf32x3_update(m, n, ld, form):
    import torch
    rng = np.random.default_rng(m + n)
    a = (rng.standard_normal((m, 32)) + 1j * rng.standard_normal((m, 32))).astype(np.complex64)
    u = (rng.standard_normal((32, n)) + 1j * rng.standard_normal((32, n))).astype(np.complex64)
    c = (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64)
    # Working-matrix layout: C and A inside one row-major array with leading
    # dimension ld (A in columns 0..31, C from column 32).
    w = np.zeros((m, ld), dtype=np.complex64)
    w[:, :32] = a
    w[:, 32:32 + n] = c
    hi, lo = pack_bt(u)
    dw = torch.from_numpy(w.view(np.float32)).cuda()
    dhi, dlo = torch.from_numpy(hi).cuda(), torch.from_numpy(lo).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    lib = nb.load()
    f = getattr(lib, form)
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_longlong,
                  C.c_longlong, C.c_void_p]
    base = dw.data_ptr()
    ok = f(base + 32 * 8, ld, base, ld, dhi.data_ptr(), dlo.data_ptr(), m, n, err.data_ptr())
    torch.cuda.synchronize()
    assert ok, lib.nec2c_cuda_last_error()
    assert int(err.item()) == 0
    out = dw.cpu().numpy().view(np.complex64)
    expect = c.astype(np.complex128) - a.astype(np.complex128) @ u.astype(np.complex128)
    scale = (np.abs(a).astype(np.float64) @ np.abs(u).astype(np.float64)).max()
    assert np.max(np.abs(out[:, 32:32 + n] - expect)) / scale < 2e-6
    # Columns outside C untouched.
    assert np.array_equal(out[:, :32], a)
    assert np.array_equal(out[:, 32 + n:], w[:, 32 + n:])


@pytest.mark.parametrize("m,n,ld", [(1100, 1300, 1340), (2047, 1024, 1090)])
def test_tf32x3_forms_agree_bitwise(m, n, ld):
    """The staged and the persistent form issue the same products in the same
    order per accumulator element, so C comes out the same bit for bit (the
    lockstep batch may take either form for a step's updates)."""
    import torch
    rng = np.random.default_rng(7 * m + n)
    w = np.zeros((m, ld), dtype=np.complex64)
    w[:, :32 + n] = (rng.standard_normal((m, 32 + n)) + 1j * rng.standard_normal((m, 32 + n))).astype(np.complex64)
    u = (rng.standard_normal((32, n)) + 1j * rng.standard_normal((32, n))).astype(np.complex64)
    hi, lo = pack_bt(u)
    lib = nb.load()
    outs = []
    for name in ("n2d_gemm_tf32x3", "n2d_gemm_tf32x3_persistent"):
        f = getattr(lib, name)
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_longlong,
                      C.c_longlong, C.c_void_p]
        dw = torch.from_numpy(w.view(np.float32).copy()).cuda()
        dhi, dlo = torch.from_numpy(hi).cuda(), torch.from_numpy(lo).cuda()
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        base = dw.data_ptr()
        assert f(base + 32 * 8, ld, base, ld, dhi.data_ptr(), dlo.data_ptr(), m, n, err.data_ptr())
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        outs.append(dw.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


# Run in a child process with NEC2C_CUDA_TC_WAIT_CYCLES=0: every update gives
# up its wait for the products at once, sets the error word, leaves C as it
# was, still waits (bounded) for the products before freeing its tensor
# memory, and returns; the context stays usable.
TIMEOUT_CHILD = r"""
import ctypes as C, os, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
import nec2c_b200 as nb
from test_tc_update_gpu import pack_bt
rng = np.random.default_rng(5)
lib = nb.load()
for name in ("n2d_gemm_tf32x3", "n2d_gemm_tf32x3_persistent"):
    f = getattr(lib, name)
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_longlong,
                  C.c_longlong, C.c_void_p]
for name, (m, n, ld) in (("n2d_gemm_tf32x3", (300, 517, 600)), ("n2d_gemm_tf32x3_persistent", (1100, 1300, 1340))):
    f = getattr(lib, name)
    w = np.zeros((m, ld), dtype=np.complex64)
    w[:, :32 + n] = (rng.standard_normal((m, 32 + n)) + 1j * rng.standard_normal((m, 32 + n))).astype(np.complex64)
    u = (rng.standard_normal((32, n)) + 1j * rng.standard_normal((32, n))).astype(np.complex64)
    hi, lo = pack_bt(u)
    dw = torch.from_numpy(w.view(np.float32)).cuda()
    dhi, dlo = torch.from_numpy(hi).cuda(), torch.from_numpy(lo).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    base = dw.data_ptr()
    assert f(base + 32 * 8, ld, base, ld, dhi.data_ptr(), dlo.data_ptr(), m, n, err.data_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 1, "time-out not reported"
    assert np.array_equal(dw.cpu().numpy().view(np.complex64), w), "C changed on the time-out path"
# The split-precision factor reads the same word and fails with the reason.
k = 300
a = rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k)) + np.diag(np.full(k, 10.0))
st = np.asfortranarray(a.T.copy())
assert nb.dense_backend_set("cuda-mixed")
ok, _ = nb.factor_classic(st)
assert not ok and "time-out" in nb.last_error(), nb.last_error()
# So does the split-precision lockstep batch, through its batched kernel
# (small updates) and the per-matrix persistent kernel (four large systems).
f32b = lib.n2d_lu_factor32_batch
f32b.restype = C.c_int
f32b.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
for sizes in ((300, 200), (1200, 1200, 1200, 1200)):
    cnt = len(sizes)
    mats = []
    for q, nq in enumerate(sizes):
        aq = np.zeros((nq, nq), dtype=np.complex64)
        aq[:, :] = rng.standard_normal((nq, nq)) + 1j * rng.standard_normal((nq, nq)) + np.diag(np.full(nq, 10.0))
        mats.append(torch.from_numpy(aq.view(np.float32)).cuda())
    pivs = [torch.zeros(nq, dtype=torch.int32, device="cuda") for nq in sizes]
    info = (C.c_int * cnt)()
    ok = f32b((C.c_void_p * cnt)(*[t.data_ptr() for t in mats]), (C.c_longlong * cnt)(*sizes),
              (C.c_longlong * cnt)(*sizes), (C.c_void_p * cnt)(*[t.data_ptr() for t in pivs]), cnt, 0, info)
    torch.cuda.synchronize()
    assert not ok and "time-out" in nb.last_error(), nb.last_error()
# The context is still usable: the FP64 factor runs and is right.
assert nb.dense_backend_set("cuda")
st = np.asfortranarray(a.T.copy())
ok, piv = nb.factor_classic(st)
assert ok, nb.last_error()
print("time-out path ok")
"""


def test_update_timeout_reported():
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, NEC2C_CUDA_TC_WAIT_CYCLES="0")
    r = subprocess.run([sys.executable, "-c", TIMEOUT_CHILD, root], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "time-out path ok" in r.stdout
