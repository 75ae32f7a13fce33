"""Allocation-free dense factor (nec2c_cuda_dense_factor_device_static)
against the classic factor entry point.

Callers that own all of a GPU's memory through their own pool, or that cannot
afford cudaMalloc's device synchronisation mid-run, use the allocation-free
variant; it must give the same pivots and factors as the classic factor
(within the dense tests' tolerance) on two calls in a row that share the
library's scratch array.  Named to run last, after every other test has used
the library; it also passes alone in a fresh process."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import nec2c_b200 as nb  # noqa: E402

pytestmark = pytest.mark.gpu


def _system(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return a + np.diag(np.full(n, 0.5 * np.sqrt(n)))


def _nec_storage(a, ld):
    n = a.shape[0]
    st = np.zeros((ld, n), dtype=np.complex128, order="F")
    st[:n, :n] = a.T
    return st


def _factor_static(st):
    """Factors a copy of NEC storage st (ld x n, Fortran order) held in device
    memory the test allocates; returns (ok, factors, pivots)."""
    import torch
    ld, n = st.shape
    # Column j of the Fortran array is row j of the algebraic matrix: the
    # C-ordered transpose has the same bytes.
    dev = torch.from_numpy(np.ascontiguousarray(st.T)).cuda()
    piv = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ok = nb.load().nec2c_cuda_dense_factor_device_static(n, dev.data_ptr(), ld, piv.data_ptr())
    torch.cuda.synchronize()
    return bool(ok), dev.cpu().numpy().T, piv.cpu().numpy()


def _compare(cases):
    """Static factor against the classic factor ("cuda" backend) on each
    (order, leading dimension, seed), one call after another."""
    lib = nb.load()
    assert nb.dense_backend_set("cuda")
    lib.nec2c_cuda_set_stream(None)
    for n, ld, seed in cases:
        a = _system(n, seed)
        st = _nec_storage(a, ld)
        ok_s, lu_s, piv_s = _factor_static(st)
        assert ok_s, lib.nec2c_cuda_last_error()
        st_c = st.copy(order="F")
        ok_c, piv_c = nb.factor_classic(st_c)
        assert ok_c
        assert np.array_equal(piv_s, piv_c)
        U_s, U_c = np.triu(lu_s[:n, :n].T), np.triu(st_c[:n, :n].T)
        L_s, L_c = np.tril(lu_s[:n, :n].T, -1), np.tril(st_c[:n, :n].T, -1)
        tol = max(1e-12, 2e-15 * n)
        assert np.max(np.abs(U_s - U_c)) / np.max(np.abs(U_c)) < tol
        assert np.max(np.abs(L_s - L_c)) < tol
        # The padding rows of the storage are left as they were.
        assert np.array_equal(lu_s[n:, :], st[n:, :])


def test_static_factor_matches_classic():
    _compare([(700, 703, 7), (2500, 2500, 25)])


def test_static_factor_grid_panel():
    """With the panel held to 8-CTA clusters (NEC2C_CUDA_LU_CLUSTER8=1, read
    once per process, hence the child process), order 2500 takes the grid
    panel, whose candidate slots also live in the static array."""
    env = dict(os.environ, NEC2C_CUDA_LU_CLUSTER8="1")
    r = subprocess.run([sys.executable, os.path.abspath(__file__)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "grid panel ok" in r.stdout


def test_static_factor_rejects_large_order():
    lib = nb.load()
    n = 4097
    # Rejected on the size alone, before any device pointer is used.
    assert not lib.nec2c_cuda_dense_factor_device_static(n, C.c_void_p(16), n, C.c_void_p(16))
    assert b"maximum" in lib.nec2c_cuda_last_error()


if __name__ == "__main__":
    _compare([(2500, 2500, 25), (2100, 2101, 21)])
    print("grid panel ok")
