"""The plan entry point's argument checks and byte accounting against the
reference's vie_fft_create (vie_fft.c:378-398), on the CPU.  Both are decided
before any device call: a plan the reference accepts under a byte limit
passes them here too (and then stops only for want of a GPU), and one it
refuses is refused here, before the device is touched."""
import ctypes as C

import numpy as np
import pytest

import cases
import nec2c_b200 as nb
import oracle_lib

needs_ref = pytest.mark.skipif(not oracle_lib.reference_available(),
                               reason="oracle/_ref not built (needs the reference tree)")


def ours(shape, xyz, h, k, eps, limit):
    lib = nb.load()
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.uintp))
    out = C.c_void_p()
    near = nb.NEAR_FN(lambda *a: 0)
    ok = lib.nec2c_cuda_vie_fft_create(C.byref(out), (C.c_size_t * 3)(*shape), xyz.size // 3,
                                       xyz.ctypes.data_as(C.POINTER(C.c_size_t)), h, k, eps.real, eps.imag,
                                       limit, near, None)
    assert not ok and not out.value      # no device here: never a plan
    return nb.last_error()


def reference_bytes(shape, xyz, h, k, eps, limit=1 << 40):
    r = oracle_lib.reference()
    r.ref_fft_backend_set(b"builtin")
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.uintp))
    p = r.ref_fft_create((C.c_size_t * 3)(*shape), xyz.size // 3, xyz.ctypes.data_as(C.POINTER(C.c_size_t)),
                         h, k, eps.real, eps.imag, limit)
    if not p:
        return None
    b = r.ref_fft_bytes(p)
    r.ref_fft_destroy(p)
    return b


VALID = [
    ((1, 1, 1), [0, 0, 0], 0.25, 0.2, 3 + 0j),
    (cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 0.25, 0.8, 3 - 0.4j),
    (cases.FAR_SHAPE, cases.FAR_XYZ, 0.25, 4.0, 2 - 0.1j),
    ((7, 6, 5), cases.random_lattice((7, 6, 5), 0.6, seed=3), 0.25, 0.3, 5 - 1j),
]


@needs_ref
@pytest.mark.parametrize("case", VALID)
def test_byte_accounting_matches_reference(case):
    shape, xyz, h, k, eps = case
    need = reference_bytes(shape, xyz, h, k, eps)
    assert need
    assert reference_bytes(shape, xyz, h, k, eps, need - 1) is None
    assert reference_bytes(shape, xyz, h, k, eps, need) == need
    assert "byte limit" in ours(shape, xyz, h, k, eps, need - 1)
    assert "byte limit" not in ours(shape, xyz, h, k, eps, need)


INVALID = [
    ((1, 1, 1), [0, 0, 0], 1.0, 1.5, 3 + 0j),          # k h > 1
    ((1, 1, 1), [0, 0, 0], 0.25, 0.2, 0.5 + 0j),       # Re eps < 1
    ((1, 1, 1), [0, 0, 0], 0.25, 0.2, 3 + 0.1j),       # active material
    ((1, 1, 1), [0, 0, 0], -0.25, 0.2, 3 + 0j),        # negative pitch
    ((1, 1, 1), [0, 0, 0], 0.25, float("nan"), 3 + 0j),
    ((1, 1, 1), [0, 0, 0], 0.25, -0.2, 3 + 0j),        # negative wavenumber
    ((0, 1, 1), [0, 0, 0], 0.25, 0.2, 3 + 0j),         # empty axis
]


@needs_ref
@pytest.mark.parametrize("case", INVALID)
def test_invalid_arguments_refused_like_reference(case):
    shape, xyz, h, k, eps = case
    assert reference_bytes(shape, xyz, h, k, eps) is None
    err = ours(shape, xyz, h, k, eps, 1 << 40)
    assert "invalid" in err, err


def test_dense_entry_points_check_arguments_first():
    """dense_backend.c's LAPACK-branch conventions, decided before any device
    call: no right-hand sides is success, order 0 or a short leading
    dimension is a failure with the reason set."""
    lib = nb.load()
    a = np.zeros((4, 4), dtype=np.complex128)
    piv = np.zeros(4, dtype=np.int32)
    rhs = np.zeros(4, dtype=np.complex128)
    p = lambda arr: arr.ctypes.data
    assert lib.nec2c_cuda_dense_solve_classic_many(4, p(a), 4, p(piv), p(rhs), 4, 0) == 1
    assert not lib.nec2c_cuda_dense_factor_classic(0, p(a), 4, p(piv))
    assert "order 0" in nb.last_error()
    assert not lib.nec2c_cuda_dense_factor_classic(4, p(a), 3, p(piv))
    assert "leading dimension" in nb.last_error()
    assert not lib.nec2c_cuda_dense_solve_classic_many(4, p(a), 4, p(piv), p(rhs), 3, 1)
    assert "stride" in nb.last_error()
    assert not lib.nec2c_cuda_dense_solve_row_major(None, p(rhs), 4)
    assert "row-major" in nb.last_error()
    assert not lib.nec2c_cuda_dense_backend_set(b"lapack")
    assert "unknown dense backend" in nb.last_error()
