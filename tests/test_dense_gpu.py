"""CUDA dense LU (factr/solve and the row-major builtin solve) against the
oracle: same pivots, same U, solutions within 1e-10 relative."""
import numpy as np
import pytest

import nec2c_b200 as nb
from oracle_lib import oracle, ptr

pytestmark = pytest.mark.gpu


def nec_storage(a, ld):
    """NEC's transposed column-major storage of the algebraic matrix a."""
    n = a.shape[0]
    st = np.zeros((ld, n), dtype=np.complex128, order="F")
    st[:n, :n] = a.T
    return st


def mom_like(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return a + np.diag(np.full(n, 0.5 * np.sqrt(n)))


def test_kat():
    """tests/dense_backend_test.c:16-33, classic storage with ld 5 and two RHS."""
    a = np.array([[4 + 1j, 1 - 2j, 0.5], [2, 5 + 0.5j, -1j], [-1 + 1j, 0.25, 3 - 1j]])
    x1 = np.array([1 + 2j, -0.5 + 1j, 2 - 0.25j])
    x2 = np.array([-1j, 2 + 0.5j, -1.0])
    assert nb.dense_backend_set("cuda")
    st = nec_storage(a, 5)
    ok, piv = nb.factor_classic(st)
    assert ok
    rhs = np.zeros((5, 2), dtype=np.complex128, order="F")
    rhs[:3, 0] = a @ x1
    rhs[:3, 1] = a @ x2
    assert nb.solve_classic_many(st, piv, rhs)
    assert np.max(np.abs(rhs[:3, 0] - x1)) < 1e-12 and np.max(np.abs(rhs[:3, 1] - x2)) < 1e-12
    ok, b = nb.solve_row_major(a, a @ x1)
    assert ok and np.max(np.abs(b - x1)) < 1e-12


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 100, 257, 700, 2500, 4100])
def test_factor_matches_oracle(n):
    a = mom_like(n, n)
    ld = n + 5
    st = nec_storage(a, ld)
    st_o = st.copy(order="F")
    assert nb.dense_backend_set("cuda")
    ok, piv = nb.factor_classic(st)
    assert ok
    piv_o = np.zeros(n, dtype=np.int32)
    assert oracle().oracle_factr(n, ptr(st_o), ptr(piv_o), ld)
    assert np.array_equal(piv, piv_o)
    # Ours: the LU row-major in NEC's storage (the Fortran view is its
    # transpose); the oracle's factr output is the column-major LU.
    U = np.triu(st[:n, :n].T)
    U_o = np.triu(st_o[:n, :n])
    # Blocked and column-by-column elimination sum in different orders; the
    # rounding difference grows with the order.
    assert np.max(np.abs(U - U_o)) / np.max(np.abs(U_o)) < max(1e-12, 2e-15 * n)
    rng = np.random.default_rng(1000 + n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = a @ x
    rhs = np.zeros((ld, 1), dtype=np.complex128, order="F")
    rhs[:n, 0] = b
    assert nb.solve_classic_many(st, piv, rhs)
    bo = np.ascontiguousarray(b.copy())
    oracle().oracle_solve(n, ptr(st_o), ptr(piv_o), ptr(bo), ld)
    assert np.linalg.norm(rhs[:n, 0] - bo) / np.linalg.norm(bo) < 1e-10
    # solve from re-uploaded factors (no device cache)
    nb.load().nec2c_cuda_dense_release()
    rhs2 = np.zeros((ld, 1), dtype=np.complex128, order="F")
    rhs2[:n, 0] = b
    assert nb.solve_classic_many(st, piv, rhs2)
    assert np.array_equal(rhs2, rhs)


@pytest.mark.parametrize("n", [1, 5, 40, 300])
def test_row_major_matches_oracle(n):
    a = mom_like(n, 50 + n)
    rng = np.random.default_rng(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ok, x = nb.solve_row_major(a, b)
    ao, bo = np.ascontiguousarray(a.copy()), np.ascontiguousarray(b.copy())
    assert ok and oracle().oracle_row_major_solve(ptr(ao), ptr(bo), n)
    assert np.linalg.norm(x - bo) / np.linalg.norm(bo) < 1e-10


def test_singular_rejected():
    a = np.zeros((4, 4), dtype=np.complex128)
    a[0, 0] = 1
    st = nec_storage(a, 4)
    ok, _ = nb.factor_classic(st)
    assert not ok
    ok, _ = nb.solve_row_major(a, np.ones(4))
    assert not ok


@pytest.mark.parametrize("n", [1, 33, 300, 1984, 2500])
def test_split_precision_refined_solve(n):
    """"cuda-mixed": FP32 factors with the tensor-core update, FP64 refinement
    in the solve; the solution matches the oracle's FP64 solve to 1e-10
    relative, reached by refinement (no FP64 fallback)."""
    a = mom_like(n, 7 * n)
    ld = n + 3
    st = nec_storage(a, ld)
    assert nb.dense_backend_set("cuda-mixed")
    try:
        ok, piv = nb.factor_classic(st)
        assert ok, nb.load().nec2c_cuda_last_error()
        rng = np.random.default_rng(n)
        x = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
        rhs = np.zeros((ld, 3), dtype=np.complex128, order="F")
        rhs[:n] = a @ x
        assert nb.solve_classic_many(st, piv, rhs)
        steps = nb.load().nec2c_cuda_dense_last_refinement()
        assert steps >= 1
        ao = nec_storage(a, ld).copy(order="F")
        po = np.zeros(n, dtype=np.int32)
        assert oracle().oracle_factr(n, ptr(ao), ptr(po), ld)
        for j in range(3):
            bo = np.ascontiguousarray((a @ x)[:, j].copy())
            oracle().oracle_solve(n, ptr(ao), ptr(po), ptr(bo), ld)
            assert np.linalg.norm(rhs[:n, j] - bo) / np.linalg.norm(bo) < 1e-10
        # The factors written back are the FP32 factors: the product of the
        # unit-lower and upper parts reproduces the row-interchanged matrix
        # to FP32 accuracy.
        lu = st[:n, :n].T
        L = np.tril(lu, -1) + np.eye(n)
        U = np.triu(lu)
        pa = a.copy()
        for i in range(n):
            q = piv[i] - 1
            if q != i:
                pa[[i, q]] = pa[[q, i]]
        assert np.max(np.abs(L @ U - pa)) / np.max(np.abs(a)) < 1e-4 * max(1.0, np.sqrt(n) / 10)
    finally:
        nb.dense_backend_set("cuda")
        nb.load().nec2c_cuda_dense_release()


def test_batched_ragged_matches_oracle():
    """Ragged batch (wire-block sized systems in one launch, plus two above
    the one-launch limit): per system the same pivots as factr, U to the dense
    tests' tolerance, the solution within 1e-12 of the oracle's; a singular
    system in the batch is reported without disturbing the others."""
    sizes = [1, 2, 11, 21, 33, 41, 64, 17, 65, 100]
    systems, ref = [], []
    for k, n in enumerate(sizes):
        a = mom_like(n, 900 + k)
        if k == 7:
            a[:, 3] = 0.0            # singular
        ld = n + (k % 3)
        st = nec_storage(a, ld)
        rng = np.random.default_rng(k)
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        b = np.ascontiguousarray(a @ x)
        systems.append((st, b.copy()))
        ref.append((a, st.copy(order="F"), b, ld))
    assert nb.dense_backend_set("cuda")
    ok, status, pivs = nb.solve_batched(systems)
    assert not ok                      # the singular one
    for k, (n, (st, xb), piv, (a, st0, b, ld)) in enumerate(zip(sizes, systems, pivs, ref)):
        if k == 7:
            assert status[k] == 0
            continue
        assert status[k] == 1, k
        po = np.zeros(n, dtype=np.int32)
        assert oracle().oracle_factr(n, ptr(st0), ptr(po), ld)
        assert np.array_equal(piv, po), k
        U, U_o = np.triu(st[:n, :n].T), np.triu(st0[:n, :n])
        assert np.max(np.abs(U - U_o)) / np.max(np.abs(U_o)) < 1e-12, k
        bo = b.copy()
        oracle().oracle_solve(n, ptr(st0), ptr(po), ptr(bo), ld)
        assert np.linalg.norm(xb - bo) / np.linalg.norm(bo) < 1e-12, k


def test_split_precision_reference_call_order():
    """"cuda-mixed" in the reference's call order: factrs factors every
    symmetry block (row blocks of one storage, matrix.c:1424-1435), netwk then
    factors its network matrix (network.c:505), and only afterwards solves
    the blocks (solves, matrix.c:1683-1701) and the network matrix (solve,
    network.c:550).  Every solution is within 1e-10 of the oracle's FP64
    solve, each reached by refinement."""
    nop, npb, nn = 4, 150, 40
    nrow = nop * npb
    blocks = [mom_like(npb, 60 + k) for k in range(nop)]
    st = np.zeros((nrow, npb), dtype=np.complex128, order="F")
    for k, a in enumerate(blocks):
        st[k * npb:(k + 1) * npb, :] = a.T
    cmn_a = mom_like(nn, 77)
    cmn = nec_storage(cmn_a, nn + 2)
    ip = np.zeros(nrow, dtype=np.int32)
    lib = nb.load()
    assert nb.dense_backend_set("cuda-mixed")
    try:
        # factrs: factr(np, &a[kk*np], &ip[kk*np], nrow) per block.
        itemsize = st.itemsize
        for k in range(nop):
            assert lib.nec2c_cuda_dense_factor_classic(npb, st.ctypes.data + k * npb * itemsize, nrow,
                                                       ip.ctypes.data + k * npb * 4), nb.last_error()
        ok, ipn = nb.factor_classic(cmn)
        assert ok
        rng = np.random.default_rng(5)
        for k, a in enumerate(blocks):
            x = rng.standard_normal(npb) + 1j * rng.standard_normal(npb)
            b = np.zeros(nrow, dtype=np.complex128)
            b[k * npb:(k + 1) * npb] = a @ x
            assert lib.nec2c_cuda_dense_solve_classic_many(npb, st.ctypes.data + k * npb * itemsize, nrow,
                                                           ip.ctypes.data + k * npb * 4,
                                                           b.ctypes.data + k * npb * itemsize, nrow, 1), \
                nb.last_error()
            assert lib.nec2c_cuda_dense_last_refinement() >= 1
            ao = nec_storage(a, npb).copy(order="F")
            po = np.zeros(npb, dtype=np.int32)
            assert oracle().oracle_factr(npb, ptr(ao), ptr(po), npb)
            bo = np.ascontiguousarray(a @ x)
            oracle().oracle_solve(npb, ptr(ao), ptr(po), ptr(bo), npb)
            got = b[k * npb:(k + 1) * npb]
            assert np.linalg.norm(got - bo) / np.linalg.norm(bo) < 1e-10, k
        xn = rng.standard_normal(nn) + 1j * rng.standard_normal(nn)
        rhs = np.zeros((nn + 2, 1), dtype=np.complex128, order="F")
        rhs[:nn, 0] = cmn_a @ xn
        assert nb.solve_classic_many(cmn, ipn, rhs)
        assert lib.nec2c_cuda_dense_last_refinement() >= 1
        assert np.linalg.norm(rhs[:nn, 0] - xn) / np.linalg.norm(xn) < 1e-10
        # Once the device copies are dropped, a split-precision solve is
        # refused rather than returned at FP32 accuracy.
        lib.nec2c_cuda_dense_release()
        rhs[:nn, 0] = cmn_a @ xn
        assert not nb.solve_classic_many(cmn, ipn, rhs)
        assert "factor it again" in nb.last_error()
    finally:
        nb.dense_backend_set("cuda")
        lib.nec2c_cuda_dense_release()
