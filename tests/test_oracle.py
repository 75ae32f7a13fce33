"""Pins the CPU oracle: against the reference compiled from its own sources
(oracle/_ref) on identical inputs, and against the reference's known-answer
data.  CPU only."""
import ctypes as C

import numpy as np
import pytest

import cases
import oracle_lib
from oracle_lib import OraclePlan, OracleHybrid, Report, oracle, ptr

needs_ref = pytest.mark.skipif(not oracle_lib.reference_available(),
                               reason="oracle/_ref not built (needs the reference tree)")

VIE_CASES = [
    ("vie_k0.2", (1, 1, 1), [0, 0, 0], 3.0),
    ("vie_k0", cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 3.0),
    ("vie_k0.8", cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 3.0),
    ("vie_k4", cases.FAR_SHAPE, cases.FAR_XYZ, 3.0),
    ("vie_k0.2", (1, 1, 1), [0, 0, 0], 1.0),
    ("vie_k0.2", (1, 1, 1), [0, 0, 0], 3 - 0.4j),
    ("vie_k0.8", cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 3 - 0.4j),
]


def ref_plan(shape, xyz, h, k, eps):
    r = oracle_lib.reference()
    r.ref_fft_backend_set(b"builtin")
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.uintp))
    p = r.ref_fft_create((C.c_size_t * 3)(*shape), xyz.size // 3,
                         xyz.ctypes.data_as(C.POINTER(C.c_size_t)), h, k, complex(eps).real,
                         complex(eps).imag, 1 << 40)
    assert p
    return p


@needs_ref
@pytest.mark.parametrize("case", VIE_CASES)
def test_matvec_matches_reference(near_tables, case):
    name, shape, xyz, eps = case
    h, k, table = near_tables[name]
    r = oracle_lib.reference()
    rp = ref_plan(shape, xyz, h, k, eps)
    op = OraclePlan(shape, xyz, h, k, eps, table)
    n = op.n
    for x in [cases.probe_vector(n)] + [np.eye(n, dtype=np.complex128)[j] * (1 + 2j) for j in range(n)]:
        x = np.ascontiguousarray(x)
        y_ref = np.empty(n, dtype=np.complex128)
        r.ref_fft_apply(rp, ptr(x), ptr(y_ref))
        assert np.array_equal(op.apply(x), y_ref)
        p_ref = np.empty(n, dtype=np.complex128)
        r.ref_fft_precondition(rp, ptr(x), ptr(p_ref))
        assert np.array_equal(op.precondition(x), p_ref)
    r.ref_fft_destroy(rp)


@needs_ref
def test_matvec_heterogeneous_matches_reference(near_tables):
    h, k, table = near_tables["rand_k0.3"]
    shape = (7, 6, 5)
    xyz = cases.random_lattice(shape, 0.6, seed=3)
    eps = cases.random_eps(xyz.size // 3, seed=4)
    r = oracle_lib.reference()
    rp = ref_plan(shape, xyz, h, k, 3.0)
    op = OraclePlan(shape, xyz, h, k, 3.0, table)
    for c, e in enumerate(eps):
        assert r.ref_fft_set_permittivity(rp, c, e.real, e.imag)
        assert op.set_permittivity(c, e)
    x = cases.probe_vector(op.n)
    y_ref = np.empty(op.n, dtype=np.complex128)
    r.ref_fft_apply(rp, ptr(x), ptr(y_ref))
    assert np.array_equal(op.apply(x), y_ref)
    b = y_ref.copy()
    ok1, x1, rep1 = op.gmres(b, rtol=1e-10)
    x2 = np.zeros_like(b)
    rep2 = Report()
    ok2 = r.ref_fft_gmres(rp, ptr(b), ptr(x2), 30, 300, 1e-10, 0.0, C.byref(rep2))
    assert ok1 and ok2
    assert rep1["iterations"] == rep2.iterations and rep1["restarts"] == rep2.restarts
    assert np.array_equal(x1, x2)
    r.ref_fft_destroy(rp)


@needs_ref
def test_fixture_tensors_match_reference(near_tables):
    """The committed near tensors are what the reference's vie_cuboid_n gives."""
    r = oracle_lib.reference()
    out = np.empty(9, dtype=np.complex128)
    for name in ("vie_k0.8", "c0", "m9_tree"):
        h, k, table = near_tables[name]
        assert len(table) == 13
        for v, t in table.items():
            assert r.ref_near_tensor(None, (C.c_size_t * 3)(*v), h, k, ptr(out))
            assert np.array_equal(out, t)


@needs_ref
def test_operator_matches_dense_reference_kernel(near_tables):
    """tests/vie_fft_test.c:19-34: product vs the dense vie_cuboid_n operator at 2e-8."""
    h, k, table = near_tables["vie_k0.8"]
    shape, xyz, er = cases.SPARSE_SHAPE, np.array(cases.SPARSE_XYZ), 3 - 0.4j
    cells = xyz.size // 3
    n = 3 * cells
    a = np.zeros((n, n), dtype=np.complex128)
    r = oracle_lib.reference()
    blk = np.empty(9, dtype=np.complex128)
    for c in range(cells):
        for d in range(cells):
            tc = np.ascontiguousarray(h * xyz[3 * c:3 * c + 3].astype(float))
            sc = np.ascontiguousarray(h * xyz[3 * d:3 * d + 3].astype(float))
            assert r.ref_pair_tensor(ptr(tc), ptr(sc), h, k, ptr(blk))
            a[3 * c:3 * c + 3, 3 * d:3 * d + 3] = -(er - 1) * blk.reshape(3, 3) + (np.eye(3) * er if c == d else 0)
    op = OraclePlan(shape, xyz, h, k, er, table)
    x = cases.probe_vector(n)
    b = a @ x
    y = op.apply(x)
    assert np.max(np.abs(y - b) / np.maximum(1, np.abs(b))) < 2e-8
    ok, sol, rep = op.gmres(b, rtol=1e-11, maxit=150)
    assert ok and np.max(np.abs(sol - x)) < 2e-8


def test_spectrum_symmetry(near_tables):
    """Green spectrum components are even/odd in each axis as the tensor is."""
    h, k, table = near_tables["vie_k0.8"]
    op = OraclePlan(cases.SPARSE_SHAPE, cases.SPARSE_XYZ, h, k, 3.0, table)
    P = op.padded
    s = op.spectrum().reshape(6, *P)
    flip = lambda a, ax: np.roll(np.flip(a, axis=ax), 1, axis=ax)
    for comp in range(3):
        for ax in range(3):
            assert np.allclose(s[comp], flip(s[comp], ax), atol=1e-12)
    assert np.allclose(s[3], -flip(s[3], 0), atol=1e-12)   # xy odd in x


# ---------------------------------------------------------------- dense
def kat_system():
    """tests/dense_backend_test.c:16-33."""
    a = np.array([[4 + 1j, 1 - 2j, 0.5], [2, 5 + 0.5j, -1j], [-1 + 1j, 0.25, 3 - 1j]])
    x = np.array([1 + 2j, -0.5 + 1j, 2 - 0.25j])
    return a, x, a @ x


def test_row_major_kat():
    a, x, b = kat_system()
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert oracle().oracle_row_major_solve(ptr(a), ptr(b), 3)
    assert np.max(np.abs(b - x)) < 1e-12


def test_classic_kat():
    a, x, b = kat_system()
    storage = np.zeros((5, 3), dtype=np.complex128, order="F")
    storage[:3, :3] = a.T          # NEC transposed storage, leading dimension 5
    piv = np.zeros(3, dtype=np.int32)
    assert oracle().oracle_factr(3, ptr(storage), ptr(piv), 5)
    bb = np.ascontiguousarray(b)
    oracle().oracle_solve(3, ptr(storage), ptr(piv), ptr(bb), 5)
    assert np.max(np.abs(bb - x)) < 1e-12


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 7, 64, 129])
def test_factr_matches_reference(n):
    rng = np.random.default_rng(n)
    ld = n + 3
    st = np.zeros((ld, n), dtype=np.complex128, order="F")
    st[:n] = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    st2 = st.copy(order="F")
    p1 = np.zeros(n, dtype=np.int32)
    p2 = np.zeros(n, dtype=np.int32)
    oracle().oracle_factr(n, ptr(st), ptr(p1), ld)
    oracle_lib.reference().ref_factr(n, ptr(st2), ptr(p2), ld)
    assert np.array_equal(p1, p2) and np.array_equal(st, st2)
    b1 = np.ascontiguousarray(rng.standard_normal(n) + 1j * rng.standard_normal(n))
    b2 = b1.copy()
    oracle().oracle_solve(n, ptr(st), ptr(p1), ptr(b1), ld)
    oracle_lib.reference().ref_solve(n, ptr(st2), ptr(p2), ptr(b2), ld)
    assert np.array_equal(b1, b2)


@needs_ref
@pytest.mark.parametrize("n", [1, 5, 40])
def test_row_major_matches_reference(n):
    rng = np.random.default_rng(10 + n)
    a = np.ascontiguousarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    b = np.ascontiguousarray(rng.standard_normal(n) + 1j * rng.standard_normal(n))
    a2, b2 = a.copy(), b.copy()
    assert oracle().oracle_row_major_solve(ptr(a), ptr(b), n)
    assert oracle_lib.reference().ref_row_major_solve(ptr(a2), ptr(b2), n)
    assert np.array_equal(b, b2)


# ---------------------------------------------------------------- GMRES
MAP = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))


def _gmres(n, apply, prec, b, x, restart=30, maxit=300, rtol=1e-12, atol=0.0):
    o = oracle()
    o.oracle_gmres.argtypes = [C.c_size_t, MAP, C.c_void_p, MAP, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_size_t, C.c_size_t, C.c_double, C.c_double, C.POINTER(Report)]
    o.oracle_gmres.restype = C.c_int
    rep = Report()
    ok = o.oracle_gmres(n, apply, None, prec if prec else MAP(), None, ptr(b), ptr(x), restart, maxit,
                        rtol, atol, C.byref(rep))
    return ok, rep


def _wrap(fn, n):
    def cb(ctx, xi, yo):
        x = np.ctypeslib.as_array(xi, shape=(2 * n,)).view(np.complex128)
        y = np.ctypeslib.as_array(yo, shape=(2 * n,)).view(np.complex128)
        return fn(x, y)
    return MAP(cb)


def stencil(x, y):
    """vie_iterative_test.c:38-49."""
    y[:] = (3 + 0.2j) * x
    y[1:] += (0.3 - 0.1j) * x[:-1]
    y[:-1] += (-0.5 + 0.3j) * x[1:]
    return 1


def test_gmres_matrix_free_restart():
    """vie_iterative_test.c:51-72."""
    n = 40
    i = np.arange(n)
    expected = np.sin(i) + 1j * np.cos(0.4 * i)
    b = np.empty(n, dtype=np.complex128)
    stencil(expected, b)
    x = np.zeros(n, dtype=np.complex128)
    op = _wrap(stencil, n)
    ok, rep = _gmres(n, op, None, b, x, restart=3)
    assert ok and rep.restarts > 0 and rep.relative_residual <= 1e-12
    assert np.max(np.abs(x - expected)) < 1e-10
    ok, rep = _gmres(n, op, None, b, x, restart=3)
    assert ok and rep.iterations == 0
    x[:] = 0
    ok, rep = _gmres(n, op, None, b, x, restart=3, maxit=1)
    assert not ok and rep.status == 1 and rep.iterations == 1


def test_gmres_failure_statuses():
    """vie_iterative_test.c:94-134 (subset)."""
    n = 3
    b = np.array([1 + 1j, 2 - 1j, -3 + 2j])
    ident = _wrap(lambda x, y: (y.__setitem__(slice(None), x), 1)[1], n)
    zero = _wrap(lambda x, y: (y.__setitem__(slice(None), 0), 1)[1], n)
    fail = _wrap(lambda x, y: 0, n)
    x = np.zeros(n, dtype=np.complex128)
    ok, rep = _gmres(n, ident, None, b, x)
    assert ok and rep.iterations == 1
    x[:] = 0
    ok, rep = _gmres(n, zero, None, np.array([1, 0, 0], dtype=np.complex128), x)
    assert not ok and rep.status == 2
    ok, rep = _gmres(n, fail, None, b, np.zeros(n, dtype=np.complex128))
    assert not ok and rep.status == 3
    ok, rep = _gmres(n, ident, fail, b, np.zeros(n, dtype=np.complex128))
    assert not ok and rep.status == 3


def test_hybrid_oracle_conductor_only():
    """dielectric_fft_test.c:167-170: no cells, two conductor rows."""
    blocks = np.array([2, 0, 0, 3], dtype=np.complex128)
    h = OracleHybrid(None, 2, 0, blocks)
    x = np.array([1 + 1j, 2 - 1j])
    y = h.apply(x)
    assert np.abs(y[0] - 2 * x[0]) + np.abs(y[1] - 3 * x[1]) < 1e-14


def fibonacci_directions(count, seed=0):
    """The reference's 974-point sphere quadrature rule (dielectric_solver.c:153-176)."""
    golden = np.pi * (3 - np.sqrt(5))
    i = np.arange(count)
    z = 1 - 2 * (i + 0.5) / count
    r = np.sqrt(np.maximum(0, 1 - z * z))
    return np.stack([r * np.cos(golden * i), r * np.sin(golden * i), z], axis=1)


@needs_ref
def test_radiation_amplitude_matches_reference():
    """dielectric_radiation_amplitude (free space) of random cells and currents,
    oracle restatement against the reference compiled here, 1e-13 relative."""
    rng = np.random.default_rng(31)
    h, k0 = 0.01, 6.28
    idx = rng.integers(0, 20, size=(300, 3))
    centers = 0.3 + h * idx
    current = rng.standard_normal(900) + 1j * rng.standard_normal(900)
    for d in list(fibonacci_directions(24)) + [np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0])]:
        a = oracle_lib.radiation_amplitude(centers, h, current, k0, d)
        r = oracle_lib.radiation_amplitude(centers, h, current, k0, d, use_reference=True)
        assert np.max(np.abs(a - r)) <= 1e-13 * np.max(np.abs(r))


@needs_ref
@pytest.mark.parametrize("pec,gap", [(False, 0.0), (True, 0.0), (True, 0.125)])
def test_hybrid_matches_reference(near_tables, pec, gap):
    """The hybrid [C B; D V] operator, its preconditioner and GMRES on it, the
    reference's through its own dielectric_fft_prepare(_pec) /
    dielectric_fft_entry / dielectric_fft_get_operator, against the oracle
    restatement on the same cells and blocks: bit-identical, in free space and
    with PEC images (bottom gap 0 and half a cell)."""
    from test_hybrid_gpu import lattice
    from test_vie_batch_gpu import hybrid_blocks
    h, k, table = near_tables["diel_k0.5"]
    idx = cases.random_lattice((4, 3, 3), 0.7, seed=17).reshape(-1, 3).astype(float)
    centers = np.ascontiguousarray(0.1 + h * idx)
    centers[:, 2] = gap + h / 2 + h * idx[:, 2]
    cells = len(centers)
    eps = cases.random_eps(cells, seed=18, er=(2.0, 5.0))
    c, v = 4, 3 * cells
    blocks, n = hybrid_blocks(c, v, 19)
    r = oracle_lib.reference()
    r.ref_fft_backend_set(b"builtin")
    rs = r.ref_hybrid_create(cells, ptr(centers), h, ptr(np.ascontiguousarray(eps)), c, ptr(blocks), k,
                             1 if pec else 0)
    assert rs
    shape, xyz = lattice(centers, h, pec)
    op = OraclePlan(shape, xyz, h, k, eps[0], table)
    for i, e in enumerate(eps):
        for q in ([i, cells + i] if pec else [i]):
            assert op.set_permittivity(q, e)
    oh = OracleHybrid(op, c, v, blocks, pec)
    rng = np.random.default_rng(20)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y_ref, p_ref = np.empty(n, dtype=np.complex128), np.empty(n, dtype=np.complex128)
    assert r.ref_hybrid_apply(rs, ptr(x), ptr(y_ref))
    assert r.ref_hybrid_precondition(rs, ptr(x), ptr(p_ref))
    assert np.array_equal(oh.apply(x), y_ref)
    ok, p = oh.precondition(x)
    assert ok and np.array_equal(p, p_ref)
    b = y_ref.copy()
    ok1, x1, rep1 = oh.gmres(b, rtol=1e-10)
    x2 = np.zeros_like(b)
    rep2 = Report()
    ok2 = r.ref_hybrid_gmres(rs, ptr(b), ptr(x2), 30, 300, 1e-10, 0.0, C.byref(rep2))
    assert ok1 and ok2
    assert rep1["iterations"] == rep2.iterations and rep1["restarts"] == rep2.restarts
    assert np.array_equal(x1, x2)
    r.ref_hybrid_destroy(rs)


@needs_ref
@pytest.mark.parametrize("gap,pec", [(0.0, False), (0.0, True), (0.125, True)])
def test_hybrid_against_dense_reference_kernel(near_tables, gap, pec):
    """tests/dielectric_fft_test.c:8-46: two cells of two materials, the
    product against the dense operator of the reference's pair tensors
    (vie_cuboid_n, or vie_cuboid_pec_n over the ground plane) at 2e-7, and
    GMRES recovering x to 1e-10."""
    from test_hybrid_gpu import lattice
    h, k, table = near_tables["diel_k0.5"]
    centers = np.array([(0.0, 0.0, 0.125 + gap), (0.25, -0.25, 0.375 + gap)])
    eps = [3 - 0.2j, 2 - 0.4j]
    shape, xyz = lattice(centers, h, pec)
    op = OraclePlan(shape, xyz, h, k, eps[0], table)
    for i, e in enumerate(eps):
        for q in ([i, 2 + i] if pec else [i]):
            assert op.set_permittivity(q, e)
    oh = OracleHybrid(op, 0, 6, np.zeros(1, dtype=np.complex128), pec)
    j = np.arange(6)
    x = np.sin(1 + j) + 1j * np.cos(0.3 * j)
    expected = np.repeat(eps, 3) * x
    r = oracle_lib.reference()
    pair = r.ref_pair_tensor_pec if pec else r.ref_pair_tensor
    block = np.empty(9, dtype=np.complex128)
    for a in range(2):
        for b in range(2):
            assert pair(ptr(np.ascontiguousarray(centers[a])), ptr(np.ascontiguousarray(centers[b])), h, k,
                        ptr(block))
            expected[3 * a:3 * a + 3] -= (eps[a] - 1) * (block.reshape(3, 3) @ x[3 * b:3 * b + 3])
    y = oh.apply(x)
    assert np.max(np.abs(y - expected)) < 2e-7
    ok, sol, rep = oh.gmres(y)
    assert ok and np.max(np.abs(sol - x)) < 1e-10


def _ref_gmres(n, apply, prec, b, x, restart=30, maxit=300, rtol=1e-12, atol=0.0):
    r = oracle_lib.reference()
    r.ref_callback_gmres.argtypes = [C.c_size_t, MAP, C.c_void_p, MAP, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_size_t, C.c_size_t, C.c_double, C.c_double, C.POINTER(Report)]
    rep = Report()
    ok = r.ref_callback_gmres(n, apply, None, prec if prec else MAP(), None, ptr(b), ptr(x), restart, maxit,
                              rtol, atol, C.byref(rep))
    return ok, rep


@needs_ref
def test_gmres_statuses_match_reference():
    """vie_iterative_test.c's operators (matrix-free stencil, identity, zero,
    failing and non-finite callbacks) and invalid inputs, run by the oracle
    and by the reference's vie_gmres on the same callbacks: same return
    value, the same report field by field, and the same x, bit for bit."""
    n = 40
    i = np.arange(n)
    b40 = np.zeros(n, dtype=np.complex128)
    stencil(np.sin(i) + 1j * np.cos(0.4 * i), b40)
    b3 = np.array([1 + 1j, 2 - 1j, -3 + 2j])

    def nan_map(x, y):
        y[:] = x
        y[0] = np.nan
        return 1
    ident = _wrap(lambda x, y: (y.__setitem__(slice(None), x), 1)[1], 3)
    runs = [
        (40, _wrap(stencil, 40), None, b40, {"restart": 3}),
        (40, _wrap(stencil, 40), None, b40, {"restart": 3, "maxit": 1}),
        (40, _wrap(stencil, 40), None, b40, {"restart": 40, "rtol": 1e-6}),
        (40, _wrap(stencil, 40), None, b40, {"restart": 5, "rtol": 0.0, "atol": 1e-9}),
        (3, ident, None, b3, {}),
        (3, _wrap(lambda x, y: (y.__setitem__(slice(None), 0), 1)[1], 3), None,
         np.array([1, 0, 0], dtype=np.complex128), {}),
        (3, _wrap(lambda x, y: 0, 3), None, b3, {}),
        (3, ident, _wrap(lambda x, y: 0, 3), b3, {}),
        (3, _wrap(nan_map, 3), None, b3, {}),
        (3, ident, None, b3, {"restart": 0}),
        (3, ident, None, b3, {"maxit": 0}),
        (3, ident, None, b3, {"rtol": 0.0, "atol": 0.0}),
        (3, ident, None, b3, {"rtol": -1.0}),
        (3, ident, None, np.zeros(3, dtype=np.complex128), {}),
    ]
    for n, apply, prec, b, kw in runs:
        x1 = np.zeros(n, dtype=np.complex128)
        x2 = np.zeros(n, dtype=np.complex128)
        ok1, rep1 = _gmres(n, apply, prec, b, x1, **kw)
        ok2, rep2 = _ref_gmres(n, apply, prec, b, x2, **kw)
        assert ok1 == ok2, kw
        d1, d2 = rep1.as_dict(), rep2.as_dict()
        for f in d1:
            assert d1[f] == d2[f] or (np.isnan(d1[f]) and np.isnan(d2[f])), (kw, f, d1, d2)
        assert np.array_equal(x1, x2, equal_nan=True), kw
