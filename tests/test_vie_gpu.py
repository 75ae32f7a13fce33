"""CUDA volume operator and device GMRES against the oracle (FP64 form: 1e-12
relative; FP32 mixed form: 1e-5 relative L2), on the reference's own test
lattices, seeded random lattices and the reference's published M9 results."""
import numpy as np
import pytest

import cases
import nec2c_b200 as nb
from oracle_lib import OraclePlan

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12      # relative to the largest output entry
FP32_TOL = 1e-5       # relative L2 (mixed form)

VIE_CASES = [
    ("vie_k0.2", (1, 1, 1), [0, 0, 0], 3.0),
    ("vie_k0", cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 3.0),
    ("vie_k0.8", cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 3.0),
    ("vie_k4", cases.FAR_SHAPE, cases.FAR_XYZ, 3.0),
    ("vie_k0.2", (1, 1, 1), [0, 0, 0], 1.0),
    ("vie_k0.2", (1, 1, 1), [0, 0, 0], 3 - 0.4j),
    ("vie_k0.8", cases.SPARSE_SHAPE, cases.SPARSE_XYZ, 3 - 0.4j),
]


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("case", VIE_CASES)
def test_matvec_reference_lattices(near_tables, case):
    name, shape, xyz, eps = case
    h, k, table = near_tables[name]
    op = OraclePlan(shape, xyz, h, k, eps, table)
    gp = nb.VolumePlan(shape, xyz, h, k, eps, table)
    n = op.n
    probes = [cases.probe_vector(n)] + [np.eye(n, dtype=np.complex128)[j] * (1 + 2j) for j in range(n)]
    for x in probes:
        assert rel_max(gp.apply(x), op.apply(x)) < FP64_TOL
        assert rel_max(gp.precondition(x), op.precondition(x)) < 1e-15
    g = int(np.prod(op.padded))
    assert rel_max(gp.spectrum(g), op.spectrum() / g) < FP64_TOL
    assert gp.bytes() > 0


@pytest.mark.parametrize("shape,fill,seed", [((7, 6, 5), 0.6, 1), ((12, 9, 17), 0.5, 2),
                                             ((24, 24, 24), 0.9, 3), ((2, 31, 3), 1.0, 4)])
def test_matvec_random_lattices(near_tables, shape, fill, seed):
    h, k, table = near_tables["rand_k0.3"]
    xyz = cases.random_lattice(shape, fill, seed)
    eps = cases.random_eps(xyz.size // 3, seed + 100)
    op = OraclePlan(shape, xyz, h, k, 3.0, table)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
    gm = nb.VolumePlan(shape, xyz, h, k, 3.0, table, mixed=True)
    for c, e in enumerate(eps):
        assert op.set_permittivity(c, e) and gp.set_permittivity(c, e) and gm.set_permittivity(c, e)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(op.n) + 1j * rng.standard_normal(op.n)
    y = op.apply(x)
    assert rel_max(gp.apply(x), y) < FP64_TOL
    assert rel_l2(gm.apply(x), y) < FP32_TOL
    assert rel_max(gp.precondition(x), op.precondition(x)) < 1e-15


def test_invalid_plans_rejected(near_tables):
    """tests/vie_fft_test.c:50-54, 69-74: the same arguments are refused."""
    h, k, table = near_tables["vie_k0.2"]
    with pytest.raises(RuntimeError):
        nb.VolumePlan(cases.SPARSE_SHAPE, cases.SPARSE_XYZ, .25, .2, 3, table, byte_limit=1)
    with pytest.raises(RuntimeError):
        nb.VolumePlan(cases.SPARSE_SHAPE, [0, 0, 0, 0, 0, 0], .25, .2, 3, table)
    with pytest.raises(RuntimeError):
        nb.VolumePlan((1, 1, 1), cases.SPARSE_XYZ, .25, .2, 3, table)
    with pytest.raises(RuntimeError):
        nb.VolumePlan((1, 1, 1), [0, 0, 0], .25, 5, 3, table)
    with pytest.raises(RuntimeError):
        nb.VolumePlan((1, 1, 1), [0, 0, 0], .25, .2, 3 + .4j, table)
    gp = nb.VolumePlan((1, 1, 1), [0, 0, 0], .25, .2, 3, table)
    assert not gp.set_permittivity(1, 2)
    assert not gp.set_permittivity(0, 3 + .1j)
    assert not gp.set_permittivity(0, complex("nan"))
    assert gp.set_permittivity(0, 1 - .4j)


@pytest.mark.parametrize("case", VIE_CASES)
def test_gmres_matches_oracle(near_tables, case):
    """vie_fft_test.c:36-39: recover x to 2e-8 at rtol 1e-11, same iterations as the oracle."""
    name, shape, xyz, eps = case
    h, k, table = near_tables[name]
    op = OraclePlan(shape, xyz, h, k, eps, table)
    gp = nb.VolumePlan(shape, xyz, h, k, eps, table)
    x = cases.probe_vector(op.n)
    b = op.apply(x)
    ok_o, xo, ro = op.gmres(b, rtol=1e-11, maxit=150)
    ok_g, xg, rg = gp.gmres(b, rtol=1e-11, maxit=150)
    assert ok_o and ok_g
    assert rg["status"] == 0 and rg["iterations"] == ro["iterations"]
    assert rg["relative_residual"] <= 1e-11
    assert np.max(np.abs(xg - x)) < 2e-8
    assert rel_max(xg, xo) < 1e-9


def test_gmres_random_lattice_and_statuses(near_tables):
    h, k, table = near_tables["rand_k0.3"]
    shape = (12, 9, 17)
    xyz = cases.random_lattice(shape, 0.5, 7)
    eps = cases.random_eps(xyz.size // 3, 8)
    op = OraclePlan(shape, xyz, h, k, 3.0, table)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
    for c, e in enumerate(eps):
        op.set_permittivity(c, e)
        gp.set_permittivity(c, e)
    rng = np.random.default_rng(9)
    b = rng.standard_normal(op.n) + 1j * rng.standard_normal(op.n)
    ok_o, xo, ro = op.gmres(b, restart=10, rtol=1e-10)
    ok_g, xg, rg = gp.gmres(b, restart=10, rtol=1e-10)
    assert ok_o and ok_g and rg["iterations"] == ro["iterations"] and rg["restarts"] == ro["restarts"]
    assert rel_l2(xg, xo) < 1e-9
    # iteration limit is explicit and keeps the measured residual
    ok, x1, r1 = gp.gmres(b, restart=10, maxit=3, rtol=1e-10)
    assert not ok and r1["status"] == 1 and r1["iterations"] == 3
    assert r1["relative_residual"] > 1e-10
    # already-converged initial guess
    ok, x2, r2 = gp.gmres(b, x0=xg, restart=10, rtol=1e-8)
    assert ok and r2["iterations"] == 0
    # non-finite right-hand side
    bad = b.copy()
    bad[5] = np.nan
    ok, _, r3 = gp.gmres(bad)
    assert not ok and r3["status"] == 6
    # invalid options
    ok, _, r4 = gp.gmres(b, restart=0)
    assert not ok and r4["status"] == 4


def test_m9_skeleton_published_currents(near_tables, reference_golden):
    """tests/m9-fft-skeleton-1e-8.txt: iterations and integrated currents."""
    shape, xyz, h, k, rhs = cases.m9_model(full=False)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, near_tables["m9_tree"][2])
    for tol in ("1e-8", "1e-10"):
        gold = reference_golden["skeleton_" + tol]
        ok, sol, rep = gp.gmres(rhs, rtol=float(tol), maxit=150)
        assert ok and rep["iterations"] == gold["iterations"]
        cur = cases.integrated_current(sol, h)
        for d in range(3):
            want = complex(*gold["integrated_normalized_current_%d" % d])
            assert abs(cur[d] - want) <= 2e-11 + 1e-9 * abs(want), (d, cur[d], want)


def test_m9_tree_published_currents(near_tables, reference_golden):
    """tests/m9-fft-tree-1e-8.txt: 9432 cells, 28296 unknowns."""
    shape, xyz, h, k, rhs = cases.m9_model(full=True)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, near_tables["m9_tree"][2])
    gold = reference_golden["tree_1e-8"]
    ok, sol, rep = gp.gmres(rhs, rtol=1e-8, maxit=150)
    assert ok and rep["iterations"] == gold["iterations"]
    cur = cases.integrated_current(sol, h)
    for d in range(3):
        want = complex(*gold["integrated_normalized_current_%d" % d])
        assert abs(cur[d] - want) <= 1e-10 + 1e-9 * abs(want), (d, cur[d], want)
    # the mixed form reaches the same solution to the FP32 operator accuracy
    gm = nb.VolumePlan(shape, xyz, h, k, 3.0, near_tables["m9_tree"][2], mixed=True)
    ok, solm, rep = gm.gmres(rhs, rtol=1e-8, maxit=150)
    assert ok and rel_l2(solm, sol) < 1e-5


def test_gmres_large_system_paths(near_tables):
    """A 40^3 lattice (192,000 unknowns): the FP64 form's multi-element MGS
    kernel matches the oracle iterate for iterate (3 iterations), and the mixed
    form's CGS2 sweeps reach the FP64 solution to the FP32 operator accuracy."""
    h, k, table = near_tables["c0"]
    shape = (40, 40, 40)
    xyz = cases.random_lattice(shape, 1.0, 11)
    eps = cases.random_eps(xyz.size // 3, 12, er=(2.0, 4.0))
    op = OraclePlan(shape, xyz, h, k, 3.0, table)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
    gm = nb.VolumePlan(shape, xyz, h, k, 3.0, table, mixed=True)
    for c, e in enumerate(eps):
        op.set_permittivity(c, e)
        gp.set_permittivity(c, e)
        gm.set_permittivity(c, e)
    rng = np.random.default_rng(13)
    b = rng.standard_normal(op.n) + 1j * rng.standard_normal(op.n)
    _, xo, ro = op.gmres(b, restart=30, maxit=3, rtol=1e-12)
    _, xg, rg = gp.gmres(b, restart=30, maxit=3, rtol=1e-12)
    assert rg["iterations"] == ro["iterations"] == 3
    assert rel_l2(xg, xo) < 1e-10
    assert abs(rg["residual_norm"] - ro["residual_norm"]) <= 1e-9 * ro["residual_norm"]
    ok64, x64, r64 = gp.gmres(b, restart=30, maxit=400, rtol=1e-8)
    okm, xm, rm = gm.gmres(b, restart=30, maxit=400, rtol=1e-8)
    assert ok64 and okm and r64["relative_residual"] <= 1e-8 and rm["relative_residual"] <= 1e-8
    assert rel_l2(xm, x64) < 1e-6


def test_radiation_amplitude(near_tables):
    """Far-field amplitude of a cell current (dielectric_solver.c:90-150, free
    space) on the device against the oracle restatement (pinned to the
    reference in test_oracle.py): 1e-12 relative to the largest amplitude."""
    import oracle_lib
    from test_oracle import fibonacci_directions
    h, k, table = near_tables["rand_k0.3"]
    shape = (12, 9, 17)
    xyz = cases.random_lattice(shape, 0.5, 41)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
    rng = np.random.default_rng(42)
    cur = rng.standard_normal(gp.n) + 1j * rng.standard_normal(gp.n)
    origin = (0.37, -1.25, 2.5)
    dirs = np.concatenate([fibonacci_directions(97), np.eye(3), -np.eye(3)])
    got = gp.radiation(cur, dirs, origin)
    centers = np.asarray(origin) + h * xyz.reshape(-1, 3).astype(np.float64)
    want = np.array([oracle_lib.radiation_amplitude(centers, h, cur, k, d) for d in dirs])
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
