"""CUDA hybrid [C B; D V] operator (dielectric_fft.c) against the oracle, with
and without the PEC image embedding, and its device GMRES."""
import numpy as np
import pytest

import cases
import nec2c_b200 as nb
from oracle_lib import OracleHybrid, OraclePlan

pytestmark = pytest.mark.gpu


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def lattice(centers, h, pec):
    """Lattice indices and shape as dielectric_fft.c:109-154 infers them."""
    c = np.asarray(centers, dtype=float)
    origin = c.min(axis=0)
    idx = np.rint((c - origin) / h).astype(np.int64)
    shape = idx.max(axis=0) + 1
    if not pec:
        return [int(s) for s in shape], idx.reshape(-1).astype(np.uintp)
    gap = int(round(2 * (origin[2] - 0.5 * h) / h))
    nz = int(shape[2])
    phys = idx.copy()
    img = idx.copy()
    img[:, 2] = nz - 1 - idx[:, 2]
    phys[:, 2] += nz + gap
    shape[2] = 2 * nz + gap
    return [int(s) for s in shape], np.concatenate([phys.reshape(-1), img.reshape(-1)]).astype(np.uintp)


def material_case(near_tables, gap, pec):
    """tests/dielectric_fft_test.c:8-46 geometry: two cells, two materials."""
    h, k, table = near_tables["diel_k0.5"]
    centers = [(0.0, 0.0, 0.125 + gap), (0.25, -0.25, 0.125 + gap + 0.25)]
    eps = [3 - 0.2j, 2 - 0.4j]
    shape, xyz = lattice(centers, h, pec)
    op = OraclePlan(shape, xyz, h, k, eps[0], table)
    gp = nb.VolumePlan(shape, xyz, h, k, eps[0], table)
    cells = len(centers)
    for i, e in enumerate(eps):
        for p in ([i, cells + i] if pec else [i]):
            assert op.set_permittivity(p, e) and gp.set_permittivity(p, e)
    return op, gp, 3 * cells


@pytest.mark.parametrize("gap,pec", [(0.0, False), (0.0, True), (0.125, True)])
def test_material_cases(near_tables, gap, pec):
    op, gp, v = material_case(near_tables, gap, pec)
    oh = OracleHybrid(op, 0, v, np.zeros(1, dtype=np.complex128), pec)
    gh = nb.HybridSystem(gp, 0, v, pec)
    gh.set_blocks(np.zeros(1, dtype=np.complex128))
    x = np.array([np.sin(1 + j) + 1j * np.cos(0.3 * j) for j in range(v)])
    assert rel_max(gh.apply(x), oh.apply(x)) < 1e-12
    y = oh.apply(x)
    ok, sol, rep = gh.gmres(y)
    assert ok and np.max(np.abs(sol - x)) < 1e-10


def test_conductor_rows_and_preconditioner(near_tables):
    """dielectric_fft_test.c:140-158: two cells plus two conductor rows."""
    h, k, table = near_tables["diel_k0.5"]
    shape, xyz = lattice([(0.0, 0.0, 0.0), (0.25, 0.0, 0.0)], h, False)
    op = OraclePlan(shape, xyz, h, k, 3.0, table)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
    c, v = 2, 6
    n = c + v
    blocks = np.zeros(c * n + v * c, dtype=np.complex128)
    for i in range(n):
        for j in range(n):
            if i < c or j < c:
                val = (4 + 1j) if i == j else 0.002 * (1 + i + 2 * j) + 0.003j * (2 + i - j)
                if i < c:
                    blocks[i * n + j] = val
                else:
                    blocks[c * n + (i - c) * c + j] = val
    oh = OracleHybrid(op, c, v, blocks)
    gh = nb.HybridSystem(gp, c, v)
    gh.set_blocks(blocks)
    x = np.array([np.sin(0.5 * i) + 1j * np.cos(0.3 * i) for i in range(n)])
    b = gh.apply(x)
    assert rel_max(b, oh.apply(x)) < 1e-12
    ok, sol, rep = gh.gmres(b)
    ok_o, solo, repo = oh.gmres(b)
    assert ok and ok_o and rep["iterations"] == repo["iterations"]
    assert np.max(np.abs(sol - x)) < 1e-10
    okp, plain = gh.precondition(b)
    assert okp and np.max(np.abs(plain[:2] - b[:2] / (4 + 1j))) < 1e-14


def test_conductors_only():
    """dielectric_fft_test.c:167-170."""
    gh = nb.HybridSystem(None, 2, 0)
    gh.set_blocks(np.array([2, 0, 0, 3], dtype=np.complex128))
    x = np.array([1 + 1j, 2 - 1j])
    y = gh.apply(x)
    assert abs(y[0] - 2 * x[0]) + abs(y[1] - 3 * x[1]) < 1e-14


def test_zero_conductor_diagonal_fails_preconditioner():
    gh = nb.HybridSystem(None, 2, 0)
    gh.set_blocks(np.array([0, 1, 1, 3], dtype=np.complex128))
    ok, _ = gh.precondition(np.ones(2, dtype=np.complex128))
    assert not ok and "diagonal entry is zero" in nb.last_error()
    ok, _, rep = gh.gmres(np.ones(2, dtype=np.complex128))
    assert not ok and rep["status"] == 3


def test_dipole_plus_cube_random_blocks(near_tables):
    """A 16^3 cube beside 21 wire unknowns, with seeded
    synthetic conductor blocks, against the oracle at rtol 1e-12."""
    h, k, table = near_tables["c0"]
    shape = (16, 16, 16)
    xyz = cases.random_lattice(shape, 1.0, 0)
    op = OraclePlan(shape, xyz, h, k, 4 - 0.1j, table)
    gp = nb.VolumePlan(shape, xyz, h, k, 4 - 0.1j, table)
    c, v = 21, op.n
    n = c + v
    rng = np.random.default_rng(21)
    top = (rng.standard_normal((c, n)) + 1j * rng.standard_normal((c, n))) * 1e-3
    top[np.arange(c), np.arange(c)] = 50 + 20j + rng.standard_normal(c)
    cross = (rng.standard_normal((v, c)) + 1j * rng.standard_normal((v, c))) * 1e-3
    blocks = np.concatenate([top.reshape(-1), cross.reshape(-1)])
    oh = OracleHybrid(op, c, v, blocks)
    gh = nb.HybridSystem(gp, c, v)
    gh.set_blocks(blocks)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert rel_max(gh.apply(x), oh.apply(x)) < 1e-12
    b = oh.apply(x)
    ok_o, xo, ro = oh.gmres(b, rtol=1e-12)
    ok_g, xg, rg = gh.gmres(b, rtol=1e-12)
    assert ok_o and ok_g and rg["iterations"] == ro["iterations"]
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-9
