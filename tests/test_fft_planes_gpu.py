"""Fused yz-plane passes (fft_plane.cuh) against the oracle and against the
five-pass form of the same plan.

The plane passes apply when the padded y and z axes are one length P = 2Q with
Q in {16, 32, 64}; they replace the z and y passes on each side of the x pass.
On lattices of each Q (cells shuffled, so the cell order is not the box
order), with the plane passes pinned (set_planes) and with the
five-pass form pinned, the product matches the oracle at the volume tests'
tolerances (FP64 1e-12 relative to the largest entry, FP32 1e-5 relative L2),
the Jacobi-preconditioned product GMRES runs on matches too, and GMRES
converges to the same solution either way."""
import numpy as np
import pytest

import cases
import nec2c_b200 as nb
from oracle_lib import OraclePlan

pytestmark = pytest.mark.gpu

# (shape, fill, seed): Q = 16, 32, 64 in y and z.
SHAPES = [((5, 16, 9), 0.8, 21), ((3, 30, 20), 0.7, 22), ((4, 64, 40), 0.5, 23)]


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def pin(plan, fp64, planes):
    assert plan.set_planes(planes, fp64=fp64), nb.last_error()
    assert plan.planes(fp64=fp64) == int(planes)


@pytest.mark.parametrize("shape,fill,seed", SHAPES)
def test_plane_passes_match_oracle(near_tables, shape, fill, seed):
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
    y, px = op.apply(x), op.precondition(x)
    b = op.apply(np.ones(op.n, dtype=np.complex128))
    sols = {}
    for planes in (True, False):
        # The mixed plan's FP64 transforms (its true residuals) follow its
        # FP64 choice.
        for plan, fp64 in ((gp, True), (gm, False), (gm, True)):
            pin(plan, fp64, planes)
        assert rel_max(gp.apply(x), y) < 1e-12
        assert rel_l2(gm.apply(x), y) < 1e-5
        assert rel_max(gp.precondition(x), px) < 1e-15
        ok, sol, rep = gp.gmres(b, rtol=1e-10, maxit=600)
        assert ok and rep["relative_residual"] <= 1e-10, rep
        sols[planes] = sol
        ok, sol_m, rep_m = gm.gmres(b, rtol=1e-9, maxit=600)
        assert ok and rep_m["relative_residual"] <= 1e-9, rep_m
        assert rel_l2(sol_m, sol) < 1e-7
    assert rel_l2(sols[True], sols[False]) < 1e-8
    gp.close()
    gm.close()


def test_plane_passes_refused_where_not_applicable(near_tables):
    """A lattice whose padded y and z differ keeps the five passes: the
    choice reads -1 and pinning the plane passes is refused."""
    h, k, table = near_tables["rand_k0.3"]
    shape = (6, 9, 20)            # padded y 32, z 64
    xyz = cases.random_lattice(shape, 0.8, 31)
    gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
    assert gp.planes(fp64=True) == -1
    assert not gp.set_planes(True, fp64=True)
    assert "plane" in nb.last_error()
    assert gp.set_planes(False, fp64=True)
    assert gp.planes(fp64=True) == -1
    gp.close()
