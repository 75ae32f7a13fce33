"""FFT pass schedule (tile height and radix split of the five matvec passes).

Every schedule computes the same transform, so the product must match the
oracle at the volume tests' tolerances whatever the schedule: FP64 form 1e-12
relative to the largest entry, FP32 form 1e-5 relative L2.  Checked for the
schedule the tuner measured, for the heuristic, and pass by pass for every
radix split on offer at the smallest, a middle and the largest tile height,
on two lattices whose padded axes cover every length with two splits
(16, 32, 64, 128) on every pass kind.  Pinned schedules outside the offer
are refused and leave the schedule as it was."""
import numpy as np
import pytest

import cases
import nec2c_b200 as nb
from oracle_lib import OraclePlan

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5
SPLITS = {16: (16, 4), 32: (8, 4), 64: (8, 16), 128: (16, 8)}
SHAPES = [((40, 9, 5), 0.7, 11), ((9, 20, 40), 0.7, 12)]


def padded(n):
    p = 1
    while p < 2 * n - 1:
        p *= 2
    return p


def pass_length(shape, i):
    P = [padded(n) for n in shape]
    return P[2] if i in (0, 4) else (P[0] if i == 2 else P[1])


def heights(shape, i, elem):
    """The heights the tuner tries (and set_schedule accepts)."""
    L = pass_length(shape, i)
    if i in (0, 4):
        cols = shape[0] * shape[1]
        return [nl for nl in range(3, 97, 3)
                if 2 * (nl + 1) * L * elem <= 100 * 1024 and (i == 0 or -(-cols // (nl // 3)) <= 65536)]
    ncomp = 3 if i == 2 else 1
    return [nl for nl in (1, 2, 4, 8, 16, 32, 64) if L * ncomp * nl * elem <= 100 * 1024]


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def build(near_tables, shape, fill, seed):
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
    return op, gp, gm, x, op.apply(x)


def check(plan, fp64, x, y):
    if fp64:
        assert rel_max(plan.apply(x), y) < FP64_TOL
    else:
        assert rel_l2(plan.apply(x), y) < FP32_TOL


@pytest.mark.parametrize("shape,fill,seed", SHAPES)
def test_tuned_schedule_within_offer(near_tables, shape, fill, seed):
    assert nb.fft_autotune_enabled()
    op, gp, gm, x, y = build(near_tables, shape, fill, seed)
    check(gp, True, x, y)
    check(gm, False, x, y)
    for plan, precs in ((gp, (True,)), (gm, (False, True))):
        for fp64 in precs:
            measured, sched = plan.schedule(fp64=fp64)
            assert measured
            plan.tune(0)
            _, heuristic = plan.schedule(fp64=fp64)
            for i, ((nl, r1), (nl_h, _)) in enumerate(zip(sched, heuristic)):
                L = pass_length(shape, i)
                assert r1 in SPLITS.get(L, (r1,)) and L % r1 == 0
                # The tuner keeps the heuristic height unless a candidate wins.
                assert nl == nl_h or nl in heights(shape, i, 16 if fp64 else 8)
            plan.tune(1)      # the shape's cached choice comes back
            assert plan.schedule(fp64=fp64) == (True, sched)
    # Heuristic, then timed afresh: same product within tolerance.
    for plan, fp64 in ((gp, True), (gm, False)):
        plan.tune(0)
        assert not plan.schedule(fp64=fp64)[0]
        check(plan, fp64, x, y)
        plan.tune(2)
        assert plan.schedule(fp64=fp64)[0]
        check(plan, fp64, x, y)


@pytest.mark.parametrize("shape,fill,seed", SHAPES)
def test_every_split_and_height_matches_oracle(near_tables, shape, fill, seed):
    op, gp, gm, x, y = build(near_tables, shape, fill, seed)
    for plan, fp64 in ((gp, True), (gm, False)):
        plan.tune(0)
        _, base = plan.schedule(fp64=fp64)
        elem = 16 if fp64 else 8
        tried = 0
        for i in range(5):
            offer = heights(shape, i, elem)
            picks = sorted({offer[0], offer[len(offer) // 2], offer[-1]})
            for r1 in SPLITS.get(pass_length(shape, i), (base[i][1],)):
                for nl in picks:
                    sched = list(base)
                    sched[i] = (nl, r1)
                    assert plan.set_schedule(sched, fp64=fp64), nb.last_error()
                    assert plan.schedule(fp64=fp64) == (True, sched)
                    check(plan, fp64, x, y)
                    tried += 1
        assert tried >= 5 * 3
    # GMRES after a pinned schedule (the captured cycle is rebuilt).
    b = op.apply(np.ones(op.n, dtype=np.complex128))
    ok, sol, rep = gp.gmres(b, rtol=1e-10, maxit=400)
    assert ok and rep["relative_residual"] <= 1e-10


def test_pinned_schedule_refused_outside_offer(near_tables):
    shape = SHAPES[0][0]
    op, gp, gm, x, y = build(near_tables, shape, 0.7, 11)
    before = gp.schedule(fp64=True)
    _, base = before
    bad = list(base)
    bad[0] = (4, base[0][1])                 # z pass: not whole lattice columns
    assert not gp.set_schedule(bad, fp64=True)
    assert "lines per tile" in nb.last_error()
    bad = list(base)
    bad[1] = (3, base[1][1])                 # strided pass: not a power of two
    assert not gp.set_schedule(bad, fp64=True)
    bad = list(base)
    bad[2] = (base[2][0], 2)                 # 2 x 64 is not a split on offer
    assert not gp.set_schedule(bad, fp64=True)
    assert "radix" in nb.last_error()
    bad = list(base)
    bad[1] = (128, base[1][1])               # above the largest height (64)
    assert not gp.set_schedule(bad, fp64=True)
    assert gp.schedule(fp64=True) == before
    # An FP64 plan has no FP32 schedule.
    with pytest.raises(RuntimeError):
        gp.schedule(fp64=False)
    assert not gp.set_schedule(base, fp64=False)
    check(gp, True, x, y)
