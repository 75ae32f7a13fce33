"""Ragged batch of volume plans (nec2c_cuda_vie_batch_*, nec2c_cuda_gmres_batch).

The batched product runs the same tile bodies as a single plan's product, on
taller tiles and inlined into other kernels (the compiler may fuse a
multiply-add differently), so each plan's slice of the batched product, under
the tuned and under every pinned batch schedule, equals the plan's own
product (default radix split) to rounding (1e-14 of the largest entry in
FP64, 1e-6 with FP32 transforms), and the FP64 form matches the oracle to
1e-12 relative to the largest entry.  Batched GMRES
solves each system with vie_gmres's per-system semantics: every system's
true relative residual meets the tolerance, the solution matches the oracle's
GMRES solution (FP64 form: 1e-8 relative at rtol 1e-11; FP32 transforms:
1e-5 at rtol 1e-8, the volume tests' mixed tolerance), and statuses are
per system (a zero right-hand side converges at once, an iteration limit
or a non-finite right-hand side stops only its own system)."""
import ctypes as C

import numpy as np
import pytest

import cases
import nec2c_b200 as nb
from oracle_lib import OracleHybrid, OraclePlan

pytestmark = pytest.mark.gpu

# Ragged lattices: padded axes from 1 to 256 (every line length of the batch).
LATTICES = [((7, 6, 5), 0.6, 1), ((12, 9, 17), 0.5, 2), ((1, 1, 1), 1.0, 3), ((16, 16, 16), 1.0, 4),
            ((40, 3, 2), 0.8, 5), ((2, 31, 3), 1.0, 6), ((5, 4, 33), 0.7, 7), ((3, 2, 70), 0.9, 8),
            ((66, 2, 2), 0.8, 9)]


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make(near_tables, mixed, lattices=LATTICES, oracle=True):
    h, k, table = near_tables["rand_k0.3"]
    plans, oracles = [], []
    for shape, fill, seed in lattices:
        xyz = cases.random_lattice(shape, fill, seed)
        eps = cases.random_eps(xyz.size // 3, seed + 50, er=(2.0, 6.0))
        gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table, mixed=mixed)
        op = OraclePlan(shape, xyz, h, k, 3.0, table) if oracle else None
        for c, e in enumerate(eps):
            assert gp.set_permittivity(c, e)
            if op:
                assert op.set_permittivity(c, e)
        plans.append(gp)
        oracles.append(op)
    return plans, oracles


@pytest.mark.parametrize("mixed", [False, True])
def test_batched_product_equals_each_plan(near_tables, mixed):
    import torch
    plans, oracles = make(near_tables, mixed)
    for p in plans:
        p.tune(0)          # default radix split, as in the batched passes
    batch = nb.VolumeBatch(plans)
    assert batch.order == sum(p.n for p in plans)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(batch.order) + 1j * rng.standard_normal(batch.order)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    assert nb.load().nec2c_cuda_vie_batch_apply_device(batch.h, C.c_void_p(xd.data_ptr()),
                                                       C.c_void_p(yd.data_ptr())), nb.last_error()
    own = [p.apply(x[batch.offsets[q]:batch.offsets[q + 1]]) for q, p in enumerate(plans)]
    tuned = batch.schedule()
    assert all(-1 <= a <= 1 and b in (0, 1) for a, b in tuned)
    # The tuned schedule, then every height scale and radix split pinned.
    for sched in (tuned, [(0, 1)] * 5, [(-1, 0)] * 4 + [(0, 0)], [(1, 1)] * 5, [(-1, 1)] * 4 + [(1, 0)]):
        assert batch.set_schedule(sched), nb.last_error()
        assert batch.schedule() == list(sched)
        yd.zero_()
        assert nb.load().nec2c_cuda_vie_batch_apply_device(batch.h, C.c_void_p(xd.data_ptr()),
                                                           C.c_void_p(yd.data_ptr())), nb.last_error()
        y = yd.cpu().numpy()
        for q, (p, op) in enumerate(zip(plans, oracles)):
            xs = x[batch.offsets[q]:batch.offsets[q + 1]]
            ys = y[batch.offsets[q]:batch.offsets[q + 1]]
            assert rel_max(ys, own[q]) < (1e-6 if mixed else 1e-14), (q, sched)
            ref = op.apply(xs)
            if mixed:
                assert rel_l2(ys, ref) < 1e-5
            else:
                assert rel_max(ys, ref) < 1e-12
    assert not batch.set_schedule([(2, 0)] * 5)       # out of range: refused, schedule kept
    assert batch.schedule() == [(-1, 1)] * 4 + [(1, 0)]
    batch.close()


@pytest.mark.parametrize("mixed,rtol,tol", [(False, 1e-11, 1e-8), (True, 1e-8, 1e-5)])
def test_batched_gmres_matches_oracle(near_tables, mixed, rtol, tol):
    plans, oracles = make(near_tables, mixed)
    batch = nb.VolumeBatch(plans)
    rng = np.random.default_rng(5)
    bs = [rng.standard_normal(p.n) + 1j * rng.standard_normal(p.n) for p in plans]
    ok, xs, reps = batch.gmres(bs, rtol=rtol, maxit=600)
    assert ok, (reps, nb.last_error())
    for q, (p, op) in enumerate(zip(plans, oracles)):
        assert reps[q]["status"] == 0
        assert reps[q]["relative_residual"] <= rtol
        # True residual of the returned solution, from the oracle's product.
        r = bs[q] - op.apply(xs[q])
        assert np.linalg.norm(r) <= 1.01 * rtol * np.linalg.norm(bs[q])
        ok_o, xo, ro = op.gmres(bs[q], rtol=1e-12, maxit=600)
        assert ok_o
        assert rel_l2(xs[q], xo) < tol
        # The single-plan solve takes about as many iterations.
        ok_s, xsingle, rs = p.gmres(bs[q], rtol=rtol, maxit=600)
        assert ok_s and abs(rs["iterations"] - reps[q]["iterations"]) <= max(3, rs["iterations"] // 10)
    batch.close()


def test_per_system_statuses(near_tables):
    lat = [((7, 6, 5), 0.6, 1), ((8, 8, 8), 1.0, 2), ((6, 6, 6), 0.9, 3), ((5, 9, 3), 1.0, 4)]
    plans, oracles = make(near_tables, False, lat)
    batch = nb.VolumeBatch(plans)
    rng = np.random.default_rng(9)
    bs = [rng.standard_normal(p.n) + 1j * rng.standard_normal(p.n) for p in plans]
    bs[1][:] = 0                      # zero right-hand side: converged at once
    bs[3][2] = np.nan                 # non-finite right-hand side
    ok, xs, reps = batch.gmres(bs, rtol=1e-10, maxit=500)
    assert not ok
    assert reps[0]["status"] == 0 and reps[0]["relative_residual"] <= 1e-10
    assert reps[1]["status"] == 0 and reps[1]["iterations"] == 0 and np.all(xs[1] == 0)
    assert reps[2]["status"] == 0
    assert reps[3]["status"] == 6     # VIE_ITERATIVE_NONFINITE
    # An iteration limit stops only the systems that reach it.
    bs[3][2] = 1.0
    ok, xs, reps = batch.gmres(bs, rtol=1e-12, maxit=7, restart=5)
    for q in (0, 2, 3):
        assert reps[q]["status"] == 1 and reps[q]["iterations"] == 7   # VIE_ITERATIVE_LIMIT
        assert reps[q]["restarts"] == 1
    assert reps[1]["status"] == 0
    # A good initial guess converges at the first true residual.
    ok, xs2, reps2 = batch.gmres(bs, x0s=[op.gmres(b, rtol=1e-13, maxit=800)[1] for op, b in zip(oracles, bs)],
                                 rtol=1e-9, maxit=50)
    assert ok and all(r["iterations"] == 0 for r in reps2)
    batch.close()


def test_batch_refuses_bad_plan_lists(near_tables):
    h, k, table = near_tables["rand_k0.3"]
    plans, _ = make(near_tables, False, [((7, 6, 5), 0.6, 1)], oracle=False)
    mixed, _ = make(near_tables, True, [((6, 5, 4), 0.6, 2)], oracle=False)
    with pytest.raises(RuntimeError):
        nb.VolumeBatch(plans + mixed)                 # FP64 and FP32 transforms
    assert "mix" in nb.last_error()
    with pytest.raises(RuntimeError):
        nb.VolumeBatch(plans + plans)                 # the same plan twice
    big = nb.VolumePlan((140, 1, 1), cases.random_lattice((140, 1, 1), 1.0, 3), h, k, 3.0, table)
    with pytest.raises(RuntimeError):
        nb.VolumeBatch([big])                         # padded axis 512 > 256
    assert "exceeds" in nb.last_error()
    b = nb.VolumeBatch(plans)
    ok, _, reps = b.gmres([np.ones(plans[0].n)], restart=31)    # restart above 30
    assert not ok and reps[0]["status"] == 4 and "at most 30" in nb.last_error()
    ok, xs, reps = b.gmres([np.ones(plans[0].n)], restart=40, maxit=20)   # cycle capped by maxit
    assert reps[0]["status"] in (0, 1) and 0 < reps[0]["iterations"] <= 20
    b.close()


# ------------------------------------------------------------ hybrid systems
def hybrid_blocks(c, v, seed):
    """[C|B] (c x n) then D (v x c), row-major: a diagonally dominant wire
    block C with weak couplings B and D to the volume unknowns."""
    rng = np.random.default_rng(seed)
    n = c + v
    cm = 0.1 * (rng.standard_normal((c, c)) + 1j * rng.standard_normal((c, c)))
    cm += np.diag(np.full(c, 4.0 + 1.0j))
    bm = 0.01 * (rng.standard_normal((c, v)) + 1j * rng.standard_normal((c, v)))
    dm = 0.01 * (rng.standard_normal((v, c)) + 1j * rng.standard_normal((v, c)))
    return np.concatenate([np.concatenate([cm, bm], axis=1).reshape(-1), dm.reshape(-1)]), n


def make_hybrids(near_tables, mixed, specs):
    """specs: (shape, fill, seed, conductors); plus one PEC-imaged system."""
    from test_hybrid_gpu import material_case
    h, k, table = near_tables["rand_k0.3"]
    gh, oh, keep = [], [], []
    for shape, fill, seed, c in specs:
        xyz = cases.random_lattice(shape, fill, seed)
        eps = cases.random_eps(xyz.size // 3, seed + 70, er=(2.0, 6.0))
        gp = nb.VolumePlan(shape, xyz, h, k, 3.0, table, mixed=mixed)
        op = OraclePlan(shape, xyz, h, k, 3.0, table)
        for i, e in enumerate(eps):
            assert gp.set_permittivity(i, e) and op.set_permittivity(i, e)
        v = 3 * (xyz.size // 3)
        blocks, n = hybrid_blocks(c, v, seed + 80)
        g = nb.HybridSystem(gp, c, v)
        g.set_blocks(blocks)
        gh.append(g)
        oh.append(OracleHybrid(op, c, v, blocks))
        keep += [gp, op]
    if not mixed:
        op, gp, v = material_case(near_tables, 0.0, True)
        blocks, n = hybrid_blocks(5, v, 99)
        g = nb.HybridSystem(gp, 5, v, pec=True)
        g.set_blocks(blocks)
        gh.append(g)
        oh.append(OracleHybrid(op, 5, v, blocks, True))
        keep += [gp, op]
    return gh, oh, keep


HYB = [((6, 5, 4), 0.8, 1, 21), ((8, 8, 8), 1.0, 2, 11), ((5, 4, 3), 1.0, 3, 41), ((12, 9, 17), 0.4, 4, 2)]


@pytest.mark.parametrize("mixed", [False, True])
def test_hybrid_batch_product(near_tables, mixed):
    import torch
    gh, oh, keep = make_hybrids(near_tables, mixed, HYB)
    batch = nb.VolumeBatch(hybrids=gh)
    assert batch.order == sum(g.n for g in gh)
    rng = np.random.default_rng(21)
    x = rng.standard_normal(batch.order) + 1j * rng.standard_normal(batch.order)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    assert nb.load().nec2c_cuda_vie_batch_apply_device(batch.h, C.c_void_p(xd.data_ptr()),
                                                       C.c_void_p(yd.data_ptr())), nb.last_error()
    y = yd.cpu().numpy()
    for q, (g, o) in enumerate(zip(gh, oh)):
        xs, ys = x[batch.offsets[q]:batch.offsets[q + 1]], y[batch.offsets[q]:batch.offsets[q + 1]]
        if mixed:
            assert rel_l2(ys, o.apply(xs)) < 1e-5, q
        else:
            assert rel_max(ys, g.apply(xs)) < 1e-14, q
            assert rel_max(ys, o.apply(xs)) < 1e-12, q
    batch.close()


@pytest.mark.parametrize("mixed,rtol,tol", [(False, 1e-11, 1e-8), (True, 1e-8, 1e-5)])
def test_hybrid_batch_gmres(near_tables, mixed, rtol, tol):
    gh, oh, keep = make_hybrids(near_tables, mixed, HYB)
    batch = nb.VolumeBatch(hybrids=gh)
    rng = np.random.default_rng(8)
    bs = [rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n) for g in gh]
    ok, xs, reps = batch.gmres(bs, rtol=rtol, maxit=600)
    assert ok, (reps, nb.last_error())
    for q, (g, o) in enumerate(zip(gh, oh)):
        assert reps[q]["status"] == 0 and reps[q]["relative_residual"] <= rtol
        r = bs[q] - o.apply(xs[q])
        assert np.linalg.norm(r) <= 1.01 * rtol * np.linalg.norm(bs[q])
        ok_o, xo, _ = o.gmres(bs[q], rtol=1e-12, maxit=600)
        assert ok_o and rel_l2(xs[q], xo) < tol
        ok_s, _, rs = g.gmres(bs[q], rtol=rtol, maxit=600)
        assert ok_s and abs(rs["iterations"] - reps[q]["iterations"]) <= max(3, rs["iterations"] // 10)
    batch.close()


def test_hybrid_batch_unpreconditionable_system(near_tables):
    """A zero conductor diagonal stops that system with the callback status
    (dielectric_fft.c:77-81), as the single solve does; the others converge."""
    gh, oh, keep = make_hybrids(near_tables, False, HYB[:2])
    blocks, n = hybrid_blocks(HYB[1][3], gh[1].n - HYB[1][3], 5)
    blocks[0] = 0                       # C_00 = 0
    gh[1].set_blocks(blocks)
    batch = nb.VolumeBatch(hybrids=gh)
    bs = [np.ones(g.n, dtype=np.complex128) for g in gh]
    ok, xs, reps = batch.gmres(bs, rtol=1e-10, maxit=300)
    _, _, single = gh[1].gmres(bs[1], rtol=1e-10, maxit=300)
    assert not ok
    assert reps[0]["status"] == 0
    assert reps[1]["status"] == single["status"] == 3     # VIE_ITERATIVE_CALLBACK_FAILED
    batch.close()
