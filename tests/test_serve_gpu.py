"""Request server (nec2c_cuda_server_*): dense and volume solves submitted
together run concurrently on worker streams, and each result is the same as
when the request runs alone (bitwise: every kernel on the path reduces in a
fixed order).  Dense solutions match numpy's FP64 solve to 1e-10 relative;
the split-precision server's match the FP64 server's to 1e-10 relative.  The
admission budget holds at every instant."""
import numpy as np
import pytest

import cases
import nec2c_b200 as nb

pytestmark = pytest.mark.gpu


def dense_case(n, seed, k=2):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a += np.diag(np.full(n, 0.5 * np.sqrt(n)))
    ld = n + 3
    st = np.zeros((ld, n), dtype=np.complex128, order="F")
    st[:n, :n] = a.T
    x = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    rhs = np.zeros((n + 1, k), dtype=np.complex128, order="F")
    rhs[:n] = a @ x
    return a, st, rhs


def volume_cases(near_tables):
    out = []
    for name, shape, fill, seed in (("rand_k0.3", (12, 9, 17), 0.5, 7), ("c0", (16, 16, 16), 1.0, 3)):
        h, k, table = near_tables[name]
        xyz = cases.random_lattice(shape, fill, seed)
        eps = cases.random_eps(xyz.size // 3, seed + 1, er=(2.0, 4.0))
        plan = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
        for c, e in enumerate(eps):
            plan.set_permittivity(c, e)
        rng = np.random.default_rng(seed + 2)
        b = rng.standard_normal(plan.n) + 1j * rng.standard_normal(plan.n)
        out.append((plan, b))
    return out


def submit_all(server, dense, volume):
    """Interleaved dense and volume requests (each volume plan twice)."""
    reqs, outs = [], []
    vol = [(p, b) for p, b in volume] * 2
    for i in range(max(len(dense), len(vol))):
        if i < len(dense):
            _, st, rhs = dense[i]
            out = rhs.copy(order="F")
            reqs.append(server.dense(st, out))
            outs.append(out)
        if i < len(vol):
            plan, b = vol[i]
            x = np.zeros_like(b)
            reqs.append(server.volume(plan, b, x, rtol=1e-10, maxit=500))
            outs.append(x)
    return reqs, outs


def max_concurrent_bytes(reqs):
    events = sorted([(r.started_s, r.footprint) for r in reqs] + [(r.finished_s, -r.footprint) for r in reqs],
                    key=lambda e: (e[0], e[1]))
    cur = peak = 0
    for _, d in events:
        cur += d
        peak = max(peak, cur)
    return peak


def test_same_alone_and_in_the_mix(near_tables):
    dense = [dense_case(n, 100 + n) for n in (40, 200, 513, 1100, 777)]
    volume = volume_cases(near_tables)
    # Alone: one worker, each request waited for before the next is queued.
    alone = nb.Server(slots=1)
    ref = []
    for i in range(len(dense)):
        _, st, rhs = dense[i]
        out = rhs.copy(order="F")
        r = alone.dense(st, out)
        assert alone.wait(r), r.error
        ref.append(("dense", out, r))
    for plan, b in volume:
        x = np.zeros_like(b)
        r = alone.volume(plan, b, x, rtol=1e-10, maxit=500)
        assert alone.wait(r), r.error
        ref.append(("volume", x, r))
    alone.close()
    # In the mix: four workers, everything queued at once.
    mix = nb.Server(slots=4)
    reqs, outs = submit_all(mix, dense, volume)
    mix.drain()
    for r in reqs:
        assert r.done and r.status, r.error
    # Requests overlapped on the device.
    overlaps = sum(1 for a in reqs for b in reqs
                   if a is not b and a.started_s < b.finished_s and b.started_s < a.finished_s)
    assert overlaps > 0
    assert max_concurrent_bytes(reqs) <= mix.budget()
    # Same plan never in flight twice.
    vol_reqs = [r for r in reqs if r.kind == nb.REQUEST_VOLUME]
    for a in vol_reqs:
        for b in vol_reqs:
            if a is not b and a.plan == b.plan:
                assert a.finished_s <= b.started_s or b.finished_s <= a.started_s
    mix.close()
    di = vi = 0
    for r, out in zip(reqs, outs):
        if r.kind == nb.REQUEST_DENSE:
            kind, expect, rr = ref[di]
            di += 1
            a = dense[di - 1][0]
            assert kind == "dense" and np.array_equal(out, expect)
            sol = np.linalg.solve(a, (dense[di - 1][2])[: a.shape[0]])
            assert np.linalg.norm(out[: a.shape[0]] - sol) / np.linalg.norm(sol) < 1e-10
        else:
            kind, expect, rr = ref[len(dense) + (vi % len(volume))]
            vi += 1
            assert kind == "volume" and np.array_equal(out, expect)
            assert r.report.iterations == rr.report.iterations
            assert r.report.relative_residual <= 1e-10


def test_split_precision_server_matches_fp64():
    dense = [dense_case(n, 300 + n, k=3) for n in (64, 600, 1500)]
    outs = {}
    for split in (False, True):
        srv = nb.Server(slots=3, split=split)
        res = []
        reqs = []
        for a, st, rhs in dense:
            out = rhs.copy(order="F")
            reqs.append(srv.dense(st, out))
            res.append(out)
        srv.drain()
        for r in reqs:
            assert r.status, r.error
            if split:
                assert r.report.iterations >= 1   # refinement steps, no FP64 fallback
        srv.close()
        outs[split] = res
    for (a, _, _), x64, xs in zip(dense, outs[False], outs[True]):
        n = a.shape[0]
        assert np.linalg.norm(xs[:n] - x64[:n]) / np.linalg.norm(x64[:n]) < 1e-10


def test_budget_limits_concurrency():
    dense = [dense_case(n, 500 + n, k=1) for n in (900, 1000, 950, 1024)]
    big = max(n for n in (900, 1000, 950, 1024))
    budget = 16 * big * big + (1 << 20)      # room for one of these at a time
    srv = nb.Server(slots=4, budget=budget)
    assert srv.budget() == budget
    reqs = []
    for a, st, rhs in dense:
        reqs.append(srv.dense(st, rhs.copy(order="F")))
    srv.drain()
    for r in reqs:
        assert r.status, r.error
        assert r.footprint <= budget
    assert max_concurrent_bytes(reqs) <= budget
    srv.close()


def test_rejects_malformed_requests():
    srv = nb.Server(slots=1)
    import ctypes as C
    r = nb.Request()
    r.kind = 7
    assert not nb.load().nec2c_cuda_server_submit(srv.h, C.byref(r))
    r.kind = nb.REQUEST_VOLUME          # neither plan nor system
    assert not nb.load().nec2c_cuda_server_submit(srv.h, C.byref(r))
    r.kind = nb.REQUEST_DENSE           # no matrix
    assert not nb.load().nec2c_cuda_server_submit(srv.h, C.byref(r))
    srv.close()


def test_batch_requests_in_the_mix(near_tables):
    """A batch request (every system of a plan batch solved at once) gives the
    same result in a concurrent mix with dense requests as the batch solved
    directly (bitwise: fixed-order reductions), and its summary report is
    the worst of its systems'."""
    h, k, table = near_tables["rand_k0.3"]
    plans = []
    for shape, fill, seed in (((7, 6, 5), 0.6, 1), ((8, 8, 8), 1.0, 2), ((12, 9, 17), 0.5, 3)):
        xyz = cases.random_lattice(shape, fill, seed)
        p = nb.VolumePlan(shape, xyz, h, k, 3.0, table, mixed=True)
        for c, e in enumerate(cases.random_eps(xyz.size // 3, seed + 9, er=(2.0, 5.0))):
            p.set_permittivity(c, e)
        plans.append(p)
    batch = nb.VolumeBatch(plans)
    rng = np.random.default_rng(77)
    b = rng.standard_normal(batch.order) + 1j * rng.standard_normal(batch.order)
    ok, direct, reps = batch.gmres(batch.split(b), rtol=1e-9, maxit=400)
    assert ok
    dense = [dense_case(n, 900 + n) for n in (300, 700)]
    srv = nb.Server(slots=3)
    x = np.zeros_like(b)
    rb = srv.batch(batch, b, x, rtol=1e-9, maxit=400)
    outs = []
    for a, st, rhs in dense:
        out = rhs.copy(order="F")
        outs.append((a, rhs, out, srv.dense(st, out)))
    srv.drain()
    assert rb.status, rb.error
    for q, part in enumerate(batch.split(x)):
        assert np.array_equal(part, direct[q])
        assert rb.system_reports[q].iterations == reps[q]["iterations"]
    assert rb.report.status == 0
    assert rb.report.iterations == max(r["iterations"] for r in reps)
    assert rb.report.relative_residual == max(r["relative_residual"] for r in reps)
    for a, rhs, out, r in outs:
        assert r.status
        sol = np.linalg.solve(a, rhs[: a.shape[0]])
        assert np.linalg.norm(out[: a.shape[0]] - sol) / np.linalg.norm(sol) < 1e-10
    srv.close()
    batch.close()


def test_requests_sharing_a_plan_never_overlap(near_tables):
    """A plan is not reentrant, and a hybrid system or a batch runs on its
    systems' plans: requests that reach one plan by any of these routes run
    one after the other, and each result is the one it gives alone
    (bitwise)."""
    from test_vie_batch_gpu import hybrid_blocks
    h, k, table = near_tables["rand_k0.3"]
    plans = []
    for shape, fill, seed in (((7, 6, 5), 0.6, 21), ((8, 8, 8), 1.0, 22), ((6, 9, 4), 0.7, 23)):
        xyz = cases.random_lattice(shape, fill, seed)
        p = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
        for c, e in enumerate(cases.random_eps(xyz.size // 3, seed + 9, er=(2.0, 5.0))):
            p.set_permittivity(c, e)
        plans.append(p)
    p1, p2, p3 = plans
    blocks, n = hybrid_blocks(9, p3.n, 31)
    hyb = nb.HybridSystem(p3, 9, p3.n)
    hyb.set_blocks(blocks)
    b12, b13 = nb.VolumeBatch([p1, p2]), nb.VolumeBatch([p1, p3])
    rng = np.random.default_rng(41)

    def rhs(m):
        return rng.standard_normal(m) + 1j * rng.standard_normal(m)
    work = [("plan", p1, rhs(p1.n)), ("batch", b12, rhs(b12.order)), ("plan", p2, rhs(p2.n)),
            ("system", hyb, rhs(hyb.n)), ("batch", b13, rhs(b13.order)), ("plan", p3, rhs(p3.n)),
            ("plan", p1, rhs(p1.n))]
    uses = {"plan": lambda op: {id(op)}, "system": lambda op: {id(op.plan)},
            "batch": lambda op: {id(p) for p in op.plans}}

    def submit(srv, kind, op, b):
        x = np.zeros_like(b)
        if kind == "batch":
            return srv.batch(op, b, x, rtol=1e-9, maxit=400), x
        return srv.volume(op, b, x, rtol=1e-9, maxit=400), x

    alone = nb.Server(slots=1)
    ref = []
    for kind, op, b in work:
        r, x = submit(alone, kind, op, b)
        assert alone.wait(r), r.error
        ref.append(x)
    alone.close()
    mix = nb.Server(slots=4)
    got = [submit(mix, kind, op, b) for kind, op, b in work]
    mix.drain()
    for (r, x), expect in zip(got, ref):
        assert r.status and r.report.status == 0, r.error
        assert np.array_equal(x, expect)
    shared = 0
    for i, (ki, oi, _) in enumerate(work):
        for j, (kj, oj, _) in enumerate(work):
            if i < j and uses[ki](oi) & uses[kj](oj):
                shared += 1
                a, b = got[i][0], got[j][0]
                assert a.finished_s <= b.started_s or b.finished_s <= a.started_s
    assert shared >= 8
    # p2 and the hybrid system (on p3) share nothing: free to overlap.
    assert not uses["plan"](p2) & uses["system"](hyb)
    mix.close()
    for o in (b12, b13, hyb, *plans):
        o.close()


def test_submit_rejections_say_why():
    """A request the server refuses at submission leaves the reason in
    nec2c_cuda_last_error, and nothing is queued."""
    srv = nb.Server(slots=1)
    for kind, why in ((99, "unknown request kind 99"), (nb.REQUEST_VOLUME, "exactly one of plan"),
                      (nb.REQUEST_BATCH, "batch request needs"), (nb.REQUEST_DENSE, "dense request needs")):
        r = nb.Request()
        r.kind = kind
        with pytest.raises(RuntimeError, match=why):
            srv._submit(r, ())
    srv.drain()
    srv.close()


def test_queued_volume_requests_merge(near_tables):
    """Continuous batching: volume requests on the systems of a registered
    batch that queue behind busy workers run as one batched solve.  Each
    merged request gets its own system's result: the one the whole batch
    gives that system solved directly (to 1e-12: per-system reductions in a
    fixed order), converged to the request's tolerance."""
    h, k, table = near_tables["rand_k0.3"]
    plans = []
    for shape, fill, seed in (((7, 6, 5), 0.6, 51), ((8, 8, 8), 1.0, 52), ((12, 9, 17), 0.5, 53),
                              ((6, 9, 4), 0.7, 54)):
        xyz = cases.random_lattice(shape, fill, seed)
        p = nb.VolumePlan(shape, xyz, h, k, 3.0, table)
        for c, e in enumerate(cases.random_eps(xyz.size // 3, seed + 9, er=(2.0, 5.0))):
            p.set_permittivity(c, e)
        plans.append(p)
    batch = nb.VolumeBatch(plans)
    rng = np.random.default_rng(61)
    bs = [rng.standard_normal(p.n) + 1j * rng.standard_normal(p.n) for p in plans]
    ok, direct, reps = batch.gmres(bs, rtol=1e-10, maxit=400)
    assert ok
    srv = nb.Server(slots=2)
    srv.merge(batch)
    dense = [dense_case(2048, 990 + i, k=1) for i in range(2)]
    blockers = [srv.dense(st, rhs.copy(order="F")) for _, st, rhs in dense]   # both workers busy
    xs = [np.zeros_like(b) for b in bs]
    reqs = [srv.volume(p, b, x, rtol=1e-10, maxit=400) for p, b, x in zip(plans, bs, xs)]
    srv.drain()
    assert all(r.status for r in blockers)
    assert max(r.merged for r in reqs) >= 2, [r.merged for r in reqs]
    for q, (r, x) in enumerate(zip(reqs, xs)):
        assert r.status, r.error
        assert r.report.status == 0 and r.report.relative_residual <= 1e-10
        if r.merged > 1:
            assert r.report.iterations == reps[q]["iterations"]
            assert np.max(np.abs(x - direct[q])) <= 1e-12 * np.max(np.abs(direct[q]))
        else:
            ok_s, xs_, rs = plans[q].gmres(bs[q], rtol=1e-10, maxit=400)
            assert np.linalg.norm(x - xs_) <= 1e-8 * np.linalg.norm(xs_)
    srv.close()
    batch.close()
