"""Host logic of the request server (nec2c_b200/host/serve.c) on the CPU.

The server's own source is compiled with a fake device layer
(tests/serve_fake.c): each fake solve holds the volume plans its request runs
on for a few milliseconds and counts every overlap on one plan.  Checked here:
exclusivity per plan (directly, through hybrid systems and in batches) while
independent requests overlap, admission by device footprint, a request larger
than the budget running alone after being passed at most `slots` times, the
default budget (the reserve rule of concurrency.c:131-136) and the submission
checks."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import nec2c_b200 as nb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GIB = 1 << 30


@pytest.fixture(scope="module")
def fake():
    build = os.path.join(ROOT, "tests", "_build")
    os.makedirs(build, exist_ok=True)
    out = os.path.join(build, "libserve_fake.so")
    subprocess.run(["gcc", "-O1", "-std=gnu11", "-fPIC", "-shared", "-pthread", "-o", out,
                    os.path.join(ROOT, "nec2c_b200", "host", "serve.c"),
                    os.path.join(ROOT, "tests", "serve_fake.c")], check=True)
    lib = C.CDLL(out)
    vp, sz = C.c_void_p, C.c_size_t
    lib.fake_reset.argtypes = [C.c_long, sz]
    lib.fake_plan.argtypes = [sz]
    lib.fake_plan.restype = vp
    lib.fake_hybrid.argtypes = [vp, sz]
    lib.fake_hybrid.restype = vp
    lib.fake_batch.argtypes = [vp, sz]
    lib.fake_batch.restype = vp
    lib.fake_hybrid_batch.argtypes = [vp, sz]
    lib.fake_hybrid_batch.restype = vp
    lib.nec2c_cuda_server_merge_batch.argtypes = [vp, vp]
    lib.nec2c_cuda_server_merge_dense.argtypes = [vp, sz]
    lib.fake_release.argtypes = [vp]
    lib.nec2c_cuda_server_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, sz, C.c_int]
    lib.nec2c_cuda_server_submit.argtypes = [vp, C.POINTER(nb.Request)]
    lib.nec2c_cuda_server_wait.argtypes = [vp, C.POINTER(nb.Request)]
    lib.nec2c_cuda_server_drain.argtypes = [vp]
    lib.nec2c_cuda_server_budget.argtypes = [vp]
    lib.nec2c_cuda_server_budget.restype = sz
    lib.nec2c_cuda_server_destroy.argtypes = [vp]
    lib.nec2c_cuda_last_error.restype = C.c_char_p
    return lib


class Server:
    def __init__(self, lib, slots, budget=0):
        self.lib, self.h, self.keep = lib, C.c_void_p(), []
        assert lib.nec2c_cuda_server_create(C.byref(self.h), 0, slots, budget, 0)

    def submit(self, r, *arrays):
        self.keep.append((r, arrays))
        ok = self.lib.nec2c_cuda_server_submit(self.h, C.byref(r))
        if not ok:
            self.keep.pop()
        return ok

    def dense(self, n):
        r = nb.Request()
        r.kind = nb.REQUEST_DENSE
        r.order = r.ld = r.rhs_stride = n
        r.rhs_count = 1
        m = np.zeros(1, dtype=np.complex128)
        rhs = np.zeros(n, dtype=np.complex128)
        r.matrix, r.rhs = m.ctypes.data, rhs.ctypes.data
        assert self.submit(r, m, rhs)
        return r, rhs

    def volume(self, plan=None, system=None, n=0, restart=30):
        r = nb.Request()
        r.kind = nb.REQUEST_VOLUME
        r.plan, r.system = plan, system
        b = np.arange(1, n + 1) * (1 + 1j) + len(self.keep)
        x = np.zeros(n, dtype=np.complex128)
        r.b, r.x = b.ctypes.data, x.ctypes.data
        r.options = nb.GmresOptions(restart, 300, 1e-12, 0.0)
        assert self.submit(r, b, x)
        return r, (b, x)

    def batch(self, batch, k, n):
        r = nb.Request()
        r.kind = nb.REQUEST_BATCH
        r.batch = batch
        b = np.arange(1, n + 1) * (2 - 1j)
        x = np.zeros(n, dtype=np.complex128)
        reps = (nb.GmresReport * k)()
        r.b, r.x = b.ctypes.data, x.ctypes.data
        r.reports = C.cast(reps, C.c_void_p)
        r.options = nb.GmresOptions(30, 300, 1e-12, 0.0)
        assert self.submit(r, b, x, reps)
        return r, (b, x, reps)

    def drain(self):
        self.lib.nec2c_cuda_server_drain(self.h)

    def close(self):
        self.lib.nec2c_cuda_server_destroy(self.h)


def overlap(a, b):
    return a.started_s < b.finished_s and b.started_s < a.finished_s


def test_exclusive_per_plan_through_systems_and_batches(fake):
    fake.fake_reset(3000, 10 * GIB)
    orders = (30, 60, 90)
    p1, p2, p3 = plans = [fake.fake_plan(n) for n in orders]
    hyb = fake.fake_hybrid(p3, 5)
    b12 = fake.fake_batch((C.c_void_p * 2)(p1, p2), 2)
    b13 = fake.fake_batch((C.c_void_p * 2)(p1, p3), 2)
    srv = Server(fake, slots=4)
    reqs = []
    for _ in range(3):
        reqs.append((srv.volume(plan=p1, n=30), {p1}))
        reqs.append((srv.batch(b12, 2, 90), {p1, p2}))
        reqs.append((srv.volume(plan=p2, n=60), {p2}))
        reqs.append((srv.volume(system=hyb, n=95), {p3}))
        reqs.append((srv.batch(b13, 2, 120), {p1, p3}))
        reqs.append((srv.volume(plan=p3, n=90), {p3}))
        reqs.append((srv.dense(64), set()))
    srv.drain()
    assert fake.fake_violations() == 0
    assert fake.fake_peak() >= 2                       # independent requests overlapped
    for (r, data), _ in reqs:
        assert r.done and r.status, r.error
        if r.kind == nb.REQUEST_DENSE:
            assert data[0] == 64
        else:
            assert r.report.status == 0
            assert np.array_equal(data[1], data[0])     # x received b
        if r.kind == nb.REQUEST_BATCH:
            assert [rep.iterations for rep in data[2]] == [1, 2]
            assert r.report.iterations == 2 and r.report.operator_applications == 2 + 3
    shared = 0
    for i, ((a, _), ua) in enumerate(reqs):
        for (b, _), ub in reqs[i + 1:]:
            if ua & ub:
                shared += 1
                assert not overlap(a, b)
    assert shared > 20
    srv.close()
    for o in (b12, b13, hyb, *plans):
        fake.fake_release(o)


def footprint(n):
    return n * n * 16 + n * 16 + n * 4 + 4096


def test_admission_by_footprint(fake):
    fake.fake_reset(3000, 10 * GIB)
    n = 256
    budget = 2 * footprint(n) + footprint(n) // 2           # room for two at a time
    srv = Server(fake, slots=4, budget=budget)
    reqs = [srv.dense(n)[0] for _ in range(8)]
    srv.drain()
    assert all(r.status and r.footprint == footprint(n) for r in reqs)
    assert fake.fake_peak() == 2
    events = sorted([(r.started_s, r.footprint) for r in reqs] + [(r.finished_s, -r.footprint) for r in reqs],
                    key=lambda e: (e[0], e[1]))
    cur = peak = 0
    for _, d in events:
        cur += d
        peak = max(peak, cur)
    assert peak <= budget
    srv.close()


def test_oversized_request_runs_alone_after_at_most_slots_passes(fake):
    fake.fake_reset(5000, 10 * GIB)
    slots = 2
    budget = 4 * footprint(100)
    srv = Server(fake, slots=slots, budget=budget)
    first = srv.dense(100)[0]
    big = srv.dense(1000)[0]                                # 16 MB: above the budget
    rest = [srv.dense(100)[0] for _ in range(10)]
    srv.drain()
    assert big.status and big.footprint > budget
    assert big.skipped <= slots
    for r in [first] + rest:
        assert r.status and not overlap(r, big)
    assert sum(1 for r in rest if r.started_s < big.started_s) <= slots
    srv.close()


def test_default_budget_keeps_the_reserve(fake):
    for free, expect in ((10 * GIB, 8 * GIB), (2 * GIB, 1 * GIB)):
        fake.fake_reset(0, free)
        srv = Server(fake, slots=1)
        assert fake.nec2c_cuda_server_budget(srv.h) == expect
        srv.close()


def test_submission_checks(fake):
    fake.fake_reset(0, 10 * GIB)
    srv = Server(fake, slots=1)
    for kind, why in ((99, b"unknown request kind 99"), (nb.REQUEST_VOLUME, b"exactly one of plan"),
                      (nb.REQUEST_BATCH, b"batch request needs"), (nb.REQUEST_DENSE, b"dense request needs")):
        r = nb.Request()
        r.kind = kind
        assert not srv.submit(r)
        assert why in fake.nec2c_cuda_last_error()
    bad = C.c_void_p()
    assert not fake.nec2c_cuda_server_create(C.byref(bad), 0, 0, 0, 0)
    assert b"slots must be" in fake.nec2c_cuda_last_error()
    srv.close()


def test_queued_volume_requests_merge(fake):
    """Continuous batching: volume requests that queue up behind busy workers
    on systems of a registered batch run as one batched solve; the same
    system twice, other GMRES options, or a system outside the batch run
    alone; merged runs keep plan and batch exclusivity."""
    fake.fake_reset(20000, 10 * GIB)
    plans = [fake.fake_plan(40 + q) for q in range(8)]
    hyb = [fake.fake_hybrid(p, 3) for p in plans]
    batch = fake.fake_hybrid_batch((C.c_void_p * 8)(*hyb), 8)
    lone = fake.fake_hybrid(fake.fake_plan(50), 2)
    srv = Server(fake, slots=2)
    assert fake.nec2c_cuda_server_merge_batch(srv.h, batch)
    assert not fake.nec2c_cuda_server_merge_batch(srv.h, batch)
    assert b"already registered" in fake.nec2c_cuda_last_error()
    blockers = [srv.dense(64)[0] for _ in range(2)]          # both workers busy
    reqs = [(q, srv.volume(system=hyb[q], n=43 + q)) for q in range(8)]
    again = srv.volume(system=hyb[0], n=43)                   # system 0 a second time
    other = srv.volume(system=hyb[5], n=48, restart=40)       # other GMRES options
    alone = srv.volume(system=lone, n=52)                     # not in a registered batch
    whole = srv.batch(batch, 8, sum(43 + q for q in range(8)))
    srv.drain()
    assert fake.fake_violations() == 0
    assert fake.fake_merged_runs() >= 1 and fake.fake_merged_peak() >= 7
    for q, (r, (b, x)) in reqs:
        assert r.done and r.status, r.error
        assert np.array_equal(x, b)
        if r.merged > 1:
            assert r.report.iterations == q + 1               # its own system's report
    assert sum(1 for _, (r, _) in reqs if r.merged > 1) >= 7
    for r, (b, x) in (again, other, alone):
        assert r.status and np.array_equal(x, b)
    assert not overlap(again[0], reqs[0][1][0])
    assert other[0].merged == 1 and alone[0].merged == 1
    members = [r for _, (r, _) in reqs] + [again[0], other[0]]
    assert whole[0].status and all(not overlap(whole[0], r) for r in members)
    assert all(r.status for r in blockers)
    srv.close()
    for o in (batch, lone, *hyb, *plans):
        fake.fake_release(o)


def test_queued_dense_requests_merge(fake):
    """Dense requests that queue behind busy workers run as lockstep batches
    of one size class (orders up to 256, 512, 1024, 2048, 4096), at most the
    registered count per batch and within the device budget; each request
    gets its own result; orders above the batch limit do not merge, and a
    split-precision server's merged requests report their refinement steps."""
    fake.fake_reset(20000, 10 * GIB)
    assert not fake.nec2c_cuda_server_merge_dense(None, 4)
    assert b"null server" in fake.nec2c_cuda_last_error()
    srv = Server(fake, slots=2)
    assert not fake.nec2c_cuda_server_merge_dense(srv.h, 70000)
    assert b"at most 65535" in fake.nec2c_cuda_last_error()
    assert fake.nec2c_cuda_server_merge_dense(srv.h, 4)
    blockers = [srv.dense(64)[0] for _ in range(2)]           # both workers busy
    orders = [300, 400, 500, 310, 320, 1000, 700, 900, 5000, 2000, 1500, 330]
    reqs = [(n, srv.dense(n)) for n in orders]
    srv.drain()
    assert fake.fake_dense_runs() >= 2 and fake.fake_dense_peak() == 4
    assert fake.fake_dense_mixed_classes() == 0
    for n, (r, rhs) in reqs:
        assert r.done and r.status, r.error
        assert rhs[0] == n                                    # its own result
    big = dict((n, r) for n, (r, _) in reqs)[5000]
    assert big.merged == 1                                    # above the batch limit
    assert sum(1 for _, (r, _) in reqs if r.merged > 1) >= 6
    assert all(r.status for r in blockers)
    srv.close()

    # The budget bounds a merged run: room for two of order 300 at a time.
    fake.fake_reset(20000, 10 * GIB)
    budget = 2 * footprint(300) + footprint(300) // 2
    srv = Server(fake, slots=1, budget=budget)
    assert fake.nec2c_cuda_server_merge_dense(srv.h, 8)
    first = srv.dense(64)[0]
    rest = [srv.dense(300)[0] for _ in range(6)]
    srv.drain()
    assert fake.fake_dense_peak() == 2
    assert all(r.status and r.merged <= 2 for r in rest)
    srv.close()

    # A split-precision server merges too; its requests report the
    # refinement steps of their lockstep run.
    fake.fake_reset(20000, 10 * GIB)
    split = Server(fake, slots=1)
    fake.nec2c_cuda_server_destroy(split.h)
    assert fake.nec2c_cuda_server_create(C.byref(split.h), 0, 1, 0, 1)
    assert fake.nec2c_cuda_server_merge_dense(split.h, 4)
    first = split.dense(64)[0]
    rest = [split.dense(300) for _ in range(3)]
    split.drain()
    assert all(r.status for r, _ in rest) and max(r.merged for r, _ in rest) >= 2
    assert all(r.report.iterations == 3 for r, _ in rest if r.merged > 1)
    assert first.status
    split.close()
