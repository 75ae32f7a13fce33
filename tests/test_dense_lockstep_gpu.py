"""Lockstep batch of FP64 factorisations (one launch per kernel and panel
step for every system of a ragged batch), through the C ABI: each system's
pivots and factors bit for bit those of its own classic factorisation (the
kernels are the same), its solution within 1e-12 of its own classic solve
and of the oracle; a singular system is reported without disturbing the
others; orders above the batch limit take the classic path.  Then the
request server's dense merging: queued requests of one size class run as
lockstep batches with each result equal to the same request served alone."""
import numpy as np
import pytest

import nec2c_b200 as nb
from oracle_lib import oracle, ptr
from test_dense_gpu import mom_like, nec_storage

pytestmark = pytest.mark.gpu


def test_lockstep_batch_matches_single():
    assert nb.dense_backend_set("cuda")
    cap = nb.load().nec2c_cuda_dense_batch_max_order()
    assert cap in (2048, 4096)
    sizes = [65, 100, 257, 300, 511, 700, 1100, 300, 2100, 2500, 40, 5000]
    sizes = [n for n in sizes if n <= cap or n == 5000]
    systems, ref = [], []
    for k, n in enumerate(sizes):
        a = mom_like(n, 1200 + k)
        if k == 7:
            a[:, 5] = 0.0            # singular
        ld = n + (k % 4)
        st = nec_storage(a, ld)
        rng = np.random.default_rng(50 + k)
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        b = np.ascontiguousarray(a @ x)
        systems.append((st, b.copy()))
        ref.append((a, st.copy(order="F"), b, ld, x))
    ok, status, pivs = nb.solve_batched(systems)
    assert not ok                    # the singular one
    for k, (n, (st, xb), piv, (a, st0, b, ld, x)) in enumerate(zip(sizes, systems, pivs, ref)):
        if k == 7:
            assert status[k] == 0
            continue
        assert status[k] == 1, (k, nb.last_error())
        single = st0.copy(order="F")
        ok1, p1 = nb.factor_classic(single)
        assert ok1, nb.last_error()
        assert np.array_equal(piv, p1), (k, n)
        if 64 < n <= cap:            # lockstep batch: the classic kernels, bit for bit
            assert np.array_equal(st[:n, :n], single[:n, :n]), (k, n)
        else:                        # the one-launch small-system kernel / the classic path
            assert np.max(np.abs(st[:n, :n] - single[:n, :n])) / np.max(np.abs(single[:n, :n])) < 1e-12, (k, n)
        xs = np.zeros((ld, 1), dtype=np.complex128, order="F")
        xs[:n, 0] = b
        assert nb.solve_classic_many(single, p1, xs)
        assert np.linalg.norm(xb - xs[:n, 0]) / np.linalg.norm(xs[:n, 0]) < 1e-12, (k, n)
        assert np.linalg.norm(xb - x) / np.linalg.norm(x) < 1e-9, (k, n)
        if n <= 700:
            po = np.zeros(n, dtype=np.int32)
            assert oracle().oracle_factr(n, ptr(st0), ptr(po), ld)
            assert np.array_equal(piv, po), (k, n)
            bo = b.copy()
            oracle().oracle_solve(n, ptr(st0), ptr(po), ptr(bo), ld)
            assert np.linalg.norm(xb - bo) / np.linalg.norm(bo) < 1e-12, (k, n)
    nb.load().nec2c_cuda_dense_release()


def test_server_merges_dense_requests():
    assert nb.dense_backend_set("cuda")
    orders = [300, 320, 400, 480, 350, 300, 700, 900, 1000, 600, 290, 310, 1800, 1200, 64, 200]
    mats, rhss = [], []
    for k, n in enumerate(orders):
        a = mom_like(n, 1400 + k)
        mats.append(np.asfortranarray(a.T))
        rng = np.random.default_rng(80 + k)
        rhss.append(np.asfortranarray((a @ (rng.standard_normal(n) + 1j * rng.standard_normal(n))).reshape(n, 1)))

    def serve(merge, slots):
        srv = nb.Server(slots=slots)
        if merge:
            srv.merge_dense(merge)
        outs, reqs = [], []
        for m, b in zip(mats, rhss):
            o = b.copy(order="F")
            reqs.append(srv.dense(m, o))
            outs.append(o)
        srv.drain()
        res = [(bool(r.status), int(r.merged)) for r in reqs]
        srv.close()
        return outs, res

    alone, res1 = serve(0, 1)
    assert all(ok and m == 1 for ok, m in res1)
    for _ in range(2):               # twice: the batch state starts clean every run
        merged, res2 = serve(6, 2)
        assert all(ok for ok, _ in res2)
        assert max(m for _, m in res2) >= 2
        for k, (x, y) in enumerate(zip(merged, alone)):
            assert np.linalg.norm(x - y) / np.linalg.norm(y) < 1e-12, (k, orders[k])


@pytest.mark.parametrize("sizes", [(70, 257, 300, 1100, 2100, 33), (1500, 1700, 1600, 1550)])
def test_split_lockstep_matches_single(sizes):
    """Split-precision lockstep batch (FP32 storage, tensor-core 3xTF32
    updates) against n2d_lu_factor32 on each matrix alone: pivots and FP32
    factors bit for bit (the same kernel bodies), ragged orders in one batch.
    The second batch's large early updates take the persistent tensor-core
    kernel per matrix, which gives the staged kernel's results bit for bit."""
    import ctypes as C
    import torch
    lib = nb.load()
    cap = lib.nec2c_cuda_dense_batch_max_order()
    single = lib.n2d_lu_factor32
    single.restype = C.c_int
    single.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    batch = lib.n2d_lu_factor32_batch
    batch.restype = C.c_int
    batch.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    sizes = [n for n in sizes if n <= cap]
    mats, pivs, works, lds = [], [], [], []
    for k, n in enumerate(sizes):
        ld = n + (n & 1) + 2 * (k % 2)
        a = np.zeros((n, ld), dtype=np.complex64)
        a[:, :n] = mom_like(n, 1600 + k)
        mats.append(a)
        lds.append(ld)
        works.append(torch.from_numpy(a.view(np.float32)).cuda())
        pivs.append(torch.zeros(n, dtype=torch.int32, device="cuda"))
    count = len(sizes)
    info = (C.c_int * count)()
    ok = batch((C.c_void_p * count)(*[w.data_ptr() for w in works]), (C.c_longlong * count)(*sizes),
               (C.c_longlong * count)(*lds), (C.c_void_p * count)(*[p.data_ptr() for p in pivs]), count, 0, info)
    torch.cuda.synchronize()
    assert ok, nb.last_error()
    for k, n in enumerate(sizes):
        assert info[k] == 0
        w1 = torch.from_numpy(mats[k].view(np.float32)).cuda()
        p1 = torch.zeros(n, dtype=torch.int32, device="cuda")
        i1 = C.c_int(0)
        assert single(w1.data_ptr(), n, lds[k], p1.data_ptr(), 0, C.byref(i1)), nb.last_error()
        torch.cuda.synchronize()
        assert i1.value == 0
        assert torch.equal(pivs[k], p1), (k, n)
        assert torch.equal(works[k], w1), (k, n)


def test_split_server_merges_with_refinement():
    """A split-precision server merging dense requests: every solution within
    1e-10 of the exact one (FP64 refinement of the tensor-core factors), the
    merged requests reporting their refinement steps."""
    orders = [300, 320, 400, 480, 350, 700, 900, 1000, 600, 1800, 1300, 200]
    mats, rhss, xs = [], [], []
    for k, n in enumerate(orders):
        a = mom_like(n, 1700 + k)
        mats.append(np.asfortranarray(a.T))
        rng = np.random.default_rng(90 + k)
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        xs.append(x)
        rhss.append(np.asfortranarray((a @ x).reshape(n, 1)))
    srv = nb.Server(slots=2, split=True)
    srv.merge_dense(6)
    outs, reqs = [], []
    for m, b in zip(mats, rhss):
        o = b.copy(order="F")
        reqs.append(srv.dense(m, o))
        outs.append(o)
    srv.drain()
    assert all(r.status for r in reqs), [r.error for r in reqs]
    assert max(r.merged for r in reqs) >= 2
    for k, (o, x, r) in enumerate(zip(outs, xs, reqs)):
        assert np.linalg.norm(o[:, 0] - x) / np.linalg.norm(x) < 1e-10, (k, orders[k])
        if r.merged > 1:
            assert r.report.iterations >= 1, k
    srv.close()


@pytest.mark.parametrize("split", [False, True])
def test_lockstep_small_orders(split):
    """Orders at and around one panel (1, 2, 5, 31, 32, 33, 64, 65) in one
    lockstep batch, as the server's smallest size class can hold them: each
    bit for bit its own factorisation (FP64 or split precision)."""
    import ctypes as C
    import torch
    lib = nb.load()
    if split:
        one, many, dt = lib.n2d_lu_factor32, lib.n2d_lu_factor32_batch, np.complex64
    else:
        one, many, dt = lib.n2d_lu_factor, lib.n2d_lu_factor_batch, np.complex128
    many.restype = C.c_int
    many.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    one.restype = C.c_int
    if split:
        one.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    else:
        one.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
    sizes = [1, 2, 5, 31, 32, 33, 64, 65]
    host, dev, piv, lds = [], [], [], []
    for k, n in enumerate(sizes):
        ld = n + (n & 1)
        a = np.zeros((n, ld), dtype=dt)
        a[:, :n] = mom_like(n, 1800 + k)
        host.append(a)
        lds.append(ld)
        dev.append(torch.from_numpy(a.view(np.float32 if split else np.float64)).cuda())
        piv.append(torch.zeros(n, dtype=torch.int32, device="cuda"))
    count = len(sizes)
    info = (C.c_int * count)()
    assert many((C.c_void_p * count)(*[d.data_ptr() for d in dev]), (C.c_longlong * count)(*sizes),
                (C.c_longlong * count)(*lds), (C.c_void_p * count)(*[p.data_ptr() for p in piv]), count, 0, info), \
        nb.last_error()
    torch.cuda.synchronize()
    for k, n in enumerate(sizes):
        assert info[k] == 0
        d1 = torch.from_numpy(host[k].view(np.float32 if split else np.float64)).cuda()
        p1 = torch.zeros(n, dtype=torch.int32, device="cuda")
        i1 = C.c_int(0)
        ok = (one(d1.data_ptr(), n, lds[k], p1.data_ptr(), 0, C.byref(i1)) if split else
              one(d1.data_ptr(), n, lds[k], p1.data_ptr(), 0, 0, C.byref(i1)))
        torch.cuda.synchronize()
        assert ok and i1.value == 0, nb.last_error()
        assert torch.equal(piv[k], p1), (k, n)
        assert torch.equal(dev[k], d1), (k, n)
