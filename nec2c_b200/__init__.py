"""ctypes view of libnec2c_cuda.so for the test harness and the benchmark.

The product is the C ABI in include/nec2c_cuda.h; this module only loads the
in-tree library and wraps its entry points with numpy arrays.  It has no CPU
fallback: importing it without the built library, or calling a compute entry
point without a CUDA device, raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnec2c_cuda.so")

NEAR_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_size_t), C.c_double, C.c_double,
                      C.POINTER(C.c_double))

STATUS = ["converged", "iteration limit", "Krylov breakdown", "operator/preconditioner failure",
          "invalid input", "workspace allocation/size failure", "nonfinite arithmetic"]


class GmresOptions(C.Structure):
    _fields_ = [("restart", C.c_size_t), ("maximum_iterations", C.c_size_t),
                ("relative_tolerance", C.c_double), ("absolute_tolerance", C.c_double)]


class GmresReport(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_size_t),
                ("operator_applications", C.c_size_t), ("restarts", C.c_size_t),
                ("residual_norm", C.c_double), ("relative_residual", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Request(C.Structure):
    """nec2c_cuda_request (include/nec2c_cuda.h)."""
    _fields_ = [("kind", C.c_int), ("order", C.c_size_t), ("ld", C.c_size_t), ("rhs_count", C.c_size_t),
                ("rhs_stride", C.c_size_t), ("matrix", C.c_void_p), ("rhs", C.c_void_p), ("plan", C.c_void_p),
                ("system", C.c_void_p), ("b", C.c_void_p), ("x", C.c_void_p), ("options", GmresOptions),
                ("status", C.c_int), ("done", C.c_int), ("skipped", C.c_uint), ("report", GmresReport),
                ("footprint", C.c_size_t), ("queued_s", C.c_double), ("started_s", C.c_double),
                ("finished_s", C.c_double), ("error", C.c_char * 128), ("batch", C.c_void_p),
                ("reports", C.c_void_p), ("merged", C.c_size_t)]


REQUEST_DENSE, REQUEST_VOLUME, REQUEST_BATCH = 1, 2, 3

_lib = None


def load():
    """Loads the in-tree library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libnec2c_cuda.so is not built (run __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    vp, sz, dbl, i = C.c_void_p, C.c_size_t, C.c_double, C.c_int
    sigs = {
        "nec2c_cuda_available": (i, []),
        "nec2c_cuda_last_error": (C.c_char_p, []),
        "nec2c_cuda_set_stream": (None, [vp]),
        "nec2c_cuda_set_device": (i, [i]),
        "nec2c_cuda_launch_count": (C.c_ulonglong, []),
        "nec2c_cuda_vie_fft_backend_set": (i, [C.c_char_p]),
        "nec2c_cuda_vie_fft_backend_name": (C.c_char_p, []),
        "nec2c_cuda_vie_fft_create": (i, [C.POINTER(vp), C.POINTER(sz), sz, C.POINTER(sz), dbl, dbl,
                                          dbl, dbl, sz, NEAR_FN, vp]),
        "nec2c_cuda_vie_fft_set_permittivity": (i, [vp, sz, dbl, dbl]),
        "nec2c_cuda_vie_fft_destroy": (None, [vp]),
        "nec2c_cuda_vie_fft_bytes": (sz, [vp]),
        "nec2c_cuda_vie_fft_device_bytes": (sz, [vp]),
        "nec2c_cuda_vie_fft_order": (sz, [vp]),
        "nec2c_cuda_vie_fft_apply": (i, [vp, vp, vp]),
        "nec2c_cuda_vie_fft_precondition": (i, [vp, vp, vp]),
        "nec2c_cuda_vie_fft_apply_device": (i, [vp, vp, vp]),
        "nec2c_cuda_vie_fft_spectrum": (i, [vp, vp]),
        "nec2c_cuda_vie_fft_radiation_device": (i, [vp, C.POINTER(dbl), vp, sz, vp, vp]),
        "nec2c_cuda_vie_fft_autotune": (None, [i]),
        "nec2c_cuda_vie_fft_autotune_enabled": (i, []),
        "nec2c_cuda_vie_fft_tune": (i, [vp, i]),
        "nec2c_cuda_vie_fft_schedule": (i, [vp, i, C.POINTER(i), C.POINTER(i)]),
        "nec2c_cuda_vie_fft_set_schedule": (i, [vp, i, C.POINTER(i), C.POINTER(i)]),
        "nec2c_cuda_vie_fft_planes": (i, [vp, i]),
        "nec2c_cuda_vie_fft_set_planes": (i, [vp, i, i]),
        "nec2c_cuda_vie_batch_create": (i, [C.POINTER(vp), C.POINTER(vp), sz]),
        "nec2c_cuda_vie_batch_destroy": (None, [vp]),
        "nec2c_cuda_hybrid_batch_create": (i, [C.POINTER(vp), C.POINTER(vp), sz]),
        "nec2c_cuda_vie_batch_order": (sz, [vp]),
        "nec2c_cuda_vie_batch_systems": (sz, [vp]),
        "nec2c_cuda_vie_batch_offset": (sz, [vp, sz]),
        "nec2c_cuda_vie_batch_apply_device": (i, [vp, vp, vp]),
        "nec2c_cuda_vie_batch_schedule": (i, [vp, C.POINTER(i), C.POINTER(i)]),
        "nec2c_cuda_vie_batch_set_schedule": (i, [vp, C.POINTER(i), C.POINTER(i)]),
        "nec2c_cuda_gmres_batch_device": (i, [vp, vp, vp, vp, vp]),
        "nec2c_cuda_gmres_batch": (i, [vp, C.POINTER(vp), C.POINTER(vp), vp, vp]),
        "nec2c_cuda_hybrid_create": (i, [C.POINTER(vp), vp, sz, sz, i]),
        "nec2c_cuda_hybrid_destroy": (None, [vp]),
        "nec2c_cuda_hybrid_set_blocks": (i, [vp, vp]),
        "nec2c_cuda_hybrid_order": (sz, [vp]),
        "nec2c_cuda_hybrid_apply": (i, [vp, vp, vp]),
        "nec2c_cuda_hybrid_precondition": (i, [vp, vp, vp]),
        "nec2c_cuda_gmres_plan": (i, [vp, vp, vp, vp, vp]),
        "nec2c_cuda_gmres_hybrid": (i, [vp, vp, vp, vp, vp]),
        "nec2c_cuda_gmres_plan_device": (i, [vp, vp, vp, vp, vp]),
        "nec2c_cuda_gmres_hybrid_device": (i, [vp, vp, vp, vp, vp]),
        "nec2c_cuda_dense_backend_set": (i, [C.c_char_p]),
        "nec2c_cuda_dense_backend_name": (C.c_char_p, []),
        "nec2c_cuda_dense_factor_classic": (i, [sz, vp, sz, vp]),
        "nec2c_cuda_dense_factor_device_static": (i, [sz, vp, sz, vp]),
        "nec2c_cuda_dense_last_refinement": (i, []),
        "nec2c_cuda_dense_solve_batched": (i, [sz, vp, vp, vp, vp, vp, vp]),
        "nec2c_cuda_server_create": (i, [C.POINTER(vp), i, i, sz, i]),
        "nec2c_cuda_server_submit": (i, [vp, C.POINTER(Request)]),
        "nec2c_cuda_server_wait": (i, [vp, C.POINTER(Request)]),
        "nec2c_cuda_server_drain": (i, [vp]),
        "nec2c_cuda_server_budget": (sz, [vp]),
        "nec2c_cuda_server_destroy": (None, [vp]),
        "nec2c_cuda_server_merge_dense": (i, [vp, sz]),
        "nec2c_cuda_dense_batch_max_order": (sz, []),
        "nec2c_cuda_dense_solve_classic": (i, [sz, vp, sz, vp, vp]),
        "nec2c_cuda_dense_solve_classic_many": (i, [sz, vp, sz, vp, vp, sz, sz]),
        "nec2c_cuda_dense_solve_row_major": (i, [vp, vp, sz]),
        "nec2c_cuda_dense_release": (None, []),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def set_fft_autotune(enable):
    """Turns the measured FFT schedule of new plans on or off (process-wide)."""
    load().nec2c_cuda_vie_fft_autotune(int(bool(enable)))


def fft_autotune_enabled():
    return bool(load().nec2c_cuda_vie_fft_autotune_enabled())


def last_error():
    return load().nec2c_cuda_last_error().decode()


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _cvec(x):
    return np.ascontiguousarray(x, dtype=np.complex128)


def table_near(table):
    """Near-tensor callback backed by a {(a, b, c): 9 complex} mapping."""
    def cb(ctx, off, h, k, out):
        key = (off[0], off[1], off[2])
        t = table.get(key)
        if t is None:
            return 0
        arr = np.asarray(t, dtype=np.complex128).reshape(9)
        for e in range(9):
            out[2 * e] = arr[e].real
            out[2 * e + 1] = arr[e].imag
        return 1
    return NEAR_FN(cb)


class VolumePlan:
    """A CUDA volume FFT plan (vie_fft_create with backend "cuda"/"cuda-mixed")."""

    def __init__(self, shape, xyz, pitch, k0, eps, near, byte_limit=1 << 62, mixed=False):
        lib = load()
        if not lib.nec2c_cuda_vie_fft_backend_set(b"cuda-mixed" if mixed else b"cuda"):
            raise RuntimeError("backend selection failed")
        self._near = near if isinstance(near, NEAR_FN) else table_near(near)
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.uintp).reshape(-1))
        self.cells = xyz.size // 3
        sh = (C.c_size_t * 3)(*shape)
        self.h = C.c_void_p()
        ok = lib.nec2c_cuda_vie_fft_create(C.byref(self.h), sh, self.cells,
                                           xyz.ctypes.data_as(C.POINTER(C.c_size_t)), pitch, k0,
                                           complex(eps).real, complex(eps).imag, byte_limit,
                                           self._near, None)
        if not ok:
            self.h = None
            raise RuntimeError("nec2c_cuda_vie_fft_create failed: " + last_error())
        self.n = 3 * self.cells

    def close(self):
        if self.h:
            load().nec2c_cuda_vie_fft_destroy(self.h)
            self.h = None

    __del__ = close

    def set_permittivity(self, cell, eps):
        return bool(load().nec2c_cuda_vie_fft_set_permittivity(self.h, cell, complex(eps).real,
                                                                complex(eps).imag))

    def apply(self, x):
        x = _cvec(x)
        y = np.empty_like(x)
        if not load().nec2c_cuda_vie_fft_apply(self.h, _ptr(x), _ptr(y)):
            raise RuntimeError("apply failed: " + last_error())
        return y

    def precondition(self, x):
        x = _cvec(x)
        y = np.empty_like(x)
        if not load().nec2c_cuda_vie_fft_precondition(self.h, _ptr(x), _ptr(y)):
            raise RuntimeError("precondition failed: " + last_error())
        return y

    def spectrum(self, grid):
        out = np.empty(6 * grid, dtype=np.complex128)
        if not load().nec2c_cuda_vie_fft_spectrum(self.h, _ptr(out)):
            raise RuntimeError("spectrum failed: " + last_error())
        return out

    def radiation(self, current, directions, origin=(0.0, 0.0, 0.0)):
        """Far-field amplitudes (count x 3) of the cell current (3 x cells)
        towards unit directions (count x 3)."""
        import torch
        cur = torch.from_numpy(_cvec(current)).cuda()
        dirs = np.ascontiguousarray(directions, dtype=np.float64).reshape(-1, 3)
        out = np.empty((dirs.shape[0], 3), dtype=np.complex128)
        org = (C.c_double * 3)(*origin)
        if not load().nec2c_cuda_vie_fft_radiation_device(self.h, org, C.c_void_p(cur.data_ptr()), dirs.shape[0],
                                                          _ptr(dirs), _ptr(out)):
            raise RuntimeError("radiation failed: " + last_error())
        return out

    def tune(self, measure=1):
        """Re-plans the FFT pass schedule: 0 heuristic, 1 timed (shape cache),
        2 timed afresh."""
        if not load().nec2c_cuda_vie_fft_tune(self.h, measure):
            raise RuntimeError("tune failed: " + last_error())

    def schedule(self, fp64=False):
        """(measured, [(lines per tile, R1), ...] for the five passes)."""
        tiles, r1 = (C.c_int * 5)(), (C.c_int * 5)()
        r = load().nec2c_cuda_vie_fft_schedule(self.h, int(bool(fp64)), tiles, r1)
        if r < 0:
            raise RuntimeError("schedule: no such precision on this plan")
        return bool(r), list(zip(tiles, r1))

    def set_schedule(self, passes, fp64=False):
        """Pins [(lines per tile, R1)] x 5; returns False when refused."""
        tiles = (C.c_int * 5)(*[int(t) for t, _ in passes])
        r1 = (C.c_int * 5)(*[int(r) for _, r in passes])
        return bool(load().nec2c_cuda_vie_fft_set_schedule(self.h, int(bool(fp64)), tiles, r1))

    def planes(self, fp64=False):
        """1: fused yz-plane passes in use, 0: five passes, -1: not applicable."""
        return load().nec2c_cuda_vie_fft_planes(self.h, int(bool(fp64)))

    def set_planes(self, planes, fp64=False):
        return bool(load().nec2c_cuda_vie_fft_set_planes(self.h, int(bool(fp64)), int(bool(planes))))

    def bytes(self):
        return load().nec2c_cuda_vie_fft_bytes(self.h)

    def device_bytes(self):
        return load().nec2c_cuda_vie_fft_device_bytes(self.h)

    def gmres(self, b, x0=None, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        return _gmres(load().nec2c_cuda_gmres_plan, self.h, b, x0, restart, maxit, rtol, atol)


def _gmres(fn, handle, b, x0, restart, maxit, rtol, atol):
    b = _cvec(b)
    x = np.zeros_like(b) if x0 is None else _cvec(x0).copy()
    opts = GmresOptions(restart, maxit, rtol, atol)
    rep = GmresReport()
    ok = fn(handle, _ptr(b), _ptr(x), C.byref(opts), C.byref(rep))
    return bool(ok), x, rep.as_dict()


class VolumeBatch:
    """Ragged batch of VolumePlans solved together (nec2c_cuda_vie_batch_*)."""

    def __init__(self, plans=None, hybrids=None):
        """A batch of VolumePlans, or (hybrids=) of HybridSystems."""
        self.plans = list(plans if hybrids is None else hybrids)   # must outlive the batch
        lib = load()
        arr = (C.c_void_p * len(self.plans))(*[p.h.value for p in self.plans])
        self.h = C.c_void_p()
        create = lib.nec2c_cuda_vie_batch_create if hybrids is None else lib.nec2c_cuda_hybrid_batch_create
        if not create(C.byref(self.h), arr, len(self.plans)):
            self.h = None
            raise RuntimeError("batch create failed: " + last_error())
        self.order = lib.nec2c_cuda_vie_batch_order(self.h)
        self.offsets = [lib.nec2c_cuda_vie_batch_offset(self.h, q) for q in range(len(self.plans) + 1)]

    def close(self):
        if self.h:
            load().nec2c_cuda_vie_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def schedule(self):
        """[(tile height scale, radix variant)] x 5 of the batched passes."""
        sc, va = (C.c_int * 5)(), (C.c_int * 5)()
        load().nec2c_cuda_vie_batch_schedule(self.h, sc, va)
        return list(zip(sc, va))

    def set_schedule(self, passes):
        sc = (C.c_int * 5)(*[int(a) for a, _ in passes])
        va = (C.c_int * 5)(*[int(b) for _, b in passes])
        return bool(load().nec2c_cuda_vie_batch_set_schedule(self.h, sc, va))

    def split(self, v):
        return [v[self.offsets[q]:self.offsets[q + 1]] for q in range(len(self.plans))]

    def gmres(self, bs, x0s=None, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        """(ok, [x_q], [report dict]) of vie_gmres on every plan at once."""
        K = len(self.plans)
        bs = [_cvec(b) for b in bs]
        xs = [np.zeros_like(b) for b in bs] if x0s is None else [_cvec(x).copy() for x in x0s]
        bp = (C.c_void_p * K)(*[b.ctypes.data for b in bs])
        xp = (C.c_void_p * K)(*[x.ctypes.data for x in xs])
        opts = GmresOptions(restart, maxit, rtol, atol)
        reps = (GmresReport * K)()
        ok = load().nec2c_cuda_gmres_batch(self.h, bp, xp, C.byref(opts), reps)
        return bool(ok), xs, [r.as_dict() for r in reps]


class HybridSystem:
    """The [C B; D V] operator of dielectric_fft.c on the device."""

    def __init__(self, plan, conductors, volume_unknowns, pec=False):
        lib = load()
        self.plan = plan
        self.h = C.c_void_p()
        if not lib.nec2c_cuda_hybrid_create(C.byref(self.h), plan.h if plan else None, conductors,
                                            volume_unknowns, 1 if pec else 0):
            self.h = None
            raise RuntimeError("hybrid create failed: " + last_error())
        self.n = conductors + volume_unknowns

    def close(self):
        if self.h:
            load().nec2c_cuda_hybrid_destroy(self.h)
            self.h = None

    __del__ = close

    def set_blocks(self, blocks):
        self._blocks = _cvec(blocks)
        if not load().nec2c_cuda_hybrid_set_blocks(self.h, _ptr(self._blocks)):
            raise RuntimeError("set_blocks failed: " + last_error())

    def apply(self, x):
        x = _cvec(x)
        y = np.empty_like(x)
        if not load().nec2c_cuda_hybrid_apply(self.h, _ptr(x), _ptr(y)):
            raise RuntimeError("apply failed: " + last_error())
        return y

    def precondition(self, x):
        x = _cvec(x)
        y = np.empty_like(x)
        ok = load().nec2c_cuda_hybrid_precondition(self.h, _ptr(x), _ptr(y))
        return bool(ok), y

    def gmres(self, b, x0=None, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        return _gmres(load().nec2c_cuda_gmres_hybrid, self.h, b, x0, restart, maxit, rtol, atol)


def dense_backend_set(name):
    return bool(load().nec2c_cuda_dense_backend_set(name.encode()))


def factor_classic(storage, ld=None):
    """Factors NEC's transposed storage (a Fortran-ordered ld x n complex array) in place."""
    n = storage.shape[1]
    ld = storage.shape[0] if ld is None else ld
    assert storage.dtype == np.complex128 and storage.flags.f_contiguous
    piv = np.zeros(n, dtype=np.int32)
    ok = load().nec2c_cuda_dense_factor_classic(n, _ptr(storage), ld, _ptr(piv))
    return bool(ok), piv


def solve_classic_many(storage, piv, rhs, ld=None):
    n = storage.shape[1]
    ld = storage.shape[0] if ld is None else ld
    assert rhs.dtype == np.complex128 and rhs.flags.f_contiguous
    ok = load().nec2c_cuda_dense_solve_classic_many(n, _ptr(storage), ld, _ptr(piv), _ptr(rhs),
                                                   rhs.shape[0], rhs.shape[1])
    return bool(ok)


def solve_row_major(a, b):
    a = _cvec(a)
    b = _cvec(b).copy()
    ok = load().nec2c_cuda_dense_solve_row_major(_ptr(a), _ptr(b), b.size)
    return bool(ok), b


class Server:
    """Request server (nec2c_cuda_server_*): requests run concurrently on
    worker threads with their own streams, admitted by device footprint."""

    def __init__(self, slots=4, budget=0, split=False, device=0):
        self.h = C.c_void_p()
        if not load().nec2c_cuda_server_create(C.byref(self.h), device, slots, budget, 1 if split else 0):
            self.h = None
            raise RuntimeError("server create failed: " + last_error())
        self._keep = {}

    def budget(self):
        return load().nec2c_cuda_server_budget(self.h)

    def dense(self, storage, rhs):
        """Queues a dense solve of NEC storage (Fortran ld x n) for rhs
        (Fortran ld_rhs x k, overwritten with the solutions)."""
        assert storage.dtype == np.complex128 and storage.flags.f_contiguous
        assert rhs.dtype == np.complex128 and rhs.flags.f_contiguous
        r = Request()
        r.kind = REQUEST_DENSE
        r.order, r.ld = storage.shape[1], storage.shape[0]
        r.rhs_count, r.rhs_stride = rhs.shape[1], rhs.shape[0]
        r.matrix, r.rhs = _ptr(storage), _ptr(rhs)
        self._submit(r, (storage, rhs))
        return r

    def volume(self, op, b, x, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        """Queues GMRES on a VolumePlan or HybridSystem; x is the initial guess
        and receives the solution."""
        r = Request()
        r.kind = REQUEST_VOLUME
        if isinstance(op, VolumePlan):
            r.plan = op.h
        else:
            r.system = op.h
        r.b, r.x = _ptr(b), _ptr(x)
        r.options = GmresOptions(restart, maxit, rtol, atol)
        self._submit(r, (op, b, x))
        return r

    def batch(self, batch, b, x, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        """Queues GMRES on every system of a VolumeBatch; b and x are the
        concatenated vectors in batch order (x: initial guess and result).
        The request's .reports array holds one report per system."""
        r = Request()
        r.kind = REQUEST_BATCH
        r.batch = batch.h
        r.b, r.x = _ptr(b), _ptr(x)
        reps = (GmresReport * len(batch.plans))()
        r.reports = C.cast(reps, C.c_void_p)
        r.options = GmresOptions(restart, maxit, rtol, atol)
        r.system_reports = reps
        self._submit(r, (batch, b, x, reps))
        return r

    def merge(self, batch):
        """Registers a VolumeBatch whose systems' queued volume requests the
        server may merge into one batched solve."""
        if not load().nec2c_cuda_server_merge_batch(self.h, batch.h):
            raise RuntimeError("merge registration failed: " + last_error())

    def merge_dense(self, max_systems):
        """Lets the server merge queued dense requests of one size class into
        lockstep batches of at most max_systems (FP64 server only)."""
        if not load().nec2c_cuda_server_merge_dense(self.h, max_systems):
            raise RuntimeError("dense merging refused: " + last_error())

    def _submit(self, r, keep):
        self._keep[C.addressof(r)] = (r, keep)
        if not load().nec2c_cuda_server_submit(self.h, C.byref(r)):
            del self._keep[C.addressof(r)]
            raise RuntimeError("submit rejected: " + last_error())

    def wait(self, r):
        ok = load().nec2c_cuda_server_wait(self.h, C.byref(r))
        self._keep.pop(C.addressof(r), None)
        return bool(ok)

    def drain(self):
        load().nec2c_cuda_server_drain(self.h)
        self._keep.clear()

    def close(self):
        if self.h:
            load().nec2c_cuda_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    __del__ = close


def solve_batched(systems):
    """Factors and solves a ragged batch [(storage, rhs), ...] in place
    (storage: Fortran ld x n NEC storage; rhs: n complex); returns
    (all_ok, status list, pivots list)."""
    count = len(systems)
    orders = (C.c_size_t * count)(*[st.shape[1] for st, _ in systems])
    lds = (C.c_size_t * count)(*[st.shape[0] for st, _ in systems])
    mats = (C.c_void_p * count)()
    rhs = (C.c_void_p * count)()
    pivs = [np.zeros(st.shape[1], dtype=np.int32) for st, _ in systems]
    pp = (C.c_void_p * count)()
    for k, (st, b) in enumerate(systems):
        assert st.dtype == np.complex128 and st.flags.f_contiguous
        assert b.dtype == np.complex128 and b.flags.c_contiguous
        mats[k], rhs[k], pp[k] = _ptr(st), _ptr(b), _ptr(pivs[k])
    status = (C.c_int * count)()
    ok = load().nec2c_cuda_dense_solve_batched(count, orders, mats, lds, pp, rhs, status)
    return bool(ok), list(status), pivs
