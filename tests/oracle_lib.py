"""ctypes bindings of the CPU oracle (oracle/lib/liboracle.so) and, when it has
been built here, of the reference compiled from its own sources
(oracle/_ref/libnec2c_ref.so).  Test infrastructure only."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "lib", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libnec2c_ref.so")

NEAR_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_size_t), C.c_double, C.c_double,
                      C.POINTER(C.c_double))


class Report(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_size_t),
                ("operator_applications", C.c_size_t), ("restarts", C.c_size_t),
                ("residual_norm", C.c_double), ("relative_residual", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_oracle = None
_ref = None


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: make -C oracle oracle")
        o = C.CDLL(ORACLE_SO)
        vp, sz, dbl, i = C.c_void_p, C.c_size_t, C.c_double, C.c_int
        o.oracle_plan_create.argtypes = [C.POINTER(vp), C.POINTER(sz), sz, C.POINTER(sz), dbl, dbl,
                                         dbl, dbl, NEAR_FN, vp]
        o.oracle_plan_create.restype = i
        o.oracle_plan_destroy.argtypes = [vp]
        o.oracle_plan_set_permittivity.argtypes = [vp, sz, dbl, dbl]
        o.oracle_plan_set_permittivity.restype = i
        o.oracle_plan_padded.argtypes = [vp, i]
        o.oracle_plan_padded.restype = sz
        o.oracle_plan_spectrum.argtypes = [vp, vp]
        o.oracle_plan_self.argtypes = [vp, vp]
        for f in ("oracle_plan_apply", "oracle_plan_precondition"):
            getattr(o, f).argtypes = [vp, vp, vp]
            getattr(o, f).restype = i
        o.oracle_far_kernel.argtypes = [C.POINTER(sz), dbl, dbl, vp]
        o.oracle_far_kernel.restype = i
        o.oracle_hybrid_create.argtypes = [C.POINTER(vp), vp, sz, sz, vp, i]
        o.oracle_hybrid_create.restype = i
        o.oracle_hybrid_destroy.argtypes = [vp]
        for f in ("oracle_hybrid_apply", "oracle_hybrid_precondition"):
            getattr(o, f).argtypes = [vp, vp, vp]
            getattr(o, f).restype = i
        for f in ("oracle_plan_gmres", "oracle_hybrid_gmres"):
            getattr(o, f).argtypes = [vp, vp, vp, sz, sz, dbl, dbl, C.POINTER(Report)]
            getattr(o, f).restype = i
        o.oracle_factr.argtypes = [i, vp, vp, i]
        o.oracle_factr.restype = i
        o.oracle_solve.argtypes = [i, vp, vp, vp, i]
        o.oracle_row_major_solve.argtypes = [vp, vp, sz]
        o.oracle_row_major_solve.restype = i
        o.oracle_radiation_amplitude.argtypes = [sz, vp, dbl, vp, dbl, vp, vp]
        _oracle = o
    return _oracle


def reference_available():
    return os.path.exists(REF_SO)


def reference():
    global _ref
    if _ref is None:
        r = C.CDLL(REF_SO)
        vp, sz, dbl, i = C.c_void_p, C.c_size_t, C.c_double, C.c_int
        r.ref_near_tensor.argtypes = [vp, C.POINTER(sz), dbl, dbl, vp]
        r.ref_near_tensor.restype = i
        r.ref_pair_tensor.argtypes = [vp, vp, dbl, dbl, vp]
        r.ref_pair_tensor.restype = i
        r.ref_pair_tensor_pec.argtypes = [vp, vp, dbl, dbl, vp]
        r.ref_pair_tensor_pec.restype = i
        r.ref_fft_backend_set.argtypes = [C.c_char_p]
        r.ref_fft_create.argtypes = [C.POINTER(sz), sz, C.POINTER(sz), dbl, dbl, dbl, dbl, sz]
        r.ref_fft_create.restype = vp
        r.ref_fft_destroy.argtypes = [vp]
        r.ref_fft_bytes.argtypes = [vp]
        r.ref_fft_bytes.restype = sz
        r.ref_fft_set_permittivity.argtypes = [vp, sz, dbl, dbl]
        r.ref_fft_set_permittivity.restype = i
        for f in ("ref_fft_apply", "ref_fft_precondition"):
            getattr(r, f).argtypes = [vp, vp, vp]
            getattr(r, f).restype = i
        r.ref_fft_gmres.argtypes = [vp, vp, vp, sz, sz, dbl, dbl, C.POINTER(Report)]
        r.ref_fft_gmres.restype = i
        r.ref_dense_gmres.argtypes = [vp, sz, vp, vp, sz, sz, dbl, dbl, C.POINTER(Report)]
        r.ref_dense_gmres.restype = i
        r.ref_factr.argtypes = [i, vp, vp, i]
        r.ref_solve.argtypes = [i, vp, vp, vp, i]
        r.ref_row_major_solve.argtypes = [vp, vp, sz]
        r.ref_row_major_solve.restype = i
        r.ref_radiation_amplitude.argtypes = [sz, vp, dbl, vp, dbl, vp, vp]
        r.ref_radiation_amplitude.restype = i
        r.ref_hybrid_create.argtypes = [sz, vp, dbl, vp, sz, vp, dbl, i]
        r.ref_hybrid_create.restype = vp
        r.ref_hybrid_destroy.argtypes = [vp]
        for f in ("ref_hybrid_apply", "ref_hybrid_precondition"):
            getattr(r, f).argtypes = [vp, vp, vp]
            getattr(r, f).restype = i
        r.ref_hybrid_gmres.argtypes = [vp, vp, vp, sz, sz, dbl, dbl, C.POINTER(Report)]
        r.ref_hybrid_gmres.restype = i
        r.ref_callback_gmres.restype = i
        _ref = r
    return _ref


def near_from_table(table):
    def cb(ctx, off, h, k, out):
        t = table.get((off[0], off[1], off[2]))
        if t is None:
            return 0
        arr = np.asarray(t, dtype=np.complex128).reshape(9)
        for e in range(9):
            out[2 * e] = arr[e].real
            out[2 * e + 1] = arr[e].imag
        return 1
    return NEAR_FN(cb)


class OraclePlan:
    def __init__(self, shape, xyz, h, k, eps, near_table):
        o = oracle()
        self._near = near_from_table(near_table)
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.uintp).reshape(-1))
        self.cells = xyz.size // 3
        self.h = C.c_void_p()
        ok = o.oracle_plan_create(C.byref(self.h), (C.c_size_t * 3)(*shape), self.cells,
                                  xyz.ctypes.data_as(C.POINTER(C.c_size_t)), h, k,
                                  complex(eps).real, complex(eps).imag, self._near, None)
        if not ok:
            self.h = None
            raise RuntimeError("oracle plan create failed")
        self.padded = [o.oracle_plan_padded(self.h, d) for d in range(3)]
        self.n = 3 * self.cells

    def __del__(self):
        if getattr(self, "h", None):
            oracle().oracle_plan_destroy(self.h)

    def set_permittivity(self, cell, eps):
        return bool(oracle().oracle_plan_set_permittivity(self.h, cell, complex(eps).real,
                                                          complex(eps).imag))

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty_like(x)
        oracle().oracle_plan_apply(self.h, ptr(x), ptr(y))
        return y

    def precondition(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty_like(x)
        oracle().oracle_plan_precondition(self.h, ptr(x), ptr(y))
        return y

    def spectrum(self):
        g = int(np.prod(self.padded))
        out = np.empty(6 * g, dtype=np.complex128)
        oracle().oracle_plan_spectrum(self.h, ptr(out))
        return out

    def gmres(self, b, x0=None, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
        rep = Report()
        ok = oracle().oracle_plan_gmres(self.h, ptr(b), ptr(x), restart, maxit, rtol, atol,
                                        C.byref(rep))
        return bool(ok), x, rep.as_dict()


class OracleHybrid:
    def __init__(self, plan, c, v, blocks, pec=False):
        o = oracle()
        self.plan = plan
        self.blocks = np.ascontiguousarray(blocks, dtype=np.complex128)
        self.h = C.c_void_p()
        if not o.oracle_hybrid_create(C.byref(self.h), plan.h if plan else None, c, v,
                                      ptr(self.blocks), 1 if pec else 0):
            raise RuntimeError("oracle hybrid create failed")
        self.n = c + v

    def __del__(self):
        if getattr(self, "h", None):
            oracle().oracle_hybrid_destroy(self.h)

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty_like(x)
        oracle().oracle_hybrid_apply(self.h, ptr(x), ptr(y))
        return y

    def precondition(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty_like(x)
        ok = oracle().oracle_hybrid_precondition(self.h, ptr(x), ptr(y))
        return bool(ok), y

    def gmres(self, b, x0=None, restart=30, maxit=300, rtol=1e-12, atol=0.0):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
        rep = Report()
        ok = oracle().oracle_hybrid_gmres(self.h, ptr(b), ptr(x), restart, maxit, rtol, atol,
                                          C.byref(rep))
        return bool(ok), x, rep.as_dict()


def sorted_offsets(shape):
    s = sorted(shape, reverse=True)
    out = []
    for a in range(s[0]):
        for b in range(min(a, s[1] - 1) + 1):
            for c in range(min(b, s[2] - 1) + 1):
                out.append((a, b, c))
    return out


def far_failures(shape, h, k):
    """Sorted offsets where the far-pair quadrature does not certify a value."""
    o = oracle()
    fails = []
    out = np.empty(9, dtype=np.complex128)
    for v in sorted_offsets(shape):
        if not o.oracle_far_kernel((C.c_size_t * 3)(*v), h, k, ptr(out)):
            fails.append(v)
    return fails


def radiation_amplitude(centers, h, current, k0, direction, use_reference=False):
    """3 complex amplitudes (oracle restatement, or the reference itself)."""
    c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1)
    j = np.ascontiguousarray(current, dtype=np.complex128)
    d = np.ascontiguousarray(direction, dtype=np.float64)
    out = np.zeros(3, dtype=np.complex128)
    if use_reference:
        assert reference().ref_radiation_amplitude(c.size // 3, ptr(c), h, ptr(j), k0, ptr(d), ptr(out))
    else:
        oracle().oracle_radiation_amplitude(c.size // 3, ptr(c), h, ptr(j), k0, ptr(d), ptr(out))
    return out
