"""Wire <-> volume coupling blocks on the GPU (nec2c_cuda_coupling_*) against
the reference's own kernels on the same inputs (oracle/_ref/libdw_shim.so:
dielectric_wire.c compiled with the reference, its static
dw_assemble_wire_to_volume and dw_point_cuboid_n called directly).

Geometry: the dipole-plus-cube model at 300 MHz (a 21-segment half-wave
dipole, radius 1 mm, 0.1 lambda from a 0.2 lambda cube of 16^3 cells); a
sample of the cube's cells (the near face, the far face, corners), in free
space and over a perfect ground (the model raised above the plane).  Sources
are seeded: for each conductor unknown the sine, cosine and constant
coefficients of three neighbouring segments, as NEC's basis spreads a unit
current, the rest exactly zero (the reference skips those segments).  The
blocks agree to 1e-12 relative to their largest entry."""
import ctypes as C
import math
import os

import numpy as np
import pytest

import nec2c_b200 as nb

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libdw_shim.so")
C0 = 299792458.0
EPS0 = 8.8541878128e-12


class WireModel(C.Structure):
    _fields_ = [("segments", C.c_size_t), ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("length", C.c_void_p), ("radius", C.c_void_p), ("cab", C.c_void_p), ("sab", C.c_void_p),
                ("salp", C.c_void_p), ("wavelength", C.c_double), ("rkh", C.c_double), ("pec_ground", C.c_int)]


def shim():
    if not os.path.exists(SHIM):
        raise RuntimeError("oracle/_ref/libdw_shim.so is not built (make -C oracle reference)")
    s = C.CDLL(SHIM)
    vp, sz, dbl, i = C.c_void_p, C.c_size_t, C.c_double, C.c_int
    s.shim_point_cuboid_n.argtypes = [vp, vp, vp, dbl, i, i, vp]
    s.shim_wire_to_volume.argtypes = [i, vp, dbl, dbl, i, i, sz, vp, sz, vp, vp, vp, dbl, dbl, vp]
    return s


def model(pec):
    lam = C0 / 300e6
    n = 21
    z0 = (0.05 + 0.25) if pec else 0.0          # dipole centre height (wavelengths)
    zc = (4 * 0.2 / 16 / 2 + 0.1) * lam if pec else 0.0   # cube centre height (m)
    seg = np.zeros((n, 8))
    for i in range(n):
        seg[i] = [0.0, 0.0, z0 - 0.25 + (i + 0.5) * 0.5 / n, 0.5 / n, 0.001 / lam, 0.0, 0.0, 1.0]
    h = 0.2 * lam / 16
    idx = [(ix, iy, iz) for ix in (0, 1, 7, 15) for iy in (0, 8, 15) for iz in (0, 5, 15)]
    centers = np.array([[0.1 * lam + (ix + 0.5) * h, -0.1 * lam + (iy + 0.5) * h, zc - 0.1 * lam + (iz + 0.5) * h]
                        for ix, iy, iz in idx])
    sizes = np.full_like(centers, h)
    return lam, seg, centers, sizes


def sources(n, columns, seed):
    rng = np.random.default_rng(seed)
    src = np.zeros((columns, n, 3), dtype=np.complex128)
    for j in range(columns):
        c = int(rng.integers(0, n))
        for s in range(max(0, c - 1), min(n, c + 2)):
            src[j, s] = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    return src


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("pec", [False, True])
def test_wire_to_volume_matches_reference(pec):
    lam, seg, centers, sizes = model(pec)
    n, cells, columns = len(seg), len(centers), 6
    src = sources(n, columns, 7 + pec)
    rng = np.random.default_rng(3)
    chi = (rng.uniform(1, 5, cells) - 1j * rng.uniform(0, 0.5, cells)).astype(np.complex128)
    k0, omega = 2 * math.pi / lam, 2 * math.pi * 300e6
    ref = np.zeros((columns, 3 * cells), dtype=np.complex128)
    segc = np.ascontiguousarray(seg)
    assert shim().shim_wire_to_volume(n, segc.ctypes.data, lam, 1.0, 2 if pec else 1, 1, columns,
                                      src.ctypes.data, cells, centers.ctypes.data, sizes.ctypes.data,
                                      chi.ctypes.data, k0, omega, ref.ctypes.data)
    cols = [np.ascontiguousarray(seg[:, k]) for k in range(8)]
    w = WireModel(n, *[c.ctypes.data for c in cols[:5]], cols[5].ctypes.data, cols[6].ctypes.data,
                  cols[7].ctypes.data, lam, 1.0, int(pec))
    got = np.zeros_like(ref)
    lib = nb.load()
    lib.nec2c_cuda_coupling_wire_to_volume.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                                       C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
    assert lib.nec2c_cuda_coupling_wire_to_volume(C.byref(w), columns, src.ctypes.data, cells, centers.ctypes.data,
                                                  sizes.ctypes.data, chi.ctypes.data, omega,
                                                  got.ctypes.data), nb.last_error()
    assert np.all(np.isfinite(got))
    assert rel(got, ref) < 1e-12


@pytest.mark.parametrize("pec", [False, True])
def test_volume_to_wire_matches_reference(pec):
    lam, seg, centers, sizes = model(pec)
    n, cells = len(seg), len(centers)
    obs = np.ascontiguousarray(seg[:, :3] * lam)
    tangent = np.ascontiguousarray(seg[:, 5:8])
    k0, omega = 2 * math.pi / lam, 2 * math.pi * 300e6
    ref = np.zeros((n, 3 * cells), dtype=np.complex128)
    s = shim()
    out18 = np.zeros(18)
    for w in range(n):
        for c in range(cells):
            assert s.shim_point_cuboid_n(obs[w].ctypes.data, np.ascontiguousarray(centers[c]).ctypes.data,
                                         np.ascontiguousarray(sizes[c]).ctypes.data, k0, 2 if pec else 1, 1,
                                         out18.ctypes.data)
            d = (out18[0::2] + 1j * out18[1::2]).reshape(3, 3)
            # dielectric_wire.c:1186-1198: tangent-tested, divided by i omega eps0.
            ref[w, 3 * c:3 * c + 3] = (tangent[w] @ d) / (1j * omega * EPS0)
    got = np.zeros_like(ref)
    lib = nb.load()
    lib.nec2c_cuda_coupling_volume_to_wire.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                                       C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]
    assert lib.nec2c_cuda_coupling_volume_to_wire(n, obs.ctypes.data, tangent.ctypes.data, cells,
                                                  centers.ctypes.data, sizes.ctypes.data, k0, omega, int(pec),
                                                  got.ctypes.data), nb.last_error()
    assert rel(got, ref) < 1e-12


def test_invalid_arguments_refused():
    lib = nb.load()
    lib.nec2c_cuda_coupling_volume_to_wire.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                                       C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]
    out = np.zeros(3, dtype=np.complex128)
    one = np.ones(3)
    assert not lib.nec2c_cuda_coupling_volume_to_wire(1, one.ctypes.data, one.ctypes.data, 1, one.ctypes.data,
                                                      one.ctypes.data, 1.0, -1.0, 0, out.ctypes.data)
    assert "invalid" in nb.last_error()
