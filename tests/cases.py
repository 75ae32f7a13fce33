"""Shared input builders for the parity tests (seeded, reproducible)."""
import math

import numpy as np

C0 = 299792458.0

# tests/vie_fft_test.c:45-60 lattices (pitch 0.25)
SPARSE_SHAPE = (5, 3, 2)
SPARSE_XYZ = [0, 0, 0, 4, 2, 1, 1, 0, 0, 0, 1, 0, 0, 0, 1, 1, 1, 1]
FAR_SHAPE = (9, 5, 3)
FAR_XYZ = [0, 0, 0, 8, 4, 2, 4, 1, 0]

# tools/m9_fft_benchmark.c:37-39 boxes [x0,y0,z0,x1,y1,z1] at 0.25 m pitch.
M9_BOXES = [(11, 11, 0, 13, 13, 32), (13, 11, 22, 24, 13, 24), (11, 13, 26, 13, 24, 28),
            (0, 0, 32, 24, 24, 48)]


def probe_vector(n):
    """The reference test's probe sin(0.7 i) + i cos(0.3 i) (vie_fft_test.c:27)."""
    i = np.arange(n)
    return np.sin(0.7 * i) + 1j * np.cos(0.3 * i)


def random_lattice(shape, fill, seed):
    rng = np.random.default_rng(seed)
    pts = [(x, y, z) for x in range(shape[0]) for y in range(shape[1]) for z in range(shape[2])]
    keep = rng.random(len(pts)) < fill
    sel = [p for p, k in zip(pts, keep) if k]
    rng.shuffle(sel)
    return np.array(sel, dtype=np.uintp).reshape(-1)


def random_eps(cells, seed, er=(2.0, 10.0), tand=(0.01, 0.1)):
    rng = np.random.default_rng(seed)
    e = rng.uniform(*er, cells)
    t = rng.uniform(*tand, cells)
    return e * (1 - 1j * t)


def m9_model(full):
    """Cells and RHS of tools/m9_fft_benchmark.c (tree when full, else skeleton)."""
    shape = [24, 24, 48] if full else [13, 13, 32]
    boxes = M9_BOXES if full else M9_BOXES[:3]
    xyz = []
    for b in boxes:
        for x in range(b[0], b[3]):
            for y in range(b[1], b[4]):
                for z in range(b[2], b[5]):
                    xyz += [x - (0 if full else 11), y - (0 if full else 11), z]
    xyz = np.array(xyz, dtype=np.uintp)
    h = 0.25
    k = 2 * math.pi * 28e6 / C0
    cells = xyz.size // 3
    rhs = np.zeros(3 * cells, dtype=np.complex128)
    z = xyz[2::3].astype(np.float64)
    rhs[0::3] = 2 * np.exp(-1j * k * h * (z + 0.5)) * math.sin(k * h / 2) / (k * h / 2)
    return shape, xyz, h, k, rhs


def integrated_current(sol, h):
    return [complex(np.sum(sol[d::3]) * h ** 3) for d in range(3)]
