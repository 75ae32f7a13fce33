"""Writes tests/golden/c2_reference_solve.json: the reference's own full solve
of the 64^3-voxel inhomogeneous block (786,432 unknowns, 128^3 padded grid,
eps_r ~ U[2,10], tand ~ U[0.01,0.1], seed 2, x-polarised plane wave,
GMRES(30) to rtol 1e-6 with the iteration limit 10000), run here through the
reference's compiled vie_fft_create / vie_fft_set_permittivity / vie_gmres
(oracle/_ref/libnec2c_ref.so, builtin FFT, OpenMP).  The whole solution does
not fit a fixture, so the file keeps what a comparison needs: the report
(status, iterations, restarts, residuals), the solution's 2-norm and
infinity-norm, its sums per component, and its values at 512 seeded indices.

Takes several minutes on the CPU.  Run from the repository root:
    python tests/golden/make_c2_pin.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402  (the workload definition and the reference library loader)

SAMPLES = 512


def sample_indices(n):
    return np.sort(np.random.default_rng(12345).choice(n, SAMPLES, replace=False))


def signature(x):
    idx = sample_indices(x.size)
    return {"norm2": float(np.linalg.norm(x)), "norm_inf": float(np.max(np.abs(x))),
            "component_sums": [[float(np.sum(x[c::3]).real), float(np.sum(x[c::3]).imag)] for c in range(3)],
            "indices": idx.tolist(), "values": [[float(v.real), float(v.imag)] for v in x[idx]]}


def main():
    w = bench.workload()
    r = bench.reference_lib()
    if r is None:
        raise SystemExit("oracle/_ref/libnec2c_ref.so is not built")
    p = bench.reference_plan(r, w)
    b = np.ascontiguousarray(w["rhs"])
    x = np.zeros_like(b)
    rep = r.Rep()
    t0 = time.perf_counter()
    r.ref_fft_gmres(p, b.ctypes.data_as(bench.C.c_void_p), x.ctypes.data_as(bench.C.c_void_p), 30,
                    bench.MAXIT, 1e-6, 0.0, bench.C.byref(rep))
    seconds = time.perf_counter() - t0
    r.ref_fft_destroy(p)
    out = {"workload": bench.CONFIG["workload"], "seed": bench.SEED,
           "threads": bench.cpu_threads(), "seconds": seconds,
           "report": {"status": rep.status, "iterations": rep.iterations, "restarts": rep.restarts,
                      "operator_applications": rep.operator_applications,
                      "residual_norm": rep.residual_norm, "relative_residual": rep.relative_residual},
           "solution": signature(x)}
    with open(os.path.join(HERE, "c2_reference_solve.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out["report"]), "%.1f s" % seconds)


if __name__ == "__main__":
    main()
