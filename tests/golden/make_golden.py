"""Generates the committed fixtures under tests/golden/ (run here, where the
reference tree and oracle/_ref exist; the GPU box only reads the fixtures).

near_tensors.json
    For each (pitch, k0) case used by the tests and the benchmark: the
    certified near-pair tensor of every sorted displacement the far-pair
    quadrature leaves to the near kernel, computed by the reference's own
    vie_cuboid_n (oracle/_ref, options of vie_fft.c:344).  These are inputs to
    the operator, the part of the spectrum build that stays on the CPU.
reference_golden.json
    The reference's published results for its M9 FFT benchmark models
    (tests/m9-fft-*-1e-8.txt / -1e-10.txt), parsed from the reference files.
"""
import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

import oracle_lib  # noqa: E402

# Reference tree whose published results are read; NEC2C_REFERENCE overrides it.
REFERENCE = os.environ.get("NEC2C_REFERENCE", "/root/reference")
C0 = 299792458.0


def cases():
    lam = C0 / 300e6
    k300 = 2 * math.pi / lam
    k28 = 2 * math.pi * 28e6 / C0
    return {
        # tests/vie_fft_test.c fixtures (pitch 0.25)
        "vie_k0.2": dict(h=0.25, k=0.2, shape=(9, 5, 3)),
        "vie_k0": dict(h=0.25, k=0.0, shape=(9, 5, 3)),
        "vie_k0.8": dict(h=0.25, k=0.8, shape=(9, 5, 3)),
        "vie_k4": dict(h=0.25, k=4.0, shape=(9, 5, 3)),
        # tests/dielectric_fft_test.c (pitch 0.25, k0 0.5, PEC embedding up to z=5)
        "diel_k0.5": dict(h=0.25, k=0.5, shape=(4, 4, 8)),
        # random lattices of the GPU parity tests
        "rand_k0.3": dict(h=0.25, k=0.3, shape=(24, 24, 24)),
        # M9 benchmark models (tools/m9_fft_benchmark.c: pitch 0.25 m, 28 MHz)
        "m9_tree": dict(h=0.25, k=k28, shape=(24, 24, 48)),
        # 16^3 cube of side 0.2 lambda at 300 MHz
        "c0": dict(h=0.2 * lam / 16, k=k300, shape=(16, 16, 16)),
        # 64^3 block of side 1 lambda at 300 MHz
        "c2": dict(h=lam / 64, k=k300, shape=(64, 64, 64)),
        # 32^3 cube of side 0.2 lambda at 300 MHz (the finest pitch of the swept cubes)
        "c3_32": dict(h=0.2 * lam / 32, k=k300, shape=(32, 32, 32)),
    }


def near_tensors():
    ref = oracle_lib.reference()
    out = {}
    for name, c in cases().items():
        fails = oracle_lib.far_failures(c["shape"], c["h"], c["k"])
        rows = []
        buf = np.empty(9, dtype=np.complex128)
        for v in fails:
            import ctypes as C
            if not ref.ref_near_tensor(None, (C.c_size_t * 3)(*v), c["h"], c["k"], oracle_lib.ptr(buf)):
                raise RuntimeError("near tensor failed at %s" % (v,))
            rows.append(list(v) + [float(z) for e in buf for z in (e.real, e.imag)])
        out[name] = dict(h=c["h"], k=c["k"], shape=list(c["shape"]), tensors=rows)
        print(name, "near offsets:", len(rows), file=sys.stderr)
    return out


def parse_m9(path):
    txt = open(path).read()
    res = {}
    for key in ("iterations", "applications"):
        m = re.search(r"\b%s=(\d+)" % key, txt)
        res[key] = int(m.group(1))
    res["residual"] = float(re.search(r"residual=([0-9.e+-]+)", txt).group(1))
    for m in re.finditer(r"(integrated_normalized_current_\d|far_axis\d_component\d)=([-+0-9.e]+)([-+][0-9.e]+)j", txt):
        res[m.group(1)] = [float(m.group(2)), float(m.group(3))]
    return res


def reference_golden():
    out = {}
    for model in ("skeleton", "tree"):
        for tol in ("1e-8", "1e-10"):
            p = os.path.join(REFERENCE, "tests", "m9-fft-%s-%s.txt" % (model, tol))
            if os.path.exists(p):
                out["%s_%s" % (model, tol)] = parse_m9(p)
    return out


def main():
    with open(os.path.join(HERE, "near_tensors.json"), "w") as f:
        json.dump(near_tensors(), f)
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(reference_golden(), f, indent=1)


if __name__ == "__main__":
    main()
