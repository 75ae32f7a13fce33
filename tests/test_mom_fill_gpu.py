"""Wire MoM fill on the GPU (nec2c_cuda_mom_fill) against the reference's own
cmset, through the drop-in program.

With the CUDA dense backend selected, the drop-in program
(nec2c_b200/binding/_build/nec2c_cuda) fills the wire-wire matrix on the GPU
from the reference's own basis functions (trio).  Its test hook
NEC2C_CUDA_FILL_CHECK runs the reference's cmset on the same matrix beside
the GPU fill and prints the largest entry difference relative to the largest
entry; the two agree to 1e-12 (the same NEC-2 kernel in FP64, summed in the
reference's order).  The solved feed impedance and segment currents then
match the stock program (builtin LU and fill) to 1e-9.

Decks (tests/decks.py): the 8 x 8 dipole array of 1984 segments with seeded
loads (config 1), a 2 x 2 array over a perfect ground, and the junction
model (a four-wire junction, a bent wire, a stub, a load) in free space and
over a perfect ground."""
import os
import re

import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

CHECK = re.compile(r"MoM fill check: order (\d+), largest difference ([0-9.eE+-]+)")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _deck(kind, directory):
    if kind == "array":
        return decks.dipole_array(directory, pattern=False), 1984
    if kind == "array_pec":
        return decks.dipole_array(directory, rows=2, cols=2, pec=True), 124
    if kind == "junctions":
        return decks.junctions(directory), 40
    return decks.junctions(directory, pec=True), 40


@pytest.mark.parametrize("kind", ["array", "array_pec", "junctions", "junctions_pec"])
def test_gpu_fill_matches_reference(tmp_path, kind):
    for b in (decks.REF_BIN, decks.CUDA_BIN):
        if not os.path.exists(b):
            raise RuntimeError("%s is not built (make -C oracle reference binding)" % b)
    deck, order = _deck(kind, str(tmp_path))
    ref, _, _ = decks.run(decks.REF_BIN, deck, ["--jobs", "1", "--backend", "builtin"])
    got, _, err = decks.run(decks.CUDA_BIN, deck, ["--jobs", "1", "--backend", "cuda"],
                            env={"NEC2C_CUDA_FILL_CHECK": "1"})
    checks = CHECK.findall(err)
    assert checks, err[-2000:]
    for n, diff in checks:
        assert int(n) == order
        assert float(diff) < 1e-12, err[-2000:]
    zr, zg = decks.feed_impedance(ref), decks.feed_impedance(got)
    assert abs(zg - zr) / abs(zr) < 1e-9, (zr, zg)
    assert _rel(decks.wire_currents(got), decks.wire_currents(ref)) < 1e-9
