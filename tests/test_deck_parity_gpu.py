"""Deck-level parity: the reference program with the CUDA backend bound in
(nec2c_b200/binding/_build/nec2c_cuda: main.c's whitelists opened, the binding linked in
with --wrap, nothing else changed) against the stock reference program
(oracle/_ref/nec2c, builtin FFT and builtin LU) on the same seeded decks.

The plain FP64 form must reproduce the reference's results: the feed
impedance within 1e-9 relative, the segment and voxel currents within 1e-9
relative L2 (both solves run to -r 1e-12, where both sit on the exact solution
of the discrete system; at looser tolerances the stopping iteration, not the
arithmetic, decides the last digits).  The mixed forms (FP32 transforms, split
LU with FP64 refinement) are held to the 1e-5 current error the mixed serving
form promises, and report their Zin and gain errors the same way.

Decks (tests/decks.py):
- the dipole beside a 16^3 dielectric cube at 300 MHz in free space (FFT-GMRES
  of the hybrid [C B; D V] system, dielectric_wire.c:1296-1321);
- the same model over a perfectly conducting ground (PEC image embedding,
  dielectric_fft.c:137-154);
- the 8 x 8 dipole array of 1984 segments with seeded loads (factrs / netwk /
  solves, main.c:3106, network.c:221)."""
import os

import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

FFT_ARGS = ["-s", "fft", "-r", "1e-12", "--jobs", "1"]


def _binaries():
    for b in (decks.REF_BIN, decks.CUDA_BIN):
        if not os.path.exists(b):
            raise RuntimeError("%s is not built (make -C oracle reference binding)" % b)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _compare(ref, got, tol, gain_tol_db, index=0):
    er, eg = decks.execution(ref, index), decks.execution(got, index)
    assert eg["status"] == "ok"
    if er["feeds"]:
        zr, zg = decks.feed_impedance(ref, index), decks.feed_impedance(got, index)
        assert abs(zg - zr) / abs(zr) < tol, (zr, zg)
        assert _rel(decks.wire_currents(got, index), decks.wire_currents(ref, index)) < tol
    vr = decks.volume_currents(ref, index)
    if vr.size:
        assert _rel(decks.volume_currents(got, index), vr) < tol
    if er["far_fields"]:
        assert decks.gain_difference_db(got, ref) < gain_tol_db
    if er["solver"].get("iterations") is not None:
        assert eg["solver"]["converged"] is True


@pytest.fixture(scope="module")
def cube_free(tmp_path_factory):
    _binaries()
    deck = decks.dipole_cube(str(tmp_path_factory.mktemp("cube")))
    ref, _, _ = decks.run(decks.REF_BIN, deck, FFT_ARGS + ["--fft-backend", "builtin"])
    return deck, ref


@pytest.fixture(scope="module")
def cube_pec(tmp_path_factory):
    _binaries()
    deck = decks.dipole_cube(str(tmp_path_factory.mktemp("cube_pec")), pec=True)
    ref, _, _ = decks.run(decks.REF_BIN, deck, FFT_ARGS + ["--fft-backend", "builtin"])
    return deck, ref


@pytest.fixture(scope="module")
def array(tmp_path_factory):
    _binaries()
    deck = decks.dipole_array(str(tmp_path_factory.mktemp("array")))
    ref, _, _ = decks.run(decks.REF_BIN, deck, ["--jobs", "1", "--backend", "builtin"])
    return deck, ref


def test_dipole_cube_fp64(cube_free):
    deck, ref = cube_free
    got, _, _ = decks.run(decks.CUDA_BIN, deck, FFT_ARGS + ["--fft-backend", "cuda"])
    assert decks.execution(got)["solver"]["used"] == "fft"
    _compare(ref, got, 1e-9, 1e-7)


def test_dipole_cube_mixed(cube_free):
    deck, ref = cube_free
    got, _, _ = decks.run(decks.CUDA_BIN, deck, FFT_ARGS + ["--fft-backend", "cuda-mixed"])
    _compare(ref, got, 1e-5, 1e-3)


def test_dipole_cube_pec_fp64(cube_pec):
    deck, ref = cube_pec
    got, _, _ = decks.run(decks.CUDA_BIN, deck, FFT_ARGS + ["--fft-backend", "cuda"])
    _compare(ref, got, 1e-9, 1e-7)


def test_dipole_array_fp64(array):
    deck, ref = array
    got, _, _ = decks.run(decks.CUDA_BIN, deck, ["--jobs", "1", "--backend", "cuda"])
    _compare(ref, got, 1e-9, 1e-7)


def test_dipole_array_split_lu(array):
    """Split-precision LU with FP64 refinement: FP64 accuracy."""
    deck, ref = array
    got, _, _ = decks.run(decks.CUDA_BIN, deck, ["--jobs", "1", "--backend", "cuda-mixed"])
    _compare(ref, got, 1e-9, 1e-7)


def test_plane_wave_cube(tmp_path):
    """The volume-only solver (dielectric_solver.c:315-527): a 16^3 cube lit by
    a plane wave, FFT-GMRES of the volume operator alone."""
    _binaries()
    deck = decks.plane_wave_cube(str(tmp_path), 16)
    ref, _, _ = decks.run(decks.REF_BIN, deck, FFT_ARGS + ["--fft-backend", "builtin"])
    got, _, _ = decks.run(decks.CUDA_BIN, deck, FFT_ARGS + ["--fft-backend", "cuda"])
    _compare(ref, got, 1e-9, 1e-7)
    got, _, _ = decks.run(decks.CUDA_BIN, deck, FFT_ARGS + ["--fft-backend", "cuda-mixed"])
    _compare(ref, got, 1e-5, 1e-3)


def test_dispersive_sweep(tmp_path):
    """A frequency table material (resource version 3) swept over three
    frequencies in one run: the material law is the reference's own
    (dielectric.h:36-56, evaluated by its prepare), each frequency a new plan,
    one job at a time through the binding."""
    _binaries()
    deck = decks.dipole_cube_sweep(str(tmp_path))
    ref, _, _ = decks.run(decks.REF_BIN, deck, FFT_ARGS + ["--fft-backend", "builtin"])
    got, _, _ = decks.run(decks.CUDA_BIN, deck, FFT_ARGS + ["--fft-backend", "cuda"])
    assert len(decks.executions(got)) == len(decks.executions(ref)) == 3
    for i in range(3):
        assert decks.execution(got, i)["frequency_mhz"] == decks.execution(ref, i)["frequency_mhz"]
        _compare(ref, got, 1e-9, 1e-7, index=i)


def test_budget_refusal_identical(tmp_path):
    """dielectric_fft.c:98-108 and vie_fft_create's byte limit: a 48^3 cube
    (128^3 padded grid) exceeds the 512 MiB accounted budget, and the bound
    program refuses it exactly as the stock one does, before any solve."""
    _binaries()
    deck = decks.plane_wave_cube(str(tmp_path), 48)
    rc_ref, doc_ref, text_ref = decks.run_status(decks.REF_BIN, deck, ["-s", "fft", "--jobs", "1"])
    rc_got, doc_got, text_got = decks.run_status(decks.CUDA_BIN, deck, ["-s", "fft", "--jobs", "1",
                                                                         "--fft-backend", "cuda"])
    assert rc_ref != 0 and rc_got == rc_ref
    msg = "padded FFT exceeds memory budget"
    assert msg in text_ref and msg in text_got
    assert decks.execution(doc_got)["status"] == decks.execution(doc_ref)["status"] == "failed"
