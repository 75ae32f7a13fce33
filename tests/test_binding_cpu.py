"""The reference-side binding on the CPU (no GPU needed): the program with the
CUDA backend bound in (nec2c_b200/binding/_build/nec2c_cuda) behaves exactly like the stock
reference program when the builtin backends are selected, since every
wrapped entry point forwards to the reference's own; and selecting a CUDA
backend where no usable device exists fails loudly at the command line
instead of running on another path."""
import os
import subprocess

import numpy as np
import pytest

import decks

needs_bins = pytest.mark.skipif(not (os.path.exists(decks.REF_BIN) and os.path.exists(decks.CUDA_BIN)),
                                reason="oracle/_ref programs not built (needs the reference tree)")


def _gpu_present():
    import nec2c_b200 as nb
    try:
        return bool(nb.load().nec2c_cuda_available())
    except Exception:
        return False


@needs_bins
def test_builtin_backends_forwarded(tmp_path):
    """A small dipole-plus-cube deck (6^3 cells) through FFT-GMRES and the
    8-element array through the classic LU: identical result documents."""
    deck = decks.dipole_cube(str(tmp_path / "cube"), side_cells=6)
    args = ["-s", "fft", "-r", "1e-10", "--jobs", "1", "--threads", "2", "--fft-backend", "builtin"]
    a, _, _ = decks.run(decks.REF_BIN, deck, args)
    b, _, _ = decks.run(decks.CUDA_BIN, deck, args)
    assert decks.feed_impedance(a) == decks.feed_impedance(b)
    assert np.array_equal(decks.wire_currents(a), decks.wire_currents(b))
    assert np.array_equal(decks.volume_currents(a), decks.volume_currents(b))
    deck = decks.dipole_array(str(tmp_path / "array"), rows=2, cols=4)
    args = ["--jobs", "1", "--backend", "builtin"]
    a, _, _ = decks.run(decks.REF_BIN, deck, args)
    b, _, _ = decks.run(decks.CUDA_BIN, deck, args)
    assert decks.feed_impedance(a) == decks.feed_impedance(b)
    assert np.array_equal(decks.wire_currents(a), decks.wire_currents(b))


@needs_bins
@pytest.mark.parametrize("flag", ["--backend", "--fft-backend"])
@pytest.mark.parametrize("name", ["cuda", "cuda-mixed"])
def test_cuda_selection_without_device_fails(tmp_path, flag, name):
    if _gpu_present():
        pytest.skip("a CUDA device is present")
    deck = decks.dipole_array(str(tmp_path), rows=1, cols=2)
    p = subprocess.run([decks.CUDA_BIN, "-i", deck, "-o", str(tmp_path / "o.txt"), flag, name],
                       capture_output=True, text=True, timeout=60)
    assert p.returncode != 0
    assert "CUDA" in p.stderr and "selection failed" in p.stderr


@needs_bins
def test_stock_program_refuses_cuda_names(tmp_path):
    """The stock reference's whitelist (main.c:1409-1421) rejects the name;
    only the bound program accepts it."""
    deck = decks.dipole_array(str(tmp_path), rows=1, cols=2)
    p = subprocess.run([decks.REF_BIN, "-i", deck, "-o", str(tmp_path / "o.txt"), "--backend", "cuda"],
                       capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "requires auto, builtin, or lapack" in p.stderr
