"""Seeded NEC decks of the dipole-plus-cube and dipole-array workloads, for
the deck-level parity tests: the stock reference program (oracle/_ref/nec2c)
and the same program with the CUDA backend bound in
(nec2c_b200/binding/_build/nec2c_cuda) run the same deck, and their result
JSON documents are compared.

Coordinates are written with full double precision (repr): the reference's
FFT lattice inference accepts cubes equal to 1e-10 only
(dielectric_fft.c:121-123)."""
import json
import os
import subprocess

import numpy as np

C0 = 299792458.0
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "nec2c")
CUDA_BIN = os.path.join(ROOT, "nec2c_b200", "binding", "_build", "nec2c_cuda")

# Far-field request of both decks: theta 0..180 and phi 0..350 in 10-degree
# steps, power gain (RP card, XNDA = 1000).
PATTERN = "RP 0 19 36 1000 0 0 10 10"
# Over a ground plane the pattern covers the upper hemisphere only.
PATTERN_UPPER = "RP 0 10 36 1000 0 0 10 10"


def dipole_cube(directory, freq_mhz=300.0, side_cells=16, eps=(4.0, 0.1), pattern=True, pec=False):
    """A centre-fed z-directed half-wave dipole (radius 1 mm, 21 segments,
    1 V at segment 11) 0.1 lambda from one face of a 0.2 lambda dielectric cube
    (ER 4, EI 0.1, meshed side_cells per side), free space.  With pec the
    model stands over a perfectly conducting ground plane (GN 1): the cube's
    bottom face 4 half-cells above it (the FFT image embedding wants the gap
    on the half-cell lattice, dielectric_fft.c:137-148) and the dipole 0.05
    lambda above it.  Returns the deck path."""
    lam = C0 / (freq_mhz * 1e6)
    z0 = 0.0
    if pec:
        z0 = 4 * (0.2 * lam / side_cells) / 2 + 0.1 * lam   # cube centre height
        zw = 0.05 * lam + lam / 4                           # dipole centre height
    q = 4.0 * np.pi * 0.2 * np.sqrt(abs(complex(eps[0], -eps[1]))) / (2 * side_cells)
    # MAX_KH so that the mesher's ceil(k n L / MAX_KH) gives side_cells
    # (dielectric_mesh.c:529-571), with margin against rounding.
    max_kh = float(q * (1.0 + 1e-6))
    deck = "\n".join([
        "CM dipole beside a dielectric cube",
        "CE",
        "GW 1 21 0 0 %r 0 0 %r 0.001" % ((zw - lam / 4, zw + lam / 4) if pec else (-lam / 4, lam / 4)),
        "GE 1" if pec else "GE 0",
        "FR 0 1 0 0 %r" % freq_mhz] + (["GN 1"] if pec else []) + [
        "EX 0 1 11 0 1 0",
        'DF "cube.diel"',
        (PATTERN_UPPER if pec else PATTERN) if pattern else "XQ",
        "EN", ""])
    diel = "\n".join([
        "NEC2C-DIELECTRIC 2",
        "MATERIAL 1 ER %r EI %r" % eps,
        "REGION 1 MATERIAL 1",
        "BOX 1 %r %r %r %r %r %r" % (0.1 * lam, -0.1 * lam, z0 - 0.1 * lam, 0.3 * lam, 0.1 * lam, z0 + 0.1 * lam),
        "MESH MAX_KH %r MAX_CELLS %d" % (max_kh, side_cells ** 3),
        "END", ""])
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "cube.diel"), "w") as f:
        f.write(diel)
    path = os.path.join(directory, "dipole_cube.nec")
    with open(path, "w") as f:
        f.write(deck)
    return path


def dipole_cube_sweep(directory, freqs_mhz=(280.0, 300.0, 320.0)):
    """The dipole beside a 0.2 lambda (at 300 MHz) cube whose permittivity is
    a frequency table (resource version 3: ER 4 -> 3 -> 2 and conductivity
    0.01 -> 0.03 S/m between 260 and 340 MHz, interpolated linearly by the
    reference's material law, dielectric.h:36-56), swept over freqs_mhz in one
    run (FR card; one execution per frequency).  The mesher sizes the cells for
    the highest frequency and the table's largest permittivity."""
    lam = C0 / 300e6
    deck = "\n".join([
        "CM dipole beside a dispersive dielectric cube, frequency sweep",
        "CE",
        "GW 1 21 0 0 %r 0 0 %r 0.001" % (-lam / 4, lam / 4),
        "GE 0",
        "FR 0 %d 0 0 %r %r" % (len(freqs_mhz), freqs_mhz[0],
                              (freqs_mhz[1] - freqs_mhz[0]) if len(freqs_mhz) > 1 else 0.0),
        "EX 0 1 11 0 1 0",
        'DF "cube_table.diel"',
        "XQ",
        "EN", ""])
    diel = "\n".join([
        "NEC2C-DIELECTRIC 3",
        "MATERIAL 1 TABLE",
        "SAMPLE 1 FREQ_MHZ 260 ER 4 SIGMA .01",
        "SAMPLE 1 FREQ_MHZ 300 ER 3 SIGMA .02",
        "SAMPLE 1 FREQ_MHZ 340 ER 2 SIGMA .03",
        "REGION 1 MATERIAL 1",
        "BOX 1 %r %r %r %r %r %r" % (0.1 * lam, -0.1 * lam, -0.1 * lam, 0.3 * lam, 0.1 * lam, 0.1 * lam),
        "MESH MAX_KH 0.3 MAX_CELLS 4096",
        "END", ""])
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "cube_table.diel"), "w") as f:
        f.write(diel)
    path = os.path.join(directory, "dipole_cube_sweep.nec")
    with open(path, "w") as f:
        f.write(deck)
    return path


def plane_wave_cube(directory, side_cells, freq_mhz=300.0, eps=(4.0, 0.1)):
    """A dielectric cube of side 0.2 lambda (ER 4, EI 0.1) meshed side_cells per
    side, alone in free space, lit by an x-polarised plane wave travelling
    along z (EX 1; the volume-only solver, dielectric_solver.c:315).  Returns
    the deck path."""
    lam = C0 / (freq_mhz * 1e6)
    q = 4.0 * np.pi * 0.2 * np.sqrt(abs(complex(eps[0], -eps[1]))) / (2 * side_cells)
    deck = "\n".join([
        "CM dielectric cube in a plane wave",
        "CE",
        "GE",
        "FR 0 1 0 0 %r 0" % freq_mhz,
        "EX 1 1 1 0 0 0 0 0 0 0",
        'DF "pw.diel"',
        "XQ",
        "EN", ""])
    diel = "\n".join([
        "NEC2C-DIELECTRIC 2",
        "MATERIAL 1 ER %r EI %r" % eps,
        "REGION 1 MATERIAL 1",
        "BOX 1 %r %r %r %r %r %r" % (-0.1 * lam, -0.1 * lam, -0.1 * lam, 0.1 * lam, 0.1 * lam, 0.1 * lam),
        "MESH MAX_KH %r MAX_ASPECT 1 MAX_CELLS %d" % (float(q * (1.0 + 1e-6)), side_cells ** 3),
        "END", ""])
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "pw.diel"), "w") as f:
        f.write(diel)
    path = os.path.join(directory, "plane_wave_cube.nec")
    with open(path, "w") as f:
        f.write(deck)
    return path


def run_status(binary, deck, args, timeout=900, env=None):
    """Runs a nec2c program on a deck; returns (exit code, result JSON or None,
    printed output).  env: extra environment variables."""
    base = os.path.splitext(deck)[0] + "_" + os.path.basename(binary)
    out, res = base + ".out", base + ".json"
    p = subprocess.run([binary, "-i", deck, "-o", out, "--result-json", res] + list(args),
                       capture_output=True, text=True, timeout=timeout, cwd=os.path.dirname(deck),
                       env=dict(os.environ, **env) if env else None)
    doc = None
    if os.path.exists(res):
        with open(res) as f:
            doc = json.load(f)
    text = open(out).read() if os.path.exists(out) else ""
    return p.returncode, doc, text + p.stderr


def dipole_array(directory, rows=8, cols=8, segments=31, seed=1, freq_mhz=300.0, pattern=True, pec=False):
    """rows x cols parallel z-directed half-wave dipoles at 0.5 lambda pitch in
    the xy plane, radius lambda/1000, free space (pec: raised 0.3 lambda
    above a perfectly conducting ground, GN 1).  Element (3, 3) (the last
    row or column of a smaller array) is driven
    with 1 V at its centre segment; every other element carries a seeded
    resistive load of 50 +- 10 ohm at its centre segment.  Returns the deck
    path."""
    lam = C0 / (freq_mhz * 1e6)
    rng = np.random.default_rng(seed)
    mid = segments // 2 + 1
    z0 = 0.55 * lam if pec else 0.0
    lines = ["CM %dx%d dipole array, seed %d" % (rows, cols, seed), "CE"]
    tag = 0
    driven = None
    for r in range(rows):
        for c in range(cols):
            tag += 1
            x, y = c * 0.5 * lam, r * 0.5 * lam
            # %.12g keeps a card within NEC's 132-character line limit.
            lines.append("GW %d %d %.12g %.12g %.12g %.12g %.12g %.12g %.12g"
                         % (tag, segments, x, y, z0 - lam / 4, x, y, z0 + lam / 4, lam / 1000))
            if (r, c) == (min(3, rows - 1), min(3, cols - 1)):
                driven = tag
    lines += ["GE 1" if pec else "GE 0"]
    tag = 0
    for r in range(rows):
        for c in range(cols):
            tag += 1
            if tag != driven:
                lines.append("LD 0 %d %d %d %r 0 0" % (tag, mid, mid, float(rng.uniform(40.0, 60.0))))
    lines += ["FR 0 1 0 0 %r" % freq_mhz] + (["GN 1"] if pec else []) + ["EX 0 %d %d 0 1 0" % (driven, mid),
              (PATTERN_UPPER if pec else PATTERN) if pattern else "XQ", "EN", ""]
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "dipole_array.nec")
    with open(path, "w") as f:
        f.write("\n".join(lines))
    return path


def junctions(directory, freq_mhz=300.0, pec=False):
    """Wires meeting at junctions, for the basis functions a junction gives
    (NEC's trio over several connected segments): a vertical half-wave
    dipole in two wires, two horizontal quarter-wave arms from its centre
    (a four-wire junction), a bent wire continuing the first arm, a short
    stub off the second, radius lambda/500; 1 V at the lower wire's middle
    segment, a 75 ohm load on the bent wire.  pec: raised 0.4 lambda above a
    perfectly conducting ground (GN 1).  Returns the deck path."""
    lam = C0 / (freq_mhz * 1e6)
    z0 = 0.4 * lam if pec else 0.0
    a = lam / 500
    q = lam / 4
    wires = [(1, 9, 0, 0, z0 - q, 0, 0, z0), (2, 9, 0, 0, z0, 0, 0, z0 + q),
             (3, 7, 0, 0, z0, q, 0, z0), (4, 7, 0, 0, z0, 0, q, z0),
             (5, 5, q, 0, z0, q, 0.6 * q, z0 + 0.3 * q), (6, 3, 0, q, z0, -0.2 * q, q, z0 - 0.25 * q)]
    lines = ["CM junctions", "CE"]
    for tag, nseg, x1, y1, z1, x2, y2, z2 in wires:
        lines.append("GW %d %d %.12g %.12g %.12g %.12g %.12g %.12g %.12g" % (tag, nseg, x1, y1, z1, x2, y2, z2, a))
    lines += ["GE 1" if pec else "GE 0", "LD 0 5 3 3 75 0 0", "FR 0 1 0 0 %r" % freq_mhz]
    lines += (["GN 1"] if pec else []) + ["EX 0 1 5 0 1 0", PATTERN_UPPER if pec else PATTERN, "EN", ""]
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "junctions.nec")
    with open(path, "w") as f:
        f.write("\n".join(lines))
    return path


def run(binary, deck, args, timeout=900, env=None):
    """Runs a nec2c program on a deck; returns (result JSON, wall seconds,
    stderr).  env: extra environment variables."""
    import time
    base = os.path.splitext(deck)[0] + "_" + os.path.basename(binary)
    out, res = base + ".out", base + ".json"
    t0 = time.perf_counter()
    p = subprocess.run([binary, "-i", deck, "-o", out, "--result-json", res] + list(args),
                       capture_output=True, text=True, timeout=timeout, cwd=os.path.dirname(deck),
                       env=dict(os.environ, **env) if env else None)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError("%s failed (%d): %s" % (os.path.basename(binary), p.returncode, p.stderr[-2000:]))
    with open(res) as f:
        return json.load(f), wall, p.stderr


def executions(doc):
    return doc["jobs"][0]["executions"]


def execution(doc, index=0):
    return executions(doc)[index]


def feed_impedance(doc, index=0):
    z = execution(doc, index)["feeds"][0]["impedance_ohm"]
    return complex(z["re"], z["im"])


def wire_currents(doc, index=0):
    return np.array([complex(w["current_a"]["re"], w["current_a"]["im"])
                     for w in execution(doc, index)["wire_currents"]])


def volume_currents(doc, index=0):
    vc = execution(doc, index)["volume_currents"]
    if not vc or not vc["rows"]:
        return np.zeros(0, dtype=np.complex128)
    cols = vc["columns"]
    idx = [cols.index(n) for n in ("jx_re_a_per_m2", "jx_im_a_per_m2", "jy_re_a_per_m2", "jy_im_a_per_m2",
                                    "jz_re_a_per_m2", "jz_im_a_per_m2")]
    a = np.array([[row[i] for i in idx] for row in vc["rows"]], dtype=np.float64)
    return (a[:, 0::2] + 1j * a[:, 1::2]).ravel()


ETA0 = 376.730313412


def gains_db(doc):
    """Power gain in dB, 4 pi |r E|^2 / (2 eta0 P_in), of every far-field
    direction the deck asked for (the documents give r E per direction and
    the power the feed accepts)."""
    e = execution(doc)
    p_in = e["feeds"][0]["accepted_power_w"]
    out = []
    for block in e["far_fields"]:
        for smp in block["samples"]:
            re2 = sum(smp[k]["re"] ** 2 + smp[k]["im"] ** 2 for k in ("r_e_theta", "r_e_phi"))
            out.append(4 * np.pi * re2 / (2 * ETA0 * p_in))
    g = np.array(out, dtype=np.float64)
    with np.errstate(divide="ignore"):
        return 10 * np.log10(g)


def gain_difference_db(a, b, window_db=30.0):
    """Largest |gain_a - gain_b| in dB over the directions within window_db of
    the peak (nulls, where dB differences mean nothing, are left out)."""
    ga, gb = gains_db(a), gains_db(b)
    keep = ga >= ga.max() - window_db
    return float(np.max(np.abs(ga[keep] - gb[keep])))
