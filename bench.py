#!/usr/bin/env python
"""Benchmark of the nec2c CUDA backend on one B200 (replicas on N GPUs).

Workload: a 64x64x64-voxel block of side 1 lambda at
300 MHz (786,432 complex unknowns, 128^3 padded FFT grid), per-voxel
eps_r ~ U[2,10] and loss tangent ~ U[0.01,0.1] (seeded), x-polarised plane
wave excitation, GMRES(30) to rtol 1e-6 (iteration limit 10000, the CLI's
maximum: the reference default of 300 does not reach 1e-6 here).  A step is one solve on a
device-resident plan in the mixed form (FP32 transforms, FP64 Arnoldi, Givens
and true residual); its current error against the plain FP64 GPU form is
reported beside the throughput.  Synthetic, seeded inputs stand in for the
reference's decks (it publishes no dataset).

Roofline: the FFT matvec (scatter, five fused transform passes, gather) timed
with CUDA events on the launching stream, L2 flushed between launches, against
the algorithmic bytes s*(6C + 18G) per product (s = 8 B per complex FP32).

Reference arm (--impl reference): the reference nec2c's own builtin FFT plan
and vie_gmres (oracle/_ref, compiled from its sources) on the host cores.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

C0 = 299792458.0
SEED = 2
MAXIT = 10000
# dram__bytes_read.sum + dram__bytes_write.sum per FP32 matvec on this
# workload, summed over its five kernels, from the ncu capture summarised in
# profiles/fft_matvec_c2_64cube.md (the intermediate grids stay in L2).
MATVEC_TRAFFIC_BYTES = 118.2e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fft-schedule", default=None,
                    help="JSON file of the c2 plans' FFT pass schedules: written by the first run "
                         "that names it, pinned by later runs (a run under ncu would otherwise "
                         "tune on serialised, slowed launches)")
    ap.add_argument("--lu-systems", type=int, default=0,
                    help="lu_batch profiling mode: one batch of this many systems of order --lu-order "
                         "(0: the default table of orders and batch sizes)")
    ap.add_argument("--lu-order", type=int, default=1984,
                    help="lu profiling mode: order of the seeded MoM-like matrix (config 1: 1984)")
    ap.add_argument("--c4-arms", default=None,
                    help="serving_c4 profiling mode: a long-stream run of only these arms (mixed[,plain]): "
                         "the mixed form saturated and under Poisson arrivals, the plain FP64 form on the "
                         "first --c4-plain-requests requests")
    ap.add_argument("--c4-rates", default=None,
                    help="serving_c4 profiling mode: comma-separated Poisson rates as fractions of the "
                         "mixed form's saturated request rate")
    ap.add_argument("--c4-plain-requests", type=int, default=None,
                    help="serving_c4 long-stream run: requests of the plain FP64 arm (a prefix of the stream)")
    ap.add_argument("--requests", type=int, default=400,
                    help="serving_c4 profiling mode: requests in the stream (config 4 names 10,000)")
    ap.add_argument("--planes", type=int, choices=[0, 1], default=None,
                    help="profiling driver: pin the fused yz-plane passes on (1) or off (0) in both "
                         "c2 plans instead of the tuner's choice")
    ap.add_argument("--only", choices=["matvec", "solve", "lu", "lu_batch", "serving", "serving_c4", "volume_batch",
                                       "coupling"],
                    help="profiling driver: build the plans, run --steps FP32 and FP64 products "
                         "(matvec) or --steps mixed solves (solve), or factor the 1984-unknown dense "
                         "matrix --steps times in each LU form (lu), run the serving stream "
                         "(serving), the 192-system dipole-plus-cube batch (volume_batch) or the wire-volume "
                         "coupling blocks of the dipole-plus-cube model --steps times (coupling); print "
                         "timings and exit")
    return ap.parse_args()


def workload():
    lam = C0 / 300e6
    n = 64
    h, k = lam / n, 2 * math.pi / lam
    g = np.arange(n)
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3).astype(np.uintp)
    cells = xyz.shape[0]
    rng = np.random.default_rng(SEED)
    er = rng.uniform(2.0, 10.0, cells)
    tand = rng.uniform(0.01, 0.1, cells)
    eps = er * (1 - 1j * tand)
    rhs = np.zeros(3 * cells, dtype=np.complex128)
    z = xyz[:, 2].astype(np.float64)
    rhs[0::3] = 2 * np.exp(-1j * k * h * (z + 0.5)) * math.sin(k * h / 2) / (k * h / 2)
    return dict(shape=(n, n, n), xyz=xyz.reshape(-1), h=h, k=k, eps=eps, rhs=rhs, cells=cells,
                padded=128, grid=128 ** 3)


def near_table():
    with open(os.path.join(ROOT, "tests", "golden", "near_tensors.json")) as f:
        raw = json.load(f)["c2"]
    table = {}
    for row in raw["tensors"]:
        v = np.array(row[3:])
        table[tuple(int(t) for t in row[:3])] = v[0::2] + 1j * v[1::2]
    return table


def near_tables_all():
    """{case: (h, k, table)} of every case in tests/golden/near_tensors.json."""
    with open(os.path.join(ROOT, "tests", "golden", "near_tensors.json")) as f:
        raw = json.load(f)
    out = {}
    for name, c in raw.items():
        table = {}
        for row in c["tensors"]:
            vals = np.array(row[3:], dtype=np.float64)
            table[tuple(int(t) for t in row[:3])] = vals[0::2] + 1j * vals[1::2]
        out[name] = (c["h"], c["k"], table)
    return out


class Clocks:
    """nvidia-smi sampler over the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [t.strip() for t in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------ reference arm
def reference_lib():
    so = os.path.join(ROOT, "oracle", "_ref", "libnec2c_ref.so")
    if not os.path.exists(so):
        return None
    r = C.CDLL(so)
    vp, sz, dbl, i = C.c_void_p, C.c_size_t, C.c_double, C.c_int
    r.ref_fft_backend_set.argtypes = [C.c_char_p]
    r.ref_fft_create.argtypes = [C.POINTER(sz), sz, C.POINTER(sz), dbl, dbl, dbl, dbl, sz]
    r.ref_fft_create.restype = vp
    r.ref_fft_set_permittivity.argtypes = [vp, sz, dbl, dbl]
    r.ref_fft_destroy.argtypes = [vp]

    class Rep(C.Structure):
        _fields_ = [("status", C.c_int), ("iterations", C.c_size_t),
                    ("operator_applications", C.c_size_t), ("restarts", C.c_size_t),
                    ("residual_norm", C.c_double), ("relative_residual", C.c_double)]
    r.Rep = Rep
    r.ref_fft_gmres.argtypes = [vp, vp, vp, sz, sz, dbl, dbl, C.POINTER(Rep)]
    r.ref_fft_gmres.restype = i
    return r


def reference_plan(r, w):
    r.ref_fft_backend_set(b"builtin")
    xyz = np.ascontiguousarray(w["xyz"])
    p = r.ref_fft_create((C.c_size_t * 3)(*w["shape"]), w["cells"],
                         xyz.ctypes.data_as(C.POINTER(C.c_size_t)), w["h"], w["k"],
                         w["eps"][0].real, w["eps"][0].imag, 1 << 40)
    if not p:
        raise RuntimeError("reference plan build failed")
    for c, e in enumerate(w["eps"]):
        r.ref_fft_set_permittivity(p, c, e.real, e.imag)
    return p


def reference_solve(r, p, w, maxit=MAXIT):
    b = np.ascontiguousarray(w["rhs"])
    x = np.zeros_like(b)
    rep = r.Rep()
    t0 = time.perf_counter()
    r.ref_fft_gmres(p, b.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p), 30, maxit, 1e-6,
                    0.0, C.byref(rep))
    return time.perf_counter() - t0, rep


def cpu_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


SAMPLE_ITERATIONS = 30


def cpu_baseline(w, full_iterations):
    """The reference on a bounded sample: one 30-iteration restart cycle of its
    vie_gmres on this workload (plan build untimed, all host threads), scaled
    to a full solve of full_iterations iterations."""
    r = reference_lib()
    if r is None:
        return None
    p = reference_plan(r, w)
    t, rep = reference_solve(r, p, w, maxit=SAMPLE_ITERATIONS)
    r.ref_fft_destroy(p)
    per_iter = t / max(rep.iterations, 1)
    return {"value": 1.0 / (per_iter * full_iterations), "unit": "solves/s", "cores": cpu_threads(),
            "kind": "reference",
            "sample": "reference vie_gmres (builtin FFT, OpenMP) for %d iterations (%.2f s incl. the "
                      "initial true residual), scaled to the %d iterations of a full solve (the reference's "
                      "own full solve takes the same count: tests/golden/c2_reference_solve.json)"
                      % (rep.iterations, t, full_iterations),
            "c0_deck": reference_c0_deck()}


def reference_c0_deck():
    """The stock reference program (oracle/_ref/nec2c) on BASELINE config 0
    end to end, -s fft -r 1e-6, all host threads: the time the drop-in
    program's deck_c0_dropin line compares with."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import tempfile
    import decks
    if not os.path.exists(decks.REF_BIN):
        return None
    deck = decks.dipole_cube(tempfile.mkdtemp())
    doc, wall, _ = decks.run(decks.REF_BIN, deck, ["-s", "fft", "-r", "1e-6", "--jobs", "1"])
    z = decks.feed_impedance(doc)
    return {"wall_s": wall, "threads": os.cpu_count(), "zin_ohm": [z.real, z.imag],
            "iterations": decks.execution(doc)["solver"]["iterations"]}


def run_reference(args, rank, world):
    """The reference's own CPU code on this workload (its builtin FFT plan and
    vie_gmres, OpenMP over all host threads).  After the warm-up steps
    (1-iteration solves) it runs ONE full solve to rtol 1e-6, timed as a
    whole, which gives the reference's own iteration count and solve time.
    Each timed step is then a bounded sample, one 30-iteration restart cycle;
    value scales the samples' per-iteration time to the full solve's measured
    iteration count, and ms_per_step is the samples' own measured time."""
    if rank != 0:
        return 0
    w = workload()
    r = reference_lib()
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return 0
    t_plan = time.perf_counter()
    p = reference_plan(r, w)
    t_plan = time.perf_counter() - t_plan
    for _ in range(args.warmup):
        reference_solve(r, p, w, maxit=1)          # warm-up: one iteration each
    t_full, rep_full = reference_solve(r, p, w)
    if rep_full.status != 0:
        raise RuntimeError("reference full solve did not converge: status %d" % rep_full.status)
    full_iterations = int(rep_full.iterations)
    sample_s, per_iter = [], []
    for _ in range(args.steps):
        t, rep = reference_solve(r, p, w, maxit=SAMPLE_ITERATIONS)
        sample_s.append(t)
        per_iter.append(t / max(rep.iterations, 1))
    r.ref_fft_destroy(p)
    solve_s = [t * full_iterations for t in per_iter]
    v = len(solve_s) / sum(solve_s)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(sample_s) / len(sample_s),
        "step": "one %d-iteration GMRES restart cycle of the reference (a bounded sample of a solve); "
                "value scales the samples to the measured iteration count of the full solve"
                % SAMPLE_ITERATIONS,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": config_for(world),
        "full_solve": {"seconds": t_full, "iterations": full_iterations, "restarts": int(rep_full.restarts),
                       "relative_residual": rep_full.relative_residual, "solves_per_s": 1.0 / t_full,
                       "plan_build_s": t_plan},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cpu_threads(), "kind": "reference",
                         "sample": "one full reference solve (%d iterations, %.1f s) measured, then per "
                                   "step the reference vie_gmres (builtin FFT, OpenMP) for %d "
                                   "iterations, scaled to the full solve's %d iterations; warm-up "
                                   "steps are 1-iteration solves"
                                   % (full_iterations, t_full, SAMPLE_ITERATIONS, full_iterations)},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "latency_ms": {"p50": 1e3 * statistics.median(solve_s), "p99": 1e3 * max(solve_s)}}))
    return 0


METRIC = ("VIE solves/s at rel.err<=1e-5 vs the FP64 GPU form (64^3 inhomogeneous VIE, "
          "GMRES(30) rtol 1e-6); FFT matvec HBM GB/s")
CONFIG = {"workload": "c2: 64^3-voxel inhomogeneous dielectric block, side 1 lambda at 300 MHz, "
                      "786432 unknowns, 128^3 padded grid, eps_r~U[2,10], tand~U[0.01,0.1], "
                      "x-polarised plane wave, GMRES(30) rtol 1e-6",
          "seed": SEED, "precision": "mixed: FP32 transforms; FP64 vectors, Arnoldi, Givens, "
                                      "true residual",
          "l2": "solve working set > L2 (Krylov basis 390 MB); matvec timings flush L2 (256 MB write)"}


def config_for(world):
    """The workload dict both arms print (the same for both, so their lines
    compare): one device per process, replicas across processes."""
    return dict(CONFIG, parallelism="replicas" if world > 1 else "single device")


# ------------------------------------------------------------ replicas
def max_over_ranks(ms, world, device):
    """The slowest rank's device time (replicas: every rank runs the whole
    workload on its own GPU; the job takes as long as the slowest)."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, steps, total_ms):
    """Whole-job solves/s: every rank solved `steps` systems in at most
    total_ms."""
    return world * steps / (total_ms * 1e-3)


# ------------------------------------------------------------------ our arm
def pin_schedules(path, nb, plan_m, plan_d):
    """Saves the tuned pass schedules of the c2 plans to path, or pins the ones
    saved there by an earlier run of the same command."""
    if not path:
        return
    plans = {"mixed_fp32": (plan_m, False), "mixed_fp64": (plan_m, True), "plain_fp64": (plan_d, True)}
    if os.path.exists(path):
        with open(path) as f:
            saved = json.load(f)
        for key, (plan, fp64) in plans.items():
            if not plan.set_schedule([tuple(e) for e in saved[key]], fp64=fp64):
                raise RuntimeError("cannot pin the saved schedule: " + nb.last_error())
        return
    with open(path, "w") as f:
        json.dump({key: plan.schedule(fp64=fp64)[1] for key, (plan, fp64) in plans.items()}, f)


def far_field_error(lib, nb, plan, x_a, x_b, w, count=974):
    """Scattered far field of two solutions of the same plan (device vectors),
    over the reference's 974-point sphere rule (dielectric_solver.c:153-176):
    the largest intensity difference in dB over the directions within 30 dB
    of the pattern's peak, and the relative difference of the scattered power
    (the rule's sum of intensities)."""
    golden = math.pi * (3 - math.sqrt(5))
    i = np.arange(count)
    z = 1 - 2 * (i + 0.5) / count
    r = np.sqrt(np.maximum(0, 1 - z * z))
    dirs = np.ascontiguousarray(np.stack([r * np.cos(golden * i), r * np.sin(golden * i), z], axis=1))
    h = w["h"]
    origin = (C.c_double * 3)(0.5 * h, 0.5 * h, 0.5 * h)
    inten = []
    for x in (x_a, x_b):
        amp = np.empty((count, 3), dtype=np.complex128)
        if not lib.nec2c_cuda_vie_fft_radiation_device(plan.h, origin, C.c_void_p(x.data_ptr()), count,
                                                       dirs.ctypes.data_as(C.c_void_p),
                                                       amp.ctypes.data_as(C.c_void_p)):
            raise RuntimeError("radiation failed: " + nb.last_error())
        inten.append(np.sum(np.abs(amp) ** 2, axis=1))
    a, b = inten
    keep = b >= 1e-3 * b.max()
    return {"directions": count, "max_db_error": float(np.max(np.abs(10 * np.log10(a[keep] / b[keep])))),
            "scattered_power_rel_err": float(abs(a.sum() - b.sum()) / b.sum())}


def run_ours(args, rank, world, local_rank):
    import torch
    import nec2c_b200 as nb

    torch.cuda.set_device(local_rank)
    lib = nb.load()
    if not lib.nec2c_cuda_set_device(local_rank) or not lib.nec2c_cuda_available():
        raise RuntimeError("CUDA backend unavailable: " + nb.last_error())
    stream = torch.cuda.current_stream()
    lib.nec2c_cuda_set_stream(C.c_void_p(stream.cuda_stream))
    if args.only == "lu":
        return lu_driver(args, nb, torch, stream)
    if args.only == "lu_batch":
        kw = {}
        if args.lu_systems:
            kw = {"orders": (args.lu_order,), "counts": (args.lu_systems,), "reps": max(1, args.steps)}
        print(json.dumps({"profile": "lu_batch", "lockstep_factor": lockstep_factor_bench(nb, torch, stream, **kw)}))
        return 0
    if args.only == "serving":
        print(json.dumps({"profile": "serving", "serving_c4": serving_bench(nb, torch)}))
        return 0
    if args.only == "serving_c4":
        rates = tuple(float(r) for r in args.c4_rates.split(",")) if args.c4_rates else (0.3, 0.5, 0.7, 0.9, 1.1)
        arms = set(args.c4_arms.split(",")) if args.c4_arms else None
        print(json.dumps({"profile": "serving_c4", "serving_c4_stream": serving_stream_c4(
            nb, torch, args.requests, rates=rates, arms=arms, plain_requests=args.c4_plain_requests)}))
        return 0
    if args.only == "coupling":
        print(json.dumps({"profile": "coupling", "coupling_c0": coupling_bench(nb, args.steps)}))
        return 0
    if args.only == "volume_batch":
        print(json.dumps({"profile": "volume_batch", "batched_volume_c3": volume_batch_bench(nb, torch, stream)}))
        return 0
    w = workload()
    table = near_table()

    def make_plan(mixed):
        t0 = time.perf_counter()
        p = nb.VolumePlan(w["shape"], w["xyz"], w["h"], w["k"], w["eps"][0], table, mixed=mixed)
        for c, e in enumerate(w["eps"]):
            if not p.set_permittivity(c, e):
                raise RuntimeError("permittivity rejected")
        torch.cuda.synchronize()
        return p, time.perf_counter() - t0

    plan_m, build_s = make_plan(True)
    plan_d, _ = make_plan(False)
    pin_schedules(args.fft_schedule, nb, plan_m, plan_d)
    n = plan_m.n
    if args.only:
        return profile_driver(args, lib, nb, torch, stream, plan_m, plan_d, w)
    b_dev = torch.from_numpy(w["rhs"]).to("cuda")
    x_dev = torch.zeros(n, dtype=torch.complex128, device="cuda")
    opts = nb.GmresOptions(30, MAXIT, 1e-6, 0.0)

    def solve_dev(plan, x):
        x.zero_()
        rep = nb.GmresReport()
        ok = lib.nec2c_cuda_gmres_plan_device(plan.h, C.c_void_p(b_dev.data_ptr()),
                                              C.c_void_p(x.data_ptr()), C.byref(opts), C.byref(rep))
        if not ok:
            raise RuntimeError("solve failed: %s %s" % (rep.as_dict(), nb.last_error()))
        return rep

    for _ in range(args.warmup):
        solve_dev(plan_m, x_dev)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches0 = lib.nec2c_cuda_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with Clocks(local_rank) as clk:
        torch.cuda.synchronize()
        for e0, e1 in ev:
            e0.record(stream)
            rep = solve_dev(plan_m, x_dev)
            e1.record(stream)
        torch.cuda.synchronize()
    launches = lib.nec2c_cuda_launch_count() - launches0
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total_ms = max_over_ranks(sum(step_ms), world, "cuda")
    iterations = rep.iterations
    x_mixed = x_dev.clone()

    # Plain FP64 form on the same solve, and the current error against it.
    solve_dev(plan_d, x_dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rep64 = solve_dev(plan_d, x_dev)
    e1.record(stream)
    torch.cuda.synchronize()
    fp64_ms = e0.elapsed_time(e1)
    rel_err = float(torch.linalg.norm(x_mixed - x_dev) / torch.linalg.norm(x_dev))
    far = far_field_error(lib, nb, plan_m, x_mixed, x_dev, w)

    # e2e through the public C ABI with pinned host buffers (H2D + D2H inside).
    b_host = torch.from_numpy(w["rhs"]).pin_memory()
    x_host = torch.zeros(n, dtype=torch.complex128).pin_memory()
    e2e_ms = []
    for _ in range(max(1, args.steps)):
        x_host.zero_()
        rep_h = nb.GmresReport()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ok = lib.nec2c_cuda_gmres_plan(plan_m.h, C.c_void_p(b_host.data_ptr()),
                                       C.c_void_p(x_host.data_ptr()), C.byref(opts), C.byref(rep_h))
        e1.record(stream)
        torch.cuda.synchronize()
        if not ok:
            raise RuntimeError("host-vector solve failed")
        e2e_ms.append(e0.elapsed_time(e1))

    # Matvec roofline: device products, L2 flushed between launches.
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    xv = torch.randn(n, dtype=torch.complex128, device="cuda")
    yv = torch.empty_like(xv)

    def time_matvec(plan, reps=20):
        out = []
        for i in range(reps + 3):
            flush.zero_()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            lib.nec2c_cuda_vie_fft_apply_device(plan.h, C.c_void_p(xv.data_ptr()),
                                                C.c_void_p(yv.data_ptr()))
            a1.record(stream)
            torch.cuda.synchronize()
            if i >= 3:
                out.append(a0.elapsed_time(a1))
        return statistics.median(out)

    mv32_ms = time_matvec(plan_m)
    mv64_ms = time_matvec(plan_d)
    planes32, planes64 = plan_m.planes(fp64=False), plan_d.planes(fp64=True)
    # Both product forms on the same plans: the fused plane passes (three
    # launches) and the five passes.
    forms = {}
    for key, plan, fp64, chosen in (("fp32", plan_m, False, planes32), ("fp64", plan_d, True, planes64)):
        if chosen < 0:
            continue
        forms[key] = {}
        for planes in (1, 0):
            plan.set_planes(planes, fp64=fp64)
            forms[key]["planes_ms" if planes else "five_pass_ms"] = time_matvec(plan)
        plan.set_planes(chosen, fp64=fp64)
    # The measured pass schedule against the heuristic one on the same plan.
    tuned32, tuned64 = plan_m.schedule(fp64=False)[1], plan_d.schedule(fp64=True)[1]
    plan_m.tune(0)
    plan_d.tune(0)
    heur32, heur64 = plan_m.schedule(fp64=False)[1], plan_d.schedule(fp64=True)[1]
    mv32_heur_ms = time_matvec(plan_m)
    mv64_heur_ms = time_matvec(plan_d)
    plan_m.tune(1)
    plan_d.tune(1)
    schedule = {
        "passes": ["z fwd + scatter", "y fwd", "x fwd + product + x inv", "y inv", "z inv + epilogue"],
        "fp32": {"tuned": tuned32, "heuristic": heur32, "tuned_ms": mv32_ms, "heuristic_ms": mv32_heur_ms},
        "fp64": {"tuned": tuned64, "heuristic": heur64, "tuned_ms": mv64_ms, "heuristic_ms": mv64_heur_ms},
        "entry": "[lines per tile, R1]",
        "planes_in_use": {"fp32": planes32, "fp64": planes64},
        "forms_ms": forms,
    }
    C_, G_ = w["cells"], w["grid"]
    bytes32 = 8 * (6 * C_ + 18 * G_)
    bytes64 = 16 * (6 * C_ + 18 * G_)
    peak, peak_kind = peaks()
    achieved = bytes32 / (mv32_ms * 1e-3) / 1e9

    # Dense LU of 1984 unknowns, both forms.
    dense = dense_bench(nb, torch, stream)
    # Lockstep batches of 16 dense factorisations (FP64 and split precision)
    # against one factorisation at a time, resident matrices.
    lockstep = lockstep_factor_bench(nb, torch, stream, orders=(1000, 2608), counts=(16,), reps=2)
    # 192 small wire blocks, ragged batch in one launch.
    batched = batched_bench(nb, torch)
    # 192-system dipole-plus-cube sweep, ragged batch of plans.
    volume_batch = volume_batch_bench(nb, torch, stream)
    # Mixed dense and volume serving stream (bounded), both forms.
    serving = serving_stream_c4(nb, torch) if world == 1 else None
    # Config 0 end to end through the drop-in program, and its two coupling
    # blocks through the C ABI (rank 0 only).
    deck_c0 = deck_bench() if rank == 0 else None
    coupling = coupling_bench(nb, 10) if rank == 0 else None
    lib.nec2c_cuda_set_stream(C.c_void_p(stream.cuda_stream))

    if rank != 0:
        return 0
    cpu = None if (args.no_cpu_baseline or world > 1) else cpu_baseline(w, rep64.iterations)
    value = replica_rate(world, args.steps, total_ms)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 transforms / c128 Krylov",
        "data": "synthetic", "config": config_for(world),
        "iterations": iterations, "rel_err_vs_fp64_gpu": rel_err, "far_field_vs_fp64_gpu": far,
        "latency_ms": {"p50": statistics.median(step_ms), "p99": max(step_ms)},
        "fp64_form": {"solves_per_s": 1e3 / fp64_ms, "iterations": rep64.iterations,
                      "ms": fp64_ms},
        "plan_build_s": build_s,
        "e2e": {"value": world * 1e3 / statistics.median(e2e_ms), "unit": "solves/s",
                "h2d_bytes_per_step": 2 * 16 * n, "d2h_bytes_per_step": 16 * n},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": MATVEC_TRAFFIC_BYTES,
                     "kernel": ("FFT matvec, FP32: fused yz-plane forward (scatter), x pass with the "
                                "spectrum product, fused yz-plane inverse (epilogue)" if planes32 == 1 else
                                "FFT matvec (scatter + 5 transform passes + gather), FP32"),
                     "algorithmic_bytes": bytes32, "ms": mv32_ms},
        "matvec_fp64": {"ms": mv64_ms, "achieved_gbs": bytes64 / (mv64_ms * 1e-3) / 1e9},
        "fft_schedule": schedule,
        "dense_lu_c1": dense,
        "lockstep_lu": lockstep,
        "batched_wire_blocks_c3": batched,
        "batched_volume_c3": volume_batch,
        "serving_c4": serving,
        "deck_c0_dropin": deck_c0,
        "coupling_c0": coupling,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0


def profile_driver(args, lib, nb, torch, stream, plan_m, plan_d, w):
    n = plan_m.n
    if args.planes is not None:
        for plan, precs in ((plan_m, (False, True)), (plan_d, (True,))):
            for fp64 in precs:
                if not plan.set_planes(args.planes, fp64=fp64):
                    raise RuntimeError(nb.last_error())
    x = torch.randn(n, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    # The products (or solves) sit in an NVTX range "products", so a launch
    # list can leave out the plan build and its schedule timing:
    #   ncu --nvtx --nvtx-include "products]" ...
    torch.cuda.nvtx.range_push("products")
    t0 = time.perf_counter()
    if args.only == "matvec":
        for plan in (plan_m, plan_d):
            for _ in range(args.steps):
                if not lib.nec2c_cuda_vie_fft_apply_device(plan.h, C.c_void_p(x.data_ptr()),
                                                           C.c_void_p(y.data_ptr())):
                    raise RuntimeError(nb.last_error())
    else:
        b = torch.from_numpy(w["rhs"]).to("cuda")
        opts = nb.GmresOptions(30, MAXIT, 1e-6, 0.0)
        for _ in range(args.steps):
            y.zero_()
            rep = nb.GmresReport()
            if not lib.nec2c_cuda_gmres_plan_device(plan_m.h, C.c_void_p(b.data_ptr()),
                                                    C.c_void_p(y.data_ptr()), C.byref(opts),
                                                    C.byref(rep)):
                raise RuntimeError(nb.last_error())
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    elapsed = time.perf_counter() - t0
    timed = {}
    if args.only == "matvec":
        # Event-timed products outside the NVTX range, L2 flushed before each.
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        for key, plan in (("fp32_us", plan_m), ("fp64_us", plan_d)):
            out = []
            for i in range(23):
                flush.zero_()
                a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a0.record(stream)
                lib.nec2c_cuda_vie_fft_apply_device(plan.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))
                a1.record(stream)
                torch.cuda.synchronize()
                if i >= 3:
                    out.append(1e3 * a0.elapsed_time(a1))
            timed[key] = statistics.median(out)
    print(json.dumps({"profile": args.only, "steps": args.steps, "s": elapsed, "products": timed,
                      "fft_schedule": {"fp32": plan_m.schedule(fp64=False)[1],
                                       "fp64": plan_d.schedule(fp64=True)[1],
                                       "planes": [plan_m.planes(fp64=False), plan_d.planes(fp64=True)]}}))
    return 0


def c1_matrix(n=1984):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a += np.diag(np.full(n, 0.5 * math.sqrt(n)))
    return a


def device_factor(nb, torch, stream, a, form, reps):
    """Factors a resident copy of a (reps + 1 times, the first untimed) with
    the device LU of the given form, then solves one right-hand side with the
    factors (reps + 1 times, the first untimed); returns the fastest factor
    and solve times in ms."""
    lib = nb.load()
    n = a.shape[0]
    if form == "cuda":
        f = lib.n2d_lu_factor
        f.restype, f.argtypes = C.c_int, [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int, C.c_int,
                                          C.POINTER(C.c_int)]
        src = torch.from_numpy(a).cuda()
        ld = n
    else:
        f = lib.n2d_lu_factor32
        f.restype, f.argtypes = C.c_int, [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int,
                                          C.POINTER(C.c_int)]
        ld = n + (n & 1)
        a32 = np.zeros((n, ld), dtype=np.complex64)
        a32[:, :n] = a
        src = torch.from_numpy(a32).cuda()
    work = src.clone()
    piv = torch.zeros(n, dtype=torch.int32, device="cuda")
    ts = []
    for i in range(reps + 1):
        work.copy_(src)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        info = C.c_int(0)
        e0.record(stream)
        ok = (f(work.data_ptr(), n, ld, piv.data_ptr(), 0, 0, C.byref(info)) if form == "cuda" else
              f(work.data_ptr(), n, ld, piv.data_ptr(), 0, C.byref(info)))
        e1.record(stream)
        torch.cuda.synchronize()
        if not ok or info.value:
            raise RuntimeError("device factor failed: " + nb.last_error())
        if i:
            ts.append(e0.elapsed_time(e1))
    sf = lib.n2d_lu_solve if form == "cuda" else lib.n2d_lu_solve32
    sf.restype, sf.argtypes = C.c_int, [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_void_p,
                                        C.c_longlong, C.c_longlong]
    rhs = torch.ones(n, dtype=torch.complex128, device="cuda")
    ss = []
    for i in range(reps + 1):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ok = sf(work.data_ptr(), n, ld, piv.data_ptr(), rhs.data_ptr(), n, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        if not ok:
            raise RuntimeError("device solve failed: " + nb.last_error())
        if i:
            ss.append(e0.elapsed_time(e1))
    return min(ts), min(ss)


def lu_driver(args, nb, torch, stream):
    a = c1_matrix(args.lu_order)
    out = {form: device_factor(nb, torch, stream, a, form, max(1, args.steps)) for form in ("cuda", "cuda-mixed")}
    print(json.dumps({"profile": "lu", "order": a.shape[0],
                      "device_factor_ms": {f: t[0] for f, t in out.items()},
                      "device_solve_ms": {f: t[1] for f, t in out.items()}}))
    return 0


def lockstep_factor_bench(nb, torch, stream, orders=(250, 1000, 2608), counts=(1, 4, 16), reps=3):
    """Lockstep batch of FP64 factorisations against one factorisation at a
    time, on device-resident copies of seeded MoM-like matrices: device ms per
    batch (CUDA events, fastest of reps after a warm-up) and the achieved
    factorisation rate (8n^3/3 flops each)."""
    lib = nb.load()
    single = lib.n2d_lu_factor
    single.restype, single.argtypes = C.c_int, [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int,
                                                C.c_int, C.POINTER(C.c_int)]
    batch = lib.n2d_lu_factor_batch
    batch.restype, batch.argtypes = C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                              C.c_void_p]
    batch32 = lib.n2d_lu_factor32_batch
    batch32.restype, batch32.argtypes = batch.restype, batch.argtypes
    out = []
    for n in orders:
        src = torch.from_numpy(c1_matrix(n)).cuda()
        for k in counts:
            work = [src.clone() for _ in range(k)]
            piv = [torch.zeros(n, dtype=torch.int32, device="cuda") for _ in range(k)]
            ptrs = (C.c_void_p * k)(*[w.data_ptr() for w in work])
            pps = (C.c_void_p * k)(*[p.data_ptr() for p in piv])
            ns = (C.c_longlong * k)(*([n] * k))
            info = (C.c_int * k)()

            def timed(fn, work, src):
                best = None
                for i in range(reps + 1):
                    for w in work:
                        w.copy_(src)
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    if not fn():
                        raise RuntimeError("factor failed: " + nb.last_error())
                    e1.record(stream)
                    torch.cuda.synchronize()
                    if i:
                        t = e0.elapsed_time(e1)
                        best = t if best is None else min(best, t)
                return best
            one = C.c_int(0)
            t_single = timed(lambda: all(single(w.data_ptr(), n, n, p.data_ptr(), 0, 0, C.byref(one))
                                         for w, p in zip(work, piv)), work, src)
            t_batch = timed(lambda: batch(ptrs, ns, ns, pps, k, 0, info), work, src)
            # Split-precision lockstep on FP32 copies (even leading dimension):
            # the factorisation alone, its refinement not included.
            ld32 = n + (n & 1)
            a32 = torch.zeros((n, 2 * ld32), dtype=torch.float32, device="cuda")
            a32.view(torch.complex64)[:, :n] = src.to(torch.complex64)
            work32 = [a32.clone() for _ in range(k)]
            ptrs32 = (C.c_void_p * k)(*[w.data_ptr() for w in work32])
            lds32 = (C.c_longlong * k)(*([ld32] * k))
            t_split = timed(lambda: batch32(ptrs32, ns, lds32, pps, k, 0, info), work32, a32)
            del work32, a32
            flops = k * 8.0 * n ** 3 / 3
            out.append({"order": n, "systems": k, "one_at_a_time_ms": t_single, "lockstep_ms": t_batch,
                        "speedup": t_single / t_batch, "lockstep_tflops": flops / (t_batch * 1e-3) / 1e12,
                        "split_lockstep_factor_ms": t_split,
                        "split_lockstep_tflops": flops / (t_split * 1e-3) / 1e12})
            del work, piv
    return out


def deck_bench():
    """BASELINE config 0 end to end through the drop-in program (nec2c with
    the CUDA backend bound in, nec2c_b200/binding/_build/nec2c_cuda): the
    21-segment dipole beside the 16^3 dielectric cube at 300 MHz, FFT-GMRES to
    -r 1e-6, once with --fft-backend cuda (plain FP64) and once with
    cuda-mixed (FP32 transforms).  Reports the wall time and the program's own
    phase timings, and the mixed form's errors against the FP64 form: feed
    impedance, segment and voxel currents (relative L2) and far-field gain
    (dB, directions within 30 dB of the peak).  Host work: the matrix fill
    and the wire-volume coupling stay on the CPU as in the reference."""
    import tempfile
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import decks
    if not os.path.exists(decks.CUDA_BIN):
        return {"unavailable": "drop-in program not built (make -C oracle binding)"}
    out = {"workload": "c0: 21-segment half-wave dipole 0.1 lambda from a 0.2 lambda cube (16^3 cells, "
                       "eps_r 4 - 0.1j), 300 MHz, -s fft -r 1e-6", "threads": os.cpu_count()}
    d = tempfile.mkdtemp()
    deck = decks.dipole_cube(d)
    docs = {}
    for name in ("cuda", "cuda-mixed"):
        timing = os.path.join(d, name + ".timing.json")
        doc, wall, _ = decks.run(decks.CUDA_BIN, deck, ["-s", "fft", "-r", "1e-6", "--jobs", "1",
                                                        "--fft-backend", name, "--timing-json", timing])
        with open(timing) as f:
            phases = {p["name"]: p["seconds"] for p in json.load(f)["phases"]}
        e = decks.execution(doc)
        z = decks.feed_impedance(doc)
        docs[name] = doc
        out[name] = {"wall_s": wall, "phases_s": phases, "zin_ohm": [z.real, z.imag],
                     "iterations": e["solver"]["iterations"], "true_residual": e["solver"]["true_residual"]}
    a, b = docs["cuda-mixed"], docs["cuda"]
    za, zb = decks.feed_impedance(a), decks.feed_impedance(b)
    wa, wb = decks.wire_currents(a), decks.wire_currents(b)
    va, vb = decks.volume_currents(a), decks.volume_currents(b)
    out["mixed_vs_fp64"] = {"zin_rel_err": abs(za - zb) / abs(zb),
                            "wire_current_rel_l2": float(np.linalg.norm(wa - wb) / np.linalg.norm(wb)),
                            "voxel_current_rel_l2": float(np.linalg.norm(va - vb) / np.linalg.norm(vb)),
                            "gain_db_max_abs": decks.gain_difference_db(a, b)}
    return out


class WireModel(C.Structure):
    """nec2c_cuda_wire_model (include/nec2c_cuda.h)."""
    _fields_ = [("segments", C.c_size_t), ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("length", C.c_void_p), ("radius", C.c_void_p), ("cab", C.c_void_p), ("sab", C.c_void_p),
                ("salp", C.c_void_p), ("wavelength", C.c_double), ("rkh", C.c_double), ("pec_ground", C.c_int)]


def coupling_bench(nb, reps):
    """The two wire-volume coupling blocks of the dipole-plus-cube model
    (21 segments, 16^3 cells, 21 conductor unknowns whose
    basis spreads over three segments each, seeded coefficients) through the
    C ABI, reps times after one untimed call; host wall time per call
    (uploads, kernels, download)."""
    lam = C0 / 300e6
    n = 21
    seg = np.zeros((n, 8))
    for i in range(n):
        seg[i] = [0.0, 0.0, -0.25 + (i + 0.5) * 0.5 / n, 0.5 / n, 0.001 / lam, 0.0, 0.0, 1.0]
    h = 0.2 * lam / 16
    g = (np.arange(16) + 0.5) * h
    X, Y, Z = np.meshgrid(0.1 * lam + g, -0.1 * lam + g, -0.1 * lam + g, indexing="ij")
    centers = np.ascontiguousarray(np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1))
    sizes = np.full_like(centers, h)
    cells = len(centers)
    rng = np.random.default_rng(1)
    src = np.zeros((n, n, 3), dtype=np.complex128)
    for j in range(n):
        for s in range(max(0, j - 1), min(n, j + 2)):
            src[j, s] = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    chi = np.full(cells, 3.0 - 0.1j)
    lib = nb.load()
    vp = C.c_void_p
    lib.nec2c_cuda_coupling_wire_to_volume.argtypes = [vp, C.c_size_t, vp, C.c_size_t, vp, vp, vp, C.c_double, vp]
    lib.nec2c_cuda_coupling_volume_to_wire.argtypes = [C.c_size_t, vp, vp, C.c_size_t, vp, vp, C.c_double,
                                                       C.c_double, C.c_int, vp]
    cols = [np.ascontiguousarray(seg[:, k]) for k in range(8)]
    w = WireModel(n, *[c.ctypes.data for c in cols], lam, 1.0, 0)
    w2v = np.zeros((n, 3 * cells), dtype=np.complex128)
    v2w = np.zeros((n, 3 * cells), dtype=np.complex128)
    obs = np.ascontiguousarray(seg[:, :3] * lam)
    tan = np.ascontiguousarray(seg[:, 5:8])
    k0, om = 2 * math.pi / lam, 2 * math.pi * 300e6
    t_w2v, t_v2w = [], []
    for rep in range(reps + 1):
        t0 = time.perf_counter()
        if not lib.nec2c_cuda_coupling_wire_to_volume(C.byref(w), n, src.ctypes.data, cells, centers.ctypes.data,
                                                      sizes.ctypes.data, chi.ctypes.data, om, w2v.ctypes.data):
            raise RuntimeError(nb.last_error())
        t1 = time.perf_counter()
        if not lib.nec2c_cuda_coupling_volume_to_wire(n, obs.ctypes.data, tan.ctypes.data, cells,
                                                      centers.ctypes.data, sizes.ctypes.data, k0, om, 0,
                                                      v2w.ctypes.data):
            raise RuntimeError(nb.last_error())
        t2 = time.perf_counter()
        if rep:
            t_w2v.append(t1 - t0)
            t_v2w.append(t2 - t1)
    return {"segments": n, "cells": cells, "unknowns": n, "wire_to_volume_ms": 1e3 * statistics.median(t_w2v),
            "volume_to_wire_ms": 1e3 * statistics.median(t_v2w)}


def dense_bench(nb, torch, stream):
    """Dense solve of 1984 unknowns (one right-hand side) in the
    FP64 form and the split-precision form (FP32 tensor-core factors + FP64
    refinement), through the classic C ABI with host buffers, plus the device
    factor alone on resident matrices."""
    a = c1_matrix()
    n = a.shape[0]
    xe = np.random.default_rng(11).standard_normal(n) + 1j * np.random.default_rng(12).standard_normal(n)
    b = a @ xe
    lib = nb.load()
    out = {"order": n, "flops": 8 * n ** 3 / 3,
           "note": "factor + solve through the classic C ABI (host buffers); device_factor_ms: "
                   "factorisation of a resident matrix alone"}
    sols = {}
    for form in ("cuda", "cuda-mixed"):
        nb.dense_backend_set(form)
        times = []
        for _ in range(3):
            st = np.asfortranarray(a.T.copy())
            rhs = np.asfortranarray(b.reshape(n, 1).copy())
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ok, piv = nb.factor_classic(st)
            ok = ok and nb.solve_classic_many(st, piv, rhs)
            times.append(time.perf_counter() - t0)
            if not ok:
                raise RuntimeError("dense solve failed: " + nb.last_error())
        sols[form] = rhs[:, 0].copy()
        t = min(times)
        out[form] = {"ms": 1e3 * t, "solves_per_s": 1 / t, "gflops": out["flops"] / t / 1e9,
                     "rel_err_vs_exact": float(np.linalg.norm(rhs[:, 0] - xe) / np.linalg.norm(xe))}
        if form == "cuda-mixed":
            out[form]["refinement_steps"] = int(lib.nec2c_cuda_dense_last_refinement())
    nb.dense_backend_set("cuda")
    lib.nec2c_cuda_dense_release()
    out["cuda-mixed"]["rel_err_vs_fp64_gpu"] = float(
        np.linalg.norm(sols["cuda-mixed"] - sols["cuda"]) / np.linalg.norm(sols["cuda"]))
    # Device factor alone (resident matrices, CUDA events).
    for form in ("cuda", "cuda-mixed"):
        out[form]["device_factor_ms"], out[form]["device_solve_ms"] = device_factor(nb, torch, stream, a, form, 3)
    return out


def batched_bench(nb, torch):
    """Small wire blocks: 128 frequencies of the 21-segment dipole
    plus 64 dipoles of 11-41 segments (seeded), each block factored and solved:
    the ragged batch in one call against one classic factor + solve per block."""
    rng = np.random.default_rng(6)
    sizes = [21] * 128 + [int(v) for v in rng.integers(11, 42, 64)]
    mats = []
    for k, n in enumerate(sizes):
        r = np.random.default_rng(1000 + k)
        a = r.standard_normal((n, n)) + 1j * r.standard_normal((n, n))
        a += np.diag(np.full(n, 0.5 * math.sqrt(n)))
        mats.append((np.asfortranarray(a.T), np.ascontiguousarray(a @ (r.standard_normal(n) + 0j))))

    def batch():
        sy = [(st.copy(order="F"), b.copy()) for st, b in mats]
        t0 = time.perf_counter()
        ok, status, _ = nb.solve_batched(sy)
        t = time.perf_counter() - t0
        if not ok:
            raise RuntimeError("batched solve failed")
        return t, sy

    def one_by_one():
        sy = [(st.copy(order="F"), b.copy().reshape(-1, 1).copy(order="F")) for st, b in mats]
        t0 = time.perf_counter()
        for st, b in sy:
            ok, piv = nb.factor_classic(st)
            if not ok or not nb.solve_classic_many(st, piv, b):
                raise RuntimeError("classic solve failed")
        return time.perf_counter() - t0, sy

    nb.dense_backend_set("cuda")
    batch()
    tb, sb = min((batch() for _ in range(3)), key=lambda r: r[0])
    one_by_one()
    ts, ss = min((one_by_one() for _ in range(2)), key=lambda r: r[0])
    nb.load().nec2c_cuda_dense_release()
    err = max(float(np.linalg.norm(x1 - x2[:, 0]) / np.linalg.norm(x2[:, 0])) for (_, x1), (_, x2) in zip(sb, ss))
    return {"systems": len(sizes), "orders": "128 x 21 + 64 in 11..41",
            "one_launch": {"ms": 1e3 * tb, "solves_per_s": len(sizes) / tb},
            "one_call_each": {"ms": 1e3 * ts, "solves_per_s": len(sizes) / ts},
            "max_rel_diff": err, "note": "host buffers through the C ABI, wall clock"}


def volume_batch_bench(nb, torch, stream):
    """A frequency and geometry sweep in one batch of dipole-plus-cube systems.

    The batch holds 192 systems.  The first 128 are one model at 128
    frequencies uniform in 100-400 MHz: a cube of 16^3 cells, 0.2 lambda at
    300 MHz, eps_r = 4 - 0.1j, beside a 21-segment dipole.  The other 64 are
    seeded cubes of 8^3-32^3 cells (0.2 lambda at 300 MHz, eps_r ~ U[2,8],
    tan d = 0.05), each beside a dipole of 11-41 segments.  Each system is the
    hybrid [C B; D V] operator, driven by a 1 V source at the dipole's centre
    and an x-polarised plane wave on the cube, and solved with GMRES(30) to
    rtol 1e-6.

    - Every plan's far pairs are quadratured on the GPU at its own frequency.
    - The 13 near-pair tensors come from the golden table of the nearest
      lattice, reused at every frequency.  The wire blocks are seeded
      diagonally dominant complex matrices with weak wire-cube couplings.  Both belong to the caller (the
      reference's certified quadrature and its wire/coupling fill), which
      bench.py may not run.
    - Timed: the whole batch in one nec2c_cuda_gmres_batch_device call, in both
      forms (FP32 transforms, and the plain FP64 form), against one device
      GMRES call per system.  CUDA events on the launching stream.
    - Served (FP32 transforms): the sweep submitted to an 8-worker request
      server from host buffers, one request per system against batch
      requests; the makespan is read from the requests' own clocks."""
    tabs = near_tables_all()
    lam = C0 / 300e6
    rng = np.random.default_rng(7)
    specs = [(16, 2 * math.pi * f / C0, "c0", 4 - 0.1j, 21) for f in np.linspace(100e6, 400e6, 128)]
    for n in rng.choice([8, 12, 16, 24, 32], 64):
        specs.append((int(n), 2 * math.pi / lam, "c0" if n <= 16 else "c3_32", rng.uniform(2, 8) * (1 - 0.05j),
                      int(rng.integers(11, 42))))
    lib = nb.load()

    blocks = []
    for q, (n, k, tab, eps, c) in enumerate(specs):
        v = 3 * n ** 3
        r = np.random.default_rng(5000 + q)
        cm = r.standard_normal((c, c)) + 1j * r.standard_normal((c, c))
        cm += np.diag(np.full(c, 2.0 * math.sqrt(c)))
        bm = 0.01 * (r.standard_normal((c, v)) + 1j * r.standard_normal((c, v)))
        dm = 0.01 * (r.standard_normal((v, c)) + 1j * r.standard_normal((v, c)))
        blocks.append(np.concatenate([np.concatenate([cm, bm], axis=1).reshape(-1), dm.reshape(-1)]))

    def build(mixed):
        systems, rhs, keep = [], [], []
        for q, (n, k, tab, eps, c) in enumerate(specs):
            h = 0.2 * lam / n
            g = np.arange(n)
            xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1).astype(np.uintp)
            p = nb.VolumePlan((n, n, n), xyz, h, k, eps, tabs[tab][2], mixed=mixed)
            v = 3 * n ** 3
            hs = nb.HybridSystem(p, c, v)
            hs.set_blocks(blocks[q])
            b = np.zeros(c + v, dtype=np.complex128)
            b[c // 2] = 1.0
            z = xyz[2::3].astype(np.float64)
            b[c::3] = 2 * np.exp(-1j * k * h * (z + 0.5)) * math.sin(k * h / 2) / (k * h / 2)
            systems.append(hs)
            rhs.append(b)
            keep.append(p)
        return systems, rhs, keep

    t0 = time.perf_counter()
    sys_m, rhs, keep_m = build(True)
    build_s = time.perf_counter() - t0
    sys_d, _, keep_d = build(False)
    opts = nb.GmresOptions(30, 3000, 1e-6, 0.0)
    out = {"systems": len(specs),
           "model": "dipole (11-41 segments) beside a cube: 128 x 16^3 (100-400 MHz) + 64 random in "
                    "{8,12,16,24,32}^3",
           "unknowns": int(sum(s.n for s in sys_m)), "plan_build_s_fp32": build_s}

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    def served(systems, rhs, slots=8):
        """The same sweep through the request server from host buffers:
        one request per system, against batch requests of 24 systems (eight
        requests that the workers run side by side) and of all 192.  Each
        layout runs twice; the faster makespan (first queued to last
        finished, host copies included) is kept."""
        res = {"slots": slots}
        srv = nb.Server(slots=slots)
        for name, per in (("one_request_per_system", 1), ("batch_requests_of_24", 24),
                          ("one_batch_request", len(systems))):
            groups = [list(range(i, min(i + per, len(systems)))) for i in range(0, len(systems), per)]
            batches = [] if per == 1 else [nb.VolumeBatch(hybrids=[systems[q] for q in g]) for g in groups]
            bvecs = [np.concatenate([rhs[q] for q in g]) for g in groups]
            best = None
            for _ in range(2):
                xs = [np.zeros_like(b) for b in bvecs]
                if per == 1:
                    reqs = [srv.volume(systems[g[0]], b, x, restart=30, maxit=3000, rtol=1e-6)
                            for g, b, x in zip(groups, bvecs, xs)]
                else:
                    reqs = [srv.batch(bt, b, x, restart=30, maxit=3000, rtol=1e-6)
                            for bt, b, x in zip(batches, bvecs, xs)]
                srv.drain()
                for r in reqs:
                    if not r.status or r.report.status != 0:
                        raise RuntimeError("served sweep failed: %s (status %d)" % (r.error.decode(),
                                                                                   r.report.status))
                ms = 1e3 * (max(r.finished_s for r in reqs) - min(r.queued_s for r in reqs))
                best = ms if best is None else min(best, ms)
            res[name] = {"requests": len(groups), "makespan_ms": best,
                         "solves_per_s": 1e3 * len(systems) / best}
            for bt in batches:
                bt.close()
        srv.close()
        return res

    sols = {}
    for form, systems, keep in (("fp32_transforms", sys_m, keep_m), ("fp64", sys_d, keep_d)):
        batch = nb.VolumeBatch(hybrids=systems)
        b_dev = torch.from_numpy(np.concatenate(rhs)).cuda()
        x_dev = torch.zeros_like(b_dev)
        reps = (nb.GmresReport * len(systems))()

        def solve_batch():
            x_dev.zero_()
            return lib.nec2c_cuda_gmres_batch_device(batch.h, C.c_void_p(b_dev.data_ptr()),
                                                     C.c_void_p(x_dev.data_ptr()), C.byref(opts), reps)
        # The first (untimed) solve of the FP32-transform batch sits in an NVTX
        # range "batch_solve" for launch lists:
        #   ncu --nvtx --nvtx-include "batch_solve]" ... --only volume_batch
        if form == "fp32_transforms":
            torch.cuda.nvtx.range_push("batch_solve")
        timed(solve_batch)
        if form == "fp32_transforms":
            torch.cuda.nvtx.range_pop()
        ms, ok = min((timed(solve_batch) for _ in range(2)), key=lambda t: t[0])
        if not ok:
            raise RuntimeError("batched solve failed: %s %s" % (
                nb.last_error(), sorted(set((r.status, r.iterations) for r in reps))[:8]))
        sols[form] = x_dev.cpu().numpy()
        its = [r.iterations for r in reps]
        schedule = batch.schedule()
        batch.close()
        bs = [torch.from_numpy(b).cuda() for b in rhs]
        x = torch.zeros(max(b.numel() for b in bs), dtype=torch.complex128, device="cuda")

        def one_by_one():
            ok = 1
            for s, b in zip(systems, bs):
                x.zero_()
                ok &= lib.nec2c_cuda_gmres_hybrid_device(s.h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                                                         C.byref(opts), C.byref(nb.GmresReport()))
            return ok
        timed(one_by_one)
        ms1, ok1 = timed(one_by_one)
        if not ok1:
            raise RuntimeError("per-system solve failed: " + nb.last_error())
        if form == "fp32_transforms":
            out["served"] = served(systems, rhs)
        out[form] = {"one_batch": {"ms": ms, "solves_per_s": 1e3 * len(systems) / ms},
                     "one_call_per_system": {"ms": ms1, "solves_per_s": 1e3 * len(systems) / ms1},
                     "iterations": {"min": int(min(its)), "max": int(max(its)), "mean": float(np.mean(its))},
                     "batch_schedule": {"passes": ["z fwd", "y fwd", "x product", "y inv", "z inv"],
                                        "tile_scale_and_radix_variant": schedule}}
        for s in systems:
            s.close()
        for p in keep:
            p.close()
    off = np.cumsum([0] + [b.size for b in rhs])
    out["max_rel_err_fp32_transforms_vs_fp64"] = max(
        float(np.linalg.norm(sols["fp32_transforms"][a:b] - sols["fp64"][a:b]) / np.linalg.norm(sols["fp64"][a:b]))
        for a, b in zip(off[:-1], off[1:]))
    out["batch_fp32_vs_plain_fp64_one_call_per_system"] = (
        out["fp32_transforms"]["one_batch"]["solves_per_s"] / out["fp64"]["one_call_per_system"]["solves_per_s"])
    return out


# Serving stream (bounded): 60% wire-only dense MoM solves of
# 200-3000 unknowns (log-uniform), 40% volume solves on resident plans of two
# lattices (0.2-lambda cubes voxelised 16^3 and 32^3 at 300 MHz, eps_r~U[2,10],
# tand 0.05) with GMRES(30) to rtol 1e-6, two resident replicas per lattice.
# One solve per request (one frequency).  Request matrices and right-hand sides
# are page-locked host buffers, as a serving front end keeps them.
SERVE_REQUESTS = 96
SERVE_SLOTS = 8


def serving_bench(nb, torch):
    rng = np.random.default_rng(4)
    table_all = near_tables_all()
    sizes = sorted(set(int(round(math.exp(v))) for v in rng.uniform(math.log(200), math.log(3000), 10)))
    def pinned(arr):
        """A page-locked copy of arr (same layout): a serving front end keeps
        its request buffers pinned, so uploads run at DMA speed."""
        t = torch.empty(arr.size, dtype=torch.complex128, pin_memory=True)
        v = t.numpy()
        out = np.lib.stride_tricks.as_strided(v, shape=arr.shape,
                                               strides=arr.strides if arr.flags.f_contiguous or arr.flags.c_contiguous
                                               else None)
        out[...] = arr
        return out, t

    keep = []
    pool = []
    for i, n in enumerate(sizes):
        r = np.random.default_rng(100 + i)
        a = r.standard_normal((n, n)) + 1j * r.standard_normal((n, n))
        a += np.diag(np.full(n, 0.5 * math.sqrt(n)))
        st, t1 = pinned(np.asfortranarray(a.T))
        x = r.standard_normal(n) + 1j * r.standard_normal(n)
        rhs, t2 = pinned(np.asfortranarray((a @ x).reshape(n, 1)))
        keep += [t1, t2]
        pool.append((st, rhs))
    lam = C0 / 300e6
    geoms = []
    for name, nside in (("c0", 16), ("c3_32", 32)):
        h, k, table = table_all[name]
        g = np.arange(nside)
        xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1).astype(np.uintp)
        cells = nside ** 3
        r = np.random.default_rng(200 + nside)
        eps = r.uniform(2.0, 10.0, cells) * (1 - 0.05j)
        bvec = np.zeros(3 * cells, dtype=np.complex128)
        z = xyz[2::3].astype(np.float64)
        bvec[0::3] = 2 * np.exp(-1j * k * h * (z + 0.5)) * math.sin(k * h / 2) / (k * h / 2)
        geoms.append(((nside,) * 3, xyz, h, k, eps, table, bvec))
    kinds = rng.random(SERVE_REQUESTS) < 0.6
    picks = rng.integers(0, 1 << 30, SERVE_REQUESTS)

    def plans(mixed):
        out = []
        for shape, xyz, h, k, eps, table, bvec in geoms:
            for _ in range(2):   # two resident replicas per lattice
                p = nb.VolumePlan(shape, xyz, h, k, eps[0], table, mixed=mixed)
                for c, e in enumerate(eps):
                    p.set_permittivity(c, e)
                out.append((p, bvec))
        return out

    def run(split, gaps, slots=SERVE_SLOTS, fp32_plans=None):
        ps = plans(split if fp32_plans is None else fp32_plans)
        srv = nb.Server(slots=slots, split=split)
        # warm-up: one request of each kind per plan / a mid-size matrix
        # Warm-up: every plan once, and enough concurrent dense requests that
        # every worker thread has set up its stream state before timing.
        warm = [srv.volume(p, b, np.zeros_like(b), rtol=1e-6, maxit=2000) for p, b in ps]
        for _ in range(2 * slots):
            st, rhs = pool[len(pool) // 2]
            warm.append(srv.dense(st, rhs.copy(order="F")))
        srv.drain()
        reqs, outs = [], []
        # Page-locked result buffers of the dense requests, allocated before
        # the stream starts (a front end recycles them).
        bufs = {i: pinned(pool[picks[i] % len(pool)][1]) for i in range(SERVE_REQUESTS) if kinds[i]}
        t0 = time.perf_counter()
        for i in range(SERVE_REQUESTS):
            if gaps is not None:
                target = t0 + gaps[i]
                while time.perf_counter() < target:
                    time.sleep(min(1e-3, max(0.0, target - time.perf_counter())))
            if kinds[i]:
                st, rhs = pool[picks[i] % len(pool)]
                o = bufs[i][0]
                o[...] = rhs
                reqs.append(srv.dense(st, o))
            else:
                p, b = ps[picks[i] % len(ps)]
                o = np.zeros_like(b)
                reqs.append(srv.volume(p, b, o, rtol=1e-6, maxit=2000))
            outs.append(o)
        srv.drain()
        for r in reqs:
            if not r.status:
                raise RuntimeError("serving request failed: " + r.error.decode())
        first = min(r.queued_s for r in reqs)
        last = max(r.finished_s for r in reqs)
        lat = sorted(1e3 * (r.finished_s - r.queued_s) for r in reqs)
        res = {"solves_per_s": len(reqs) / (last - first),
               "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
               "makespan_s": last - first}
        for kind, name in ((nb.REQUEST_DENSE, "dense"), (nb.REQUEST_VOLUME, "volume")):
            svc = [1e3 * (r.finished_s - r.started_s) for r in reqs if r.kind == kind]
            res[name + "_service_ms_mean"] = sum(svc) / max(1, len(svc))
        srv.close()
        for p, _ in ps:
            p.close()
        return res, outs

    lib = nb.load()
    l0 = lib.nec2c_cuda_launch_count()
    out = {"requests": SERVE_REQUESTS, "dense": int(kinds.sum()), "volume": int((~kinds).sum()),
           "slots": SERVE_SLOTS, "dense_orders": sizes,
           "lattices": ["16^3 (12288 unknowns)", "32^3 (98304 unknowns)"]}
    sat = {}
    for split in (False, True):
        sat[split], outs = run(split, None)
        again, _ = run(split, None)
        if again["solves_per_s"] > sat[split]["solves_per_s"]:
            sat[split] = again
        if split:
            outs_m = outs
        else:
            outs_d = outs
    err = max(float(np.linalg.norm(m - d) / np.linalg.norm(d)) for m, d in zip(outs_m, outs_d))
    out["saturation"] = {"fp64": sat[False], "mixed": sat[True]}
    # FP32 volume plans with the FP64 LU for the dense requests: at these
    # orders the LU is panel-bound in both forms and the split form's
    # refinement only adds latency.
    out["saturation"]["fp32_volume_fp64_lu"] = max((run(False, None, fp32_plans=True)[0] for _ in range(2)),
                                                    key=lambda r: r["solves_per_s"])
    # The plain FP64 GPU form: one request at a time, FP64 plans and LU.
    plain, _ = run(False, None, slots=1)
    out["plain_fp64_one_at_a_time"] = plain
    out["mixed_serving_vs_plain_fp64"] = sat[True]["solves_per_s"] / plain["solves_per_s"]
    out["fp32_volume_fp64_lu_serving_vs_plain_fp64"] = (out["saturation"]["fp32_volume_fp64_lu"]["solves_per_s"] /
                                                         plain["solves_per_s"])
    rate = 0.7 * sat[True]["solves_per_s"]
    gaps = np.cumsum(np.random.default_rng(5).exponential(1.0 / rate, SERVE_REQUESTS))
    pois = {}
    for split in (False, True):
        pois[split], _ = run(split, gaps)
    out["poisson"] = {"rate_per_s": rate, "fp64": pois[False], "mixed": pois[True]}
    out["mixed_vs_fp64_solves_per_s"] = sat[True]["solves_per_s"] / sat[False]["solves_per_s"]
    out["max_rel_err_mixed_vs_fp64"] = err
    out["gpu_launches"] = int(lib.nec2c_cuda_launch_count() - l0)
    return out


# Most dense requests of one size class in one lockstep batch.
DENSE_MERGE = 16


def serving_stream_c4(nb, torch, requests=400, sizes_per_model=16, rates=(0.3, 0.5, 0.7, 0.9, 1.1),
                      lattices=(8, 16, 24, 32, 48), seed=11, arms=None, plain_requests=None):
    """BASELINE config 4 shaped stream through the request server.

    Requests: 60% dense MoM models (orders log-uniform in 200-3000, ten orders
    with three seeded matrices each standing for their frequencies), 40%
    dipole-plus-dielectric VIE models over a perfectly conducting ground plane
    (PEC image embedding): cubes of 8^3-48^3 cells (0.2 lambda at 300 MHz,
    eps_r ~ U[2,10], tan d 0.05) raised one cell above the plane, each beside a
    dipole of 11-41 segments, every model resident on the device at 16
    frequencies (280-355 MHz).  Each request asks for F in {1, 2, 4, 8, 16}
    distinct frequencies of its model and is submitted as F solve requests
    (one per frequency); its latency runs from the first being queued to the
    last being done.

    Forms (16 workers): `mixed` = FP32 transforms and the split-precision LU,
    the server merging queued volume requests on one model's frequencies into
    one batched solve (each model's 16 frequency systems are one registered
    batch) and queued dense requests of one size class into one lockstep
    factorisation (at most DENSE_MERGE) of FP32 copies on the tensor cores,
    refined in FP64; `mixed_unmerged` = the same without merging;
    `mixed_fp64_lu` = merged, FP32 transforms with the FP64 LU; `fp64` = FP64
    transforms and LU, merged; `plain_fp64_one_at_a_time` = FP64, one worker, no merging.  Saturation:
    everything queued at once.  Poisson: request arrivals at the given
    fractions of the mixed form's saturated request rate (the sweep shows
    where p99 latency diverges).  Seeded synthetic matrices, lattices and
    wire blocks stand in for the reference's decks; the near-pair tensors
    come from the golden table whose cell size is nearest."""
    rng = np.random.default_rng(seed)
    tabs = near_tables_all()
    lam = C0 / 300e6
    slots = 16

    def pinned(arr):
        t = torch.empty(arr.size, dtype=torch.complex128, pin_memory=True)
        out = np.lib.stride_tricks.as_strided(t.numpy(), shape=arr.shape, strides=arr.strides)
        out[...] = arr
        return out, t

    keep = []
    orders = sorted(set(int(round(math.exp(v))) for v in rng.uniform(math.log(200), math.log(3000), 10)))
    dense_pool = []
    for i, n in enumerate(orders):
        mats = []
        for f in range(3):
            r = np.random.default_rng(300 + 7 * i + f)
            a = r.standard_normal((n, n)) + 1j * r.standard_normal((n, n))
            a += np.diag(np.full(n, 0.5 * math.sqrt(n)))
            st, t1 = pinned(np.asfortranarray(a.T))
            x = r.standard_normal(n) + 1j * r.standard_normal(n)
            rhs, t2 = pinned(np.asfortranarray((a @ x).reshape(n, 1)))
            keep += [t1, t2]
            mats.append((st, rhs))
        dense_pool.append(mats)

    freqs = np.linspace(280e6, 355e6, sizes_per_model)
    specs = []
    for m, n in enumerate(lattices):
        r = np.random.default_rng(400 + m)
        h = 0.2 * lam / n
        tab = min(("c0", "c2", "c3_32"), key=lambda t: abs(tabs[t][0] - h))
        specs.append(dict(n=int(n), c=int(r.integers(11, 42)), eps=r.uniform(2, 10) * (1 - 0.05j),
                          tab=tab, seed=500 + m))

    def build_models(mixed):
        models = []
        for sp in specs:
            n, c = sp["n"], sp["c"]
            h = 0.2 * lam / n
            g = np.arange(n)
            xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
            # PEC image embedding: physical cells one cell (two half cells)
            # above the plane, their images below; lattice index as
            # dielectric_fft.c:137-154 lays it out (gap of 2 half cells).
            phys = xyz.copy()
            phys[:, 2] += n + 2
            img = xyz.copy()
            img[:, 2] = n - 1 - xyz[:, 2]
            lat = np.concatenate([phys, img]).astype(np.uintp).reshape(-1)
            shape = (n, n, 2 * n + 2)
            v = 3 * n ** 3
            r = np.random.default_rng(sp["seed"])
            cm = r.standard_normal((c, c)) + 1j * r.standard_normal((c, c))
            cm += np.diag(np.full(c, 2.0 * math.sqrt(c)))
            bm = 0.01 * (r.standard_normal((c, v)) + 1j * r.standard_normal((c, v)))
            dm = 0.01 * (r.standard_normal((v, c)) + 1j * r.standard_normal((v, c)))
            blocks = np.concatenate([np.concatenate([cm, bm], axis=1).reshape(-1), dm.reshape(-1)])
            systems, plans, rhs = [], [], []
            for f in freqs:
                k = 2 * math.pi * f / C0
                p = nb.VolumePlan(shape, lat, h, k, sp["eps"], tabs[sp["tab"]][2], mixed=mixed)
                hs = nb.HybridSystem(p, c, v, pec=True)
                hs.set_blocks(blocks)
                b = np.zeros(c + v, dtype=np.complex128)
                b[c // 2] = 1.0
                z = xyz[:, 2].astype(np.float64)
                b[c::3] = 2 * np.exp(-1j * k * h * (z + 0.5)) * math.sin(k * h / 2) / (k * h / 2)
                plans.append(p)
                systems.append(hs)
                rhs.append(b)
            # Every frequency of the model in one batch, registered with the
            # server: queued requests on its systems merge into one solve.
            models.append(dict(plans=plans, systems=systems, rhs=rhs,
                               batch=nb.VolumeBatch(hybrids=systems)))
        return models

    nreq = requests
    kinds = rng.random(nreq) < 0.6
    fsel = rng.choice([1, 2, 4, 8, 16], nreq)
    picks = rng.integers(0, 1 << 30, nreq)
    # The frequencies each request asks for: F distinct ones of its model's 16.
    fsets = [np.sort(rng.choice(len(freqs), int(F), replace=False)) for F in fsel]

    def run(models, split, slots_, gaps, merge, only=None, limit=None):
        srv = nb.Server(slots=slots_, split=split)
        if merge:
            for mdl in models:
                srv.merge(mdl["batch"])
            # Queued dense requests of one size class factor in lockstep (on a
            # split-precision server: FP32 tensor-core factors, FP64 refinement).
            srv.merge_dense(DENSE_MERGE)
        # Warm every worker (stream state, kernel attributes) and every system.
        for mdl in models:
            for hs, b in zip(mdl["systems"], mdl["rhs"]):
                srv.volume(hs, b, np.zeros_like(b), rtol=1e-6, maxit=3000)
        for _ in range(2 * slots_):
            st, rhs = dense_pool[len(dense_pool) // 2][0]
            srv.dense(st, rhs.copy(order="F"))
        srv.drain()
        groups = []
        sols = {}   # a solution per (kind, model, frequency), for the error between forms
        t0 = time.perf_counter()
        for i in range(nreq):
            if gaps is not None:
                target = t0 + gaps[i]
                while time.perf_counter() < target:
                    time.sleep(min(1e-3, max(0.0, target - time.perf_counter())))
            subs = []
            if (only is not None and bool(kinds[i]) != only) or (limit is not None and i >= limit):
                continue
            if kinds[i]:
                pi = picks[i] % len(dense_pool)
                mats = dense_pool[pi]
                for f in fsets[i]:
                    st, rhs = mats[f % len(mats)]
                    out = rhs.copy(order="F")
                    subs.append(srv.dense(st, out))
                    sols[("dense", pi, int(f) % len(mats))] = out
            else:
                mi = picks[i] % len(models)
                mdl = models[mi]
                for f in fsets[i]:
                    b = mdl["rhs"][f]
                    x = np.zeros_like(b)
                    subs.append(srv.volume(mdl["systems"][f], b, x, rtol=1e-6, maxit=3000))
                    sols[("volume", mi, int(f))] = x
            groups.append((kinds[i], subs, i))
        srv.drain()
        lat, merged, dmerged = [], [], []
        service = {"dense_s": 0.0, "volume_s": 0.0}
        per_size = {}
        for dense_req, subs, i in groups:
            size = ("order %d" % orders[picks[i] % len(dense_pool)] if dense_req
                    else "%d^3" % specs[picks[i] % len(models)]["n"])
            for r in subs:
                if not r.status or (r.kind != nb.REQUEST_DENSE and r.report.status != 0):
                    raise RuntimeError("c4 stream request failed: %s (status %d)" % (r.error.decode(),
                                                                                    r.report.status))
                (dmerged if dense_req else merged).append(r.merged)
                # Worker time per kind (merged requests share one run: counted once).
                if r.merged <= 1 or r.footprint:
                    service["dense_s" if dense_req else "volume_s"] += r.finished_s - r.started_s
                    per_size[size] = per_size.get(size, 0.0) + r.finished_s - r.started_s
            lat.append(1e3 * (max(r.finished_s for r in subs) - min(r.queued_s for r in subs)))
        first = min(r.queued_s for _, subs, _ in groups for r in subs)
        last = max(r.finished_s for _, subs, _ in groups for r in subs)
        solves = int(sum(len(subs) for _, subs, _ in groups))
        srv.close()
        lat.sort()
        service["per_size_s"] = per_size
        return {"requests": len(groups), "solves": solves, "solves_per_s": solves / (last - first),
                "requests_per_s": len(groups) / (last - first), "makespan_s": last - first,
                "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                "volume_solves_merged_mean": float(np.mean(merged)) if merged else None,
                "dense_solves_merged_mean": float(np.mean(dmerged)) if dmerged else None,
                "worker_time": service}, sols

    t0 = time.perf_counter()
    m32 = build_models(True)
    m64 = build_models(False)
    out = {"requests": nreq, "dense_fraction": float(kinds.mean()), "frequencies_per_request": [1, 2, 4, 8, 16],
           "mean_frequencies": float(fsel.mean()), "dense_orders": orders,
           "vie_lattices_over_pec_ground": ["%d^3" % n for n in lattices], "frequencies_per_model": len(freqs),
           "slots": slots, "setup_s": time.perf_counter() - t0,
           "device_gb_in_use_after_setup": (lambda f: (f[1] - f[0]) / 1e9)(torch.cuda.mem_get_info())}
    sat = {}
    if arms is not None:
        # A long stream: the mixed form at saturation and under Poisson
        # arrivals, and (arms holding "plain") the plain FP64 form on the
        # first plain_requests requests; its throughput per solve does not
        # depend on the stream's length.
        sat["mixed"], _ = run(m32, True, slots, None, True)
        out["saturation"] = sat
        if "plain" in arms:
            pl, _ = run(m64, False, 1, None, False, None, plain_requests)
            pl["first_requests"] = plain_requests
            out["plain_fp64_one_at_a_time"] = pl
            out["mixed_vs_plain_fp64"] = sat["mixed"]["solves_per_s"] / pl["solves_per_s"]
    else:
        runs = [run(m32, True, slots, None, True) for _ in range(2)]
        sat["mixed"], sols_mixed = max(runs, key=lambda r: r[0]["solves_per_s"])
        sat["mixed_unmerged"], _ = run(m32, True, slots, None, False)
        sat["mixed_fp64_lu"], sols_fp64lu = run(m32, False, slots, None, True)
        runs = [run(m64, False, slots, None, True) for _ in range(2)]
        sat["fp64"], sols_fp64 = max(runs, key=lambda r: r[0]["solves_per_s"])
        plain, sols_plain = run(m64, False, 1, None, False)

        def rel_err(a, b):
            return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))

        def worst(sols, ref, kind):
            errs = [rel_err(v, ref[k]) for k, v in sols.items() if k[0] == kind and k in ref]
            return max(errs) if errs else None
        # Current error of each form against the plain FP64 form on the same
        # systems (volume: GMRES to rtol 1e-6 in both, so the difference is
        # the solver's tolerance as much as the precision).
        out["error_vs_plain_fp64"] = {
            "mixed": {"volume_current": worst(sols_mixed, sols_plain, "volume"),
                      "dense_current": worst(sols_mixed, sols_plain, "dense")},
            "mixed_fp64_lu": {"volume_current": worst(sols_fp64lu, sols_plain, "volume"),
                              "dense_current": worst(sols_fp64lu, sols_plain, "dense")},
            "fp64_merged": {"volume_current": worst(sols_fp64, sols_plain, "volume"),
                            "dense_current": worst(sols_fp64, sols_plain, "dense")}}
        out["saturation"] = sat
        out["plain_fp64_one_at_a_time"] = plain
        # Each kind of request alone (the same requests), both forms: where
        # the mixed stream's time goes; volume requests also unmerged.
        out["by_kind"] = {}
        for name, only in (("dense", True), ("volume", False)):
            mx, _ = run(m32, True, slots, None, True, only)
            pl, _ = run(m64, False, 1, None, False, only)
            out["by_kind"][name] = {"mixed": mx, "plain_fp64_one_at_a_time": pl,
                                    "mixed_vs_plain_fp64": mx["solves_per_s"] / pl["solves_per_s"]}
            if not only:
                out["by_kind"][name]["mixed_unmerged"], _ = run(m32, True, slots, None, False, only)
        out["mixed_vs_plain_fp64"] = sat["mixed"]["solves_per_s"] / plain["solves_per_s"]
        out["mixed_fp64_lu_vs_plain_fp64"] = sat["mixed_fp64_lu"]["solves_per_s"] / plain["solves_per_s"]
        out["fp64_batched_vs_plain_fp64"] = sat["fp64"]["solves_per_s"] / plain["solves_per_s"]
    sweep = []
    for frac in rates:
        rate = frac * sat["mixed"]["requests_per_s"]
        gaps = np.cumsum(np.random.default_rng(13).exponential(1.0 / rate, nreq))
        res, _ = run(m32, True, slots, gaps, True)
        res["offered_requests_per_s"] = rate
        res["fraction_of_saturation"] = frac
        sweep.append(res)
    out["poisson_mixed"] = sweep
    for ms in (m32, m64):
        for mdl in ms:
            mdl["batch"].close()
            for hs in mdl["systems"]:
                hs.close()
            for p in mdl["plans"]:
                p.close()
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            return run_reference(args, rank, world)
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
