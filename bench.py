#!/usr/bin/env python
"""Benchmark of the unstaggered generalized-momentum PIC step on one plasma.

Workload (the 512x512 Weibel configuration): 2D periodic grid 512x512 over
[0, 2pi/0.3)^2, 256 electrons per cell (67,108,864 particles) at uniform
random positions with a bi-Maxwellian in normalized momentum (thermal spread
0.02c in x, 0.2c in y), fixed uniform ion background n0 = 1, quadratic
B-spline, dt = 0.05, FP64 throughout.  A step is one pass of the hot path
over all particles.

The headline line times the explicit spectral BDF1/IAEM step (continuity-
consistent charge update, diagnostics -- energy history, gauge / Gauss /
continuity residuals -- every step as the reference's run loop does).  Its
"implicit" object times the implicit energy-conserving orbit-averaged
GM-HC-CN step (Anderson outer iteration on the mesh current to 1e-11, local
particle fixed points to 1e-12, knot-split orbits, Nyquist projection: the
reference's manuscript deck in 2D) on the same plasma.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  value = whole-job particle-steps/s with inputs resident
in HBM; e2e = the same metric through the public API from pinned host
buffers (upload, start-up fields, K steps with a diagnostics row read back
each step, particle state read back); roofline = the dominant kernel against
the measured HBM copy bandwidth; cpu_baseline = the reference's own CPU code
(oracle/_ref, compiled from the reference sources) on a bounded sample of the
same workload.  N > 1 runs N independent replicas (the method runs on one
GPU; it has no cross-GPU exchange).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
WORKLOADS = {
    "weibel512": dict(nx=512, ny=512, ppc=256, L=2 * np.pi / 0.3, dt=0.05, method="bdf1",
                      charge_update="conserving", uth=(0.02, 0.2, 0.0), seed=2026),
    "weibel64": dict(nx=64, ny=64, ppc=64, L=2 * np.pi / 0.3, dt=0.05, method="bdf1",
                     charge_update="conserving", uth=(0.02, 0.2, 0.0), seed=2026),
    # profiling case: same grid and physics, 16 e-/cell (370 MB of particle state)
    "weibel512_ppc16": dict(nx=512, ny=512, ppc=16, L=2 * np.pi / 0.3, dt=0.05, method="bdf1",
                            charge_update="conserving", uth=(0.02, 0.2, 0.0), seed=2026),
    # profiling case with the bench workload's cell occupancy pattern (several
    # warps per cell): 256x256 grid, 64 e-/cell (4,194,304 particles, 370 MB)
    "weibel256_ppc64": dict(nx=256, ny=256, ppc=64, L=2 * np.pi / 0.3, dt=0.05, method="bdf1",
                            charge_update="conserving", uth=(0.02, 0.2, 0.0), seed=2026),
    # the same Weibel decks advanced by the implicit orbit-averaged GM-HC-CN step
    "weibel512_implicit": dict(nx=512, ny=512, ppc=256, L=2 * np.pi / 0.3, dt=0.05, method="cn_orbit",
                               charge_update="-", uth=(0.02, 0.2, 0.0), seed=2026),
    "weibel64_implicit": dict(nx=64, ny=64, ppc=64, L=2 * np.pi / 0.3, dt=0.05, method="cn_orbit",
                              charge_update="-", uth=(0.02, 0.2, 0.0), seed=2026),
    "weibel512_ppc16_implicit": dict(nx=512, ny=512, ppc=16, L=2 * np.pi / 0.3, dt=0.05,
                                     method="cn_orbit", charge_update="-", uth=(0.02, 0.2, 0.0),
                                     seed=2026),
}
# Solver settings of the implicit workloads: the reference's manuscript deck
# (Project3/inputs/manuscript/weibel_main_dt02_T100.txt) in 2D (nz = 1, Lz = 1).
IMPLICIT_DECK = dict(Lz=1.0, kappa=1.0, sigma1=1.0, sigma2=1.0, n0=1.0, spline_order=2,
                     orbit_quad_order=8, split_orbit_at_knots=True, nyquist_projection=True,
                     nonlinear_solver="anderson_quasi_newton", nonlinear_rtol=1e-11,
                     nonlinear_atol=1e-13, nonlinear_max_iter=80, anderson_memory=4,
                     anderson_start=2, anderson_damping=0.5, anderson_regularization=1e-12,
                     anderson_growth_limit=1.2, uniform_local_rtol=1e-12, uniform_local_atol=1e-14,
                     uniform_local_max_iter=64, uniform_local_damping=1.0)
# Algorithmic HBM bytes per particle per step of the fused push kernel: the
# FP64 particle state x, y, P(3), v(3), v_prev(3) read once and written once.
ALG_BYTES_PER_PARTICLE = 176
# The mixed form's push kernel: cell (int32), offsets (2), P (3), v (3),
# v_prev (3) in FP32 read (48 B), the same less P_z written (44 B).
ALG_BYTES_PER_PARTICLE_MIXED = 92
# Diagnostics columns whose mixed-vs-FP64 difference the bench line reports.
MIXED_ERROR_COLUMNS = ("field_energy", "kinetic_energy", "total_energy", "Bz_l2", "E_l2", "J_l2", "rho_l2")
# Reference CPU sample: same grid, 16 electrons per cell, timed step loop.
REF_SAMPLE_PPC = 16
REF_SAMPLE_STEPS = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="upic", choices=["upic", "reference"])
    ap.add_argument("--workload", default="weibel512", choices=sorted(WORKLOADS))
    ap.add_argument("--diag-stride", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision companion run of an explicit workload")
    ap.add_argument("--implicit-workload", default="weibel512_implicit",
                    help="implicit-method workload reported beside an explicit headline ('none' skips)")
    ap.add_argument("--implicit-steps", type=int, default=3,
                    help="timed steps of the implicit companion run (at most --steps)")
    ap.add_argument("--learned-steps", type=int, default=260,
                    help="steps of the learned-vs-extrapolated first-guess comparison (0 skips; one GPU only)")
    ap.add_argument("--learned-train", type=int, default=200,
                    help="training steps of the learned first guess")
    ap.add_argument("--learned-dt", type=float, default=None,
                    help="time step of the learned-guess comparison (default: the case's 0.05)")
    ap.add_argument("--ensemble-runs", type=int, default=256,
                    help="independent runs of the ensemble comparison (0 skips; one GPU only)")
    ap.add_argument("--ensemble-steps", type=int, default=80,
                    help="steps of the ensemble comparison")
    ap.add_argument("--implicit-ensemble-runs", type=int, default=1024,
                    help="1D-2V two-stream runs of the implicit ensemble comparison (0 skips; one GPU only)")
    ap.add_argument("--implicit-ensemble-steps", type=int, default=5,
                    help="steps of the implicit ensemble comparison")
    ap.add_argument("--implicit-ensemble-max-particles", type=float, default=1e6,
                    help="largest particle count of an implicit ensemble run (log-uniform from 1e4)")
    ap.add_argument("--implicit-ensemble-check-runs", type=int, default=32,
                    help="runs stepped alone for the sequential rate and the bitwise check (0: all)")
    ap.add_argument("--large-mixed-check", action="store_true",
                    help="instead of the bench line: the 2048x2048, 64 e-/cell Weibel + beam run in FP64 and in "
                         "mixed precision (energy drift and gauge residual of both), one JSON line")
    ap.add_argument("--large-steps", type=int, default=500, help="steps of --large-mixed-check")
    return ap.parse_args()


def config_desc(w, extra=None):
    d = {"workload": f"weibel_bimaxwellian_{w['nx']}x{w['ny']}_ppc{w['ppc']}",
         "grid": [w["nx"], w["ny"]], "particles": w["nx"] * w["ny"] * w["ppc"],
         "particles_per_cell": w["ppc"], "L": w["L"], "dt": w["dt"], "method": w["method"],
         "charge_update": w["charge_update"], "shape": "quadratic B-spline",
         "precision": "fp64",
         "l2": f"inputs larger than L2 (particle state {w['ppc'] * w['nx'] * w['ny'] * 88 / 1e9:.1f} GB)"
         if w["ppc"] * w["nx"] * w["ny"] > 10_000_000 else "inputs smaller than L2",
         "parallelism": "replicas"}
    if w["method"] == "cn_orbit":
        d["implicit_deck"] = dict(IMPLICIT_DECK)
    if extra:
        d.update(extra)
    return d


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid=None):
        self.uuid = uuid
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.seek(0)
        rows = [r.split(", ") for r in self.file.read().strip().splitlines() if r.strip()]
        if self.uuid:
            mine = [r for r in rows if len(r) >= 10 and self.uuid in r[1]]
            rows = mine or rows
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 10:
                continue
            try:
                sm.append(float(r[2]))
                smax.append(float(r[3]))
            except ValueError:
                continue
            for name, val in zip(names, r[6:10]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_traffic(np_total):
    """DRAM bytes per push launch from the committed ncu capture, scaled by
    particle count (traffic grows in proportion to the particles streamed)."""
    path = os.path.join(ROOT, "profiles", "push_deposit_traffic.json")
    try:
        with open(path) as fh:
            t = json.load(fh)
        return float(t["dram_bytes_per_launch"]) * np_total / float(t["particles"])
    except Exception:
        return None


def max_over_ranks(x, dist, device):
    """Max of a per-rank scalar over all ranks (device time is taken as the
    slowest rank's); identity without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, particles_per_rank, steps, max_ms):
    """Whole-job particle-steps/s of `world` independent replicas timed by
    the slowest one."""
    return world * particles_per_rank * steps / (max_ms / 1e3)


# ---------------------------------------------------------------------------
def reference_sample(w, ppc, steps, warmup, seed):
    """Time the reference's own step loop on a sample of workload w and
    return (particle-steps/s, kind, particles, seconds, what).

    Explicit workloads: Project2's run loop (oracle/_ref/libref_p2.so, or the
    oracle port when the reference build is absent) on the same grid with
    ppc electrons per cell.  Implicit workloads: Project3's
    nonlinear_step_orbit loop (oracle/_ref/libref_p3.so) on a 64x64 sub-box
    with the workload's cell size and physics and ppc electrons per cell (the
    per-particle cost of the implicit step does not depend on the box)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    # inputs from the oracle's restatement of the workload generator (bit for
    # bit the product's), so this arm loads none of the product's code
    gen = ol.generate_bimaxwellian
    if w["method"] == "cn_orbit":
        lib = ol.ref_p3()
        if lib is None:
            raise RuntimeError("oracle/_ref/libref_p3.so is not built (make -C oracle ref)")
        nsub = 64
        Ls = w["L"] * nsub / w["nx"]
        d = IMPLICIT_DECK
        p = gen(nsub, nsub, Ls, Ls, ppc, w["uth"], seed=seed)
        x = np.zeros((len(p["x"]), 3))
        x[:, 0] = p["x"] - Ls / 2
        x[:, 1] = p["y"] - Ls / 2
        q = p["q"] * d["Lz"]
        m = np.abs(q)

        def prob(n_steps):
            return ol.P3Problem(nsub, nsub, Ls, Ls, w["dt"], Lz=d["Lz"], kappa=d["kappa"], order=2,
                                nq=d["orbit_quad_order"], split=True, nyquist=True,
                                nl_rtol=d["nonlinear_rtol"], nl_atol=d["nonlinear_atol"],
                                nl_maxit=d["nonlinear_max_iter"], and_damp=d["anderson_damping"],
                                loc_rtol=d["uniform_local_rtol"], loc_atol=d["uniform_local_atol"],
                                loc_maxit=d["uniform_local_max_iter"], n_steps=n_steps)
        if warmup > 0:
            ol.p3_run(lib.ref_p3_run, prob(1), x, p["v"], q, m, want_fields=False)
        out = ol.p3_run(lib.ref_p3_run, prob(steps), x, p["v"], q, m, want_fields=False)
        n = len(q)
        secs = out["seconds"]
        what = (f"serial reference nonlinear_step_orbit loop, {nsub}x{nsub} sub-box with the "
                f"workload's cell size, {ppc} e-/cell ({n} particles), {steps} steps "
                f"(mean {out['info'][:, 0].mean():.1f} outer iterations)")
        return n * steps / secs, "reference", n, secs, what
    lib = ol.ref_p2()
    kind = "reference"
    fn = lib.ref_p2_simulate if lib is not None else None
    if fn is None:
        fn = ol.oracle().o2_simulate
        kind = "port"
    p = gen(w["nx"], w["ny"], w["L"], w["L"], ppc, w["uth"], seed=seed)
    parts = {"x": p["x"], "y": p["y"], "P": p["P"], "v": p["v"], "vprev": p["v_prev"], "q": p["q"],
             "m": p["m"]}
    if warmup > 0:
        prob = ol.P2Problem(w["nx"], w["ny"], w["L"], w["L"], w["dt"], 1, True, n_steps=warmup)
        parts, _, _, _ = ol.simulate(fn, prob, parts, want_fields=False)
    prob = ol.P2Problem(w["nx"], w["ny"], w["L"], w["L"], w["dt"], 1, True, n_steps=steps)
    _, _, _, secs = ol.simulate(fn, prob, parts, want_fields=False)
    n = len(parts["x"])
    what = (f"serial reference step loop, {w['nx']}x{w['ny']} grid, {ppc} e-/cell ({n} particles), "
            f"{steps} steps with diagnostics every step")
    return n * steps / secs, kind, n, secs, what


def _ref_worker(args):
    name, ppc, steps, warmup, seed = args
    return reference_sample(WORKLOADS[name], ppc, steps, warmup, seed)


def reference_pool(name, steps, warmup, diag_stride=1):
    """The reference's CPU step on all host cores (one serial reference
    process per core, each on its own sample of workload `name`)."""
    import multiprocessing as mp
    w = WORKLOADS[name]
    cores = min(os.cpu_count() or 1, 64)
    # per-process sample: explicit 512x512 grid with 4 e-/cell (1,048,576
    # particles); implicit 64x64 sub-box with 2 e-/cell (8,192 particles)
    ppc = 2 if w["method"] == "cn_orbit" else 4
    warm = min(warmup, 1) if w["method"] == "cn_orbit" else warmup
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(name, ppc, steps, warm, 1000 + i) for i in range(cores)])
    wall = time.perf_counter() - t0
    n = res[0][2]
    slowest = max(r[3] for r in res)
    value = cores * n * steps / slowest
    sample = (f"{cores} concurrent processes, each a {res[0][4]}; value = total particle-steps / "
              f"slowest process time")
    return {"value": value, "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * slowest / steps,
            "config": config_desc(w, {"diag_stride": diag_stride}),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": res[0][1],
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}


def run_reference_arm(args):
    """--impl reference: rank 0 times the reference's own CPU step; other
    ranks exit without work."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    main = reference_pool(args.workload, args.steps, args.warmup, args.diag_stride)
    line = {"metric": METRIC, "value": main["value"], "unit": METRIC, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": main["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    for k in ("config", "cpu_baseline", "e2e", "wall_s"):
        line[k] = main[k]
    if args.implicit_workload != "none" and WORKLOADS[args.workload]["method"] != "cn_orbit":
        imp = reference_pool(args.implicit_workload, min(args.steps, args.implicit_steps), args.warmup,
                             args.diag_stride)
        imp.update({"metric": METRIC, "unit": METRIC, "impl": "reference", "dtype": "f64"})
        line["implicit"] = imp
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# Learned vs extrapolated first guess of the implicit outer iteration: a
# 256x256 periodic plasma, 128 e-/cell (8,388,608 electrons), isotropic
# Maxwellian vth = 0.05 c with a density perturbation of amplitude 0.01 at
# k = (1, 1), solved to a 1e-10 relative residual.
LEARNED_CASE = dict(nx=256, ny=256, ppc=128, L=2 * np.pi / 0.3, dt=0.05, vth=0.05, amp=0.01, seed=404)


def learned_particles(up, c):
    p = up.generate_bimaxwellian(c["nx"], c["ny"], c["L"], c["L"], c["ppc"], (c["vth"],) * 3, seed=c["seed"])
    # displacement xi = -amp k / |k|^2 sin(k.x): n = n0 (1 + amp cos(k.x)) to first order
    k = 2 * np.pi / c["L"]
    ph = k * p["x"] + k * p["y"]
    d = -c["amp"] * np.sin(ph) / (2 * k)
    p["x"] = p["x"] + d
    p["y"] = p["y"] + d
    return p


def learned_comparison(args):
    """Both first guesses on the same plasma: outer iterations per step,
    wall time per step (host clock around the solver calls, which synchronise
    every step), and the distance between the two final states."""
    import unstaggered_pic_b200 as up

    c = dict(LEARNED_CASE)
    if args.learned_dt:
        c["dt"] = args.learned_dt
    steps, train = args.learned_steps, min(args.learned_train, max(0, args.learned_steps - 3))
    window = steps - min(steps, train + 2)
    p = learned_particles(up, c)
    deck = dict(IMPLICIT_DECK)
    deck["nonlinear_rtol"] = 1e-10
    res = {}
    for pred in ("extrapolated", "learned"):
        cfg = up.ImplicitConfig(nx=c["nx"], ny=c["ny"], Lx=c["L"], Ly=c["L"], dt=c["dt"], current_predictor=pred,
                                learned_train_steps=train, **deck)
        with up.Simulation(cfg) as sim:
            sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
            sim.init_fields(False)
            t0 = time.perf_counter()
            _, info_a = sim.step_implicit(steps - window, diagnostics=False)
            t1 = time.perf_counter()
            _, info_b = (sim.step_implicit(window, diagnostics=False) if window > 0
                         else (None, np.zeros((0, info_a.shape[1]))))
            t2 = time.perf_counter()
            fields = np.stack([sim.field(f) for f in ("phi", "Ax", "Ay", "Az", "Jx", "Jy", "Jz")])
        info = np.concatenate([info_a, info_b])
        res[pred] = (info, fields, t1 - t0, t2 - t1)
    cols = up.SOLVE_INFO_COLUMNS
    out = {"workload": f"maxwellian_perturbed_{c['nx']}x{c['ny']}_ppc{c['ppc']}",
           "particles": c["nx"] * c["ny"] * c["ppc"], "steps": steps, "training_steps": train,
           "dt": c["dt"], "nonlinear_rtol": 1e-10, "data": "synthetic (seeded Maxwellian, vth 0.05, density perturbation 0.01 at "
                                              "k = (1, 1))"}
    for pred, (info, _, ta, tb) in res.items():
        it = info[:, cols.index("iterations")]
        after = info[len(info) - window:] if window > 0 else info[:0]
        used = info[:, cols.index("predictor_used")]
        out[pred] = {
            "outer_iterations_per_step": float(it.mean()),
            "outer_iterations_per_step_after_training": float(after[:, 0].mean()) if window > 0 else None,
            "ms_per_step_training_window": 1e3 * ta / max(1, steps - window),
            "ms_per_step_after_training": 1e3 * tb / window if window > 0 else None,
            "guess_error_median_after_training": (float(np.median(after[:, cols.index("guess_error")]))
                                                  if window > 0 else None),
            "steps_using_learned_guess": int((used == 2).sum()),
            "final_rms_residual_max": float(info[:, cols.index("final_rms_residual")].max()),
        }
    fe, fl = res["extrapolated"][1], res["learned"][1]
    out["final_state_max_rel_diff"] = float(max(np.max(np.abs(fl[k] - fe[k])) / (np.max(np.abs(fe[k])) + 1e-300)
                                                for k in range(len(fe))))
    return out


# Ensemble of independent explicit runs of uneven sizes (the batched
# ensemble on the explicit 2D method): per run the node count
# is drawn from {128, 256, 512, 1024} (grids 16x8, 16x16, 32x16, 32x32) and
# the particle count log-uniformly from [1e4, 1e5]; Weibel bi-Maxwellian
# plasma, dt 0.05.  Tile size and re-sort interval are autotuned per grid
# bucket on the bucket's median run.
ENSEMBLE_GRIDS = [(16, 8), (16, 16), (32, 16), (32, 32)]


def ensemble_comparison(args):
    """The runs advanced one after another with upic_step, then the same
    runs from the same start advanced together with upic_ensemble_step (one
    CUDA graph per period); particle-steps/s of both (host clock around the
    calls, which return when the work is complete) and the largest state
    difference between the two (they are bit-for-bit equal by design)."""
    import unstaggered_pic_b200 as up

    rng = np.random.default_rng(707)
    nruns, steps = args.ensemble_runs, args.ensemble_steps
    L0 = 2 * np.pi / 0.3
    runs = []
    for r in range(nruns):
        nx, ny = ENSEMBLE_GRIDS[rng.integers(len(ENSEMBLE_GRIDS))]
        npart = int(round(np.exp(rng.uniform(np.log(1e4), np.log(1e5)))))
        ppc = max(1, npart // (nx * ny))
        runs.append((nx, ny, ppc, 1000 + r))
    t0 = time.perf_counter()
    tuned = {}
    for nx, ny in ENSEMBLE_GRIDS:
        members = sorted(ppc for gx, gy, ppc, _ in runs if (gx, gy) == (nx, ny))
        if not members:
            continue
        ppc = members[len(members) // 2]
        Lx, Ly = L0 * nx / 32, L0 * ny / 32
        p = up.generate_bimaxwellian(nx, ny, Lx, Ly, ppc, (0.02, 0.2, 0.0), seed=5)
        make = lambda tile, si: up.Config(nx=nx, ny=ny, Lx=Lx, Ly=Ly, dt=0.05, method="bdf1", tile=tile,
                                          sort_interval=si)
        tile, si, _ = up.autotune_explicit(make, p, tiles=(4, 8), sort_intervals=(2, 4), steps=8)
        tuned[f"{nx}x{ny}"] = {"tile": tile, "sort_interval": si}
    t_tune = time.perf_counter() - t0

    def start_all():
        sims = []
        for nx, ny, ppc, seed in runs:
            Lx, Ly = L0 * nx / 32, L0 * ny / 32
            t = tuned[f"{nx}x{ny}"]
            sim = up.Simulation(up.Config(nx=nx, ny=ny, Lx=Lx, Ly=Ly, dt=0.05, method="bdf1", tile=t["tile"],
                                          sort_interval=t["sort_interval"]))
            p = up.generate_bimaxwellian(nx, ny, Lx, Ly, ppc, (0.02, 0.2, 0.0), seed=seed)
            sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
            sim.init_fields(False)
            sims.append(sim)
        return sims

    total = sum(nx * ny * ppc for nx, ny, ppc, _ in runs)
    seq = start_all()
    for sim in seq:
        sim.step(3, 0)
    t0 = time.perf_counter()
    for sim in seq:
        sim.step(steps, 0)
    t_seq = time.perf_counter() - t0
    ens_sims = start_all()
    for sim in ens_sims:
        sim.step(3, 0)
    ens = up.Ensemble(ens_sims)
    t0 = time.perf_counter()
    ens.step(ens.period)  # records the graph
    t_first = time.perf_counter() - t0
    left = steps - ens.period
    t0 = time.perf_counter()
    if left > 0:
        ens.step(left)
    t_ens = time.perf_counter() - t0
    diff = 0.0
    for a, b in zip(seq, ens_sims):
        pa, pb = a.get_particles(), b.get_particles()
        diff = max(diff, float(np.max(np.abs(pa["v"] - pb["v"]))))
    # the sequential runs took `steps` steps, the ensemble `steps` too
    ens.close()
    for sim in seq + ens_sims:
        sim.close()
    return {"workload": f"{nruns} independent explicit Weibel runs, grids {ENSEMBLE_GRIDS}, "
                        f"1e4-1e5 particles each (log-uniform)",
            "runs": nruns, "particles": total, "steps": steps, "period": ens.period,
            "tuned": tuned, "autotune_seconds": t_tune,
            "sequential": {"value": total * steps / t_seq, "unit": METRIC, "ms_per_step": 1e3 * t_seq / steps,
                           "what": "upic_step(run, K) for each run in turn"},
            "ensemble": {"value": total * left / t_ens if left > 0 else None, "unit": METRIC,
                         "ms_per_step": 1e3 * t_ens / left if left > 0 else None,
                         "first_period_seconds_with_capture": t_first,
                         "what": "upic_ensemble_step: one CUDA graph launch per period, every run on its own "
                                 "stream; timed after the period that records the graph"},
            "max_abs_velocity_difference": diff,
            "data": "synthetic (seeded bi-Maxwellian per run)"}


# Implicit ensemble: 1D-2V periodic two-stream runs (64 by default; the
# full-size batch is 1024 runs of up to 1e6 particles), Nx from
# {128, 256, 512, 1024}, particle count log-uniform in [1e4, 1e5],
# counter-drifting Maxwellian beams at +-v0, v0 uniform in [0.05, 0.3] c,
# vth 0.01 c, cubic splines, dt 0.1.
def implicit_ensemble_comparison(args):
    """The runs advanced one after another with upic_step_implicit, then
    the same runs together with upic_ensemble_step (a pool of host threads,
    each run on its own stream); particle-steps/s of both and the largest
    state difference (bit-for-bit equal by design)."""
    import unstaggered_pic_b200 as up

    rng = np.random.default_rng(909)
    nruns, steps = args.implicit_ensemble_runs, args.implicit_ensemble_steps
    pmax = float(args.implicit_ensemble_max_particles)
    deck = dict(IMPLICIT_DECK)
    deck["spline_order"] = 3
    runs = []
    for r in range(nruns):
        nx = int(rng.choice([128, 256, 512, 1024]))
        npart = 2 * int(round(np.exp(rng.uniform(np.log(1e4), np.log(pmax))) / 2))
        v0 = float(rng.uniform(0.05, 0.3))
        runs.append((nx, npart, v0, 3000 + r))
    # the runs stepped alone: all of them, or every k-th for a large ensemble
    ncheck = args.implicit_ensemble_check_runs or nruns
    checked = list(range(0, nruns, max(1, nruns // ncheck)))[:ncheck]

    def start_all(which=None):
        sims = []
        for nx, npart, v0, seed in (runs if which is None else [runs[i] for i in which]):
            g = np.random.default_rng(seed)
            Lx = 2 * np.pi * v0 / 0.6 * 4  # four wavelengths of the fastest-growing cold mode
            nb = npart // 2
            x = g.uniform(-Lx / 2, Lx / 2, npart)
            v = np.zeros((npart, 3))
            v[:nb, 0], v[nb:, 0] = v0, -v0
            v[:, :2] += 0.01 * g.normal(size=(npart, 2))
            q = np.full(npart, -Lx / npart)
            cfg = up.ImplicitConfig(nx=nx, ny=1, Lx=Lx, Ly=1.0, dt=0.1, **deck)
            sim = up.Simulation(cfg)
            sim.set_particles(x, np.zeros(npart), np.zeros((npart, 3)), v, v, q, np.abs(q))
            sim.init_fields(False)
            sims.append(sim)
        return sims

    total = sum(n for _, n, _, _ in runs)
    total_checked = sum(runs[i][1] for i in checked)
    seq = start_all(checked)
    t0 = time.perf_counter()
    for sim in seq:
        sim.step_implicit(steps, diagnostics=False)
    t_seq = time.perf_counter() - t0
    par = start_all()
    ens = up.Ensemble(par)
    t0 = time.perf_counter()
    ens.step(steps)
    t_ens = time.perf_counter() - t0
    diff = 0.0
    for i, a in zip(checked, seq):
        diff = max(diff, float(np.max(np.abs(a.get_particles()["v"] - par[i].get_particles()["v"]))))
    ens.close()
    for sim in seq + par:
        sim.close()
    return {"workload": f"{nruns} independent 1D-2V two-stream runs (implicit GM-HC-CN, cubic), Nx from "
                        f"{{128, 256, 512, 1024}}, 1e4-{pmax:.0e} particles each (log-uniform), v0 in [0.05, 0.3] c",
            "runs": nruns, "particles": total, "steps": steps,
            "sequential": {"value": total_checked * steps / t_seq, "unit": METRIC,
                           "ms_per_step": 1e3 * t_seq / steps, "runs": len(checked),
                           "what": "upic_step_implicit(run, K) for each run in turn"
                                   + ("" if len(checked) == nruns else
                                      f" (every {max(1, nruns // ncheck)}-th run; rate over those runs)")},
            "ensemble": {"value": total * steps / t_ens, "unit": METRIC, "ms_per_step": 1e3 * t_ens / steps,
                         "what": "upic_ensemble_step: runs on a pool of host threads, each on its own stream"},
            "max_abs_velocity_difference": diff,
            "data": "synthetic (seeded beams per run)"}


def make_simulation(up, w, precision="fp64", predictor="previous", warm=False):
    if w["method"] == "cn_orbit":
        cfg = up.ImplicitConfig(nx=w["nx"], ny=w["ny"], Lx=w["L"], Ly=w["L"], dt=w["dt"], current_predictor=predictor,
                                local_warm_start=warm, **IMPLICIT_DECK)
    else:
        cfg = up.Config(nx=w["nx"], ny=w["ny"], Lx=w["L"], Ly=w["L"], dt=w["dt"], method=w["method"],
                        charge_update=w["charge_update"], precision=precision)
    return up.Simulation(cfg)


def advance(sim, w, steps, diag_stride):
    """K steps of the workload's method; returns the implicit solve reports,
    or the explicit diagnostics rows."""
    if w["method"] == "cn_orbit":
        _, info = sim.step_implicit(steps, diagnostics=diag_stride > 0)
        return info
    return sim.step(steps, diag_stride)


# Implicit map kernel: per launch it streams x, y, P(3), v(3) of every
# particle (64 B); the final consistency launch of a step also writes the end
# state x, y, P(3), v(3), vbar(3) (88 B).
IMPLICIT_READ_BYTES = 64
IMPLICIT_WRITE_BYTES = 88


def measure(args, name, steps, warmup, world, rank, dist, dev, predictor="previous", warm=False, extras=True):
    """Device-resident and end-to-end throughput of workload `name` (one
    replica per rank), the dominant kernel's roofline and the reference CPU
    sample; returns the bench-line fields."""
    import torch
    import unstaggered_pic_b200 as up

    w = WORKLOADS[name]
    implicit = w["method"] == "cn_orbit"
    np_total = w["nx"] * w["ny"] * w["ppc"]

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(x):
        return max_over_ranks(x, dist, "cuda")

    # host inputs in pinned memory (seed differs per replica)
    p = up.generate_bimaxwellian(w["nx"], w["ny"], w["L"], w["L"], w["ppc"], w["uth"],
                                 seed=w["seed"] + rank)
    pinned = {}
    for k, a in p.items():
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        pinned[k] = t
    del p
    host = {k: t.numpy() for k, t in pinned.items()}
    sim = make_simulation(up, w, predictor=predictor, warm=warm)
    stream = torch.cuda.current_stream()
    sim.set_stream(stream.cuda_stream)

    def load():
        sim.set_particles(host["x"], host["y"], host["P"], host["v"], host["v_prev"], host["q"],
                          host["m"])

    # ---- device-resident throughput
    load()
    sim.init_fields(False)
    advance(sim, w, warmup, args.diag_stride)
    torch.cuda.synchronize()
    barrier()
    sim.profile_enable(True)
    _, _, launches0 = sim.profile_read()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    info = advance(sim, w, steps, args.diag_stride)
    e1.record(stream)
    rows64 = None if implicit else info
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_ms = allmax(e0.elapsed_time(e1))
    kern_ms, kern_n, launches1 = sim.profile_read()
    sim.profile_enable(False)
    gpu_launches = launches1 - launches0
    value = replica_throughput(world, np_total, steps, t_ms)
    peak, peak_kind = measured_hbm_peak()
    if implicit:
        alg_bytes = np_total * (IMPLICIT_READ_BYTES * kern_n + IMPLICIT_WRITE_BYTES * steps)
        achieved = alg_bytes / (kern_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                    "kernel": "implicit_map_kernel (per-particle local GM-HC solve + orbit-averaged "
                              "current deposit)",
                    "kernel_ms": kern_ms / max(kern_n, 1), "kernel_launches": kern_n,
                    "kernel_share": kern_ms / t_ms,
                    "algorithmic_bytes_per_particle_launch": IMPLICIT_READ_BYTES,
                    "note": "FP64-issue bound (local fixed point with orbit quadrature per particle "
                            "per launch); HBM fraction stated for the streamed particle state"}
        solve = {"outer_iterations_per_step": float(np.mean(info[:, 0])),
                 "map_evaluations_per_step": kern_n / steps,
                 "local_iterations_mean": float(np.mean(info[:, 5])),
                 "local_iterations_max": float(np.max(info[:, 4])),
                 "final_rms_residual_max": float(np.max(info[:, 2]))}
    else:
        push_avg_s = kern_ms / max(kern_n, 1) / 1e3
        achieved = ALG_BYTES_PER_PARTICLE * np_total / push_avg_s / 1e9
        traffic = measured_traffic(np_total)
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                    "kernel": "push_deposit_kernel (gather + IAEM push + next-step deposit)",
                    "kernel_ms": push_avg_s * 1e3, "kernel_share": kern_ms / t_ms,
                    "algorithmic_bytes_per_particle": ALG_BYTES_PER_PARTICLE}
        solve = None

    # ---- end to end through the public API from pinned host buffers
    e2e = None
    if extras and not args.no_e2e:
        # the step's result is read back into pinned host buffers, as the inputs come from them
        res = {k: torch.empty((np_total,) if k in ("x", "y") else (np_total, 3), dtype=torch.float64,
                              pin_memory=True).numpy() for k in ("x", "y", "P", "v", "v_prev")}
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        load()
        t1 = time.perf_counter()
        sim.init_fields(True)
        t2 = time.perf_counter()
        advance(sim, w, steps, 1)
        t3 = time.perf_counter()
        out = sim.get_particles(out=res)
        t4 = time.perf_counter()
        t_e2e = allmax(t4 - t0)
        phases = {"set_particles": t1 - t0, "init_fields": t2 - t1, "steps": t3 - t2, "get_particles": t4 - t3}
        del out
        ncol = len(up.IMPLICIT_DIAG_COLUMNS) + len(up.SOLVE_INFO_COLUMNS) if implicit else len(up.DIAG_COLUMNS)
        # x, y, P, v, v_prev (11 doubles); q and m cross only when they are
        # not uniform (this plasma's are: one species)
        h2d = np_total * 11 * 8 / steps
        d2h = (ncol * 8 * (steps + 1) + np_total * 11 * 8) / steps
        api = "upic_step_implicit(K)" if implicit else "upic_step(K, diagnostics every step)"
        e2e = {"value": world * np_total * steps / t_e2e, "unit": METRIC,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "seconds": t_e2e,
               "phase_seconds": phases,
               "what": f"upic_set_particles + upic_init_fields + {api} with a diagnostics row per "
                       "step + upic_get_particles, host wall clock, max over ranks"}
    sim.close()

    # ---- mixed-precision form of the explicit step on the same input
    mixed = None
    if extras and not implicit and not args.no_mixed:
        torch.cuda.empty_cache()
        msim = make_simulation(up, w, "mixed")
        msim.set_stream(stream.cuda_stream)
        msim.set_particles(host["x"], host["y"], host["P"], host["v"], host["v_prev"], host["q"], host["m"])
        msim.init_fields(False)
        advance(msim, w, warmup, args.diag_stride)
        torch.cuda.synchronize()
        barrier()
        msim.profile_enable(True)
        torch.cuda.synchronize()
        e0.record(stream)
        rows32 = advance(msim, w, steps, args.diag_stride)
        e1.record(stream)
        torch.cuda.synchronize()
        tm_ms = allmax(e0.elapsed_time(e1))
        mk_ms, mk_n, _ = msim.profile_read()
        msim.close()
        mpush_s = mk_ms / max(mk_n, 1) / 1e3
        mach = ALG_BYTES_PER_PARTICLE_MIXED * np_total / mpush_s / 1e9
        err = {}
        for col in MIXED_ERROR_COLUMNS:
            k = up.DIAG_COLUMNS.index(col)
            a, b = rows32[:, k], rows64[:, k]
            ok = np.isfinite(a) & np.isfinite(b)
            scale = float(np.max(np.abs(b[ok]))) if ok.any() else 0.0
            err[col] = float(np.max(np.abs(a[ok] - b[ok])) / scale) if scale > 0 else None
        mixed = {"value": replica_throughput(world, np_total, steps, tm_ms), "unit": METRIC,
                 "ms_per_step": tm_ms / steps, "dtype": "f32 particles, f64 field solve and energies",
                 "roofline": {"bound": "hbm", "achieved": mach, "peak": peak, "unit": "GB/s", "frac": mach / peak,
                              "kernel": "push_deposit_mixed_kernel", "kernel_ms": mpush_s * 1e3,
                              "algorithmic_bytes_per_particle": ALG_BYTES_PER_PARTICLE_MIXED},
                 "max_rel_diff_vs_fp64": err,
                 "what": f"same plasma, same {warmup} warm-up and {steps} timed steps as the FP64 run; "
                         "differences over the timed steps, relative to each column's largest FP64 value"}

    cpu = None
    if extras and rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref_ppc, ref_steps = (4, 2) if implicit else (REF_SAMPLE_PPC, REF_SAMPLE_STEPS)
            v, kind, n, secs, what = reference_sample(w, ref_ppc, ref_steps, 0, 7)
            cpu = {"value": v, "unit": METRIC, "cores": 1, "kind": kind,
                   "sample": f"{what} ({secs:.1f} s)"}
        except Exception as exc:  # the baseline is reported, not required
            cpu = {"value": None, "unit": METRIC, "cores": 1, "kind": "reference",
                   "sample": f"failed: {exc}"}

    out = {"value": value, "steps": steps, "warmup": warmup, "ms_per_step": t_ms / steps,
           "config": config_desc(w, {"diag_stride": args.diag_stride}), "roofline": roofline,
           "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches, "clocks": clk}
    if solve is not None:
        out["implicit_solve"] = solve
    if mixed is not None:
        out["mixed"] = mixed
    return out


def run_upic(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    main = measure(args, args.workload, args.steps, args.warmup, world, rank, dist, dev)
    companion = None
    if args.implicit_workload != "none" and WORKLOADS[args.workload]["method"] != "cn_orbit":
        torch.cuda.empty_cache()
        companion = measure(args, args.implicit_workload, min(args.steps, args.implicit_steps),
                            args.warmup, world, rank, dist, dev)
        # the same run with the opt-in accelerations (not in the reference):
        # extrapolated first current guess, warm-started local fixed points
        torch.cuda.empty_cache()
        opt = measure(args, args.implicit_workload, min(args.steps, args.implicit_steps), args.warmup, world,
                      rank, dist, dev, predictor="extrapolated", warm=True, extras=False)
        companion["opt_in"] = {
            "value": opt["value"], "unit": METRIC, "ms_per_step": opt["ms_per_step"],
            "implicit_solve": opt.get("implicit_solve"),
            "what": "current_predictor = extrapolated (2 J^n - J^(n-1)) and local_warm_start = 1; "
                    "same tolerances, same plasma"}
    ensemble = None
    if args.ensemble_runs > 0 and world == 1 and WORKLOADS[args.workload]["method"] != "cn_orbit":
        torch.cuda.empty_cache()
        ensemble = ensemble_comparison(args)
    implicit_ensemble = None
    if args.implicit_ensemble_runs > 0 and world == 1 and WORKLOADS[args.workload]["method"] != "cn_orbit":
        torch.cuda.empty_cache()
        implicit_ensemble = implicit_ensemble_comparison(args)
    learned = None
    if args.learned_steps > 0 and world == 1 and WORKLOADS[args.workload]["method"] != "cn_orbit":
        torch.cuda.empty_cache()
        learned = learned_comparison(args)
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": main["value"], "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic"}
    for k in ("config", "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks", "implicit_solve", "mixed"):
        if k in main:
            line[k] = main[k]
    if companion is not None:
        companion.update({"metric": METRIC, "unit": METRIC, "n_gpus": world, "dtype": "f64",
                          "method": "implicit orbit-averaged GM-HC-CN step on the same plasma"})
        line["implicit"] = companion
    if learned is not None:
        line["learned_guess"] = learned
    if ensemble is not None:
        line["ensemble"] = ensemble
    if implicit_ensemble is not None:
        line["implicit_ensemble"] = implicit_ensemble
    print(json.dumps(line))
    return 0


def large_mixed_check(args):
    """The large mixed-precision configuration on the explicit step: a
    2048x2048 periodic grid with the cell size of the 512x512 bench workload
    (L = 4 * 2 pi / 0.3), 58 electrons per cell of Weibel bi-Maxwellian
    plasma (vth 0.02, 0.2, 0 c) plus 6 per cell of a beam of density 0.1
    drifting at 0.5 c along x (268,435,456 particles), fixed ion background
    1.1, dt 0.05, run in FP64 and in mixed precision from the same seed;
    energy drift and gauge / Gauss residuals of both, every 10 steps."""
    import torch
    import unstaggered_pic_b200 as up

    torch.cuda.set_device(0)
    n, L, steps = 2048, 4 * 2 * np.pi / 0.3, args.large_steps
    u_beam = 0.5 / np.sqrt(1 - 0.25)
    a = up.generate_bimaxwellian(n, n, L, L, 58, (0.02, 0.2, 0.0), n0=1.0, seed=55)
    b = up.generate_bimaxwellian(n, n, L, L, 6, (0.02, 0.02, 0.02), udrift=(u_beam, 0.0, 0.0), n0=0.1, seed=56)
    p = {k: np.concatenate([a[k], b[k]]) for k in a}
    del a, b
    npart = len(p["x"])
    names = up.DIAG_COLUMNS
    out = {"workload": f"weibel_beam_{n}x{n}_ppc64", "particles": npart, "steps": steps, "L": L, "dt": 0.05,
           "shape": "quadratic B-spline (the explicit method's)", "data": "synthetic (seeded)"}
    rows = {}
    for prec in ("fp64", "mixed"):
        cfg = up.Config(nx=n, ny=n, Lx=L, Ly=L, dt=0.05, method="bdf1", n0=1.1, precision=prec)
        with up.Simulation(cfg) as sim:
            sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
            row0 = sim.init_fields(True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d = sim.step(steps, 10)
            el = time.perf_counter() - t0
        d = np.vstack([row0, d[9::10]])
        rows[prec] = d
        e = d[:, names.index("total_energy")]
        out[prec] = {"value": npart * steps / el, "unit": METRIC, "ms_per_step": 1e3 * el / steps,
                     "energy_drift_max": float(np.max(np.abs(e - e[0]) / abs(e[0]))),
                     "gauge_rms_max": float(np.max(d[:, names.index("gauge_rms")])),
                     "gauss_rms_max": float(np.max(d[:, names.index("gauss_rms")])),
                     "continuity_rms_start": float(d[0, names.index("continuity_rms")]),
                     "continuity_rms_max_after_start": float(np.max(d[1:, names.index("continuity_rms")])),
                     "final_field_energy": float(d[-1, names.index("field_energy")]),
                     "final_Bz_l2": float(d[-1, names.index("Bz_l2")])}
    r64, r32 = rows["fp64"], rows["mixed"]
    out["mixed_vs_fp64_max_rel_diff"] = {
        c: float(np.max(np.abs(r32[:, names.index(c)] - r64[:, names.index(c)])) /
                 (np.max(np.abs(r64[:, names.index(c)])) + 1e-300))
        for c in ("total_energy", "field_energy", "kinetic_energy", "Bz_l2", "E_l2", "J_l2")}
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.large_mixed_check:
        return large_mixed_check(args)
    return run_upic(args)


if __name__ == "__main__":
    sys.exit(main())
