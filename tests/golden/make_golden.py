"""Regenerate the golden fixtures in tests/golden/ from the reference's own code.

Runs the reference solvers Project2/spectral_pic_part3.cpp,
Project3/ec_pic_nyquist_projected.cpp and Project1/ec_pic_serial_demo.cpp
through the C-ABI harnesses oracle/_ref/libref_p2.so, libref_p3.so and
libref_p1.so (built by `make -C oracle` from the reference sources) on small
seeded inputs and saves inputs and outputs, and copies the published
validation numbers of Project2/docs/validation_summary.json and the columns
of the shipped Project1/output/landau_weak run.  The
fixtures let the oracle and the GPU path be checked where the reference
sources are absent.

    UPIC_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py        # all fixtures
    UPIC_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py p3     # implicit runs only
    UPIC_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py p1     # Project1 runs only

UPIC_REFERENCE_DIR is needed only by the fixtures that copy shipped reference
files (the published validation numbers and the shipped Project1 output).
"""
import csv
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402



def ref_path(*parts):
    """Path of a file of the reference checkout named by UPIC_REFERENCE_DIR."""
    root = os.environ.get("UPIC_REFERENCE_DIR")
    if not root or not os.path.isdir(root):
        raise SystemExit("set UPIC_REFERENCE_DIR to the reference checkout")
    return os.path.join(root, *parts)


def seeded_particles(rng, n, Lx, Ly, vth=(0.02, 0.2, 0.05), edge=True):
    """Random electrons (uniform positions, Maxwellian momenta) with q/m = -1."""
    x = rng.uniform(0, Lx, n)
    y = rng.uniform(0, Ly, n)
    if edge and n >= 8:
        # positions on and next to cell edges, the domain edge and node centres
        x[:4] = [0.0, np.nextafter(Lx, 0), Lx / 2, 0.5 * Lx / 8]
        y[:4] = [np.nextafter(Ly, 0), 0.0, 0.25 * Ly, Ly / 2]
    u = rng.normal(size=(n, 3)) * np.asarray(vth)
    gam = np.sqrt(1 + (u * u).sum(1))
    v = u / gam[:, None]
    w = Lx * Ly / n
    q = np.full(n, -w)
    m = np.full(n, w)
    P = m[:, None] * u
    vprev = v + rng.normal(size=(n, 3)) * 1e-3
    return {"x": x, "y": y, "P": P, "v": v, "vprev": vprev, "q": q, "m": m}


def main():
    lib = ol.ref_p2()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p2.so missing: run make -C oracle")
    rng = np.random.default_rng(20260101)
    nx, ny, Lx, Ly = 32, 16, 3.0, 2.0
    parts = seeded_particles(rng, 2000, Lx, Ly)
    N = nx * ny
    J = np.zeros(3 * N)
    lib.ref_p2_deposit_current(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ctypes.c_long(2000),
                               ol.ptr(parts["x"]), ol.ptr(parts["y"]), ol.ptr(parts["v"]),
                               ol.ptr(parts["q"]), ol.ptr(J))
    rho = np.zeros(N)
    lib.ref_p2_deposit_charge(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ctypes.c_double(1.0),
                              ctypes.c_long(2000), ol.ptr(parts["x"]), ol.ptr(parts["y"]),
                              ol.ptr(parts["q"]), ol.ptr(rho))
    f = rng.normal(size=N)
    gat = np.zeros(2000)
    lib.ref_p2_gather(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ol.ptr(f), ctypes.c_long(2000),
                      ol.ptr(parts["x"]), ol.ptr(parts["y"]), ol.ptr(gat))
    re = rng.normal(size=N)
    im = rng.normal(size=N)
    fre, fim = re.copy(), im.copy()
    lib.ref_p2_fft2d(nx, ny, ol.ptr(fre), ol.ptr(fim), 0)
    ire, iim = re.copy(), im.copy()
    lib.ref_p2_fft2d(nx, ny, ol.ptr(ire), ol.ptr(iim), 1)
    ddx = np.zeros(N)
    ddy = np.zeros(N)
    lib.ref_p2_spectral_derivative(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ol.ptr(f), 0, ol.ptr(ddx))
    lib.ref_p2_spectral_derivative(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ol.ptr(f), 1, ol.ptr(ddy))
    phi = np.zeros(N)
    lib.ref_p2_poisson(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ctypes.c_double(1.0), ol.ptr(rho),
                       ol.ptr(phi))
    np.savez_compressed(os.path.join(HERE, "p2_kernels.npz"), nx=nx, ny=ny, Lx=Lx, Ly=Ly,
                        **{"in_" + k: v for k, v in parts.items()}, J=J, rho=rho, f=f, gather=gat,
                        re=re, im=im, fft_re=fre, fft_im=fim, ifft_re=ire, ifft_im=iim, ddx=ddx,
                        ddy=ddy, phi=phi)

    # short runs of the step loop, every method/charge variant
    for order in (1, 2):
        for conserving in (True, False):
            prob = ol.P2Problem(16, 32, 2.5, 4.0, 0.05, order, conserving, n_steps=12)
            p = seeded_particles(rng, 1024, prob.Lx, prob.Ly)
            out, diag, fields, _ = ol.simulate(lib.ref_p2_simulate, prob, p)
            name = f"p2_run_bdf{order}_{'conserving' if conserving else 'naive'}.npz"
            np.savez_compressed(os.path.join(HERE, name), params=prob.params(), iparams=prob.iparams(),
                                **{"in_" + k: v for k, v in p.items()},
                                **{"out_" + k: v for k, v in out.items()}, diag=diag, fields=fields)

    # published validation numbers of the four Weibel decks
    with open(ref_path("Project2", "docs", "validation_summary.json")) as fh:
        summ = json.load(fh)
    runs = {k: v for k, v in summ["runs"].items() if k.startswith("weibel")}
    with open(os.path.join(HERE, "p2_weibel_published.json"), "w") as fh:
        json.dump({"source": "Project2/docs/validation_summary.json", "runs": runs}, fh, indent=1)
    p3_main()
    p1_main()
    print("fixtures written")


def p3_edge_positions(x, Lx, Ly, nx, ny):
    """Put the first particles on the domain edge, on nodes and next to them."""
    dx, dy = Lx / nx, Ly / ny
    x[:6, 0] = [-Lx / 2, np.nextafter(Lx / 2, 0), 0.0, -Lx / 2 + dx, np.nextafter(-Lx / 2 + 3 * dx, 0),
                0.5 * dx]
    x[:6, 1] = [np.nextafter(Ly / 2, 0), -Ly / 2, -Ly / 2 + 2 * dy, 0.0, 0.25 * dy,
                np.nextafter(-Ly / 2 + 5 * dy, 0)]


# Implicit (Project3) runs: (name, problem keywords, particles per cell, thermal
# spreads of u = gamma v, two species).
P3_CASES = [
    ("p3_run_o2_anderson", dict(nx=16, ny=16, Lx=2 * np.pi / 0.3, Ly=2 * np.pi / 0.3, dt=0.05, order=2,
                                nq=8, nyquist=True, n_steps=4), 8, (0.02, 0.2, 0.0), False),
    ("p3_run_o3_picard", dict(nx=16, ny=16, Lx=2 * np.pi / 0.3, Ly=2 * np.pi / 0.3, dt=0.2, order=3,
                              nq=8, nyquist=False, solver="picard", n_steps=3), 8, (0.02, 0.2, 0.0),
     False),
    ("p3_run_o1_nosplit", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, dt=0.1, order=1, nq=4,
                               split=False, nyquist=True, n_steps=3), 8, (0.05, 0.05, 0.05), False),
    ("p3_run_o4", dict(nx=8, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, dt=0.1, order=4, nq=8, nyquist=True,
                       n_steps=2), 16, (0.05, 0.05, 0.05), False),
    ("p3_run_two_species", dict(nx=16, ny=8, Lx=2 * np.pi, Ly=np.pi, dt=0.1, order=2, nq=8,
                                nyquist=True, n_steps=2, Lz=0.5), 16, (0.1, 0.05, 0.02), True),
    # 1D-2V (ny = nz = 1), cubic splines
    ("p3_run_1d_o3", dict(nx=64, ny=1, Lx=4 * np.pi, Ly=1.0, dt=0.1, order=3, nq=8, nyquist=True,
                          n_steps=3), 32, (0.1, 0.05, 0.0), False),
]


# Implicit runs that need the selective particle sub-cycling fallback (a
# small particle_local_max_iter makes some local solves fail over the full
# dt): (name, problem keywords, particles per cell, thermal spreads,
# fallback max_substeps).
P3_FALLBACK_CASES = [
    ("p3_fallback_few", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, dt=0.2, order=2, nq=8, nyquist=True,
                             n_steps=2, loc_maxit=5), 8, (0.3, 0.3, 0.0), 64),
    ("p3_fallback_some", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, dt=0.1, order=2, nq=8, nyquist=True,
                              n_steps=2, loc_maxit=4), 8, (0.5, 0.5, 0.0), 64),
    ("p3_fallback_many_o3", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, dt=0.3, order=3, nq=8, nyquist=True,
                                 n_steps=2, loc_maxit=5), 8, (0.3, 0.3, 0.1), 64),
]


# Long implicit run for the linear growth rate: 1D-2V (ny = nz = 1) cold
# relativistic two-stream instability, beams at +-0.2 c, 1024 electrons per
# beam on a quiet start with a 1e-3 density perturbation of mode 1, cubic
# splines, 250 steps of dt = 0.1 (about ten e-foldings, into saturation).
P3_LONG_CASE = ("p3_two_stream_long", dict(nx=64, ny=1, Lx=2 * np.pi / 3.0, Ly=1.0, dt=0.1, order=3, nq=8,
                                           nyquist=True, n_steps=250), 1024, 0.2, 1e-3)


def two_stream_particles(Lx, Ly, Lz, nb, v0, eps, n0=1.0):
    """Quiet-start cold beams at +-v0 on the same displaced positions:
    n = n0 (1 + eps cos(k (x + L/2))) to first order."""
    k = 2 * np.pi / Lx
    x0 = -Lx / 2 + (np.arange(nb) + 0.5) * Lx / nb
    xi = -(eps / k) * np.sin(k * (x0 + Lx / 2))
    n = 2 * nb
    x = np.zeros((n, 3))
    x[:, 0] = np.concatenate([x0 + xi, x0 + xi])
    v = np.zeros((n, 3))
    v[:nb, 0], v[nb:, 0] = v0, -v0
    q = np.full(n, -n0 * Lx * Ly * Lz / n)
    return x, v, q, np.abs(q)


def p3_long_main(lib=None):
    """Fixture of a long reference run (diagnostics of every step) whose
    linear growth rate, energy drift and gauge residual the GPU run must
    reproduce."""
    lib = lib or ol.ref_p3()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p3.so missing: run make -C oracle")
    name, kw, nb, v0, eps = P3_LONG_CASE
    prob = ol.P3Problem(**kw)
    x, v, q, m = two_stream_particles(prob.Lx, prob.Ly, prob.Lz, nb, v0, eps)
    out = ol.p3_run(lib.ref_p3_run, prob, x, v, q, m)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), dparams=prob.dparams(), iparams=prob.iparams(),
                        in_x=x, in_v=v, in_q=q, in_m=m, diag=out["diag"], info=out["info"],
                        fields=out["fields"], seconds=out["seconds"])
    print(name, "seconds", out["seconds"], "iterations", out["info"][:, 0].sum())


# Full-length run of the CPU-runnable explicit configuration: 2D Weibel on a
# 64x64 grid over [0, 2 pi / 0.3)^2, 64 electrons per cell (262,144) from the
# workloads' seeded bi-Maxwellian (vth 0.02 c in x, 0.2 c in y), quadratic
# splines, BDF1 with the conserving charge update, dt 0.05, 1000 steps.  Only
# the diagnostics rows (energy history, gauge / Gauss / continuity residuals,
# |B_z|) and the final fields are kept; the particles are regenerated from
# the seed (the generator is checked bit for bit in the CPU tests).
P2_LONG_CASE = dict(nx=64, ny=64, L=2 * np.pi / 0.3, ppc=64, uth=(0.02, 0.2, 0.0), seed=2026, dt=0.05,
                    n_steps=1000)


def p2_long_main():
    lib = ol.ref_p2()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p2.so missing: run make -C oracle")
    c = P2_LONG_CASE
    p = ol.generate_bimaxwellian(c["nx"], c["ny"], c["L"], c["L"], c["ppc"], c["uth"], seed=c["seed"])
    parts = {"x": p["x"], "y": p["y"], "P": p["P"], "v": p["v"], "vprev": p["v_prev"], "q": p["q"], "m": p["m"]}
    prob = ol.P2Problem(c["nx"], c["ny"], c["L"], c["L"], c["dt"], 1, True, n_steps=c["n_steps"])
    out, diag, fields, secs = ol.simulate(lib.ref_p2_simulate, prob, parts)
    np.savez_compressed(os.path.join(HERE, "p2_weibel64_long.npz"), params=prob.params(), iparams=prob.iparams(),
                        ppc=c["ppc"], uth=np.array(c["uth"]), seed=c["seed"], diag=diag, fields=fields,
                        out_v_checksum=np.array([out["v"].sum(), np.abs(out["v"]).sum()]), seconds=secs)
    print("p2_weibel64_long seconds", secs)


# Long implicit 2D Weibel run for the growth rate: a bi-Maxwellian hot along x
# (u_th = 0.3 c in x, 0.03 c in y, seeded), so that the Weibel modes have k
# along y (B_z(k_y), the mode Project3's diagnostics record); 16x16 grid over
# [0, 2 pi)^2, 64 electrons per cell (16,384); the manuscript deck's solver
# settings in 2D with its dt = 0.2, 200 steps: the magnetic field grows from
# the particle noise by about 30x in field energy between t = 10 and t = 24,
# then saturates.  Run on the OpenMP build of the reference
# (oracle/_ref/libref_p3_omp.so, the reference's own -fopenmp recipe) when it
# is present.
P3_WEIBEL_CASE = dict(nx=16, ny=16, L=2 * np.pi, ppc=64, uth=(0.3, 0.03, 0.0), seed=77, dt=0.2, n_steps=200)


def p3_weibel_particles(c):
    """Particles of P3_WEIBEL_CASE in Project3's box [-L/2, L/2): x (n, 3), v (n, 3), q, m."""
    p = ol.generate_bimaxwellian(c["nx"], c["ny"], c["L"], c["L"], c["ppc"], c["uth"], seed=c["seed"])
    n = len(p["x"])
    x = np.zeros((n, 3))
    x[:, 0] = p["x"] - c["L"] / 2
    x[:, 1] = p["y"] - c["L"] / 2
    return x, p["v"], p["q"], np.abs(p["q"])


def p3_weibel_main():
    omp = os.path.join(os.path.dirname(ol.REF_P3_SO), "libref_p3_omp.so")
    lib = ctypes.CDLL(omp) if os.path.exists(omp) else ol.ref_p3()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p3.so missing: run make -C oracle")
    c = P3_WEIBEL_CASE
    x, v, q, m = p3_weibel_particles(c)
    prob = ol.P3Problem(c["nx"], c["ny"], c["L"], c["L"], c["dt"], order=2, nq=8, n_steps=c["n_steps"])
    out = ol.p3_run(lib.ref_p3_run, prob, x, v, q, m)
    np.savez_compressed(os.path.join(HERE, "p3_weibel16_long.npz"), dparams=prob.dparams(), iparams=prob.iparams(),
                        ppc=c["ppc"], uth=np.array(c["uth"]), seed=c["seed"],
                        diag=out["diag"], info=out["info"], fields=out["fields"], seconds=out["seconds"],
                        threads=os.cpu_count() if os.path.exists(omp) else 1)
    print("p3_weibel16_long seconds", out["seconds"], "iterations", out["info"][:, 0].sum())


# Orbit kernels: (order, knot splitting, Gauss points)
P3_ORBIT_CASES = [(2, True, 8), (2, False, 8), (1, True, 4), (3, True, 6)]


def p3_orbit_main(lib):
    """Fixtures of the reference's orbit integrals path_average_deposit_current
    and path_average_gather_and_gradient on a 16x32 grid: 1000 orbits of up
    to ~3 cells (several knot crossings, the periodic seam), z components 0."""
    rng = np.random.default_rng(20261204)
    nx, ny, Lx, Ly = 16, 32, 5.0, 7.0
    n = 1000
    x0 = np.zeros((n, 3))
    x0[:, 0] = rng.uniform(-Lx / 2, Lx / 2, n)
    x0[:, 1] = rng.uniform(-Ly / 2, Ly / 2, n)
    p3_edge_positions(x0, Lx, Ly, nx, ny)
    vbar = rng.uniform(-0.9, 0.9, (n, 3)) / np.sqrt(3)
    dt = 2.5
    dx = dt * vbar
    dx[:, 2] = 0.0
    q = rng.uniform(-1.5, 0.5, n)
    N = nx * ny
    mesh = rng.normal(size=(3, N))
    An = rng.normal(size=(3, N))
    Anp1 = An + 0.1 * rng.normal(size=(3, N))
    out = {"x0": x0, "dx": dx, "vbar": vbar, "q": q, "mesh": mesh, "An": An, "Anp1": Anp1,
           "cases": np.array([[o, int(sp), nq] for o, sp, nq in P3_ORBIT_CASES]),
           "grid": np.array([nx, ny]), "box": np.array([Lx, Ly])}
    for k, (order, split, nq) in enumerate(P3_ORBIT_CASES):
        prob = ol.P3Problem(nx, ny, Lx, Ly, dt, order=order, nq=nq, split=split, nyquist=True)
        J = np.zeros(3 * N)
        lib.ref_p3_orbit_deposit(ol.ptr(prob.dparams()), ol.ptr(prob.iparams()), ctypes.c_long(n),
                                 ol.ptr(x0), ol.ptr(dx), ol.ptr(vbar), ol.ptr(q), ol.ptr(J))
        gat = np.zeros(3 * n)
        grad = np.zeros(9 * n)
        lib.ref_p3_orbit_gather(ol.ptr(prob.dparams()), ol.ptr(prob.iparams()), ctypes.c_long(n), ol.ptr(x0),
                                ol.ptr(dx), ol.ptr(np.ascontiguousarray(mesh)), ol.ptr(np.ascontiguousarray(An)),
                                ol.ptr(np.ascontiguousarray(Anp1)), ol.ptr(gat), ol.ptr(grad))
        out[f"J_{k}"] = J
        out[f"gathered_{k}"] = gat.reshape(n, 3)
        out[f"grad_{k}"] = grad.reshape(n, 3, 3)
    np.savez_compressed(os.path.join(HERE, "p3_orbit_kernels.npz"), **out)
    print("p3_orbit_kernels written")


def p3_main():
    """Fixtures of the implicit GM-HC-CN step from oracle/_ref/libref_p3.so."""
    lib = ol.ref_p3()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p3.so missing: run make -C oracle")
    p3_orbit_main(lib)
    for k, (name, kw, ppc, uth, two) in enumerate(P3_CASES):
        rng = np.random.default_rng(20261203 + k)
        prob = ol.P3Problem(**kw)
        x, v, q, m = ol.p3_particles(rng, prob.nx, prob.ny, ppc, prob.Lx, prob.Ly, uth=uth, Lz=prob.Lz)
        p3_edge_positions(x, prob.Lx, prob.Ly, prob.nx, prob.ny)
        if two:
            # every other particle a heavier positive species
            q[1::2] = -q[1::2]
            m[1::2] = 4.0 * m[1::2]
            v[1::2] *= 0.5
        out = ol.p3_run(lib.ref_p3_run, prob, x, v, q, m, want_step_diag=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dparams=prob.dparams(),
                            iparams=prob.iparams(), in_x=x, in_v=v, in_q=q, in_m=m,
                            **{"out_" + k: out[k] for k in ("x", "v", "P", "v_prev", "vbar")},
                            diag=out["diag"], info=out["info"], fields=out["fields"],
                            step_diag=out["step_diag"])
        print(name, "iterations", out["info"][:, 0].tolist())
    p3_fallback_main(lib)


def p3_fallback_main(lib=None):
    """Fixtures of implicit runs through the reference's selective particle
    sub-cycling fallback, with the sub-cycled step diagnostics
    (compute_subcycled_step_diagnostics) of each step."""
    lib = lib or ol.ref_p3()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p3.so missing: run make -C oracle")
    for k, (name, kw, ppc, uth, max_sub) in enumerate(P3_FALLBACK_CASES):
        rng = np.random.default_rng(20261220 + k)
        prob = ol.P3Problem(**kw)
        x, v, q, m = ol.p3_particles(rng, prob.nx, prob.ny, ppc, prob.Lx, prob.Ly, uth=uth, Lz=prob.Lz)
        lib.ref_p3_set_fallback(1, max_sub)
        try:
            out = ol.p3_run(lib.ref_p3_run, prob, x, v, q, m, want_step_diag=True)
            sel = np.zeros(4 * prob.n_steps)
            lib.ref_p3_selective_info(ol.ptr(sel), prob.n_steps)
        finally:
            lib.ref_p3_set_fallback(0, 64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dparams=prob.dparams(), iparams=prob.iparams(),
                            in_x=x, in_v=v, in_q=q, in_m=m, max_substeps=max_sub,
                            **{"out_" + c: out[c] for c in ("x", "v", "P", "v_prev", "vbar")},
                            diag=out["diag"], info=out["info"], fields=out["fields"],
                            selective=sel.reshape(prob.n_steps, 4), step_diag=out["step_diag"])
        print(name, "iterations", out["info"][:, 0].tolist(), "selective", sel.tolist())


# Non-relativistic implicit (Project1) runs: (name, problem keywords,
# particle source).  "ref": the reference's own initializer (two_stream or
# Landau); ("thermal", vth, nonuniform): seeded particles with thermal
# velocities in all three components, per-particle charges when nonuniform.
P1_CASES = [
    ("p1_run_landau_weak", dict(nx=32, ny=1, Lx=12.566370614359172, Ly=1.0, Lz=1.0, dt=0.1, order=1, nq=12,
                                picard_tol=1e-10, picard_maxit=24, n_steps=60, ppc=32, case="landau_weak",
                                landau_alpha=0.01, vth=1.0), "ref"),
    ("p1_run_landau_strong_o3", dict(nx=16, ny=2, Lx=12.566370614359172, Ly=1.0, Lz=1.0, dt=0.1, order=3,
                                     nq=12, picard_tol=1e-10, picard_maxit=30, n_steps=8, ppc=16,
                                     case="landau_strong", landau_alpha=0.5, vth=1.0), "ref"),
    ("p1_run_two_stream_o2", dict(nx=16, ny=8, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, dt=0.025, order=2,
                                  nq=16, n_steps=6, ppc=4, case="two_stream"), "ref"),
    ("p1_run_thermal_o2_nosplit", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, Lz=1.0, dt=0.1, order=2,
                                       nq=8, split=False, n_steps=4),
     ("thermal", (0.1, 0.1, 0.05), False)),
    ("p1_run_thermal_o1_weights", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=np.pi, Lz=0.5, dt=0.1, order=1, nq=6,
                                       n_steps=4), ("thermal", (0.2, 0.1, 0.1), True)),
    ("p1_run_o4_capped", dict(nx=8, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, dt=0.1, order=4, nq=8,
                              picard_maxit=3, sweep=False, n_steps=3), ("thermal", (0.05, 0.05, 0.0), False)),
]
# The reference embeds these 2D runs in 3D with nz = 1 and also splits orbits
# at z knots; the z spline is constant there, so that changes no integral,
# only the path statistics.  Runs with both knot splitting and z motion use
# orders whose z knots the particles do not reach (1 and 3), or vz = 0.


def p1_particles(rng, prob, vth, nonuniform, ppc=8):
    """Seeded particles on the Project1 box [-L/2, L/2) (z = 0): thermal
    velocities, charges summing to -n0 Lx Ly Lz, m = |q|."""
    n = prob.nx * prob.ny * ppc
    x = np.zeros((n, 3))
    x[:, 0] = rng.uniform(-prob.Lx / 2, prob.Lx / 2, n)
    x[:, 1] = rng.uniform(-prob.Ly / 2, prob.Ly / 2, n)
    p3_edge_positions(x, prob.Lx, prob.Ly, prob.nx, prob.ny)
    v = rng.normal(size=(n, 3)) * np.asarray(vth)
    w = rng.uniform(0.5, 1.5, n) if nonuniform else np.ones(n)
    q = -prob.n0 * prob.Lx * prob.Ly * prob.Lz * w / w.sum()
    return x, v, q, np.abs(q)


def p1_main():
    """Fixtures of the non-relativistic implicit Picard step from
    oracle/_ref/libref_p1.so, and the columns of the reference's shipped
    landau_weak run (Project1/output) that the harness reproduces."""
    lib = ol.ref_p1()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_p1.so missing: run make -C oracle")
    for k, (name, kw, src) in enumerate(P1_CASES):
        prob = ol.P1Problem(**kw)
        if src == "ref":
            x, v, q, m = ol.p1_init(lib, prob)
        else:
            x, v, q, m = p1_particles(np.random.default_rng(20261210 + k), prob, src[1], src[2])
        out = ol.p1_run(lib.ref_p1_run, prob, x, v, q, m)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dparams=prob.dparams(), iparams=prob.iparams(),
                            in_x=x, in_v=v, in_q=q, in_m=m,
                            **{"out_" + c: out[c] for c in ("x", "v", "P", "v_prev")},
                            diag=out["diag"], info=out["info"], fields=out["fields"], step_diag=out["step_diag"])
        print(name, len(q), "particles, iterations", out["info"][:, 0].astype(int).tolist())
    shipped = ref_path("Project1", "output", "landau_weak")
    with open(shipped + "_diagnostics.csv") as fh:
        rows = list(csv.reader(fh))
    with open(shipped + "_step_diagnostics.csv") as fh:
        srows = list(csv.reader(fh))
    # the shipped run is 300 steps long; the deck's first 60 are kept
    hdr, data = rows[0], rows[1:62]
    srows = srows[:61]
    info_cols = ["picard_iterations", "picard_current_error", "picard_velocity_error", "crossing_particles",
                 "avg_path_segments", "max_path_segments"]
    diag = np.array([[float(r[hdr.index(c)]) for c in ol.P1_DIAG_NAMES] for r in data])
    info = np.array([[float(r[hdr.index(c)]) for c in info_cols] for r in data[1:]])
    sdiag = np.array([[float(v) for v in r[2:]] for r in srows[1:]])
    np.savez_compressed(os.path.join(HERE, "p1_landau_weak_shipped.npz"), diag=diag, info=info,
                        step_diag=sdiag, diag_columns=np.array(ol.P1_DIAG_NAMES),
                        info_columns=np.array(info_cols), step_diag_columns=np.array(srows[0][2:]))
    print("p1_landau_weak_shipped written")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "p3":
        p3_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "p3_fallback":
        p3_fallback_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "p3_long":
        p3_long_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "p2_long":
        p2_long_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "p3_weibel":
        p3_weibel_main()
    elif len(sys.argv) > 1 and sys.argv[1] == "p1":
        p1_main()
    else:
        main()
