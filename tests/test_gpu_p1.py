"""GPU parity of the non-relativistic implicit orbit-averaged path
(libupic.so, UPIC_METHOD_CN_ORBIT_NONREL) against runs of the reference's own
solver (Project1/ec_pic_serial_demo.cpp picard_step_orbit through
oracle/_ref/libref_p1.so), committed as tests/golden/p1_*.npz.  The
landau_weak fixture is itself pinned to the run the reference ships
(tests/test_oracle.py).

Both sides iterate the Picard map on the particle velocities until the
relative change of the current and of the velocities falls below picard_tol
(1e-10 or 1e-11), so a converged step agrees to well below that tolerance,
not to round-off: fields and particle arrays are bounded by TOL_STEP per step
in relative terms.  The capped case stops after a fixed number of
iterations on both sides.  Round-off-level columns (Gauss and gauge
residuals, mean charge, the A-chain residual) are compared in absolute terms
against TOL_ROUNDOFF."""
import os

import numpy as np
import pytest

import unstaggered_pic_b200 as up

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_STEP = 2e-10      # relative difference per step, fields and particle state
TOL_ROUNDOFF = 1e-12  # absolute, residual diagnostics at round-off level
CASES = ["p1_run_landau_weak", "p1_run_landau_strong_o3", "p1_run_two_stream_o2", "p1_run_thermal_o2_nosplit",
         "p1_run_thermal_o1_weights", "p1_run_o4_capped"]
FIELD_ORDER = ["phi", "psi", "rho", "Ax", "Ay", "Az", "Ux", "Uy", "Uz", "Jx", "Jy", "Jz"]
FAMILIES = {0: [0], 1: [1], 2: [2], 3: [3, 4, 5], 4: [3, 4, 5], 5: [3, 4, 5], 6: [6, 7, 8], 7: [6, 7, 8],
            8: [6, 7, 8], 9: [9, 10, 11], 10: [9, 10, 11], 11: [9, 10, 11]}
DIAG_IDX = [up.IMPLICIT_DIAG_COLUMNS.index(n) for n in up.NONREL_DIAG_COLUMNS]
INFO_IDX = [up.SOLVE_INFO_COLUMNS.index(n) for n in
            ("iterations", "picard_current_error", "picard_velocity_error", "crossing_particles",
             "avg_path_segments", "max_path_segments")]
ROUNDOFF_DIAG = ("gauss_rms", "gauss_max", "gauge_rms", "mean_rho")


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)


def family_err(fields, ref, k):
    scale = max(np.max(np.abs(ref[j])) for j in FAMILIES[k])
    d = np.max(np.abs(np.asarray(fields[k]) - ref[k]))
    return float(d / scale) if scale > 0 else float(d)


def periodic_err(a, b, L):
    d = np.asarray(a) - np.asarray(b)
    d -= L * np.round(d / L)
    return float(np.max(np.abs(d))) if d.size else 0.0


def config_from(dp, ip):
    """NonrelConfig of a fixture's (dparams, iparams) (oracle_lib.P1Problem layout)."""
    assert int(ip[2]) == 1  # 2D runs (nz = 1)
    return up.NonrelConfig(nx=int(ip[0]), ny=int(ip[1]), Lx=dp[0], Ly=dp[1], Lz=dp[2], dt=dp[3], c=dp[4],
                           eps0=dp[5], mu0=dp[6], n0=dp[7], spline_order=int(ip[3]), orbit_quad_order=int(ip[4]),
                           split_orbit_at_knots=bool(ip[5]), picard_tol=dp[8], picard_max_iter=int(ip[6]),
                           final_consistency_sweep=bool(ip[7]), perturbation_mode=int(ip[9]))


def load_sim(g):
    cfg = config_from(g["dparams"], g["iparams"])
    sim = up.Simulation(cfg)
    x, v = g["in_x"], g["in_v"]
    n = len(g["in_q"])
    sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
    return sim, cfg


def compare_diag(row, ref, tol):
    """row: the 23-column implicit row; ref: Project1's 11 columns."""
    p1 = row[DIAG_IDX]
    e_abs = abs(ref[up.NONREL_DIAG_COLUMNS.index("E_mode_abs")])
    for k, name in enumerate(up.NONREL_DIAG_COLUMNS):
        a, b = p1[k], ref[k]
        if name in ROUNDOFF_DIAG:
            assert abs(a - b) < TOL_ROUNDOFF, (name, a, b)
        else:
            scale = max(abs(b), e_abs) if name.startswith("E_mode") else abs(b)
            assert abs(a - b) <= tol * scale + 1e-15, (name, a, b)


def compare_info(info, ref, tol_picard, capped):
    """Picard iterations, last errors and path statistics of each step."""
    mine = info[:, INFO_IDX]
    for s in range(len(ref)):
        it, cur, vel, cross, avg, mx = mine[s]
        rit, rcur, rvel, rcross, ravg, rmx = ref[s]
        assert abs(it - rit) <= (0 if capped else 1), (s, it, rit)
        if capped:
            # the same iterates on both sides: the errors are differences of
            # nearby iterates, equal to a relative 1e-6 of themselves
            assert abs(cur - rcur) <= 1e-6 * abs(rcur) + 1e-14, (s, cur, rcur)
            assert abs(vel - rvel) <= 1e-6 * abs(rvel) + 1e-14, (s, vel, rvel)
        else:
            assert max(cur, vel) < tol_picard and max(rcur, rvel) < tol_picard, (s, cur, vel, rcur, rvel)
        assert abs(cross - rcross) <= 1, (s, cross, rcross)
        assert mx == rmx, (s, mx, rmx)


@pytest.mark.parametrize("case", CASES)
def test_nonrel_run_matches_reference(case):
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    sim, cfg = load_sim(g)
    nsteps = int(g["iparams"][8])
    capped = not bool(g["iparams"][7])
    try:
        row0 = sim.init_fields()
        compare_diag(row0, g["diag"][0], 1e-12)
        diag, info, sd = sim.step_implicit(nsteps, step_diagnostics=True)
        for s in range(nsteps):
            compare_diag(diag[s], g["diag"][s + 1], TOL_STEP * (s + 1))
        compare_info(info, g["info"], cfg.picard_tol, capped)
        tol = TOL_STEP * nsteps
        fields = np.stack([sim.field(f) for f in FIELD_ORDER])
        ref_fields = g["fields"]
        for k, f in enumerate(FIELD_ORDER):
            err = family_err(fields, ref_fields, k)
            assert err < tol, (f, err)
        p = sim.get_particles()
        assert periodic_err(p["x"], g["out_x"][:, 0], cfg.Lx) < tol * cfg.Lx
        assert periodic_err(p["y"], g["out_x"][:, 1], cfg.Ly) < tol * cfg.Ly
        assert relerr(p["v"], g["out_v"]) < tol
        assert relerr(p["P"], g["out_P"]) < tol
        assert relerr(p["v_prev"], g["out_v_prev"]) < tol
        # step diagnostics (compute_step_diagnostics, ec_pic_serial_demo.cpp:1384)
        ref = g["step_diag"]
        npart = len(g["in_q"])
        for s in range(nsteps):
            for k, name in enumerate(up.STEP_DIAG_COLUMNS):
                a, b = sd[s, k], ref[s, k]
                if name in ("crossing_particles", "total_crossings"):
                    assert abs(a - b) <= 1, (s, name, a, b)
                elif name == "avg_path_segments":
                    assert abs(a - b) <= 1.0 / npart + 1e-15, (s, name, a, b)
                elif name == "max_path_segments":
                    assert a == b, (s, name, a, b)
                elif abs(b) < 1e-10:
                    assert abs(a - b) < TOL_ROUNDOFF, (s, name, a, b)
                else:
                    assert abs(a - b) <= TOL_STEP * (s + 1) * abs(b) + TOL_ROUNDOFF, (s, name, a, b)
    finally:
        sim.close()


def test_nonrel_energy_conserved_and_deterministic():
    """The converged knot-split scheme conserves total energy to round-off
    (the reference's landau_weak run holds it to 1e-15), and two runs from
    the same input are bitwise equal."""
    g = dict(np.load(os.path.join(GOLD, "p1_run_landau_weak.npz")))
    results = []
    for _ in range(2):
        sim, _ = load_sim(g)
        try:
            row0 = sim.init_fields()
            diag, info = sim.step_implicit(20)
            results.append((row0, diag, sim.field("Ax"), sim.get_particles()["v"]))
        finally:
            sim.close()
    row0, diag, ax, v = results[0]
    col = up.IMPLICIT_DIAG_COLUMNS.index("total_energy")
    drift = np.abs(diag[:, col] - row0[col]) / row0[col]
    assert drift.max() < 1e-12, drift.max()
    assert np.array_equal(results[1][1], diag)
    assert np.array_equal(results[1][2], ax)
    assert np.array_equal(results[1][3], v)


def test_nonrel_errors_and_empty():
    with pytest.raises(up.UpicError) as e:
        up.Simulation(up.NonrelConfig(nx=8, ny=8, picard_max_iter=0))
    assert e.value.code == -1
    for bad in (dict(c=0.0), dict(eps0=-1.0), dict(spline_order=5), dict(orbit_quad_order=33), dict(nx=12),
                dict(picard_tol=float("nan"))):
        kw = dict(nx=8, ny=8)
        kw.update(bad)
        with pytest.raises(up.UpicError) as e:
            up.Simulation(up.NonrelConfig(**kw))
        assert e.value.code == -1, bad
    cfg = up.NonrelConfig(nx=8, ny=8, dt=0.1)
    with up.Simulation(cfg) as sim:
        with pytest.raises(up.UpicError) as e:
            sim.init_fields()
        assert e.value.code == -4  # particles first
        sim.set_particles(np.zeros(0), np.zeros(0), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)),
                          np.zeros(0), np.zeros(0))
        sim.init_fields()
        diag, info = sim.step_implicit(2)
        # zero current is a fixed point: the second iterate meets the tolerance
        assert np.all(info[:, up.SOLVE_INFO_COLUMNS.index("iterations")] == 2)
        assert np.all(sim.field("phi") == 0.0)
    # speeds above c are allowed (non-relativistic method)
    g = dict(np.load(os.path.join(GOLD, "p1_run_two_stream_o2.npz")))
    cfg = config_from(g["dparams"], g["iparams"])
    with up.Simulation(cfg) as sim:
        n = 64
        rng = np.random.default_rng(3)
        x = rng.uniform(-cfg.Lx / 2, cfg.Lx / 2, n)
        y = rng.uniform(-cfg.Ly / 2, cfg.Ly / 2, n)
        v = np.zeros((n, 3))
        v[:, 0] = 1.5
        sim.set_particles(x, y, np.zeros((n, 3)), v, v, -np.ones(n) / n, np.ones(n) / n)
        sim.init_fields()
        diag, info = sim.step_implicit(1)
        assert np.all(np.isfinite(diag))
