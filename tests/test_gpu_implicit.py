"""GPU parity of the implicit orbit-averaged GM-HC-CN path (libupic.so,
UPIC_METHOD_CN_ORBIT) against runs of the reference's own solver
(Project3/ec_pic_nyquist_projected.cpp through oracle/_ref/libref_p3.so),
committed as tests/golden/p3_*.npz.

Both sides iterate the outer current map to the same mixed tolerance
(nonlinear_rtol 1e-11, nonlinear_atol 1e-13) and the particle map to
1e-12/1e-14, so a converged step agrees to about that tolerance, not to
round-off: the tests bound the relative difference of every field and
particle array by TOL_STEP per step taken.  Round-off-level diagnostics (Gauss
and gauge residuals) are compared in absolute terms against TOL_ROUNDOFF."""
import ctypes
import os

import numpy as np
import pytest

import oracle_lib as ol
import unstaggered_pic_b200 as up

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_STEP = 2e-10      # relative difference per step, fields and particle state
TOL_ROUNDOFF = 1e-12  # absolute, residual diagnostics at round-off level
CASES = ["p3_run_o2_anderson", "p3_run_o3_picard", "p3_run_o1_nosplit", "p3_run_o4",
         "p3_run_two_species", "p3_run_1d_o3"]
FIELD_ORDER = ["phi", "psi", "rho", "Ax", "Ay", "Az", "Ux", "Uy", "Uz", "Jx", "Jy", "Jz"]


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b))
    if scale == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / scale)


# Vector fields are compared against the magnitude of the whole vector: a
# component that is zero in exact arithmetic (A_z of a run with v_z = 0)
# holds only rounding noise on both sides.
FAMILIES = {0: [0], 1: [1], 2: [2], 3: [3, 4, 5], 4: [3, 4, 5], 5: [3, 4, 5], 6: [6, 7, 8], 7: [6, 7, 8],
            8: [6, 7, 8], 9: [9, 10, 11], 10: [9, 10, 11], 11: [9, 10, 11]}


def family_err(fields, ref, k):
    scale = max(np.max(np.abs(ref[j])) for j in FAMILIES[k])
    d = np.max(np.abs(np.asarray(fields[k]) - ref[k]))
    return float(d / scale) if scale > 0 else float(d)


def periodic_err(a, b, L):
    d = np.asarray(a) - np.asarray(b)
    d -= L * np.round(d / L)
    return float(np.max(np.abs(d)))


def config_from(dp, ip):
    """ImplicitConfig of a fixture's (dparams, iparams) (oracle_lib.P3Problem layout)."""
    return up.ImplicitConfig(
        nx=int(ip[0]), ny=int(ip[1]), Lx=dp[0], Ly=dp[1], Lz=dp[2], dt=dp[3], kappa=dp[4], sigma1=dp[5],
        sigma2=dp[6], n0=dp[7], spline_order=int(ip[3]), orbit_quad_order=int(ip[4]),
        split_orbit_at_knots=bool(ip[5]), nyquist_projection=bool(ip[6]),
        nonlinear_solver="picard" if ip[11] == 1 else "anderson", nonlinear_rtol=dp[8],
        nonlinear_atol=dp[9], nonlinear_max_iter=int(ip[7]), anderson_memory=int(ip[8]),
        anderson_start=int(ip[9]), anderson_damping=dp[10], anderson_regularization=dp[11],
        anderson_growth_limit=dp[12], uniform_local_rtol=dp[13], uniform_local_atol=dp[14],
        uniform_local_max_iter=int(ip[10]), uniform_local_damping=dp[15], perturbation_mode=int(ip[13]))


def load_sim(g):
    cfg = config_from(g["dparams"], g["iparams"])
    sim = up.Simulation(cfg)
    x, v = g["in_x"], g["in_v"]
    n = len(g["in_q"])
    sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
    return sim, cfg


def compare_diag(row, ref, nyquist, tol):
    names = up.IMPLICIT_DIAG_COLUMNS
    for k, name in enumerate(names):
        a, b = row[k], ref[k]
        roundoff = name in ("gauss_rms", "gauss_max", "gauge_rms", "gauge_max", "gauss_relative",
                            "gauge_relative", "mean_rho")
        if roundoff and (nyquist or abs(b) < 1e-9):
            assert abs(a - b) < TOL_ROUNDOFF * max(1.0, abs(b)) or abs(a) < 1e-11, (name, a, b)
        else:
            assert abs(a - b) <= tol * max(abs(b), 1e-300) + 1e-14, (name, a, b)


@pytest.mark.parametrize("case", CASES)
def test_implicit_run_matches_reference(case):
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    sim, cfg = load_sim(g)
    nsteps = int(g["iparams"][12])
    nyq = bool(g["iparams"][6])
    try:
        row0 = sim.init_fields()
        compare_diag(row0, g["diag"][0], nyq, 1e-12)
        diag, info = sim.step_implicit(nsteps)
        for s in range(nsteps):
            compare_diag(diag[s], g["diag"][s + 1], nyq, TOL_STEP * (s + 1))
        # same outer iteration path
        assert np.all(np.abs(info[:, 0] - g["info"][:, 0]) <= 1), (info[:, 0], g["info"][:, 0])
        assert np.all(info[:, 1] == 1.0)
        tol = TOL_STEP * nsteps
        fields = np.stack([sim.field(f) for f in FIELD_ORDER])
        for k, f in enumerate(FIELD_ORDER):
            err = family_err(fields, g["fields"], k)
            assert err < tol, (f, err)
        p = sim.get_particles()
        assert periodic_err(p["x"], g["out_x"][:, 0], cfg.Lx) < tol * cfg.Lx
        assert periodic_err(p["y"], g["out_x"][:, 1], cfg.Ly) < tol * cfg.Ly
        assert relerr(p["v"], g["out_v"]) < tol
        assert relerr(p["P"], g["out_P"]) < tol
        assert relerr(p["v_prev"], g["out_v_prev"]) < tol
    finally:
        sim.close()


def test_implicit_energy_conserved_and_deterministic():
    """Energy of the knot-split orbit-averaged scheme is conserved to the
    solver tolerance, and two runs from the same input are bitwise equal."""
    g = dict(np.load(os.path.join(GOLD, "p3_run_o2_anderson.npz")))
    results = []
    for _ in range(2):
        sim, _ = load_sim(g)
        try:
            row0 = sim.init_fields()
            diag, info = sim.step_implicit(6)
            results.append((row0, diag, sim.field("Jx"), sim.get_particles()["v"]))
        finally:
            sim.close()
    row0, diag, jx, v = results[0]
    e0 = row0[up.IMPLICIT_DIAG_COLUMNS.index("total_energy")]
    drift = np.abs(diag[:, up.IMPLICIT_DIAG_COLUMNS.index("total_energy")] - e0) / e0
    assert drift.max() < 1e-10
    assert np.array_equal(results[1][1], diag)
    assert np.array_equal(results[1][2], jx)
    assert np.array_equal(results[1][3], v)


def test_implicit_errors():
    g = dict(np.load(os.path.join(GOLD, "p3_run_o2_anderson.npz")))
    sim, cfg = load_sim(g)
    try:
        with pytest.raises(up.UpicError) as e:
            sim.step_implicit(1)
        assert e.value.code == -4  # UPIC_ERR_STATE: init_fields first
        sim.init_fields()
        with pytest.raises(up.UpicError) as e:
            sim.step(1)
        assert e.value.code == -4  # the explicit step on an implicit context
        # superluminal input velocity (gamma_from_v throws in the reference)
        n = 4
        with pytest.raises(up.UpicError) as e:
            sim.set_particles(np.zeros(n), np.zeros(n), np.zeros((n, 3)), np.full((n, 3), 0.6),
                              np.zeros((n, 3)), -np.ones(n), np.ones(n))
        assert e.value.code == -8
    finally:
        sim.close()
    # a local solve that cannot converge in one iteration fails loudly
    cfg.uniform_local_max_iter = 1
    sim = up.Simulation(cfg)
    try:
        x, v = g["in_x"], g["in_v"]
        n = len(g["in_q"])
        sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
        sim.init_fields()
        with pytest.raises(up.UpicError) as e:
            sim.step_implicit(1)
        assert e.value.code == -7  # UPIC_ERR_LOCAL_PARTICLE
        assert "maximum_iterations" in str(e.value)
    finally:
        sim.close()


def test_implicit_empty_and_bad_config():
    cfg = up.ImplicitConfig(nx=8, ny=8, dt=0.1)
    sim = up.Simulation(cfg)
    try:
        sim.set_particles(np.zeros(0), np.zeros(0), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)),
                          np.zeros(0), np.zeros(0))
        row0 = sim.init_fields()
        diag, info = sim.step_implicit(2)
        assert np.all(sim.field("phi") == 0.0)
        assert info[0, 0] == 1  # the zero current is a fixed point
    finally:
        sim.close()
    for bad in (dict(spline_order=5), dict(orbit_quad_order=0), dict(anderson_memory=5), dict(nx=12),
                dict(kappa=0.0)):
        kw = dict(nx=8, ny=8, dt=0.1)
        kw.update(bad)
        with pytest.raises(up.UpicError) as e:
            up.Simulation(up.ImplicitConfig(**kw))
        assert e.value.code == -1


@pytest.mark.skipif(not os.path.exists(ol.REF_P3_SO), reason="oracle/_ref/libref_p3.so not built")
def test_implicit_larger_case_against_reference_build():
    """A 32x32 grid, 16 particles per cell, 3 steps, compared with the
    reference build directly (when oracle/_ref travels with the tree)."""
    rng = np.random.default_rng(7)
    prob = ol.P3Problem(32, 32, 2 * np.pi / 0.3, 2 * np.pi / 0.3, 0.05, order=2, nq=8, n_steps=3)
    x, v, q, m = ol.p3_particles(rng, 32, 32, 16, prob.Lx, prob.Ly, uth=(0.02, 0.2, 0.0), Lz=prob.Lz)
    ref = ol.p3_run(ol.ref_p3().ref_p3_run, prob, x, v, q, m)
    g = {"dparams": prob.dparams(), "iparams": prob.iparams(), "in_x": x, "in_v": v, "in_q": q, "in_m": m}
    sim, cfg = load_sim(g)
    try:
        sim.init_fields()
        diag, info = sim.step_implicit(3)
        for s in range(3):
            compare_diag(diag[s], ref["diag"][s + 1], True, TOL_STEP * (s + 1))
        fields = np.stack([sim.field(f) for f in FIELD_ORDER])
        for k, f in enumerate(FIELD_ORDER):
            assert family_err(fields, ref["fields"], k) < 3 * TOL_STEP, f
    finally:
        sim.close()


ORBIT = dict(np.load(os.path.join(GOLD, "p3_orbit_kernels.npz")))
TOL_ONE = 1e-13  # one kernel-level orbit integral, relative to the field's max magnitude


@pytest.mark.parametrize("k", range(len(ORBIT["cases"])))
def test_orbit_kernels_match_reference(k):
    """upic_orbit_deposit / upic_orbit_gather against the reference's
    path_average_deposit_current and path_average_gather_and_gradient on
    orbits that cross several knots and the periodic seam."""
    g = ORBIT
    order, split, nq = (int(v) for v in g["cases"][k])
    nx, ny = (int(v) for v in g["grid"])
    Lx, Ly = (float(v) for v in g["box"])
    cfg = up.ImplicitConfig(nx=nx, ny=ny, Lx=Lx, Ly=Ly, Lz=1.0, dt=2.5, spline_order=order, orbit_quad_order=nq,
                            split_orbit_at_knots=bool(split), nyquist_projection=True)
    with up.Simulation(cfg) as sim:
        x0 = g["x0"]
        J = sim.orbit_deposit(x0[:, 0], x0[:, 1], g["dx"], g["vbar"], g["q"])
        assert relerr(J.ravel(), g[f"J_{k}"]) < TOL_ONE
        gat, grad = sim.orbit_gather(x0[:, 0], x0[:, 1], g["dx"], g["mesh"], g["An"], g["Anp1"])
        assert relerr(gat, g[f"gathered_{k}"]) < TOL_ONE
        assert relerr(grad, g[f"grad_{k}"]) < TOL_ONE
        # a second call on the same context reuses its staging buffers
        J2 = sim.orbit_deposit(x0[:, 0], x0[:, 1], g["dx"], g["vbar"], g["q"])
        assert np.array_equal(J, J2)
        # no orbits: zero current
        Z = sim.orbit_deposit(np.zeros(0), np.zeros(0), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0))
        assert np.all(Z == 0.0)


def compare_step_diag(sd, ref, np_):
    """Step diagnostics rows against the reference's: crossing counts within
    one (a path exactly on a knot), the largest path exactly, round-off
    residuals absolutely, the rest to the step tolerance."""
    for s in range(len(ref)):
        for k, name in enumerate(up.STEP_DIAG_COLUMNS):
            a, b = sd[s, k], ref[s, k]
            if name in ("crossing_particles", "total_crossings"):
                assert abs(a - b) <= 1, (s, name, a, b)
            elif name == "avg_path_segments":
                assert abs(a - b) <= 1.0 / np_ + 1e-15, (s, name, a, b)
            elif name == "max_path_segments":
                assert a == b, (s, name, a, b)
            elif abs(b) < 1e-10:
                assert abs(a - b) < TOL_ROUNDOFF, (s, name, a, b)  # round-off residuals
            else:
                assert abs(a - b) <= TOL_STEP * (s + 1) * abs(b) + TOL_ROUNDOFF, (s, name, a, b)


@pytest.mark.parametrize("case", CASES)
def test_step_diagnostics_match_reference(case):
    """upic_step_implicit's step diagnostics against the reference's
    compute_step_diagnostics of the same steps: the work/energy balances,
    the A-chain residual and the knot-crossing statistics."""
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    sim, cfg = load_sim(g)
    nsteps = int(g["iparams"][12])
    np_ = len(g["in_q"])
    try:
        sim.init_fields(diagnostics=False)  # energies of the start state computed on demand
        _, info, sd = sim.step_implicit(nsteps, diagnostics=False, step_diagnostics=True)
        assert sd.shape == (nsteps, len(up.STEP_DIAG_COLUMNS))
        compare_step_diag(sd, g["step_diag"], np_)
    finally:
        sim.close()


def test_extrapolated_predictor_same_solution():
    """current_predictor = extrapolated (2 J^n - J^(n-1)) converges to the
    reference's solution at the same tolerances, in no more outer
    iterations over the run than the reference's previous-current guess."""
    g = dict(np.load(os.path.join(GOLD, "p3_run_o2_anderson.npz")))
    nsteps = int(g["iparams"][12])
    nyq = bool(g["iparams"][6])
    iters = {}
    for pred in ("previous", "extrapolated"):
        cfg = config_from(g["dparams"], g["iparams"])
        cfg.current_predictor = pred
        sim = up.Simulation(cfg)
        x, v = g["in_x"], g["in_v"]
        n = len(g["in_q"])
        sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
        try:
            sim.init_fields()
            diag, info = sim.step_implicit(nsteps)
            for s in range(nsteps):
                compare_diag(diag[s], g["diag"][s + 1], nyq, TOL_STEP * (s + 1))
            fields = np.stack([sim.field(f) for f in FIELD_ORDER])
            for k, f in enumerate(FIELD_ORDER):
                assert family_err(fields, g["fields"], k) < TOL_STEP * nsteps, f
            iters[pred] = info[:, 0]
        finally:
            sim.close()
    assert iters["extrapolated"][0] == iters["previous"][0]  # no history on the first step
    assert iters["extrapolated"].sum() <= iters["previous"].sum(), iters


@pytest.mark.parametrize("case", ["p3_run_o2_anderson", "p3_run_o3_picard", "p3_run_two_species"])
def test_local_warm_start_same_solution(case):
    """local_warm_start = 1 (each local fixed point starts from the previous
    map evaluation's orbit velocity) converges to the reference's solution at
    the same tolerances with fewer local iterations."""
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    nsteps = int(g["iparams"][12])
    nyq = bool(g["iparams"][6])
    local = {}
    for warm in (False, True):
        cfg = config_from(g["dparams"], g["iparams"])
        cfg.local_warm_start = warm
        sim = up.Simulation(cfg)
        x, v = g["in_x"], g["in_v"]
        n = len(g["in_q"])
        sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
        try:
            sim.init_fields()
            diag, info = sim.step_implicit(nsteps)
            for s in range(nsteps):
                compare_diag(diag[s], g["diag"][s + 1], nyq, TOL_STEP * (s + 1))
            fields = np.stack([sim.field(f) for f in FIELD_ORDER])
            for k, f in enumerate(FIELD_ORDER):
                assert family_err(fields, g["fields"], k) < TOL_STEP * nsteps, f
            p = sim.get_particles()
            assert relerr(p["v"], g["out_v"]) < TOL_STEP * nsteps
            local[warm] = info[:, up.SOLVE_INFO_COLUMNS.index("local_particle_iterations_mean")]
        finally:
            sim.close()
    # the final consistency evaluation's mean local iterations drop
    assert np.all(local[True] < local[False]), local


FALLBACK_CASES = ["p3_fallback_few", "p3_fallback_some", "p3_fallback_many_o3"]


@pytest.mark.parametrize("case", FALLBACK_CASES)
def test_selective_fallback_matches_reference(case):
    """Runs where some particles' local solves fail over the full dt: with
    selective_particle_fallback the failing particles are sub-cycled (2, 4,
    ... substeps) and the outer solve restarts, as the reference's
    nonlinear_step_selective_particle_fallback does; the same particles are
    refined the same number of times, the state agrees to the solver
    tolerance, and the step diagnostics follow the reference's sub-cycled
    form (one A-chain term per sub-orbit, grid work of the accepted current)."""
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    cfg = config_from(g["dparams"], g["iparams"])
    cfg.selective_particle_fallback = True
    cfg.selective_particle_max_substeps = int(g["max_substeps"])
    nsteps = int(g["iparams"][12])
    sim, _ = None, None
    sim = up.Simulation(cfg)
    x, v = g["in_x"], g["in_v"]
    n = len(g["in_q"])
    sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
    cols = up.SOLVE_INFO_COLUMNS
    try:
        sim.init_fields()
        diag, info, sd = sim.step_implicit(nsteps, step_diagnostics=True)
        for s in range(nsteps):
            compare_diag(diag[s], g["diag"][s + 1], True, TOL_STEP * (s + 1))
        sel = g["selective"]
        got = info[:, [cols.index(c) for c in ("selective_fallback_used", "selective_refinement_restarts",
                                               "selective_refined_particles", "selective_total_particle_substeps")]]
        assert np.array_equal(got, sel), (got, sel)
        assert np.all(np.abs(info[:, 0] - g["info"][:, 0]) <= 1), (info[:, 0], g["info"][:, 0])
        compare_step_diag(sd, g["step_diag"], n)
        tol = TOL_STEP * nsteps
        fields = np.stack([sim.field(f) for f in FIELD_ORDER])
        for k, f in enumerate(FIELD_ORDER):
            assert family_err(fields, g["fields"], k) < tol, (f, family_err(fields, g["fields"], k))
        p = sim.get_particles()
        assert periodic_err(p["x"], g["out_x"][:, 0], cfg.Lx) < tol * cfg.Lx
        assert periodic_err(p["y"], g["out_x"][:, 1], cfg.Ly) < tol * cfg.Ly
        assert relerr(p["v"], g["out_v"]) < tol
        assert relerr(p["P"], g["out_P"]) < tol
        assert relerr(p["v_prev"], g["out_v_prev"]) < tol
    finally:
        sim.close()


def test_selective_fallback_limits():
    """Without the fallback a failing local solve ends the step
    (UPIC_ERR_LOCAL_PARTICLE); with max_substeps = 1 nothing can be refined
    and the step fails as the reference's exhausted fallback does."""
    g = dict(np.load(os.path.join(GOLD, "p3_fallback_some.npz")))
    x, v = g["in_x"], g["in_v"]
    n = len(g["in_q"])
    for fallback, maxsub, code, text in ((False, 64, -7, "local particle solve failed"),
                                         (True, 1, -6, "selective particle fallback reached h=dt/1")):
        cfg = config_from(g["dparams"], g["iparams"])
        cfg.selective_particle_fallback = fallback
        cfg.selective_particle_max_substeps = maxsub
        with up.Simulation(cfg) as sim:
            sim.set_particles(x[:, 0], x[:, 1], np.zeros((n, 3)), v, v, g["in_q"], g["in_m"])
            sim.init_fields()
            with pytest.raises(up.UpicError) as e:
                sim.step_implicit(1)
            assert e.value.code == code and text in str(e.value), str(e.value)
    with pytest.raises(up.UpicError) as e:
        up.Simulation(up.ImplicitConfig(nx=8, ny=8, selective_particle_fallback=True,
                                        selective_particle_max_substeps=3))
    assert e.value.code == -1


def growth_fit(amp, dt, lo, hi):
    """Least-squares slope of log(amp) against time over the steps where
    lo <= amp <= hi (the linear phase), and that window."""
    idx = np.nonzero((amp >= lo) & (amp <= hi))[0]
    t = idx * dt
    return np.polyfit(t, np.log(amp[idx]), 1)[0], idx


def test_two_stream_growth_matches_reference():
    """A long run (250 steps, about ten e-foldings into saturation) of the
    1D-2V cold relativistic two-stream instability against the reference's
    run on the same quiet start: the linear growth rate of |E_x(k_x = 1)|
    within 2%, the mode amplitude through the linear phase, and the energy
    drift and gauge residual of every step at the reference's level."""
    g = dict(np.load(os.path.join(GOLD, "p3_two_stream_long.npz")))
    sim, cfg = load_sim(g)
    nsteps = int(g["iparams"][12])
    cols = up.IMPLICIT_DIAG_COLUMNS
    try:
        row0 = sim.init_fields()
        diag, info = sim.step_implicit(nsteps)
    finally:
        sim.close()
    assert np.all(info[:, 1] == 1.0)
    ours = np.vstack([row0, diag])
    ref = g["diag"]
    k = cols.index("E_mode_abs")
    a_ref, a_gpu = ref[:, k], ours[:, k]
    # linear phase: from 4x the seeded amplitude (past the beat of the
    # excited modes) to half the final amplitude (before saturation)
    lo, hi = 4 * a_ref[0], 0.5 * a_ref.max()
    rate_ref, idx = growth_fit(a_ref, cfg.dt, lo, hi)
    rate_gpu, idx_gpu = growth_fit(a_gpu, cfg.dt, lo, hi)
    assert len(idx) >= 50 and np.all(np.diff(idx) == 1), idx
    assert np.array_equal(idx, idx_gpu)
    assert abs(rate_gpu - rate_ref) <= 0.02 * abs(rate_ref), (rate_gpu, rate_ref)
    # and the cold-beam dispersion relation 1 = wb^2/(w - k v0)^2 + wb^2/(w + k v0)^2,
    # wb^2 = (n0/2)/gamma0^3 (longitudinal mass), is met to 3%
    v0, k = 0.2, 2 * np.pi / cfg.Lx
    wb2, kv = 0.5 * (1 - v0 * v0) ** 1.5, k * v0
    w2 = np.roots([1.0, -(2 * kv * kv + 2 * wb2), kv ** 4 - 2 * wb2 * kv * kv])
    rate_theory = np.sqrt(-np.min(w2.real))
    assert abs(rate_gpu - rate_theory) <= 0.03 * rate_theory, (rate_gpu, rate_theory)
    # through the linear phase the amplitudes themselves agree closely
    lin = np.arange(idx[-1] + 1)
    assert np.max(np.abs(a_gpu[lin] - a_ref[lin]) / a_ref[lin]) < 1e-6
    # energy drift and gauge residual of every step at the reference's level
    e = cols.index("total_energy")
    drift_ref = np.abs(ref[:, e] - ref[0, e]) / ref[0, e]
    drift_gpu = np.abs(ours[:, e] - ours[0, e]) / ours[0, e]
    assert drift_gpu.max() <= max(10 * drift_ref.max(), 1e-12), (drift_gpu.max(), drift_ref.max())
    gg = cols.index("gauge_relative")
    assert np.max(ours[:, gg]) <= max(10 * np.max(ref[:, gg]), 1e-12), (np.max(ours[:, gg]), np.max(ref[:, gg]))


@pytest.mark.parametrize("order,split", [(1, True), (2, True), (2, False), (3, True), (4, True)])
def test_orbit_deposit_gather_adjoint(order, split):
    """The orbit current deposit and the orbit field gather use the same
    weights, so the particle power sum_p q vbar . <E S> equals the mesh
    power dV sum_nodes J . E to round-off (the reference's known-answer test
    test_orbit_deposit_gather_adjointness, threshold 5e-14)."""
    rng = np.random.default_rng(23 + order)
    nx = ny = 8
    L, dt, n = 2 * np.pi, 0.2, 64
    cfg = up.ImplicitConfig(nx=nx, ny=ny, Lx=L, Ly=L, Lz=L, dt=dt, spline_order=order, orbit_quad_order=18,
                            split_orbit_at_knots=split, nyquist_projection=False)
    x0 = rng.uniform(-0.5, 0.5, (n, 2)) * L
    vbar = rng.normal(size=(n, 3)) * np.array([0.35, 0.2, 0.15])
    dx = dt * vbar
    q = 0.1 * rng.normal(size=n)
    E = rng.normal(size=(3, nx * ny))
    with up.Simulation(cfg) as sim:
        J = sim.orbit_deposit(x0[:, 0], x0[:, 1], dx, vbar, q).reshape(3, -1)
        Ebar, _ = sim.orbit_gather(x0[:, 0], x0[:, 1], dx, E, E, E)
    dV = (L / nx) * (L / ny) * L
    particle = float(np.sum(q * np.sum(vbar * Ebar, axis=1)))
    mesh = float(np.sum(J * E)) * dV
    scale = abs(particle) + abs(mesh) + 1.0
    assert abs(particle - mesh) / scale < 5e-14, (particle, mesh)
