"""GPU tests of checkpoint / restart (upic_save_state, upic_load_state): a run
saved after K steps and restored into a fresh context continues bit for bit
as the uninterrupted run does, for the explicit BDF method (with a re-sort
inside the continued window and a fixed background), the implicit GM-HC-CN
method and the non-relativistic Picard method."""
import os

import numpy as np
import pytest

import unstaggered_pic_b200 as up

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ["phi", "Ax", "Ay", "Az", "rho", "Jx", "Jy", "Jz"]


def explicit_config(**kw):
    args = dict(nx=32, ny=32, Lx=2 * np.pi / 0.3, Ly=2 * np.pi / 0.3, dt=0.05, method="bdf2")
    args.update(kw)
    return up.Config(**args)


def load_explicit(sim, cfg, seed=5, ppc=8):
    p = up.generate_bimaxwellian(cfg.nx, cfg.ny, cfg.Lx, cfg.Ly, ppc, (0.02, 0.2, 0.05), seed=seed)
    sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])


def snapshot(sim, fields):
    part = sim.get_particles()
    return {**{k: v.copy() for k, v in part.items()}, **{f: sim.field(f).copy() for f in fields}}


def assert_same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("charge", ["conserving", "naive"])
def test_explicit_restart_is_bitwise(tmp_path, charge):
    cfg = explicit_config(charge_update=charge)
    path = str(tmp_path / "state.bin")
    bg = None
    if charge == "naive":
        rng = np.random.default_rng(3)
        bg = 1.0 + 0.01 * rng.normal(size=(cfg.nx, cfg.ny))
    with up.Simulation(cfg) as sim:
        load_explicit(sim, cfg)
        if bg is not None:
            sim.set_background(bg)
        sim.init_fields()
        sim.step(7)            # particles re-sorted every 4 steps: the continued window re-sorts too
        sim.save_state(path)
        rows_a = sim.step(6)
        snap_a = snapshot(sim, FIELDS)
    with up.Simulation(cfg) as sim:
        sim.load_state(path)
        assert sim.np == len(snap_a["x"])
        rows_b = sim.step(6)
        snap_b = snapshot(sim, FIELDS)
    assert np.array_equal(rows_a, rows_b, equal_nan=True)
    assert_same(snap_a, snap_b)


def implicit_sim(case):
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    dp, ip = g["dparams"], g["iparams"]
    if case.startswith("p1_"):
        cfg = up.NonrelConfig(nx=int(ip[0]), ny=int(ip[1]), Lx=dp[0], Ly=dp[1], Lz=dp[2], dt=dp[3], c=dp[4],
                              eps0=dp[5], mu0=dp[6], n0=dp[7], spline_order=int(ip[3]),
                              orbit_quad_order=int(ip[4]), split_orbit_at_knots=bool(ip[5]), picard_tol=dp[8],
                              picard_max_iter=int(ip[6]), final_consistency_sweep=bool(ip[7]),
                              perturbation_mode=int(ip[9]))
    else:
        cfg = up.ImplicitConfig(
            nx=int(ip[0]), ny=int(ip[1]), Lx=dp[0], Ly=dp[1], Lz=dp[2], dt=dp[3], kappa=dp[4], sigma1=dp[5],
            sigma2=dp[6], n0=dp[7], spline_order=int(ip[3]), orbit_quad_order=int(ip[4]),
            split_orbit_at_knots=bool(ip[5]), nyquist_projection=bool(ip[6]),
            nonlinear_solver="picard" if ip[11] == 1 else "anderson", nonlinear_rtol=dp[8],
            nonlinear_atol=dp[9], nonlinear_max_iter=int(ip[7]), anderson_memory=int(ip[8]),
            anderson_start=int(ip[9]), anderson_damping=dp[10], anderson_regularization=dp[11],
            anderson_growth_limit=dp[12], uniform_local_rtol=dp[13], uniform_local_atol=dp[14],
            uniform_local_max_iter=int(ip[10]), uniform_local_damping=dp[15], perturbation_mode=int(ip[13]))
    return g, cfg


@pytest.mark.parametrize("case", ["p3_run_two_species", "p1_run_thermal_o1_weights"])
def test_implicit_restart_is_bitwise(tmp_path, case):
    g, cfg = implicit_sim(case)
    n = len(g["in_q"])
    path = str(tmp_path / "state.bin")
    fields = FIELDS + ["psi", "Ux", "Uy", "Uz"]
    with up.Simulation(cfg) as sim:
        sim.set_particles(g["in_x"][:, 0], g["in_x"][:, 1], np.zeros((n, 3)), g["in_v"], g["in_v"], g["in_q"],
                          g["in_m"])
        sim.init_fields()
        sim.step_implicit(1)
        sim.save_state(path)
        diag_a, info_a, sd_a = sim.step_implicit(2, step_diagnostics=True)
        snap_a = snapshot(sim, fields)
    with up.Simulation(cfg) as sim:
        sim.load_state(path)
        diag_b, info_b, sd_b = sim.step_implicit(2, step_diagnostics=True)
        snap_b = snapshot(sim, fields)
    assert np.array_equal(diag_a, diag_b, equal_nan=True)
    assert np.array_equal(info_a, info_b, equal_nan=True)
    assert np.array_equal(sd_a, sd_b, equal_nan=True)
    assert_same(snap_a, snap_b)


def test_state_file_errors(tmp_path):
    cfg = explicit_config()
    path = str(tmp_path / "state.bin")
    with up.Simulation(cfg) as sim:
        load_explicit(sim, cfg, ppc=2)
        sim.init_fields()
        sim.save_state(path)
    # a different configuration
    with up.Simulation(explicit_config(dt=0.04)) as sim:
        with pytest.raises(up.UpicError) as e:
            sim.load_state(path)
        assert e.value.code == -1
    # not a state file, a truncated one, a missing one
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"not a state file at all, just bytes")
    short = tmp_path / "short.bin"
    short.write_bytes(open(path, "rb").read()[:4096])
    with up.Simulation(cfg) as sim:
        for p in (junk, short, tmp_path / "missing.bin"):
            with pytest.raises(up.UpicError) as e:
                sim.load_state(str(p))
            assert e.value.code == -2
        # the context stays usable: a good file loads afterwards
        sim.load_state(path)
        sim.step(2)
