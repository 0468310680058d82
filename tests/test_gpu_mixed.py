"""GPU tests of the mixed-precision explicit step (UPIC_PRECISION_MIXED):
FP32 particles stored as nearest node + cell-relative offset, FP32 gather,
push and deposit sums, FP64 field solve, single-word fixed-point grid
accumulation.  Checked against the FP64 step on the same input: every
diagnostic and field agrees to the stated FP32-level tolerance over 50
steps, round-off residuals (gauge, Gauss, continuity) stay at FP64
round-off, runs are bitwise reproducible, and restarts are exact."""
import numpy as np
import pytest

import unstaggered_pic_b200 as up

pytestmark = pytest.mark.gpu
STEPS = 50
# relative difference mixed vs FP64 after 50 steps, by diagnostics column
TOL_DIAG = 2e-5
TOL_FIELD = 1e-4     # fields relative to their magnitude (A, phi, J, rho)


def config(precision, **kw):
    args = dict(nx=32, ny=32, Lx=2 * np.pi / 0.3, Ly=2 * np.pi / 0.3, dt=0.05, method="bdf1",
                charge_update="conserving", precision=precision)
    args.update(kw)
    return up.Config(**args)


def run(cfg, steps=STEPS, ppc=16, seed=11):
    p = up.generate_bimaxwellian(cfg.nx, cfg.ny, cfg.Lx, cfg.Ly, ppc, (0.02, 0.2, 0.05), seed=seed)
    with up.Simulation(cfg) as sim:
        sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
        row0 = sim.init_fields()
        rows = sim.step(steps)
        fields = {f: sim.field(f) for f in ("phi", "Ax", "Ay", "Az", "rho", "Jx", "Jy", "Jz")}
        part = sim.get_particles()
    return row0, rows, fields, part, p


@pytest.mark.parametrize("method,charge", [("bdf1", "conserving"), ("bdf2", "naive")])
def test_mixed_matches_fp64(method, charge):
    r64 = run(config("fp64", method=method, charge_update=charge))
    r32 = run(config("mixed", method=method, charge_update=charge))
    names = up.DIAG_COLUMNS
    for k, name in enumerate(names):
        a, b = r32[1][:, k], r64[1][:, k]
        if np.max(np.abs(b)) < 1e-9:
            # round-off residuals of the FP64 field solve stay at round-off
            assert np.max(np.abs(a)) < 1e-9, (name, np.max(np.abs(a)))
        else:
            # (random positions put noise on the k^2 = 0 Nyquist modes, which
            # the Poisson start-up cannot represent: the Gauss and gauge
            # residuals of this input are physical, in both precisions)
            scale = np.max(np.abs(b))
            assert np.max(np.abs(a - b)) <= TOL_DIAG * scale, (name, np.max(np.abs(a - b)) / scale)
    for f in r64[2]:
        scale = np.max(np.abs(r64[2][f]))
        err = np.max(np.abs(r32[2][f] - r64[2][f])) / scale
        assert err < TOL_FIELD, (f, err)
    L = r64[4]
    dx = (r64[3]["x"] - r32[3]["x"] + 0.5 * 2 * np.pi / 0.3) % (2 * np.pi / 0.3) - 0.5 * 2 * np.pi / 0.3
    assert np.max(np.abs(dx)) < 1e-4
    assert np.max(np.abs(r32[3]["v"] - r64[3]["v"])) < 1e-4


def test_mixed_bitwise_reproducible_and_roundtrip():
    cfg = config("mixed")
    a = run(cfg, steps=12)
    b = run(cfg, steps=12)
    assert np.array_equal(a[1], b[1])
    for f in a[2]:
        assert np.array_equal(a[2][f], b[2][f])
    # no steps: positions come back to within an FP32 offset of a cell
    p = up.generate_bimaxwellian(cfg.nx, cfg.ny, cfg.Lx, cfg.Ly, 4, (0.02, 0.2, 0.05), seed=3)
    with up.Simulation(cfg) as sim:
        sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
        out = sim.get_particles()
    dx = cfg.Lx / cfg.nx
    assert np.max(np.abs(out["x"] - p["x"])) <= 2.0 ** -24 * dx * 1.01
    assert np.max(np.abs(out["y"] - p["y"])) <= 2.0 ** -24 * dx * 1.01
    assert np.allclose(out["v"], p["v"], rtol=2 ** -23, atol=0)
    assert np.allclose(out["P"], p["P"], rtol=2 ** -23, atol=0)


def test_mixed_restart_and_config_errors(tmp_path):
    cfg = config("mixed", method="bdf2")
    p = up.generate_bimaxwellian(cfg.nx, cfg.ny, cfg.Lx, cfg.Ly, 8, (0.02, 0.2, 0.05), seed=5)
    path = str(tmp_path / "mixed.state")
    with up.Simulation(cfg) as sim:
        sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
        sim.init_fields()
        sim.step(5)
        sim.save_state(path)
        rows_a = sim.step(6)
        jx_a = sim.field("Jx")
    with up.Simulation(cfg) as sim:
        sim.load_state(path)
        rows_b = sim.step(6)
        jx_b = sim.field("Jx")
    assert np.array_equal(rows_a, rows_b)
    assert np.array_equal(jx_a, jx_b)
    # the implicit methods run in FP64 only
    with pytest.raises(up.UpicError) as e:
        cfg = up.ImplicitConfig(nx=8, ny=8)
        c = cfg.to_c()
        c.precision = 1
        import ctypes
        from unstaggered_pic_b200._native import lib
        ctx = ctypes.c_void_p()
        rc = lib().upic_create(ctypes.byref(c), ctypes.byref(ctx))
        if rc != 0:
            raise up.UpicError(rc, lib().upic_last_error(None).decode())
        lib().upic_destroy(ctx)
    assert e.value.code == -1


def test_full_run_growth_rate_mixed_vs_fp64():
    """The CPU-runnable Weibel workload over its full length (64x64 grid,
    64 electrons per cell, bi-Maxwellian vth = (0.02, 0.2, 0) c, dt 0.05,
    1000 steps) in both precisions: the Weibel growth rate of |B_z| (log-
    linear fit over steps 250..650, the linear phase) agrees to 1e-4, the
    field-energy history to 1e-5 and the energy change (BDF1 damps) to
    1e-4 (measured: 8e-9, 3e-7 and 2e-6)."""
    L = 2 * np.pi / 0.3
    out = {}
    for prec in ("fp64", "mixed"):
        cfg = up.Config(nx=64, ny=64, Lx=L, Ly=L, dt=0.05, method="bdf1", charge_update="conserving", precision=prec)
        p = up.generate_bimaxwellian(64, 64, L, L, 64, (0.02, 0.2, 0.0), seed=2026)
        with up.Simulation(cfg) as sim:
            sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
            row0 = sim.init_fields()
            out[prec] = np.vstack([row0, sim.step(1000)])
    names = up.DIAG_COLUMNS
    bz, fe, te = names.index("Bz_l2"), names.index("field_energy"), names.index("total_energy")
    t = np.arange(250, 651) * 0.05
    rate = {k: np.polyfit(t, np.log(d[250:651, bz]), 1)[0] for k, d in out.items()}
    assert rate["fp64"] > 0.05, rate  # the instability grows
    assert abs(rate["mixed"] - rate["fp64"]) <= 1e-4 * rate["fp64"], rate
    d64, d32 = out["fp64"], out["mixed"]
    assert np.max(np.abs(d32[:, fe] - d64[:, fe])) <= 1e-5 * np.max(d64[:, fe])
    de64, de32 = d64[:, te] - d64[0, te], d32[:, te] - d32[0, te]
    assert np.max(np.abs(de32 - de64)) <= 1e-4 * np.max(np.abs(de64))
