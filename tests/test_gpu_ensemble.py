"""GPU tests of ensembles of independent explicit runs (upic_ensemble_*):
2D runs of uneven grid sizes, particle counts, tilings and re-sort
intervals, FP64 and mixed precision, advanced together by one CUDA graph
per period give bit for bit the state that stepping each run alone gives;
the autotuner returns one of its candidates."""
import numpy as np
import pytest

import unstaggered_pic_b200 as up

pytestmark = pytest.mark.gpu
FIELDS = ["phi", "Ax", "Ay", "Az", "rho", "Jx", "Jy", "Jz"]


def run_specs():
    """(config keywords, particles) of six uneven 2D runs: grids 16x16 to
    64x32, 4 to 16 electrons per cell, tiles 4 and 8, re-sort intervals 2
    and 4, BDF1 and BDF2, conserving and naive charge, FP64 and mixed."""
    L = 2 * np.pi / 0.3
    rows = [(16, 16, 16, dict(method="bdf1", sort_interval=2, tile=4)),
            (32, 16, 12, dict(method="bdf1", sort_interval=4, tile=8)),
            (64, 32, 4, dict(method="bdf2", sort_interval=4)),
            (32, 32, 8, dict(method="bdf1", sort_interval=2, charge_update="naive")),
            (16, 32, 10, dict(method="bdf2", sort_interval=4, tile=4)),
            (16, 16, 16, dict(method="bdf1", sort_interval=2, precision="mixed"))]
    specs = []
    for i, (nx, ny, ppc, kw) in enumerate(rows):
        Lx, Ly = L * nx / 32, L * ny / 32
        p = up.generate_bimaxwellian(nx, ny, Lx, Ly, ppc, (0.02, 0.2, 0.05), seed=40 + i)
        specs.append((dict(nx=nx, ny=ny, Lx=Lx, Ly=Ly, dt=0.05, **kw), p))
    return specs


def start(kw, p):
    sim = up.Simulation(up.Config(**kw))
    sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
    sim.init_fields(False)
    return sim


def state(sim):
    part = sim.get_particles()
    return {**part, **{f: sim.field(f) for f in FIELDS}}


def test_ensemble_matches_runs_alone():
    specs = run_specs()
    alone = [start(kw, p) for kw, p in specs]
    together = [start(kw, p) for kw, p in specs]
    try:
        with up.Ensemble(together) as ens:
            assert ens.period == 40  # lcm(5 history slots, twice the re-sort intervals 2 and 4)
            for chunk in (85, 40, 3, 80):  # graph launches, replays, remainders, recaptures at a new phase
                ens.step(chunk)
                for sim in alone:
                    sim.step(chunk, 0)
                for a, b in zip(alone, together):
                    sa, sb = state(a), state(b)
                    for k in sa:
                        assert np.array_equal(sa[k], sb[k]), (chunk, k)
                    assert a.steps_taken() == b.steps_taken()
            # a run reloaded with more particles (its buffers reallocated) and
            # restarted: the ensemble records a new graph
            kw, _ = specs[2]
            p = up.generate_bimaxwellian(kw["nx"], kw["ny"], kw["Lx"], kw["Ly"], 12, (0.02, 0.2, 0.05), seed=99)
            for sim in (alone[2], together[2]):
                sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
                sim.init_fields(False)
            ens.step(40)
            for sim in alone:
                sim.step(40, 0)
            for a, b in zip(alone, together):
                sa, sb = state(a), state(b)
                for k in sa:
                    assert np.array_equal(sa[k], sb[k]), ("reload", k)
        # the runs stay usable after the ensemble is gone
        rows = together[1].step(2)
        assert np.all(np.isfinite(rows))
    finally:
        for s in alone + together:
            s.close()


def test_ensemble_errors():
    kw, p = run_specs()[0]
    sim = start(kw, p)
    imp = up.Simulation(up.ImplicitConfig(nx=8, ny=8))
    try:
        with pytest.raises(up.UpicError):
            up.Ensemble([sim, sim])
        with pytest.raises(up.UpicError):
            up.Ensemble([sim, imp])
        with pytest.raises(up.UpicError):
            up.Ensemble([])
    finally:
        sim.close()
        imp.close()


def test_autotune_returns_a_candidate():
    L = 2 * np.pi / 0.3
    p = up.generate_bimaxwellian(64, 64, L, L, 16, (0.02, 0.2, 0.0), seed=3)
    make = lambda tile, si: up.Config(nx=64, ny=64, Lx=L, Ly=L, dt=0.05, method="bdf1", tile=tile,
                                      sort_interval=si)
    tile, si, times = up.autotune_explicit(make, p, tiles=(4, 8), sort_intervals=(2, 4), steps=4)
    assert (tile, si) in times and len(times) == 4
    assert all(t > 0 for t in times.values())


def test_contexts_with_different_windows_coexist():
    """A kernel's shared-memory limit belongs to the function: a context
    created after another with a smaller deposit window must not lower the
    limit the first one's launches need."""
    L = 2 * np.pi / 0.3
    p = up.generate_bimaxwellian(64, 64, L, L, 4, (0.02, 0.2, 0.0), seed=8)
    sims = []
    try:
        for tile in (16, 4):
            sim = up.Simulation(up.Config(nx=64, ny=64, Lx=L, Ly=L, dt=0.05, tile=tile))
            sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
            sim.init_fields(False)
            sims.append(sim)
        rows = [sim.step(3) for sim in sims]
        assert np.allclose(rows[0], rows[1], rtol=1e-11, atol=1e-14)
    finally:
        for sim in sims:
            sim.close()


IMPLICIT_DECK = dict(Lz=1.0, kappa=1.0, sigma1=1.0, sigma2=1.0, n0=1.0, orbit_quad_order=8,
                     split_orbit_at_knots=True, nyquist_projection=True, nonlinear_rtol=1e-10,
                     nonlinear_atol=1e-13, nonlinear_max_iter=80, anderson_damping=0.5,
                     uniform_local_rtol=1e-12, uniform_local_atol=1e-14, uniform_local_max_iter=64)


def two_stream_1d(nx, nb, v0, eps=1e-3):
    """1D-2V (ny = 1) cold beams at +-v0 on a quiet start, Project3 coordinates."""
    Lx = 2 * np.pi * v0 / 0.6
    k = 2 * np.pi / Lx
    x0 = -Lx / 2 + (np.arange(nb) + 0.5) * Lx / nb
    x0 = x0 - (eps / k) * np.sin(k * (x0 + Lx / 2))
    x = np.concatenate([x0, x0])
    v = np.zeros((2 * nb, 3))
    v[:nb, 0], v[nb:, 0] = v0, -v0
    q = np.full(2 * nb, -Lx / (2 * nb))
    return Lx, x, v, q, np.abs(q)


def test_implicit_ensemble_matches_runs_alone():
    """Implicit runs (1D-2V two-stream of uneven sizes, cubic splines, and a
    2D non-relativistic run) advanced on the ensemble's thread pool equal the
    same runs advanced alone, bit for bit."""
    specs = []
    for nx, nb, v0 in ((64, 512, 0.2), (128, 1500, 0.15), (32, 300, 0.3)):
        Lx, x, v, q, m = two_stream_1d(nx, nb, v0)
        cfg = dict(nx=nx, ny=1, Lx=Lx, Ly=1.0, dt=0.1, spline_order=3, **IMPLICIT_DECK)
        specs.append((up.ImplicitConfig, cfg, (np.stack([x, np.zeros_like(x), np.zeros_like(x)], 1), None, v, q, m)))
    L = 2 * np.pi
    p = up.generate_bimaxwellian(16, 16, L, L, 8, (0.05, 0.05, 0.0), seed=6)
    specs.append((up.NonrelConfig, dict(nx=16, ny=16, Lx=L, Ly=L, dt=0.05),
                  (np.stack([p["x"], p["y"], np.zeros_like(p["x"])], 1), None, p["v"], p["q"], p["m"])))

    def start_impl(cls, kw, parts):
        sim = up.Simulation(cls(**kw))
        x, _, v, q, m = parts
        sim.set_particles(x[:, 0], x[:, 1], np.zeros_like(v), v, v, q, m)
        sim.init_fields(False)
        return sim

    alone = [start_impl(*s) for s in specs]
    together = [start_impl(*s) for s in specs]
    try:
        with up.Ensemble(together) as ens:
            assert ens.period == 1
            ens.step(4)
        for sim in alone:
            sim.step_implicit(4, diagnostics=False)
        for a, b in zip(alone, together):
            sa, sb = state(a), state(b)
            for k in sa:
                assert np.array_equal(sa[k], sb[k]), k
        with pytest.raises(up.UpicError):
            up.Ensemble([alone[0], start(*run_specs()[0])])
    finally:
        for s in alone + together:
            s.close()


def test_ensemble_with_an_empty_run():
    """A run without particles (its fields still evolve) in an ensemble
    equals the same run stepped alone."""
    L = 2 * np.pi / 0.3
    p = up.generate_bimaxwellian(16, 16, L, L, 8, (0.02, 0.2, 0.0), seed=9)
    empty = {k: v[:0] for k, v in p.items()}
    sims_a, sims_b = [], []
    try:
        for parts in (p, empty):
            for lst in (sims_a, sims_b):
                sim = up.Simulation(up.Config(nx=16, ny=16, Lx=L, Ly=L, dt=0.05, sort_interval=2))
                # (an explicit context needs a particle set loaded once before
                # it accepts an empty one)
                sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
                sim.set_particles(parts["x"], parts["y"], parts["P"], parts["v"], parts["v_prev"], parts["q"],
                                  parts["m"])
                sim.init_fields(False)
                lst.append(sim)
        with up.Ensemble(sims_b) as ens:
            ens.step(25)
        for sim in sims_a:
            sim.step(25, 0)
        for a, b in zip(sims_a, sims_b):
            for f in FIELDS:
                assert np.array_equal(a.field(f), b.field(f)), f
    finally:
        for s in sims_a + sims_b:
            s.close()
