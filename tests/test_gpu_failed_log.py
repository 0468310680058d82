"""upic_failed_particle_log through the Python binding (Simulation.
failed_particle_log): the cold Weibel start whose local solves fail at two
iterations, stepped with and without the selective fallback.

With the fallback every failure event of the step is logged (restart 0, 1,
... of the layout, rows sorted by particle index inside an event, each row
the particle's solve report: reason maximum_iterations after two
iterations, residuals above the tolerance, the last iterate one damped
update past the previous); the step then converges and the log holds no
exhausted event.  Without the fallback the step fails with
UPIC_ERR_LOCAL_PARTICLE and its one event is marked exhausted."""
import numpy as np
import pytest

import unstaggered_pic_b200 as up
from unstaggered_pic_b200._native import UPIC_ERR

pytestmark = pytest.mark.gpu
COL = {n: i for i, n in enumerate(up.FAILED_LOG_COLUMNS)}
KEYS = dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, v0=0.5, weibel_B0=1e-3, particles_per_cell_pair=2,
            spline_order=3)


def start(fallback):
    s = up.p3_initial_state("weibel", Lz=1.0, **KEYS)
    cfg = up.ImplicitConfig(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, Lz=1.0, dt=0.2, spline_order=3,
                            orbit_quad_order=8, nyquist_projection=False, uniform_local_max_iter=2,
                            selective_particle_fallback=fallback)
    sim = up.Simulation(cfg)
    n = len(s["q"])
    sim.set_particles(s["x"], s["y"], np.zeros((n, 3)), s["v"], s["v"], s["q"], s["m"])
    sim.set_initial_potential(s["A"], s["U"])
    sim.init_fields(False)
    return sim, n


def check_rows(rows, n):
    assert rows.shape[1] == len(up.FAILED_LOG_COLUMNS)
    assert np.all(rows[:, COL["step"]] == 0)
    assert np.all((rows[:, COL["particle_index"]] >= 0) & (rows[:, COL["particle_index"]] < n))
    assert np.all(rows[:, COL["failure_reason"]] == up.FAILURE_REASONS.index("maximum_iterations"))
    assert np.all(rows[:, COL["local_iterations"]] == 2)
    assert np.all(rows[:, COL["final_scaled_residual"]] > 1.0)
    assert np.all(np.isfinite(rows[:, COL["first_scaled_residual"]]))
    # events: rows of one (restart, map evaluation) pair, sorted by particle
    keys = rows[:, [COL["layout_refinement_restart"], COL["map_evaluation"]]]
    for key in np.unique(keys, axis=0):
        ev = rows[np.all(keys == key, axis=1)]
        assert np.all(np.diff(ev[:, COL["particle_index"]]) > 0)
        assert np.all(ev[:, COL["failed_particles_in_event"]] == len(ev))
    # theta and h of the failing substep
    sub = rows[:, COL["assigned_substeps"]]
    k = rows[:, COL["failed_substep_zero_based"]]
    assert np.all(k < sub)
    assert np.allclose(rows[:, COL["theta0"]], k / sub) and np.allclose(rows[:, COL["theta1"]], (k + 1) / sub)
    assert np.allclose(rows[:, COL["h"]], 0.2 / sub)


def test_failed_log_with_fallback():
    sim, n = start(True)
    with sim:
        sim.step_implicit(1, diagnostics=False)
        rows = sim.failed_particle_log()
    assert len(rows) > 0
    check_rows(rows, n)
    assert np.all(rows[:, COL["event_exhausted"]] == 0)
    restarts = np.unique(rows[:, COL["layout_refinement_restart"]])
    assert restarts[0] == 0 and np.all(np.diff(restarts) == 1)
    # each restart doubles the failed particles' substeps
    first = rows[rows[:, COL["layout_refinement_restart"]] == 0]
    assert np.all(first[:, COL["assigned_substeps"]] == 1)


def test_failed_log_without_fallback():
    sim, n = start(False)
    with sim:
        with pytest.raises(up.UpicError) as e:
            sim.step_implicit(1, diagnostics=False)
        assert UPIC_ERR[e.value.code] == "UPIC_ERR_LOCAL_PARTICLE"
        rows = sim.failed_particle_log()
    assert len(rows) > 0
    check_rows(rows, n)
    assert np.all(rows[:, COL["event_exhausted"]] == 1)
    assert np.all(rows[:, COL["layout_refinement_restart"]] == 0)
    assert np.all(rows[:, COL["assigned_substeps"]] == 1)
