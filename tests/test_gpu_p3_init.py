"""Runs started from Project3's cold-instability initial states (the
two-stream and Weibel eigenmodes of initialize_two_stream_3d_linear_x :3689
and initialize_weibel_filamentation_3d :3961, on 2D grids) through the
public API -- upic_p3_initial_state, upic_set_particles,
upic_set_initial_potential, upic_init_fields, upic_step_implicit -- against
the reference's own runs from its own initialize_state (oracle/_ref/libref_p3.so).

The start state (canonical momenta with q A(x), history velocities under
E = -grad phi - U and B = curl A, Nyquist projection) agrees to rounding;
the steps agree to the solver tolerance, as the other implicit parity tests;
the Weibel eigenmode grows at the reference's rate."""
import numpy as np
import pytest

import oracle_lib as ol
import unstaggered_pic_b200 as up
from test_gpu_implicit import config_from, relerr

pytestmark = pytest.mark.gpu
TOL_STEP = 2e-10

CASES = [
    ("weibel", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, v0=0.5, weibel_B0=1e-3, particles_per_cell_pair=2,
                    spline_order=2), dict(dt=0.2, nq=8, n_steps=4)),
    ("two_stream", dict(nx=32, ny=4, Lx=2 * np.pi / 3.0, Ly=1.0, v0=0.2, two_stream_density_alpha=1e-3,
                        particles_per_cell_pair=8, spline_order=3), dict(dt=0.1, nq=8, n_steps=4)),
]


def _problem(keys, run):
    return ol.P3Problem(keys["nx"], keys["ny"], keys["Lx"], keys["Ly"], run["dt"], Lz=1.0, order=keys["spline_order"],
                        nq=run["nq"], nyquist=True, n_steps=run["n_steps"], mode=keys.get("perturbation_mode", 1))


def _start(case, keys, prob):
    s = up.p3_initial_state(case, Lz=1.0, **keys)
    sim = up.Simulation(config_from(prob.dparams(), prob.iparams()))
    n = len(s["q"])
    sim.set_particles(s["x"], s["y"], np.zeros((n, 3)), s["v"], s["v"], s["q"], s["m"])
    sim.set_initial_potential(s["A"], s["U"])
    return sim, s


@pytest.mark.parametrize("case,keys,run", CASES)
def test_instability_start_and_steps_match_reference(case, keys, run):
    lib = ol.ref_p3()
    if lib is None:
        pytest.skip("oracle/_ref/libref_p3.so is not built")
    prob = _problem(keys, run)
    ref0 = ol.p3_case_state(lib, prob, case, keys)
    ref = ol.p3_case_run(lib, prob, case, keys)
    sim, s = _start(case, keys, prob)
    d0 = sim.init_fields(True)
    start = sim.get_particles()
    # start state: P = m gamma v + q A(x), v_prev from E and B of the start fields
    assert relerr(start["P"], ref0["P"]) < 1e-13
    assert relerr(start["v_prev"], ref0["v_prev"]) < 1e-13
    for f, k in (("Ax", 0), ("Ay", 1), ("Az", 2)):
        assert np.max(np.abs(sim.field(f) - ref0["A"][k])) <= 1e-15 * max(1.0, np.max(np.abs(ref0["A"]))), f
    assert np.max(np.abs(sim.field("Ux") - ref0["U"][0])) <= 1e-15 * max(1.0, np.max(np.abs(ref0["U"])))
    # start diagnostics to rounding: the field energy of a 1e-3 perturbation
    # carries the cancellation of rho = n0 + deposited charge (5e-12); the
    # mode a case does not seed is rounding noise, held to 1e-13 of the seeded one
    modes = [up.IMPLICIT_DIAG_COLUMNS.index(c) for c in ("Bz_y_mode_abs", "E_mode_abs")]
    seeded = max(abs(ref["diag"][0, k]) for k in modes)
    for c, tol in (("field_energy", 5e-12), ("kinetic_energy", 1e-13), ("total_energy", 1e-13),
                   ("Bz_y_mode_abs", 1e-12), ("E_mode_abs", 1e-12)):
        k = up.IMPLICIT_DIAG_COLUMNS.index(c)
        assert abs(d0[k] - ref["diag"][0, k]) <= tol * abs(ref["diag"][0, k]) + 1e-13 * seeded, c
    # steps
    diag, info = sim.step_implicit(prob.n_steps)
    assert np.max(np.abs(info[:, 0] - ref["info"][:, 0])) <= 1
    for c in ("field_energy", "kinetic_energy", "total_energy"):
        k = up.IMPLICIT_DIAG_COLUMNS.index(c)
        assert relerr(diag[:, k], ref["diag"][1:, k]) < TOL_STEP * prob.n_steps, c
    # the seeded mode to the step tolerance, the other one as rounding noise
    # on the scale of the seeded one
    ks, ko = [up.IMPLICIT_DIAG_COLUMNS.index(c) for c in
              (("Bz_y_mode_abs", "E_mode_abs") if case == "weibel" else ("E_mode_abs", "Bz_y_mode_abs"))]
    assert relerr(diag[:, ks], ref["diag"][1:, ks]) < TOL_STEP * prob.n_steps
    assert np.max(np.abs(diag[:, ko] - ref["diag"][1:, ko])) <= TOL_STEP * prob.n_steps * np.max(ref["diag"][:, ks])
    names = ["phi", "psi", "rho", "Ax", "Ay", "Az", "Ux", "Uy", "Uz", "Jx", "Jy", "Jz"]
    for k, n in enumerate(names):
        scale = max(np.max(np.abs(ref["fields"][j])) for j in ((k // 3) * 3 + np.arange(3) if k >= 3 else [k]))
        assert np.max(np.abs(sim.field(n) - ref["fields"][k])) <= TOL_STEP * prob.n_steps * max(scale, 1e-30), n
    sim.close()


def test_weibel_eigenmode_grows_at_the_reference_rate():
    """40 steps of the seeded Weibel eigenmode: |B_z(k_y)| grows as the
    reference's run does (history within 1e-6), at close to the cold-fluid
    rate with the B-spline factor."""
    lib = ol.ref_p3()
    if lib is None:
        pytest.skip("oracle/_ref/libref_p3.so is not built")
    case, keys, _ = CASES[0]
    prob = _problem(keys, dict(dt=0.2, nq=8, n_steps=40))
    ref = ol.p3_case_run(lib, prob, case, keys)
    sim, s = _start(case, keys, prob)
    d0 = sim.init_fields(True)
    diag, _ = sim.step_implicit(prob.n_steps)
    sim.close()
    k = up.IMPLICIT_DIAG_COLUMNS.index("Bz_y_mode_abs")
    b = np.concatenate([[d0[k]], diag[:, k]])
    assert relerr(b, ref["diag"][:, k]) < 1e-6
    t = prob.dt * np.arange(prob.n_steps + 1)
    rate = np.polyfit(t, np.log(b), 1)[0]
    rate_ref = np.polyfit(t, np.log(ref["diag"][:, k]), 1)[0]
    assert abs(rate / rate_ref - 1) < 0.02
    assert abs(rate / s["growth_rate"] - 1) < 0.1, (rate, s["growth_rate"])
