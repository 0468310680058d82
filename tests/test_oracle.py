"""CPU tests of the oracle: pinned to the reference's own code (bit for bit)
and to the reference's published validation numbers."""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle_lib as ol

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def test_oracle_kernels_match_reference_fixtures():
    o = ol.oracle()
    g = load("p2_kernels.npz")
    nx, ny, Lx, Ly = int(g["nx"]), int(g["ny"]), float(g["Lx"]), float(g["Ly"])
    n = len(g["in_x"])
    cd = ctypes.c_double
    J = np.zeros(3 * nx * ny)
    o.o2_deposit_current(nx, ny, cd(Lx), cd(Ly), ctypes.c_long(n), ol.ptr(g["in_x"]), ol.ptr(g["in_y"]),
                         ol.ptr(g["in_v"]), ol.ptr(g["in_q"]), ol.ptr(J))
    assert np.array_equal(J, g["J"])
    rho = np.zeros(nx * ny)
    o.o2_deposit_charge(nx, ny, cd(Lx), cd(Ly), cd(1.0), ctypes.c_long(n), ol.ptr(g["in_x"]),
                        ol.ptr(g["in_y"]), ol.ptr(g["in_q"]), ol.ptr(rho))
    assert np.array_equal(rho, g["rho"])
    gat = np.zeros(n)
    o.o2_gather(nx, ny, cd(Lx), cd(Ly), ol.ptr(g["f"]), ctypes.c_long(n), ol.ptr(g["in_x"]),
                ol.ptr(g["in_y"]), ol.ptr(gat))
    assert np.array_equal(gat, g["gather"])
    for inv, kr, ki in ((0, "fft_re", "fft_im"), (1, "ifft_re", "ifft_im")):
        re, im = g["re"].copy(), g["im"].copy()
        o.o2_fft2d(nx, ny, ol.ptr(re), ol.ptr(im), inv)
        assert np.array_equal(re, g[kr]) and np.array_equal(im, g[ki])
    for d, key in ((0, "ddx"), (1, "ddy")):
        out = np.zeros(nx * ny)
        o.o2_spectral_derivative(nx, ny, cd(Lx), cd(Ly), ol.ptr(g["f"]), d, ol.ptr(out))
        assert np.array_equal(out, g[key])
    phi = np.zeros(nx * ny)
    o.o2_poisson(nx, ny, cd(Lx), cd(Ly), cd(1.0), ol.ptr(g["rho"]), ol.ptr(phi))
    assert np.array_equal(phi, g["phi"])


@pytest.mark.parametrize("name", ["p2_run_bdf1_conserving.npz", "p2_run_bdf1_naive.npz",
                                  "p2_run_bdf2_conserving.npz", "p2_run_bdf2_naive.npz"])
def test_oracle_step_loop_matches_reference_fixtures(name):
    g = load(name)
    p, ip = g["params"], g["iparams"]
    prob = ol.P2Problem(int(ip[0]), int(ip[1]), p[0], p[1], p[2], int(ip[2]), bool(ip[3]), p[3], p[4],
                        p[5], p[6], int(ip[4]), int(ip[5]))
    parts = {k[3:]: g[k] for k in g if k.startswith("in_")}
    out, diag, fields, _ = ol.simulate(ol.oracle().o2_simulate, prob, parts)
    for k in out:
        assert np.array_equal(out[k], g["out_" + k]), k
    assert np.array_equal(diag, g["diag"], equal_nan=True)
    assert np.array_equal(fields, g["fields"])


@pytest.mark.parametrize("run,order,conserving", [("weibel_bdf1_conserving", 1, True),
                                                  ("weibel_bdf2_conserving", 2, True),
                                                  ("weibel_bdf1_naive", 1, False)])
def test_oracle_reproduces_published_weibel_validation(run, order, conserving):
    """Full Project2 Weibel decks (32x32, 4 samples/cell, 160 steps) against
    Project2/docs/validation_summary.json."""
    with open(os.path.join(GOLD, "p2_weibel_published.json")) as fh:
        pub = json.load(fh)["runs"][run]
    o = ol.oracle()
    o.o2_init_weibel.restype = ctypes.c_long
    L = 6.283185307179586
    parts = ol.init_weibel(o.o2_init_weibel, 32, 32, L, L, 4)
    prob = ol.P2Problem(32, 32, L, L, 0.05, order, conserving, n_steps=160)
    _, diag, _, _ = ol.simulate(o.o2_simulate, prob, parts, want_fields=False)
    # maxima skip the initial row, as Project2/tools/validate_against_paper.py:60,75 does
    assert diag[1:, 0].max() == pub["max_gauge_rms"]
    assert diag[1:, 1].max() == pub["max_gauss_rms"]
    assert diag[1:, 2].max() == pub["max_continuity_rms"]
    assert diag[-1, 3] == pub["final_Bz_l2"]
    assert diag[-1, 10] == pub["final_total_energy"]
    assert diag[1:, 11].max() == pub["max_speed"]


def test_oracle_matches_live_reference_when_built():
    """When the reference harness is available (this container), compare a
    fresh random case directly."""
    ref = ol.ref_p2()
    if ref is None:
        pytest.skip("reference harness not built (no reference sources)")
    rng = np.random.default_rng(7)
    from golden.make_golden import seeded_particles
    prob = ol.P2Problem(8, 64, 1.0, 7.0, 0.1, 2, False, n_steps=5)
    p = seeded_particles(rng, 300, prob.Lx, prob.Ly)
    a = ol.simulate(ol.oracle().o2_simulate, prob, p)
    b = ol.simulate(ref.ref_p2_simulate, prob, p)
    for k in a[0]:
        assert np.array_equal(a[0][k], b[0][k])
    assert np.array_equal(a[1], b[1], equal_nan=True)


@pytest.mark.parametrize("case", [0, 4])
def test_implicit_fixtures_regenerate_from_reference_build(case):
    """The committed implicit-method fixtures (tests/golden/p3_*.npz) are
    outputs of the reference's own solver: rerunning the reference build on
    the stored inputs reproduces them bit for bit.  Skipped where the
    reference sources (and so oracle/_ref/libref_p3.so) are absent."""
    ref = ol.ref_p3()
    if ref is None:
        pytest.skip("reference harness not built (no reference sources)")
    from golden.make_golden import P3_CASES
    name = P3_CASES[case][0]
    g = dict(np.load(os.path.join(GOLD, name + ".npz")))
    prob = ol.P3Problem(**P3_CASES[case][1])
    assert np.array_equal(prob.dparams(), g["dparams"]) and np.array_equal(prob.iparams(), g["iparams"])
    out = ol.p3_run(ref.ref_p3_run, prob, g["in_x"], g["in_v"], g["in_q"], g["in_m"], want_step_diag=True)
    for k in ("x", "v", "P", "v_prev", "vbar"):
        assert np.array_equal(out[k], g["out_" + k]), k
    assert np.array_equal(out["diag"], g["diag"])
    assert np.array_equal(out["info"], g["info"])
    assert np.array_equal(out["fields"], g["fields"])
    assert np.array_equal(out["step_diag"], g["step_diag"])


def test_orbit_fixtures_regenerate_from_reference_build(tmp_path, monkeypatch):
    """tests/golden/p3_orbit_kernels.npz is the reference's own orbit
    integrals: regenerating it from the reference build is bit-exact."""
    ref = ol.ref_p3()
    if ref is None:
        pytest.skip("reference harness not built (no reference sources)")
    import golden.make_golden as mg
    monkeypatch.setattr(mg, "HERE", str(tmp_path))
    mg.p3_orbit_main(ref)
    a = dict(np.load(os.path.join(GOLD, "p3_orbit_kernels.npz")))
    b = dict(np.load(os.path.join(str(tmp_path), "p3_orbit_kernels.npz")))
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_p1_landau_weak_fixture_is_the_shipped_run():
    """tests/golden/p1_run_landau_weak.npz (the reference's landau_weak deck
    through oracle/_ref/libref_p1.so) carries the very numbers of the run the
    reference ships in Project1/output/landau_weak_*.csv (extracted into
    tests/golden/p1_landau_weak_shipped.npz): every diagnostics, Picard and
    step-diagnostics column of all 60 steps agrees to the last printed digit
    (17 significant digits, so bit for bit)."""
    g = dict(np.load(os.path.join(GOLD, "p1_run_landau_weak.npz")))
    s = dict(np.load(os.path.join(GOLD, "p1_landau_weak_shipped.npz")))
    assert list(s["diag_columns"]) == ol.P1_DIAG_NAMES
    assert np.array_equal(g["diag"], s["diag"], equal_nan=True)
    assert np.array_equal(g["info"], s["info"], equal_nan=True)
    assert np.array_equal(g["step_diag"], s["step_diag"], equal_nan=True)


@pytest.mark.parametrize("case", [0, 3, 5])
def test_p1_fixtures_regenerate_from_reference_build(case):
    """The committed non-relativistic fixtures (tests/golden/p1_run_*.npz)
    are outputs of the reference's own solver (Project1/ec_pic_serial_demo.cpp):
    rerunning the reference build on the stored inputs reproduces them bit
    for bit.  Skipped where oracle/_ref/libref_p1.so is absent."""
    ref = ol.ref_p1()
    if ref is None:
        pytest.skip("reference harness not built (no reference sources)")
    from golden.make_golden import P1_CASES
    name, kw, src = P1_CASES[case]
    g = dict(np.load(os.path.join(GOLD, name + ".npz")))
    prob = ol.P1Problem(**kw)
    assert np.array_equal(prob.dparams(), g["dparams"]) and np.array_equal(prob.iparams(), g["iparams"])
    if src == "ref":
        x, v, q, m = ol.p1_init(ref, prob)
        assert np.array_equal(x, g["in_x"]) and np.array_equal(v, g["in_v"]) and np.array_equal(q, g["in_q"])
    out = ol.p1_run(ref.ref_p1_run, prob, g["in_x"], g["in_v"], g["in_q"], g["in_m"])
    for k in ("x", "v", "P", "v_prev"):
        assert np.array_equal(out[k], g["out_" + k]), k
    for k in ("diag", "info", "step_diag"):
        assert np.array_equal(out[k], g[k], equal_nan=True), k
    assert np.array_equal(out["fields"], g["fields"])


@pytest.mark.parametrize("args", [
    (16, 8, 20.94, 10.47, 5, (0.02, 0.2, 0.0), (0.0, 0.0, 0.0), 1.0, 1.0, 2026),
    (32, 32, 3.0, 5.0, 3, (0.1, 0.05, 0.02), (0.577, 0.0, -0.1), 1.0, 0.1, 56),
    (256, 128, 20.94, 10.47, 3, (0.02, 0.2, 0.0), (0.0, 0.0, 0.0), 2.0, 1.0, 1000),
])
def test_oracle_generator_equals_product_generator(args):
    """The oracle's restatement of the workloads' seeded plasma gives the
    product generator's arrays bit for bit (the reference arm of bench.py
    builds its inputs from the oracle, without the product library; the
    largest case runs the product on several host threads)."""
    import unstaggered_pic_b200 as up
    nx, ny, Lx, Ly, ppc, uth, ud, c, n0, seed = args
    a = ol.generate_bimaxwellian(nx, ny, Lx, Ly, ppc, uth, udrift=ud, c=c, n0=n0, seed=seed)
    b = up.generate_bimaxwellian(nx, ny, Lx, Ly, ppc, uth, udrift=ud, c=c, n0=n0, seed=seed)
    for k in a:
        assert a[k].tobytes() == b[k].tobytes(), k


# Instability starts of Project3 (initialize_two_stream_3d_linear_x :3689,
# initialize_weibel_filamentation_3d :3961) and its Landau example
# (initialize_landau_damping_1d3d :3853) on 2D grids: the product's host
# restatement against the reference's own initialize_state, bit for bit.
P3_INIT_CASES = [
    ("weibel", dict(nx=16, ny=16, Lx=2 * np.pi, Ly=2 * np.pi, v0=0.5, weibel_B0=1e-3, particles_per_cell_pair=2,
                    spline_order=2)),
    ("weibel", dict(nx=8, ny=32, Lx=3.0, Ly=2 * np.pi / 0.7, v0=0.3, perturbation=2e-3, particles_per_cell_pair=3,
                    spline_order=3, perturbation_mode=2, weibel_finite_grid_theory=0)),
    ("two_stream", dict(nx=32, ny=4, Lx=2 * np.pi / 3.0, Ly=1.0, v0=0.2, two_stream_density_alpha=1e-3,
                        particles_per_cell_pair=8, spline_order=3)),
    ("two_stream", dict(nx=16, ny=8, Lx=2 * np.pi, Ly=2.0, v0=0.25, perturbation=0.01, tsi_transverse_seed=1e-3,
                        tsi_transverse_mode=2, particles_per_cell_pair=4, spline_order=2)),
    ("landau", dict(nx=32, ny=2, Lx=4 * np.pi, Ly=1.0, particles_per_cell_pair=16, landau_alpha=0.05,
                    spline_order=1, thermal_velocity=0.1)),
    ("landau", dict(nx=16, ny=4, Lx=2 * np.pi, Ly=3.0, particles_per_cell_pair=64, perturbation=0.3,
                    spline_order=2, thermal_velocity=0.05, perturbation_mode=2)),
]


@pytest.mark.parametrize("case,keys", P3_INIT_CASES)
def test_p3_instability_start_equals_reference(case, keys):
    lib = ol.ref_p3()
    if lib is None:
        pytest.skip("oracle/_ref/libref_p3.so is not built")
    import unstaggered_pic_b200 as up
    mine = up.p3_initial_state(case, Lz=1.0, **keys)
    # the reference's start with its Nyquist projection off, so that A and U
    # are the initializer's own
    prob = ol.P3Problem(keys["nx"], keys["ny"], keys["Lx"], keys["Ly"], 0.1, Lz=1.0, order=keys["spline_order"],
                        nyquist=False, mode=keys.get("perturbation_mode", 1))
    ref = ol.p3_case_state(lib, prob, case, keys)
    assert np.array_equal(mine["x"], ref["x"][:, 0]) and np.array_equal(mine["y"], ref["x"][:, 1])
    assert np.all(ref["x"][:, 2] == 0.0)
    for k in ("v", "q", "m", "A", "U"):
        assert np.array_equal(mine[k], ref[k]), k
    assert mine["growth_rate"] == ref["growth_rate"]
