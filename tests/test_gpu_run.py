"""GPU tests of upic_run, the deck-driven drop-in for the reference's
explicit solver CLI (Project2/spectral_pic_part3.cpp main).  The driver
reads the reference's deck keys, loads the reference's Weibel or cloud
particles, runs the step on the GPU and writes _diagnostics.csv,
_particle_sample.csv and _config_echo.txt in the reference's formats.

Checks: the CSV schemas and every value against the CPU oracle (always
present) and against the reference CLI itself run on the same deck (when
oracle/_ref/libref_p2.so was built from the reference sources).  Values
agree to TOL (relative to each column's scale); text fields and counts
exactly."""
import csv
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "unstaggered_pic_b200", "upic_run")
TOL = 1e-10


def write_deck(path, prefix, **kw):
    keys = dict(example="weibel", method="bdf2", charge_update="conserving", nx=32, ny=16, Lx=3.0, Ly=2.0,
                n_steps=30, dt=0.05, particles_per_cell=4, diagnostic_stride=4, particle_sample_count=64,
                seed=777, run_unit_tests="true", unknown_key_for_warning=1)
    keys.update(kw)
    with open(path, "w") as fh:
        fh.write("# deck written by the test\n")
        for k, v in keys.items():
            fh.write(f"{k} = {v}\n")
        fh.write(f"output_prefix = {prefix}\n")


def read_csv(path):
    with open(path) as fh:
        rows = list(csv.reader(fh))
    return rows[0], rows[1:]


def run_driver(deck):
    r = subprocess.run([RUN, deck], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


def compare_numeric(a_rows, b_rows, text_cols, tol):
    assert len(a_rows) == len(b_rows)
    ncol = len(a_rows[0])
    for k in range(ncol):
        if k in text_cols:
            assert [r[k] for r in a_rows] == [r[k] for r in b_rows], k
            continue
        a = np.array([float(r[k]) for r in a_rows])
        b = np.array([float(r[k]) for r in b_rows])
        scale = max(np.max(np.abs(b)), 1e-300)
        # round-off level columns (gauge / Gauss / continuity residuals) by level
        if scale < 1e-9:
            assert np.max(np.abs(a)) < 1e-9, k
        else:
            assert np.max(np.abs(a - b)) <= tol * scale, (k, np.max(np.abs(a - b)) / scale)


def test_usage_and_errors(tmp_path):
    r = subprocess.run([RUN], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    bad = tmp_path / "bad.txt"
    bad.write_text("nx = 12\n")
    r = subprocess.run([RUN, str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and "powers of two" in r.stderr
    r = subprocess.run([RUN, str(tmp_path / "missing.txt")], capture_output=True, text=True)
    assert r.returncode == 1 and "could not open" in r.stderr


def test_weibel_deck_matches_oracle(tmp_path):
    prefix = str(tmp_path / "gpu")
    deck = str(tmp_path / "deck.txt")
    write_deck(deck, prefix)
    r = run_driver(deck)
    assert "warning: unknown input key ignored: unknown_key_for_warning" in r.stderr
    assert "wrote " + prefix + "_diagnostics.csv" in r.stdout
    hdr, rows = read_csv(prefix + "_diagnostics.csv")
    assert hdr == ["step", "time", "requested_method", "active_method", "charge_update", "gauge_rms",
                   "gauss_rms", "continuity_rms", "Bz_l2", "B_l2", "E_l2", "rho_l2", "J_l2", "field_energy",
                   "kinetic_energy", "total_energy", "max_speed", "mean_gamma"]
    # rows at steps 0, 4, 8, ..., 28 and the last step 30
    assert [int(r[0]) for r in rows] == [0, 4, 8, 12, 16, 20, 24, 28, 30]
    assert rows[0][3] == "initial" and all(r[3] == "bdf2" for r in rows[1:])
    # the oracle: the reference's Weibel initializer and step loop, restated
    lib = ol.oracle()
    init = ol.init_weibel(lib.o2_init_weibel, 32, 16, 3.0, 2.0, 4, seed=777)
    prob = ol.P2Problem(32, 16, 3.0, 2.0, 0.05, 2, True, n_steps=30, diag_stride=4)
    out, diag, _, _ = ol.simulate(lib.o2_simulate, prob, init, want_fields=False)
    steps = [int(r[0]) for r in rows]
    for k in range(13):
        a = np.array([float(r[5 + k]) for r in rows])
        b = diag[steps, k]
        scale = max(np.max(np.abs(b)), 1e-300)
        if scale < 1e-9:
            assert np.max(np.abs(a)) < 1e-9, k
        else:
            assert np.max(np.abs(a - b)) <= TOL * scale, (k, np.max(np.abs(a - b)) / scale)
    hdr, ps = read_csv(prefix + "_particle_sample.csv")
    assert hdr == ["id", "x", "y", "x_centered", "y_centered", "vx", "vy", "vz", "q", "m", "gamma"]
    assert len(ps) == 64
    x = np.array([float(r[1]) for r in ps])
    vx = np.array([float(r[5]) for r in ps])
    assert np.max(np.abs(x - out["x"][:64])) < 1e-12
    assert np.max(np.abs(vx - out["v"][:64, 0])) < 1e-12
    echo = open(prefix + "_config_echo.txt").read()
    assert "mobile_electrons = 4096\n" in echo and "static_ions = 0\n" in echo


@pytest.mark.skipif(not os.path.exists(ol.REF_P2_SO if hasattr(ol, "REF_P2_SO") else ""),
                    reason="oracle/_ref/libref_p2.so not built")
@pytest.mark.parametrize("example,charge", [("weibel", "conserving"), ("cloud", "naive"), ("cloud", "conserving")])
def test_deck_matches_reference_cli(tmp_path, example, charge):
    """The same deck through upic_run and through the reference's own main()."""
    kw = dict(example=example, charge_update=charge, method="bdf1" if example == "cloud" else "bdf2")
    if example == "cloud":
        kw.update(nx=32, ny=32, Lx=16.0, Ly=16.0, cloud_particles=3000, cloud_sigma=1.5, cloud_thermal=0.02)
    gdeck, rdeck = str(tmp_path / "g.txt"), str(tmp_path / "r.txt")
    write_deck(gdeck, str(tmp_path / "gpu"), **kw)
    write_deck(rdeck, str(tmp_path / "ref"), **kw)
    run_driver(gdeck)
    ref = ol.ref_p2()
    ref.ref_p2_run_deck.argtypes = [ctypes.c_char_p]
    assert ref.ref_p2_run_deck(rdeck.encode()) == 0
    ha, ra = read_csv(str(tmp_path / "gpu_diagnostics.csv"))
    hb, rb = read_csv(str(tmp_path / "ref_diagnostics.csv"))
    assert ha == hb
    compare_numeric(ra, rb, text_cols={0, 2, 3, 4}, tol=TOL)
    ha, ra = read_csv(str(tmp_path / "gpu_particle_sample.csv"))
    hb, rb = read_csv(str(tmp_path / "ref_particle_sample.csv"))
    assert ha == hb
    compare_numeric(ra, rb, text_cols={0}, tol=1e-12)
    ea = [ln for ln in open(str(tmp_path / "gpu_config_echo.txt")) if not ln.startswith("output_prefix")]
    eb = [ln for ln in open(str(tmp_path / "ref_config_echo.txt")) if not ln.startswith("output_prefix")]
    assert ea == eb


# ---- Project1 decks: upic_run --nonrel -------------------------------------

def write_p1_deck(path, prefix, **kw):
    """A Project1 deck: the keys of Project1/examples/input_landau_weak.txt
    (1D Landau damping, 32x1x1) unless overridden."""
    keys = dict(test_case="landau_weak", nx=32, ny=1, nz=1, Lx=12.566370614359172, Ly=1.0, Lz=1.0, n_steps=60,
                dt=0.1, particles_per_cell=32, spline_order=1, orbit_quad_order=12, split_orbit_at_knots="true",
                c=1.0, eps0=1.0, mu0=1.0, n0=1.0, thermal_velocity=1.0, landau_alpha=0.01, perturbation_mode=1,
                theory_omega=1.4156618886, theory_gamma=-0.1533594669, picard_tol=1.0e-10, picard_max_iter=24,
                final_consistency_sweep="true", run_unit_tests="false")
    keys.update(kw)
    with open(path, "w") as fh:
        fh.write("# Project1 deck written by the test\n")
        for k, v in keys.items():
            fh.write(f"{k} = {v}\n")
        fh.write(f"output_prefix = {prefix}\n")


def run_nonrel(deck):
    r = subprocess.run([RUN, "--nonrel", deck], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


P1_DIAG_TEXT = {0}                 # step
P1_DIAG_ROUNDOFF = {2, 3, 4, 14}   # gauss_rms, gauss_max, gauge_rms, mean_rho


def compare_p1_diagnostics(ra, rb, tol, picard_tol):
    assert len(ra) == len(rb)
    cols = len(ra[0])
    for k in range(cols):
        a = np.array([float(r[k]) for r in ra])
        b = np.array([float(r[k]) for r in rb])
        if k in P1_DIAG_TEXT:
            assert [r[k] for r in ra] == [r[k] for r in rb]
        elif k == 1:  # time, same arithmetic
            assert np.array_equal(a, b)
        elif k in P1_DIAG_ROUNDOFF:
            assert np.max(np.abs(a - b)) < 1e-12, k
        elif k == 15:  # Picard iterations
            assert np.max(np.abs(a - b)) <= 1
        elif k in (16, 17):  # last Picard errors: both below the tolerance
            assert np.all(np.isnan(a[:1])) and np.all(np.isnan(b[:1]))
            assert np.all(a[1:] < picard_tol) and np.all(b[1:] < picard_tol), k
        elif k == 18:  # crossing particles
            assert np.max(np.abs(a - b)) <= 1
        elif k == 20:
            assert np.array_equal(a, b)
        else:
            both_nan = np.isnan(a) & np.isnan(b)
            assert np.array_equal(np.isnan(a), np.isnan(b)), k
            scale = max(np.max(np.abs(b[~both_nan])) if (~both_nan).any() else 0.0, 1e-300)
            d = np.abs(a - b)[~both_nan]
            assert d.size == 0 or np.max(d) <= tol * scale + 1e-15, (k, np.max(d) / scale)


def test_nonrel_usage_and_errors(tmp_path):
    deck = str(tmp_path / "d.txt")
    write_p1_deck(deck, str(tmp_path / "x"), nz=16)
    r = subprocess.run([RUN, "--nonrel", deck], capture_output=True, text=True)
    assert r.returncode == 1 and "nz = 1" in r.stderr
    write_p1_deck(deck, str(tmp_path / "x"), nx=12)
    r = subprocess.run([RUN, "--nonrel", deck], capture_output=True, text=True)
    assert r.returncode == 1 and "powers of two" in r.stderr
    write_p1_deck(deck, str(tmp_path / "x"), test_case="bump_on_tail", n_steps=1)
    r = subprocess.run([RUN, "--nonrel", deck], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown test_case" in r.stderr
    write_p1_deck(deck, str(tmp_path / "x"), landau_alpha=1.5, n_steps=1)
    r = subprocess.run([RUN, "--nonrel", deck], capture_output=True, text=True)
    assert r.returncode == 1 and "|alpha| < 1" in r.stderr


@pytest.mark.skipif(not os.path.exists(ol.REF_P1_SO), reason="oracle/_ref/libref_p1.so not built")
def test_nonrel_initial_particles_match_reference_cli(tmp_path):
    """With n_steps = 0 both programs write the start state: the two-stream
    and Landau initializers give the very same particles (all 17 digits)."""
    ref = ol.ref_p1()
    ref.ref_p1_run_deck.argtypes = [ctypes.c_char_p]
    for case, kw in (("landau_strong", dict(landau_alpha=0.5, nx=16, ny=2)),
                     ("two_stream", dict(nx=16, ny=8, Lx=6.283185307179586, Ly=6.283185307179586,
                                         Lz=6.283185307179586, particles_per_cell=3, spline_order=2))):
        g, r = str(tmp_path / f"g_{case}"), str(tmp_path / f"r_{case}")
        write_p1_deck(g + ".txt", g, test_case=case, n_steps=0, **kw)
        write_p1_deck(r + ".txt", r, test_case=case, n_steps=0, **kw)
        run_nonrel(g + ".txt")
        assert ref.ref_p1_run_deck((r + ".txt").encode()) == 0
        assert open(g + "_particle_sample.csv").read() == open(r + "_particle_sample.csv").read(), case
        assert open(g + "_config_echo.txt").read() == open(r + "_config_echo.txt").read(), case
        ha, ra = read_csv(g + "_diagnostics.csv")
        hb, rb = read_csv(r + "_diagnostics.csv")
        assert ha == hb and len(ra) == 1
        compare_p1_diagnostics(ra, rb, 1e-12, 1e-10)


@pytest.mark.skipif(not os.path.exists(ol.REF_P1_SO), reason="oracle/_ref/libref_p1.so not built")
@pytest.mark.parametrize("case", ["landau_weak", "two_stream_2d"])
def test_nonrel_deck_matches_reference_cli(tmp_path, case):
    """A Project1 deck through upic_run --nonrel and through the reference's
    own main(): every file, header and column."""
    kw = {}
    if case == "two_stream_2d":
        kw = dict(test_case="two_stream", nx=16, ny=8, Lx=6.283185307179586, Ly=6.283185307179586,
                  Lz=6.283185307179586, particles_per_cell=4, spline_order=2, orbit_quad_order=16, n_steps=8,
                  dt=0.025, picard_tol=1e-11, picard_max_iter=16, theory_omega=0.0, theory_gamma=0.0)
    g, r = str(tmp_path / "gpu"), str(tmp_path / "ref")
    write_p1_deck(g + ".txt", g, **kw)
    write_p1_deck(r + ".txt", r, **kw)
    out = run_nonrel(g + ".txt").stdout
    assert "Final total energy" in out
    ref = ol.ref_p1()
    ref.ref_p1_run_deck.argtypes = [ctypes.c_char_p]
    assert ref.ref_p1_run_deck((r + ".txt").encode()) == 0
    ha, ra = read_csv(g + "_diagnostics.csv")
    hb, rb = read_csv(r + "_diagnostics.csv")
    assert ha == hb
    nsteps = len(rb) - 1
    compare_p1_diagnostics(ra, rb, 2e-10 * nsteps, 1e-10 if case == "landau_weak" else 1e-11)
    ha, ra = read_csv(g + "_step_diagnostics.csv")
    hb, rb = read_csv(r + "_step_diagnostics.csv")
    assert ha == hb and len(ra) == len(rb) == nsteps
    for k in range(len(ha)):
        a = np.array([float(x[k]) for x in ra])
        b = np.array([float(x[k]) for x in rb])
        name = ha[k]
        if name in ("step", "time", "max_path_segments"):
            assert np.array_equal(a, b), name
        elif name in ("crossing_particles", "total_crossings"):
            assert np.max(np.abs(a - b)) <= 1, name
        elif name == "avg_path_segments":
            assert np.max(np.abs(a - b)) <= 1.5 / 1024, name
        elif np.max(np.abs(b)) < 1e-10:
            assert np.max(np.abs(a - b)) < 1e-12, name
        else:
            assert np.max(np.abs(a - b)) <= 2e-10 * nsteps * np.abs(b).max() + 1e-12, name
    ha, ra = read_csv(g + "_particle_sample.csv")
    hb, rb = read_csv(r + "_particle_sample.csv")
    assert ha == hb and len(ra) == len(rb)
    assert [x[0] for x in ra] == [x[0] for x in rb]
    for k in range(1, len(ha)):
        a = np.array([float(x[k]) for x in ra])
        b = np.array([float(x[k]) for x in rb])
        assert np.max(np.abs(a - b)) <= 1e-9 * max(np.abs(b).max(), 1.0), ha[k]
    assert open(g + "_config_echo.txt").read() == open(r + "_config_echo.txt").read()


def test_nonrel_unit_tests_pass(tmp_path):
    """run_unit_tests = true: the 2D start-up checks pass, with the
    reference's messages, on the console and in _unit_tests.txt."""
    g = str(tmp_path / "u")
    write_p1_deck(g + ".txt", g, n_steps=2, run_unit_tests="true")
    out = run_nonrel(g + ".txt").stdout
    log = open(g + "_unit_tests.txt").read()
    for line in ("R_A,p chain-rule unit test: abs_rms=", "R_A,p crossing unit test: split_abs_rms=",
                 "Initial Gauss-law unit test: gauss_rms=", "One-step Gauss-law unit test: gauss_rms=",
                 "One-step R_A,p unit test: A_chain_abs_rms=", "One-step deposit/gather work residual="):
        assert line in log and line in out, line
    assert "FAILED" not in log and "Unit tests passed." in out


# ---- Project3 decks: upic_run --p3 -------------------------------------------

def write_p3_deck(path, prefix, **kw):
    """A 2D Project3 deck (two-stream eigenmode, 16x4, five steps of dt 0.1,
    the last one shortened to the remaining time) unless overridden."""
    keys = dict(test_case="cold_relativistic_two_stream", nx=16, ny=4, nz=1, Lx=2.0943951023931953, Ly=1.0, Lz=1.0,
                n_steps=5, dt=0.1, particles_per_cell_pair=4, spline_order=2, orbit_quad_order=8, v0=0.2,
                two_stream_density_alpha=0.001, nyquist_projection="true", run_unit_tests="false")
    keys.update(kw)
    with open(path, "w") as fh:
        fh.write("# Project3 deck written by the test\n")
        for k, v in keys.items():
            fh.write(f"{k} = {v}\n")
        fh.write(f"output_prefix = {prefix}\n")


def run_p3(deck, check=True):
    r = subprocess.run([RUN, "--p3", deck], capture_output=True, text=True, timeout=900)
    if check:
        assert r.returncode == 0, r.stdout + r.stderr
    return r


# columns of the step records: integer counters of the outer solve (one
# iteration more or less is the solver tolerance's reach), the method text,
# residual-level columns (differences of converged iterates, i.e. rounding
# noise of the current amplified by the residual's smallness: the same
# order of magnitude, not the same digits), relative Gauss and gauge
# residuals (discrete identities that hold to rounding),
# wall-clock columns
P3_COUNTERS = {"nonlinear_iterations", "anderson_restarts", "anderson_steps", "picard_fallback_steps",
               "backtracked_steps", "local_particle_iterations_max", "local_iterations_max"}
P3_RESIDUALS = {"nonlinear_rms_residual", "nonlinear_max_particle_residual", "nonlinear_absolute_rms_residual",
                "observed_convergence_rate", "estimated_map_contraction", "max_scaled_particle_residual",
                "local_particle_iterations_mean", "local_iterations_mean"}
P3_NORMALIZED = {"gauss_relative": "gauss_normalization_rms", "gauge_relative": "gauge_normalization_rms"}
# path statistics: a particle ending within rounding of a spline knot may be
# counted on either side
P3_PATHS = {"crossing_particles", "total_crossings", "avg_path_segments", "max_path_segments"}
# energy changes of one step: small differences of the energies, held to
# the energies' own agreement (1e-10 of the kinetic energy)
P3_ENERGY_CHANGES = {"delta_K", "delta_W", "particle_work", "grid_work"}
P3_TEXT = {"convergence_method", "outcome", "wavevector_class", "probe_axis"}
P3_WALL = {"elapsed_wall_seconds"}


def compare_p3_csv(a_path, b_path, tol, energy=0.0, bad=None):
    """Every column of two Project3 CSV files by its kind: counters within
    one, text equal, residual-level columns within a factor 100 on rows whose
    iteration counts agree, relative Gauss / gauge residuals at rounding level
    on both sides or to 1e-6, path statistics within one crossing,
    one-step energy changes to 1e-10 of the kinetic energy (energy), knot
    jumps and representation differences (differences of nearly equal
    probes) to 1e-6, physical values to tol relative to the column's scale,
    round-off-level columns (scale below 1e-9) by level.  Mismatches are
    appended to bad (file, column, detail); without bad the first one fails."""
    own = bad is None
    bad = [] if own else bad
    name_of = os.path.basename(a_path)
    ha, ra = read_csv(a_path)
    hb, rb = read_csv(b_path)
    if ha != hb or len(ra) != len(rb):
        bad.append((name_of, "layout", (len(ha), len(hb), len(ra), len(rb))))
        assert not own, bad
        return ha, ra, rb
    if "nonlinear_iterations" in ha:
        it = ha.index("nonlinear_iterations")
        same = np.array([r1[it] == r2[it] for r1, r2 in zip(ra, rb)])
    else:
        same = np.ones(len(ra), dtype=bool)

    def check(ok, name, detail=None):
        if not ok:
            bad.append((name_of, name, detail))

    for k, name in enumerate(ha):
        if name in P3_WALL:
            continue
        if name in P3_TEXT:
            check(all(r1[k] == r2[k] or (name == "convergence_method" and not s) for r1, r2, s in zip(ra, rb, same)),
                  name)
            continue
        a = np.array([float(r[k]) for r in ra])
        b = np.array([float(r[k]) for r in rb])
        if not (np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(np.isinf(a), np.isinf(b))):
            check(False, name, "nan/inf pattern")
            continue
        fin = np.isfinite(b)
        if not fin.any():
            continue
        d = np.where(fin, np.abs(np.where(fin, a, 0.0) - np.where(fin, b, 0.0)), 0.0)
        if name in P3_COUNTERS:
            check(np.max(d[fin]) <= 1, name, float(np.max(d[fin])))
        elif name in P3_RESIDUALS:
            m = fin & same & (np.abs(b) > 1e-300) & (np.abs(a) > 1e-300)
            if m.any():
                lr = np.abs(np.log10(np.abs(a[m]) / np.abs(b[m])))
                check(np.all(lr <= 2.0), name, float(np.max(lr)))
        elif name in P3_PATHS:
            check(np.max(d[fin]) <= (0.01 if name == "avg_path_segments" else 1), name, float(np.max(d[fin])))
        elif name in P3_ENERGY_CHANGES:
            check(np.max(d[fin]) <= tol * np.max(np.abs(b[fin])) + 1e-10 * energy, name, float(np.max(d[fin])))
        elif name in P3_NORMALIZED:
            # a discrete identity's relative residual: rounding level (below
            # 1e-8) on both sides, or the same value where it is more
            norm = np.array([float(r[ha.index(P3_NORMALIZED[name])]) for r in rb])
            small = np.abs(b) < 1e-8
            check(np.all(np.abs(a[fin & small]) < 1e-8), name, "rounding level")
            m = fin & ~small & (norm > 1e-12)
            if m.any():
                check(np.max(d[m]) <= 1e-6 * np.max(np.abs(b[m])), name, float(np.max(d[m])))
        else:
            scale = np.max(np.abs(b[fin]))
            # knot jumps and representation differences are differences of
            # nearly equal probe values
            rel = 1e-6 if name.endswith("_jump") or name.endswith("_difference") else tol
            if scale < 1e-9:
                check(np.max(np.abs(a[fin])) < 1e-9, name, float(np.max(np.abs(a[fin]))))
            else:
                check(np.max(d[fin]) <= rel * scale, name, float(np.max(d[fin]) / scale))
    assert not (own and bad), bad
    return ha, ra, rb


P3_DECKS = {
    # two-stream eigenmode with a transverse seed: Nyquist projection, field
    # line probes, grid snapshots, transverse diagnostics, particle snapshots
    "two_stream": dict(field_grid_snapshots="true", field_diagnostics_interval=0.2, transverse_diagnostics="true",
                       transverse_spectrum_interval=0.25, tsi_transverse_seed=0.001,
                       particle_snapshot_times="0.1, 0.3"),
    # Weibel eigenmode, cubic splines, probes along y; local iteration limit 2
    # forces the selective sub-cycling fallback on every step
    "weibel_selective": dict(test_case="cold_relativistic_weibel", nx=16, ny=16, Lx=6.283185307179586,
                             Ly=6.283185307179586, n_steps=4, dt=0.2, particles_per_cell_pair=2, spline_order=3,
                             v0=0.5, weibel_B0=0.001, two_stream_density_alpha=-1, nyquist_projection="false",
                             field_probe_points_per_cell=4, field_diagnostics_interval=0.4,
                             selective_particle_fallback="true", particle_local_max_iter=2),
    # Project3's Landau example with the damped-Picard outer solver and a
    # theory envelope
    "landau_picard": dict(test_case="landau", nx=32, ny=2, Lx=12.566370614359172, n_steps=6, particles_per_cell_pair=16,
                          thermal_velocity=0.1, landau_alpha=0.05, spline_order=1, orbit_quad_order=12,
                          nonlinear_solver="picard", theory_gamma=-0.01, theory_omega=1.0, field_diagnostics="false",
                          two_stream_density_alpha=-1, nyquist_projection="false"),
}


def compare_failed_particles(a_path, b_path, tol=1e-9, rtol_res=0.05):
    """_failed_particle_diagnostics.csv: the same header and failure events
    (time, layout restart, map evaluation) with the same number of rows.
    Within an event the particles selected by the worst-residual rule can
    differ where residuals tie to rounding (symmetric cold plasmas, whose
    tied particles differ in sign), so each column's sorted values are
    compared: counters and reasons exactly, the rest as sorted magnitudes to
    tol of the column's largest magnitude (the residual columns,
    differences of nearly equal velocities, to rtol_res); rows of a particle
    that both sides selected are compared column by column."""
    ha, ra = read_csv(a_path)
    hb, rb = read_csv(b_path)
    assert ha == hb
    def events(rows):
        out = {}
        for x in rows:
            out.setdefault((float(x[0]), int(x[1]), int(x[2])), []).append(x)
        return out
    ea, eb = events(ra), events(rb)
    assert sorted(ea) == sorted(eb)
    exact = {"event_exhausted", "failed_particles_in_event", "assigned_substeps", "failed_substep_zero_based",
             "local_iterations", "failure_reason"}
    skip = {"time_before", "layout_refinement_restart", "map_evaluation", "particle_index", "x0_x", "x0_y"}
    residual = {"first_scaled_residual", "final_scaled_residual", "final_absolute_residual"}
    for key in ea:
        a, b = ea[key], eb[key]
        assert len(a) == len(b), key
        for j, name in enumerate(ha):
            if name in skip:
                continue
            if name in exact:
                assert sorted(x[j] for x in a) == sorted(x[j] for x in b), (key, name)
                continue
            va, vb = np.sort([abs(float(x[j])) for x in a]), np.sort([abs(float(x[j])) for x in b])
            # a vector component is held to the vector's magnitude (the z
            # components of these 2D runs are rounding noise)
            group = [k for k, n in enumerate(ha) if name[-2:] in ("_x", "_y", "_z") and n[:-2] == name[:-2]] or [j]
            scale = max(max(abs(float(x[k])) for x in b for k in group), 1e-300)
            assert np.max(np.abs(va - vb)) <= (rtol_res if name in residual else tol) * scale, (key, name)
        ia = {x[ha.index("particle_index")]: x for x in a}
        for x in b:
            y = ia.get(x[ha.index("particle_index")])
            if y is None:
                continue
            for j, name in enumerate(ha):
                if name in exact or j < 3:
                    assert x[j] == y[j], (key, name)
                elif name in residual:
                    assert abs(float(x[j]) - float(y[j])) <= rtol_res * abs(float(x[j])), (key, name)
                elif name != "particle_index":
                    assert abs(float(x[j]) - float(y[j])) <= tol * max(abs(float(x[j])), 1.0), (key, name)


@pytest.mark.skipif(not os.path.exists(ol.REF_P3_SO), reason="oracle/_ref/libref_p3.so not built")
@pytest.mark.parametrize("case", sorted(P3_DECKS))
def test_p3_deck_matches_reference_cli(tmp_path, case):
    """A 2D Project3 deck through upic_run --p3 and through the reference's
    own main(): every output file, header and column."""
    kw = P3_DECKS[case]
    g, r = str(tmp_path / "gpu"), str(tmp_path / "ref")
    write_p3_deck(g + ".txt", g, **kw)
    write_p3_deck(r + ".txt", r, **kw)
    out = run_p3(g + ".txt").stdout
    assert "Final total energy" in out
    ref = ol.ref_p3()
    ref.ref_p3_run_deck.argtypes = [ctypes.c_char_p]
    assert ref.ref_p3_run_deck((r + ".txt").encode()) == 0
    assert open(g + "_config_echo.txt").read() == open(r + "_config_echo.txt").read()
    nsteps = len(read_csv(r + "_step_diagnostics.csv")[1])
    tol = 1e-9 * max(nsteps, 1)
    bad = []
    h, ra, rb = compare_p3_csv(g + "_diagnostics.csv", r + "_diagnostics.csv", tol, bad=bad)
    energy = max(abs(float(x[h.index("kinetic_energy")])) for x in rb)
    compare_p3_csv(g + "_step_diagnostics.csv", r + "_step_diagnostics.csv", tol, energy, bad=bad)
    for f in ("_adaptive_diagnostics.csv", "_particle_inner_history.csv", "_particle_sample.csv",
              "_field_line_probe.csv", "_field_knot_jumps.csv", "_field_grid_snapshots.csv", "_velocity_moments.csv",
              "_field_spectrum.csv", "_particles_t0.10000000000000001.csv", "_particles_t0.29999999999999999.csv"):
        if os.path.exists(r + f):
            compare_p3_csv(g + f, r + f, tol, bad=bad)
    assert not bad, bad
    # every step converged with the reference's method and iteration count
    assert [x[h.index("convergence_method")] for x in ra] == [x[h.index("convergence_method")] for x in rb]
    compare_failed_particles(g + "_failed_particle_diagnostics.csv", r + "_failed_particle_diagnostics.csv")
    names = sorted(os.path.basename(p)[len("ref"):] for p in map(str, tmp_path.glob("ref_*")))
    assert names == sorted(os.path.basename(p)[len("gpu"):] for p in map(str, tmp_path.glob("gpu_*")))
    if case == "weibel_selective":
        info = {n: [float(x[h.index(n)]) for x in ra[1:]] for n in ("selective_fallback_used", "selective_n4")}
        assert all(v == 1 for v in info["selective_fallback_used"]) and max(info["selective_n4"]) > 0


@pytest.mark.skipif(not os.path.exists(ol.REF_P3_SO), reason="oracle/_ref/libref_p3.so not built")
@pytest.mark.parametrize("order", [1, 2, 3])
def test_p3_failed_particles_without_fallback(tmp_path, order):
    """The Weibel deck whose local solves fail, with the selective fallback
    off, for spline orders 1-3 (segment moments at 1 and 2, point gathers
    at 3): both runs stop at the first step, and the failing particles are
    recorded as the reference records them (one exhausted event, the 16
    worst)."""
    kw = dict(P3_DECKS["weibel_selective"], selective_particle_fallback="false", spline_order=order)
    g, r = str(tmp_path / "gpu"), str(tmp_path / "ref")
    write_p3_deck(g + ".txt", g, **kw)
    write_p3_deck(r + ".txt", r, **kw)
    out = run_p3(g + ".txt", check=False)
    assert out.returncode == 1
    ref = ol.ref_p3()
    ref.ref_p3_run_deck.argtypes = [ctypes.c_char_p]
    assert ref.ref_p3_run_deck((r + ".txt").encode()) == 1
    assert "fixed step 1 failed at t=0" in out.stderr + out.stdout
    rows = read_csv(r + "_failed_particle_diagnostics.csv")[1]
    assert 0 < len(rows) <= 16 and all(x[3] == "1" for x in rows)
    compare_failed_particles(g + "_failed_particle_diagnostics.csv", r + "_failed_particle_diagnostics.csv")


def test_p3_unit_tests_pass(tmp_path):
    """run_unit_tests = true: the 2D start-up checks pass, with the
    reference's messages, on the console and in _unit_tests.txt."""
    g = str(tmp_path / "u")
    write_p3_deck(g + ".txt", g, n_steps=1, run_unit_tests="true", field_diagnostics="false")
    out = run_p3(g + ".txt").stdout
    log = open(g + "_unit_tests.txt").read()
    for line in ("Orbit deposit/gather adjoint unit test: residual=", "Initial Gauss-law unit test: gauss_rms=",
                 "One-step Gauss-law unit test: gauss_rms=", "One-step R_A,p unit test: A_chain_abs_rms=",
                 "Small multistep energy unit test: max_rel_drift=", "Instability IC/theory unit test: ts_gamma=",
                 "Two-stream eigenmode growth unit test: gamma_fit="):
        assert line in log and line in out, line
    assert "FAILED" not in log and "Unit tests passed." in out
