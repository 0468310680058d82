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
