"""Host-side checks of upic_run's Project3 deck reader (upic_run --p3, the
drop-in for Project3/ec_pic_nyquist_projected.cpp main): deck errors and
warnings come with the reference's messages (read_config :1178-1433) and end
the run before any device work, so these run without a GPU."""
import os
import subprocess

import pytest

from test_gpu_run import RUN, run_p3, write_p3_deck

pytestmark = pytest.mark.skipif(not os.path.exists(RUN), reason="upic_run is not built")


def test_p3_usage_and_errors(tmp_path):
    """Deck errors end the run with the reference's messages before any
    device work (no GPU needed)."""
    deck = str(tmp_path / "d.txt")
    for kw, text in ((dict(nz=16), "nz = 1"), (dict(nx=12), "powers of two"),
                     (dict(adaptive_dt="true"), "manuscript runs require adaptive_dt=false"),
                     (dict(test_case="bump_on_tail"), "unknown test_case/initial_condition"),
                     (dict(nonlinear_solver="newton"), "nonlinear_solver must be picard or anderson_quasi_newton"),
                     (dict(sigma1=2.0), "Maxwell-compatible nondimensionalization"),
                     (dict(test_case="landau", particles_per_cell_pair=1), "at least two velocity samples"),
                     (dict(test_case="landau", landau_alpha=1.5), "|alpha| < 1"),
                     (dict(particle_snapshot_times="0.1, -2"), "finite and nonnegative"),
                     (dict(selective_particle_max_substeps=12), "power-of-two")):
        write_p3_deck(deck, str(tmp_path / "x"), **kw)
        r = run_p3(deck, check=False)
        assert r.returncode == 1 and text in r.stderr, (kw, r.stderr)
    write_p3_deck(deck, str(tmp_path / "x"), mystery_key=3, c=1.0, n_steps=0, nz=16)
    r = run_p3(deck, check=False)
    assert "warning: unknown input key ignored: mystery_key" in r.stderr
    assert "warning: c is deprecated" in r.stderr
    r = subprocess.run([RUN, "--p3"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
