"""upic_set_particles rejects a particle set with a non-finite position or
velocity (UPIC_ERR_NONFINITE) for every method and precision, whichever
side checks it (the explicit FP64 upload checks positions and velocities on
the device), and the context takes a valid set afterwards: the run then
equals a run on a fresh context."""
import numpy as np
import pytest

import unstaggered_pic_b200 as up
from unstaggered_pic_b200._native import UPIC_ERR

pytestmark = pytest.mark.gpu
L = 2 * np.pi / 0.3


def plasma(n=16, ppc=8, seed=3):
    return up.generate_bimaxwellian(n, n, L, L, ppc, (0.02, 0.2, 0.02), seed=seed)


def load(sim, p, shift=0.0):
    sim.set_particles(p["x"] + shift, p["y"] + shift, p["P"], p["v"], p["v_prev"], p["q"], p["m"])


CONFIGS = {
    "explicit_fp64": lambda: up.Config(nx=16, ny=16, Lx=L, Ly=L, dt=0.05),
    "explicit_mixed": lambda: up.Config(nx=16, ny=16, Lx=L, Ly=L, dt=0.05, precision="mixed"),
    "implicit": lambda: up.ImplicitConfig(nx=16, ny=16, Lx=L, Ly=L, dt=0.05),
}


@pytest.mark.parametrize("kind", sorted(CONFIGS))
@pytest.mark.parametrize("bad", ["x", "y", "vx", "vz_inf"])
def test_nonfinite_particle_is_rejected(kind, bad):
    p = plasma()
    shift = -L / 2 if kind == "implicit" else 0.0
    q = {k: np.array(v, copy=True) for k, v in p.items()}
    i = len(q["x"]) // 3
    if bad == "x":
        q["x"][i] = np.nan
    elif bad == "y":
        q["y"][i] = np.nan
    elif bad == "vx":
        q["v"][i, 0] = np.nan
    else:
        q["v"][i, 2] = np.inf
    with up.Simulation(CONFIGS[kind]()) as sim:
        with pytest.raises(up.UpicError) as e:
            load(sim, q, shift)
        assert UPIC_ERR[e.value.code] == "UPIC_ERR_NONFINITE"
        load(sim, p, shift)
        sim.init_fields(False)
        if kind == "implicit":
            sim.step_implicit(1, diagnostics=False)
        else:
            sim.step(2, 0)
        a = sim.get_particles()
    with up.Simulation(CONFIGS[kind]()) as sim:
        load(sim, p, shift)
        sim.init_fields(False)
        if kind == "implicit":
            sim.step_implicit(1, diagnostics=False)
        else:
            sim.step(2, 0)
        b = sim.get_particles()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
