"""CPU checks of the C ABI library: it loads, exports every function that
include/upic.h declares, and fails cleanly (no crash) without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from unstaggered_pic_b200 import _native
import unstaggered_pic_b200 as up

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "upic.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(upic_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in _native.SYMBOLS, f"{n} missing from the ctypes binding"


def test_abi_version_and_config_defaults():
    L = _native.lib()
    assert L.upic_abi_version() == 2
    cfg = _native.UpicConfig()
    assert L.upic_config_default(ctypes.byref(cfg)) == 0
    # reference Config defaults (spectral_pic_part3.cpp:174-231)
    assert (cfg.nx, cfg.ny, cfg.method, cfg.charge_update) == (32, 32, 1, 0)
    assert cfg.dt == 0.05 and cfg.c == 1.0 and cfg.eps0 == 1.0 and cfg.mu0 == 1.0 and cfg.n0 == 1.0
    assert abs(cfg.Lx - 2 * np.pi) < 1e-15
    # implicit-method defaults (ec_pic_nyquist_projected.cpp:837-1005)
    assert (cfg.spline_order, cfg.orbit_quad_order, cfg.split_orbit_at_knots, cfg.nyquist_projection) == \
        (2, 16, 1, 0)
    assert (cfg.nonlinear_solver, cfg.nonlinear_max_iter, cfg.anderson_memory, cfg.anderson_start,
            cfg.local_max_iter, cfg.perturbation_mode) == (0, 32, 4, 2, 24, 1)
    assert (cfg.kappa, cfg.sigma1, cfg.sigma2) == (1.0, 1.0, 1.0)
    assert (cfg.nonlinear_rtol, cfg.nonlinear_atol, cfg.anderson_damping, cfg.anderson_regularization,
            cfg.anderson_growth_limit) == (1e-12, 1e-13, 0.7, 1e-12, 1.2)
    assert (cfg.local_rtol, cfg.local_atol, cfg.local_damping) == (1e-11, 1e-13, 1.0)


def test_config_struct_layout_matches_header():
    """The ctypes mirror has the C struct's size and field offsets."""
    import subprocess
    import tempfile
    fields = [f[0] for f in _native.UpicConfig._fields_]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"upic.h\"\nint main(void){printf(\"%zu\"" + \
        "".join(' \" %zu\"' for _ in fields) + ", sizeof(upic_config)" + \
        "".join(f", offsetof(upic_config, {f})" for f in fields) + ");return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = [int(t) for t in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()]
    assert out[0] == ctypes.sizeof(_native.UpicConfig)
    for f, off in zip(fields, out[1:]):
        assert getattr(_native.UpicConfig, f).offset == off, f


@pytest.mark.parametrize("kw,code", [(dict(nx=48), -1), (dict(method="bdf3"), None),
                                     (dict(charge_update=5), -1), (dict(dt=-1.0), -1)])
def test_config_validation_errors(kw, code):
    """read_config validation (spectral_pic_part3.cpp:281-293) maps to
    UPIC_ERR_CONFIG; it is checked before any device work."""
    if kw.get("method") == "bdf3":
        with pytest.raises(KeyError):
            up.Config(**kw).to_c()
        return
    with pytest.raises(up.UpicError) as e:
        up.Simulation(up.Config(**kw))
    assert e.value.code == code


def test_create_without_gpu_fails_cleanly(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(up.UpicError) as e:
        up.Simulation(up.Config())
    assert e.value.code == -3


def test_generator_deterministic_and_distributed():
    a = up.generate_bimaxwellian(16, 8, 3.0, 2.0, 64, (0.02, 0.2, 0.05), seed=9)
    b = up.generate_bimaxwellian(16, 8, 3.0, 2.0, 64, (0.02, 0.2, 0.05), seed=9)
    c = up.generate_bimaxwellian(16, 8, 3.0, 2.0, 64, (0.02, 0.2, 0.05), seed=10)
    for k in a:
        assert np.array_equal(a[k], b[k])
    assert not np.array_equal(a["x"], c["x"])
    n = 16 * 8 * 64
    assert a["x"].shape == (n,) and a["P"].shape == (n, 3)
    assert np.all((a["x"] >= 0) & (a["x"] < 3.0)) and np.all((a["y"] >= 0) & (a["y"] < 2.0))
    # every cell holds exactly ppc particles, in cell-major order
    cell = (a["x"] // (3.0 / 16)).astype(int) * 8 + (a["y"] // (2.0 / 8)).astype(int)
    assert np.array_equal(cell, np.repeat(np.arange(16 * 8), 64))
    u = a["P"] / a["m"][:, None]  # normalized momentum gamma v / c
    assert np.allclose(u.std(0), [0.02, 0.2, 0.05], rtol=0.05)
    assert np.allclose(a["q"].sum(), -3.0 * 2.0)  # neutralizes n0 = 1
    gam = np.sqrt(1 + (u * u).sum(1))
    assert np.allclose(a["v"], u / gam[:, None], rtol=1e-15, atol=1e-18)
    assert np.array_equal(a["v"], a["v_prev"])
