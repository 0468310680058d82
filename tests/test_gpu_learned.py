"""GPU tests of the learned first guess (current_predictor = learned): the
network's tensor-core convolution and weight gradient against numpy on the
same bf16 inputs, and implicit runs that use the predictor: the same
converged solution as the reference's previous-current guess, a falling
training loss, and bit-for-bit checkpoint / restart of the trained state."""
import numpy as np
import pytest

import unstaggered_pic_b200 as up

pytestmark = pytest.mark.gpu

DECK = dict(Lz=1.0, kappa=1.0, sigma1=1.0, sigma2=1.0, n0=1.0, spline_order=2, orbit_quad_order=8,
            split_orbit_at_knots=True, nyquist_projection=True, nonlinear_solver="anderson_quasi_newton",
            nonlinear_rtol=1e-11, nonlinear_atol=1e-13, nonlinear_max_iter=80, anderson_memory=4,
            anderson_start=2, anderson_damping=0.5, anderson_regularization=1e-12, anderson_growth_limit=1.2,
            uniform_local_rtol=1e-12, uniform_local_atol=1e-14, uniform_local_max_iter=64,
            uniform_local_damping=1.0)
FIELDS = ["phi", "psi", "rho", "Ax", "Ay", "Az", "Ux", "Uy", "Uz", "Jx", "Jy", "Jz"]


def to_bf16(a):
    """float32 -> bf16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


def taps():
    return [(t // 3 - 1, t % 3 - 1) for t in range(9)]


def conv_ref(x, w, sign):
    """out[ix, iy, n] = sum_t,c x[ix + sign dx_t, iy + sign dy_t, c] w[n, t*32 + c] (periodic), float64,
    and the sum of |terms| for the tolerance."""
    xf = from_bf16(x).astype(np.float64)
    wf = from_bf16(w).astype(np.float64).reshape(32, 9, 32)
    out = np.zeros(x.shape[:2] + (32,))
    mag = np.zeros_like(out)
    for t, (dx, dy) in enumerate(taps()):
        xs = np.roll(xf, shift=(-sign * dx, -sign * dy), axis=(0, 1))
        out += xs @ wf[:, t, :].T
        mag += np.abs(xs) @ np.abs(wf[:, t, :]).T
    return out, mag


@pytest.fixture(scope="module")
def ctx():
    sim = up.Simulation(up.Config(nx=8, ny=8, Lx=1.0, Ly=1.0, dt=0.05, method="bdf1"))
    yield sim
    sim.close()


@pytest.mark.parametrize("shape", [(16, 16), (12, 10), (64, 1), (128, 64)])
@pytest.mark.parametrize("sign", [1, -1])
def test_conv_matches_numpy(ctx, shape, sign):
    """Linear mode (fp32 out): the tensor-core implicit GEMM equals the
    float64 sum of the same bf16 products to fp32 accumulation error; ReLU
    and mask modes round the same values once to bf16."""
    rng = np.random.default_rng(7 + shape[0] + sign)
    x = to_bf16(rng.normal(size=shape + (32,)))
    w = to_bf16(rng.normal(size=(32, 288)) / 17.0)
    bias = rng.normal(size=32).astype(np.float32)
    ref, mag = conv_ref(x, w, sign)
    got = ctx.guess_conv(x, w, mode="linear", sign=sign)
    assert np.all(np.abs(got - ref) <= 2e-6 * mag + 1e-30), np.max(np.abs(got - ref) / mag)
    relu = ctx.guess_conv(x, w, bias=bias, mode="relu", sign=sign)
    want = np.maximum(got + bias, 0.0).astype(np.float32)
    assert np.all(np.abs(from_bf16(relu) - want) <= 2 ** -7 * np.abs(want) + 1e-30)
    mask = to_bf16(rng.normal(size=shape + (32,)))
    masked = ctx.guess_conv(x, w, mask=mask, mode="mask", sign=sign)
    want = np.where(from_bf16(mask) > 0, got, 0.0).astype(np.float32)
    assert np.all(np.abs(from_bf16(masked) - want) <= 2 ** -7 * np.abs(want) + 1e-30)


@pytest.mark.parametrize("shape", [(16, 16), (40, 24)])
def test_wgrad_matches_numpy(ctx, shape):
    rng = np.random.default_rng(11 + shape[0])
    x = to_bf16(rng.normal(size=shape + (32,)))
    dz = to_bf16(rng.normal(size=shape + (32,)))
    gw, gb = ctx.guess_wgrad(dz, x)
    xf = from_bf16(x).astype(np.float64)
    dzf = from_bf16(dz).astype(np.float64).reshape(-1, 32)
    for t, (dx, dy) in enumerate(taps()):
        xs = np.roll(xf, shift=(-dx, -dy), axis=(0, 1)).reshape(-1, 32)
        ref = dzf.T @ xs
        mag = np.abs(dzf).T @ np.abs(xs)
        assert np.all(np.abs(gw[:, t * 32:(t + 1) * 32] - ref) <= 1e-5 * mag), t
    assert np.allclose(gb, dzf.sum(axis=0), rtol=0, atol=1e-5 * np.abs(dzf).sum(axis=0).max())


def make_sim(predictor, **kw):
    cfg = up.ImplicitConfig(nx=32, ny=32, Lx=2 * np.pi / 0.3, Ly=2 * np.pi / 0.3, dt=0.05,
                            current_predictor=predictor, **DECK, **kw)
    sim = up.Simulation(cfg)
    p = up.generate_bimaxwellian(32, 32, cfg.Lx, cfg.Ly, 16, (0.05, 0.05, 0.05), seed=31)
    sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
    sim.init_fields()
    return sim


def test_learned_predictor_same_solution():
    """The learned guess converges to the previous-current guess's solution
    at the same tolerances; the predictor's report: previous guess on the
    first step, extrapolation on the second, training from the third, the
    training loss falls."""
    nsteps, train = 24, 18
    cols = up.SOLVE_INFO_COLUMNS
    out = {}
    for pred in ("previous", "learned"):
        sim = make_sim(pred, learned_train_steps=train, learned_train_iters=8)
        try:
            _, info = sim.step_implicit(nsteps)
            out[pred] = (info, np.stack([sim.field(f) for f in FIELDS]), sim.get_particles())
        finally:
            sim.close()
    info_p, f_p, p_p = out["previous"]
    info_l, f_l, p_l = out["learned"]
    assert np.all(info_l[:, cols.index("converged")] == 1)
    for k, f in enumerate(FIELDS):
        scale = np.max(np.abs(f_p[k])) + 1e-300
        assert np.max(np.abs(f_l[k] - f_p[k])) / scale < 1e-8, f
    assert np.max(np.abs(p_l["v"] - p_p["v"])) < 1e-8 * np.max(np.abs(p_p["v"]))
    used = info_l[:, cols.index("predictor_used")]
    assert used[0] == 0 and used[1] == 1 and np.all(used[1:] >= 1)
    loss = info_l[:, cols.index("learned_loss")]
    assert np.all(np.isnan(loss[:2])) and np.all(np.isfinite(loss[2:2 + train]))
    assert np.all(np.isnan(loss[2 + train:]))
    # the first samples follow the start-up transient; past it the loss falls
    assert np.mean(loss[2 + train - 4:2 + train]) < 0.2 * np.max(loss[2:6]), loss
    lerr = info_l[:, cols.index("learned_error")]
    assert np.all(np.isnan(lerr[:3])) and np.all(np.isfinite(lerr[3:]))
    # the guess used is the better of the two on the step before, so its
    # distance is one of the two reported
    g = info_l[3:, cols.index("guess_error")]
    x = info_l[3:, cols.index("extrapolation_error")]
    assert np.all((g == x) | (g == lerr[3:]))
    # the previous-current run reports the distance of its own guess only
    assert np.all(np.isnan(info_p[:, cols.index("extrapolation_error")]))


def test_learned_predictor_restart_is_bitwise(tmp_path):
    path = str(tmp_path / "state.bin")
    kw = dict(learned_train_steps=10, learned_train_iters=2)
    sim = make_sim("learned", **kw)
    try:
        sim.step_implicit(6)
        sim.save_state(path)
        _, info_a = sim.step_implicit(4)
        fa = np.stack([sim.field(f) for f in FIELDS])
    finally:
        sim.close()
    cfg = up.ImplicitConfig(nx=32, ny=32, Lx=2 * np.pi / 0.3, Ly=2 * np.pi / 0.3, dt=0.05,
                            current_predictor="learned", **DECK, **kw)
    with up.Simulation(cfg) as sim:
        sim.load_state(path)
        _, info_b = sim.step_implicit(4)
        fb = np.stack([sim.field(f) for f in FIELDS])
    assert np.array_equal(info_a, info_b, equal_nan=True)
    assert np.array_equal(fa, fb)


class NonrelLearned(up.NonrelConfig):
    def to_c(self):
        cfg = super().to_c()
        cfg.current_predictor = up.PREDICTORS["learned"]
        return cfg


def test_learned_predictor_config_errors():
    with pytest.raises(up.UpicError):
        up.Simulation(NonrelLearned(nx=8, ny=8))
    with pytest.raises(up.UpicError):
        up.Simulation(up.ImplicitConfig(nx=8, ny=8, current_predictor="learned", learned_train_iters=0))
