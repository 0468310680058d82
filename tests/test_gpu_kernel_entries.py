"""Kernel-level push and field-update entry points against the reference's
own functions, called through oracle/_ref/libref_p3.so and libref_p2.so on
the same inputs:

- upic_push_gmhc: the GM-HC-CN particle push (solve_local_particle_substep,
  Project3/ec_pic_nyquist_projected.cpp:4930) in given fields, orders 1-4,
  with and without knot splitting;
- upic_fft_solve_cn: the field half of a map evaluation (continuity update,
  cn_potential_update :3249, grad phi_mid; :5265-5285), with and without the
  Nyquist projection;
- upic_push_iaem: the explicit method's IAEM momentum push
  (push_particles_momentum_and_velocity, Project2/spectral_pic_part3.cpp:1057).

The local fixed point stops at its own tolerance (1e-12 relative), so both
sides take the same iterates up to rounding when they take the same number
of iterations: outputs agree to TOL (relative to each array's scale)."""
import ctypes

import numpy as np
import pytest

import oracle_lib as ol
import unstaggered_pic_b200 as up
from test_gpu_implicit import config_from

pytestmark = pytest.mark.gpu
TOL = 1e-11


def ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def smooth_field(rng, nx, ny, Lx, Ly, amp, modes=3):
    """A sum of a few low Fourier modes on the node grid (x = -L/2 + i dx)."""
    x = -0.5 * Lx + Lx * np.arange(nx) / nx
    y = -0.5 * Ly + Ly * np.arange(ny) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    f = np.zeros((nx, ny))
    for _ in range(modes):
        kx, ky = rng.integers(0, 3, 2)
        ph = rng.uniform(0, 2 * np.pi)
        f += amp * rng.normal() * np.cos(2 * np.pi * (kx * X / Lx + ky * Y / Ly) + ph)
    return f


def ref_lib():
    lib = ol.ref_p3()
    if lib is None:
        pytest.skip("oracle/_ref/libref_p3.so is not built")
    return lib


@pytest.mark.parametrize("order,split", [(1, True), (2, True), (2, False), (3, True), (4, True)])
def test_push_gmhc_matches_reference(order, split):
    lib = ref_lib()
    nx, ny, Lx, Ly = 16, 8, 4.0, 2.0
    prob = ol.P3Problem(nx, ny, Lx, Ly, 0.3, order=order, nq=8, split=split, nyquist=True)
    rng = np.random.default_rng(40 + order)
    gpm = np.stack([smooth_field(rng, nx, ny, Lx, Ly, 0.3) for _ in range(2)] + [np.zeros((nx, ny))])
    An = np.stack([smooth_field(rng, nx, ny, Lx, Ly, 0.2) for _ in range(3)])
    Ae = An + np.stack([smooth_field(rng, nx, ny, Lx, Ly, 0.02) for _ in range(3)])
    n = 300
    x0 = np.zeros((n, 3))
    x0[:, 0] = rng.uniform(-Lx / 2, Lx / 2, n)
    x0[:, 1] = rng.uniform(-Ly / 2, Ly / 2, n)
    v = 0.4 * rng.uniform(-1, 1, (n, 3))
    q = np.full(n, -0.01)
    m = np.full(n, 0.01)
    P = m[:, None] * v / np.sqrt(1 - np.sum(v * v, 1))[:, None] + 0.3 * rng.normal(size=(n, 3)) * 0.01
    # the reference
    ref = {k: np.zeros((n, 3)) for k in ("x1", "P_end", "v_end", "vbar")}
    rep = np.zeros((n, 2), dtype=np.int32)
    rc = lib.ref_p3_push_gmhc(ptr(prob.dparams()), prob.iparams().ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              ctypes.c_long(n), ptr(x0), ptr(P), ptr(v), ptr(q), ptr(m),
                              ptr(np.ascontiguousarray(gpm.reshape(3, -1))), ptr(np.ascontiguousarray(An.reshape(3, -1))),
                              ptr(np.ascontiguousarray(Ae.reshape(3, -1))), ptr(ref["x1"]), ptr(ref["P_end"]),
                              ptr(ref["v_end"]), ptr(ref["vbar"]), rep.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    assert rc == 0
    with up.Simulation(config_from(prob.dparams(), prob.iparams())) as sim:
        out = sim.push_gmhc(x0[:, 0], x0[:, 1], P, v, q, m, gpm[:2], An, Ae)
        again = sim.push_gmhc(x0[:, 0], x0[:, 1], P, v, q, m, gpm[:2], An, Ae)
    assert np.array_equal(out["vbar"], again["vbar"], equal_nan=True)  # deterministic
    ok = rep[:, 1] == 0
    assert ok.sum() > 0.9 * n
    assert np.array_equal(out["report"][:, 1] == 0, ok)
    assert np.max(np.abs(out["report"][ok, 0] - rep[ok, 0])) <= 1
    same = ok & (out["report"][:, 0] == rep[:, 0])
    assert same.sum() > 0.9 * ok.sum()
    for k in ("P_end", "v_end", "vbar"):
        d = np.abs(out[k][same] - ref[k][same])
        assert np.max(d) <= TOL * np.max(np.abs(ref[k][ok])), k
    dx = out["x1"][same] - ref["x1"][same, 0]
    dy = out["y1"][same] - ref["x1"][same, 1]
    dx -= Lx * np.round(dx / Lx)
    dy -= Ly * np.round(dy / Ly)
    assert np.max(np.abs(dx)) <= TOL * Lx and np.max(np.abs(dy)) <= TOL * Ly
    assert np.all(np.isnan(out["vbar"][~ok]))


@pytest.mark.parametrize("nyquist", [True, False])
def test_fft_solve_cn_matches_reference(nyquist):
    lib = ref_lib()
    nx, ny, Lx, Ly = 16, 32, 3.0, 5.0
    prob = ol.P3Problem(nx, ny, Lx, Ly, 0.2, order=2, nyquist=nyquist)
    rng = np.random.default_rng(7)
    f = {k: rng.normal(size=(nx, ny)) for k in ("phi", "psi", "rho")}
    for k in ("A", "U", "J"):
        f[k] = rng.normal(size=(3, nx, ny))
    N = nx * ny
    ref = {"phi": np.zeros(N), "psi": np.zeros(N), "rho": np.zeros(N), "A": np.zeros(3 * N), "U": np.zeros(3 * N),
           "gpm": np.zeros(3 * N)}
    c = {k: np.ascontiguousarray(v.ravel()) for k, v in f.items()}
    rc = lib.ref_p3_fft_solve_cn(ptr(prob.dparams()), prob.iparams().ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 ptr(c["phi"]), ptr(c["psi"]), ptr(c["rho"]), ptr(c["A"]), ptr(c["U"]), ptr(c["J"]),
                                 ptr(ref["phi"]), ptr(ref["psi"]), ptr(ref["rho"]), ptr(ref["A"]), ptr(ref["U"]),
                                 ptr(ref["gpm"]))
    assert rc == 0
    with up.Simulation(config_from(prob.dparams(), prob.iparams())) as sim:
        out = sim.fft_solve_cn(f["phi"], f["psi"], f["rho"], f["A"], f["U"], f["J"])
    for k in ("phi", "psi", "rho", "A", "U"):
        b = ref[k]
        assert np.max(np.abs(out[k].ravel() - b)) <= 1e-13 * np.max(np.abs(b)), k
    g = ref["gpm"].reshape(3, N)[:2]
    assert np.max(np.abs(out["grad_phi_mid"].reshape(2, N) - g)) <= 1e-13 * np.max(np.abs(g))


def test_push_iaem_matches_reference():
    """upic_push_iaem against the reference's push_particles_momentum_and_velocity
    (spectral_pic_part3.cpp:1057) with its own spectral gradients, on random
    fields and particles (Project2 coordinates, [0, L))."""
    lib = ol.ref_p2()
    if lib is None:
        pytest.skip("oracle/_ref/libref_p2.so is not built")
    nx, ny, Lx, Ly, dt, c = 32, 16, 6.0, 3.0, 0.05, 1.0
    rng = np.random.default_rng(11)
    phi = rng.normal(size=(nx, ny))
    A = 0.3 * rng.normal(size=(3, nx, ny))
    n = 500
    x, y = rng.uniform(0, Lx, n), rng.uniform(0, Ly, n)
    v = 0.3 * rng.uniform(-1, 1, (n, 3))
    vp = v + 0.01 * rng.normal(size=(n, 3))
    q, m = np.full(n, -0.02), np.full(n, 0.02)
    P = m[:, None] * v / np.sqrt(1 - np.sum(v * v, 1))[:, None]
    ref = [np.ascontiguousarray(a).copy() for a in (P, v, vp)]
    rc = lib.ref_p2_push_iaem(nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), ctypes.c_double(dt),
                              ctypes.c_double(c), ctypes.c_long(n), ptr(np.ascontiguousarray(x)),
                              ptr(np.ascontiguousarray(y)), ptr(ref[0]), ptr(ref[1]), ptr(ref[2]),
                              ptr(np.ascontiguousarray(q)), ptr(np.ascontiguousarray(m)),
                              ptr(np.ascontiguousarray(phi.ravel())), ptr(np.ascontiguousarray(A.ravel())))
    assert rc == 0
    cfg = up.Config(nx=nx, ny=ny, Lx=Lx, Ly=Ly, dt=dt, method="bdf1", c=c)
    with up.Simulation(cfg) as sim:
        Pn, vn, wn = sim.push_iaem(x, y, P, v, vp, q, m, phi, A)
    for a, b, name in ((Pn, ref[0], "P"), (vn, ref[1], "v")):
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b)), name
    assert np.array_equal(wn, v)
    assert np.array_equal(ref[2], v)
