"""Derived field output: E and B through upic_get_field and Project3's field
grid snapshot (upic_write_field_snapshot).

The implicit method's E = -grad phi - U and B = curl A (compute_E,
spectral_curl, Project3/ec_pic_nyquist_projected.cpp:3338, :1780) are checked
against the same formulas applied in numpy (FP64 FFTs, Nyquist-zeroed wave
numbers) to the reference's own fields of the fixture run, and the explicit
method's E = -grad phi - dA/dt (BDF1) and B = curl A
(Project2/spectral_pic_part3.cpp:918-944) against numpy on two consecutive
time levels and against the step's diagnostics row (E_l2, Bz_l2, B_l2), whose
columns are parity-tested against the reference."""
import csv
import os

import numpy as np
import pytest

import unstaggered_pic_b200 as up
from test_gpu_implicit import load_sim

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


def gold(name):
    return dict(np.load(os.path.join(GOLD, name)))


def relerr(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))


def wavenumbers(n, L):
    k = np.array([0 if i == n // 2 else (i if i < n // 2 else i - n) for i in range(n)], dtype=np.float64)
    return 2 * np.pi * k / L


def ddx(f, L, axis):
    n = f.shape[axis]
    k = wavenumbers(n, L)
    shape = [1, 1]
    shape[axis] = n
    return np.fft.ifft2(1j * k.reshape(shape) * np.fft.fft2(f)).real


def test_implicit_E_B_and_snapshot(tmp_path):
    g = gold("p3_run_o2_anderson.npz")
    sim, cfg = load_sim(g)
    sim.init_fields(True)
    nsteps = int(g["iparams"][12])
    sim.step_implicit(nsteps)
    f = {n: sim.field(n) for n in up.FIELDS}
    Lx, Ly = cfg.Lx, cfg.Ly
    # against the numpy formulas on the reference's own fields of the same run
    ref = g["fields"]  # phi, psi, rho, A(3), U(3), J(3) after the last step
    phi, A, U = ref[0], ref[3:6], ref[6:9]
    Eref = [-ddx(phi, Lx, 0) - U[0], -ddx(phi, Ly, 1) - U[1], -U[2]]
    Bref = [ddx(A[2], Ly, 1), -ddx(A[2], Lx, 0), ddx(A[1], Lx, 0) - ddx(A[0], Ly, 1)]
    Emag = max(np.max(np.abs(e)) for e in Eref)
    Bmag = max(np.max(np.abs(b)) for b in Bref)
    for k, n in enumerate(("Ex", "Ey", "Ez")):
        assert np.max(np.abs(f[n] - Eref[k])) / Emag < 2e-10, n  # the step's solver tolerance
    for k, n in enumerate(("Bx", "By", "Bz")):
        assert np.max(np.abs(f[n] - Bref[k])) / Bmag < 2e-10, n
    # and against the same formulas on this run's own fields (round-off only)
    Eown = [-ddx(f["phi"], Lx, 0) - f["Ux"], -ddx(f["phi"], Ly, 1) - f["Uy"], -f["Uz"]]
    Bown = [ddx(f["Az"], Ly, 1), -ddx(f["Az"], Lx, 0), ddx(f["Ay"], Lx, 0) - ddx(f["Ax"], Ly, 1)]
    for k, n in enumerate(("Ex", "Ey", "Ez")):
        assert np.max(np.abs(f[n] - Eown[k])) / Emag < TOL, n
    for k, n in enumerate(("Bx", "By", "Bz")):
        assert np.max(np.abs(f[n] - Bown[k])) / Bmag < TOL, n
    # Project3's snapshot columns and values
    path = tmp_path / "run_field_grid_snapshots.csv"
    sim.write_field_snapshot(path, nsteps, nsteps * cfg.dt)
    sim.write_field_snapshot(path, nsteps, nsteps * cfg.dt, append=True)
    sim.close()
    with open(path) as fh:
        rows = list(csv.reader(fh))
    assert rows[0] == ("step,time,spline_order,ix,iy,iz,x,y,z,phi,psi,rho,"
                       "Ax,Ay,Az,Ux,Uy,Uz,Jx,Jy,Jz,Ex,Ey,Ez,Bx,By,Bz").split(",")
    nx, ny = cfg.nx, cfg.ny
    assert len(rows) == 1 + 2 * nx * ny
    data = np.array([[float(v) for v in r] for r in rows[1:1 + nx * ny]])
    assert np.all(data[:, 0] == nsteps) and np.all(data[:, 2] == cfg.spline_order)
    assert np.array_equal(data[:, 3], np.repeat(np.arange(nx), ny))
    assert np.array_equal(data[:, 4], np.tile(np.arange(ny), nx))
    assert np.allclose(data[:, 6], -Lx / 2 + data[:, 3] * Lx / nx, rtol=0, atol=1e-15 * Lx)
    names = ["phi", "psi", "rho", "Ax", "Ay", "Az", "Ux", "Uy", "Uz", "Jx", "Jy", "Jz", "Ex", "Ey", "Ez", "Bx",
             "By", "Bz"]
    for k, n in enumerate(names):
        assert np.array_equal(data[:, 9 + k], f[n].ravel()), n  # %.17g round-trips exactly


def test_explicit_E_B_against_numpy_and_diagnostics():
    nx, ny, L, dt = 32, 64, 2 * np.pi / 0.3, 0.05
    p = up.generate_bimaxwellian(nx, ny, L, L, 8, (0.02, 0.2, 0.0), seed=9)
    cols = {c: i for i, c in enumerate(up.DIAG_COLUMNS)}
    with up.Simulation(up.Config(nx=nx, ny=ny, Lx=L, Ly=L, dt=dt, method="bdf1")) as sim:
        sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
        row0 = sim.init_fields(True)
        # start-up: dA/dt = 0 in the step-0 row
        E0 = np.stack([sim.field(n) for n in ("Ex", "Ey", "Ez")])
        assert relerr(np.sqrt(np.mean(np.sum(E0 ** 2, axis=0))), row0[cols["E_l2"]]) < TOL
        sim.step(6, 1)
        A_prev = np.stack([sim.field(n) for n in ("Ax", "Ay", "Az")])
        row = sim.step(1, 1)[-1]
        phi = sim.field("phi")
        A = np.stack([sim.field(n) for n in ("Ax", "Ay", "Az")])
        E = np.stack([sim.field(n) for n in ("Ex", "Ey", "Ez")])
        B = np.stack([sim.field(n) for n in ("Bx", "By", "Bz")])
    At = (A - A_prev) / dt
    Eref = np.stack([-ddx(phi, L, 0) - At[0], -ddx(phi, L, 1) - At[1], -At[2]])
    Bref = np.stack([ddx(A[2], L, 1), -ddx(A[2], L, 0), ddx(A[1], L, 0) - ddx(A[0], L, 1)])
    assert relerr(E, Eref) < 1e-10  # A_t amplifies the FP64 rounding of A by 1/dt
    assert relerr(B, Bref) < TOL
    assert relerr(np.sqrt(np.mean(np.sum(E ** 2, axis=0))), row[cols["E_l2"]]) < TOL
    assert relerr(np.sqrt(np.mean(B[2] ** 2)), row[cols["Bz_l2"]]) < TOL
    assert relerr(np.sqrt(np.mean(np.sum(B ** 2, axis=0))), row[cols["B_l2"]]) < TOL


def test_snapshot_rejects_explicit_method(tmp_path):
    with up.Simulation(up.Config(nx=8, ny=8, Lx=1.0, Ly=1.0, dt=0.05)) as sim:
        p = up.generate_bimaxwellian(8, 8, 1.0, 1.0, 2, (0.02, 0.2, 0.0), seed=1)
        sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
        sim.init_fields(False)
        with pytest.raises(up.UpicError):
            sim.write_field_snapshot(tmp_path / "x.csv", 0, 0.0)


def bspline(r, x):
    """Centred cardinal B-spline of degree r and its derivative (the
    truncated-power form of the r+1-fold box convolution)."""
    from math import comb, factorial

    def B(deg, t):
        if deg == 0:
            return ((t >= -0.5) & (t < 0.5)).astype(np.float64)
        s = np.zeros_like(t)
        for k in range(deg + 2):
            s += (-1) ** k * comb(deg + 1, k) * np.maximum(t + (deg + 1) / 2 - k, 0.0) ** deg
        return s / factorial(deg)

    return B(r, x), B(r - 1, x + 0.5) - B(r - 1, x - 0.5)


def test_probe_fields_match_numpy():
    """upic_probe_fields (the shape gathers and shape gradients behind
    Project3's field line probes, evaluate_reconstructed_field_probe
    :7924) against the same sums in numpy over the run's own fields, at
    points inside and outside the box."""
    g = gold("p3_run_o2_anderson.npz")
    sim, cfg = load_sim(g)
    sim.init_fields(True)
    sim.step_implicit(2)
    order = cfg.spline_order
    nx, ny, Lx, Ly = cfg.nx, cfg.ny, cfg.Lx, cfg.Ly
    dx, dy = Lx / nx, Ly / ny
    names = ["phi", "psi", "rho", "Ax", "Ay", "Az", "Ux", "Uy", "Uz", "Jx", "Jy", "Jz", "Ex", "Ey", "Ez", "Bx", "By",
             "Bz"]
    F = np.stack([sim.field(n) for n in names])
    rng = np.random.default_rng(5)
    x = rng.uniform(-0.75 * Lx, 0.75 * Lx, 40)
    y = rng.uniform(-0.75 * Ly, 0.75 * Ly, 40)
    out = sim.probe_fields(x, y)
    assert out.shape == (40, len(up.PROBE_COLUMNS))
    want = np.zeros_like(out)
    for p in range(40):
        u, v = (x[p] + 0.5 * Lx) / dx, (y[p] + 0.5 * Ly) / dy
        il, jl = int(np.floor(u - 0.5 * (order - 1))), int(np.floor(v - 0.5 * (order - 1)))
        for a in range(order + 1):
            wx, dwx = bspline(order, np.array([u - (il + a)]))
            for b in range(order + 1):
                wy, dwy = bspline(order, np.array([v - (jl + b)]))
                node = F[:, (il + a) % nx, (jl + b) % ny]
                want[p, :18] += node * wx[0] * wy[0]
                want[p, 18] += node[0] * dwx[0] / dx * wy[0]
                want[p, 19] += node[0] * wx[0] * dwy[0] / dy
                for c in range(3):
                    want[p, 21 + 3 * c] += node[3 + c] * dwx[0] / dx * wy[0]
                    want[p, 22 + 3 * c] += node[3 + c] * wx[0] * dwy[0] / dy
    for k, name in enumerate(up.PROBE_COLUMNS):
        scale = max(np.max(np.abs(want[:, k])), 1e-30)
        assert np.max(np.abs(out[:, k] - want[:, k])) <= 1e-12 * scale + 1e-300, name
    assert np.all(out[:, [20, 23, 26, 29]] == 0.0)
