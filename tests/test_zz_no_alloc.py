"""upic_deposit_current_noalloc: the current deposit for callers that may not
allocate device memory (hosts that own all device memory through their own
allocator, or loops that cannot risk the synchronization a cudaMalloc or
cudaFree may cause).  It keeps its scratch in a fixed device array and takes
caller-owned device buffers.  Checked through the C ABI against
upic_deposit_current on two calls in a row (the second call must not see the
first call's sums), within the deposit tolerance of the other GPU tests.
This file sorts last so that a run stopping at the first failure has run
every other test first."""
import ctypes

import numpy as np
import pytest

import unstaggered_pic_b200 as up
from unstaggered_pic_b200._native import lib

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _particles(rng, n, Lx, Ly):
    x = rng.uniform(0.0, Lx, n)
    y = rng.uniform(0.0, Ly, n)
    x[:2] = [0.0, np.nextafter(Lx, 0.0)]
    y[:2] = [np.nextafter(Ly, 0.0), 0.0]
    v = rng.normal(size=(n, 3)) * np.array([0.02, 0.2, 0.05])
    q = np.full(n, -Lx * Ly / n)
    return x, y, v, q


def test_noalloc_matches_existing_deposit_twice():
    import torch
    torch.cuda.set_device(0)
    nx, ny, Lx, Ly = 64, 128, 3.0, 5.0
    rng = np.random.default_rng(42)
    sim = up.Simulation(up.Config(nx=nx, ny=ny, Lx=Lx, Ly=Ly))
    stream = torch.cuda.current_stream()
    J = torch.empty(3 * nx * ny, dtype=torch.float64, device="cuda")
    for call, n in enumerate((20000, 7000)):
        x, y, v, q = _particles(rng, n, Lx, Ly)
        ref = sim.deposit_current(x, y, v, q).ravel()
        dx, dy, dv, dq = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, y, v, q))
        J.fill_(np.nan)
        rc = lib().upic_deposit_current_noalloc(nx, ny, Lx, Ly, n, dx.data_ptr(), dy.data_ptr(),
                                                dv.data_ptr(), dq.data_ptr(), J.data_ptr(),
                                                ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, call
        torch.cuda.synchronize()
        got = J.cpu().numpy()
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err < TOL, (call, err)
    sim.close()


def _call(nx, ny, Lx, Ly, x, y, v, q, J, stream):
    import torch
    dx, dy, dv, dq = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, y, v, q))
    torch.cuda.synchronize()
    return lib().upic_deposit_current_noalloc(nx, ny, Lx, Ly, len(x), dx.data_ptr(), dy.data_ptr(),
                                              dv.data_ptr(), dq.data_ptr(), J.data_ptr(),
                                              ctypes.c_void_p(stream))


def test_noalloc_side_stream_large_then_small_grid():
    """A call on a non-default stream, a large grid that fills most of the
    fixed array, then a smaller grid: the second call must not see what the
    first left behind beyond the part it clears."""
    import torch
    torch.cuda.set_device(0)
    rng = np.random.default_rng(7)
    side = torch.cuda.Stream()
    for nx, ny, Lx, Ly, n in ((256, 256, 8.0, 8.0, 60000), (32, 64, 2.0, 3.0, 5000)):
        x, y, v, q = _particles(rng, n, Lx, Ly)
        with up.Simulation(up.Config(nx=nx, ny=ny, Lx=Lx, Ly=Ly)) as sim:
            ref = sim.deposit_current(x, y, v, q).ravel()
        J = torch.full((3 * nx * ny,), np.nan, dtype=torch.float64, device="cuda")
        rc = _call(nx, ny, Lx, Ly, x, y, v, q, J, side.cuda_stream)
        assert rc == 0, (nx, ny)
        got = J.cpu().numpy()
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err < TOL, (nx, ny, err)


def test_noalloc_nonfinite_input_is_an_error():
    """A NaN velocity or an infinite charge gives UPIC_ERR_NONFINITE and a NaN
    current, not a finite wrong one; the next clean call is exact again."""
    import torch
    torch.cuda.set_device(0)
    nx, ny, Lx, Ly = 32, 32, 2.0, 2.0
    rng = np.random.default_rng(11)
    x, y, v, q = _particles(rng, 3000, Lx, Ly)
    J = torch.zeros(3 * nx * ny, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    bad_v = v.copy()
    bad_v[17, 1] = np.nan
    assert _call(nx, ny, Lx, Ly, x, y, bad_v, q, J, stream) == -5  # UPIC_ERR_NONFINITE
    assert np.all(np.isnan(J.cpu().numpy()))
    bad_q = q.copy()
    bad_q[5] = np.inf
    assert _call(nx, ny, Lx, Ly, x, y, v, bad_q, J, stream) == -5
    assert _call(nx, ny, Lx, Ly, x, y, v, q, J, stream) == 0
    with up.Simulation(up.Config(nx=nx, ny=ny, Lx=Lx, Ly=Ly)) as sim:
        ref = sim.deposit_current(x, y, v, q).ravel()
    got = J.cpu().numpy()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < TOL


def test_noalloc_rejects_grid_beyond_capacity():
    import torch
    torch.cuda.set_device(0)
    J = torch.empty(3, dtype=torch.float64, device="cuda")
    rc = lib().upic_deposit_current_noalloc(512, 256, 1.0, 1.0, 0, None, None, None, None,
                                            J.data_ptr(), None)
    assert rc == -10  # UPIC_ERR_TOO_LARGE: 512*256 > UPIC_NOALLOC_MAX_NODES
