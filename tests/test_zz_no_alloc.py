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


def test_noalloc_rejects_grid_beyond_capacity():
    import torch
    torch.cuda.set_device(0)
    J = torch.empty(3, dtype=torch.float64, device="cuda")
    rc = lib().upic_deposit_current_noalloc(512, 256, 1.0, 1.0, 0, None, None, None, None,
                                            J.data_ptr(), None)
    assert rc == -10  # UPIC_ERR_TOO_LARGE: 512*256 > UPIC_NOALLOC_MAX_NODES
