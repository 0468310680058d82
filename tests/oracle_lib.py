"""ctypes bindings to the CPU oracle (oracle/liboracle.so) and to the reference
harness (oracle/_ref/libref_p2.so).  Test infrastructure only: these are the
checkers, never the product path."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_P2_SO = os.path.join(ROOT, "oracle", "_ref", "libref_p2.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def ptr(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_ip)
    raise TypeError(a.dtype)


def _load(path):
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


def oracle():
    lib = _load(ORACLE_SO)
    if lib is None:
        raise RuntimeError("oracle/liboracle.so missing: run make -C oracle")
    return lib


def ref_p2():
    """The reference's own code; None when it was not built (no sources)."""
    return _load(REF_P2_SO)


class P2Problem:
    """Explicit BDF/IAEM run description shared by the oracle and the reference
    harness (argument contract of ref_p2_simulate / o2_simulate)."""

    def __init__(self, nx, ny, Lx, Ly, dt, bdf_order=1, conserving=True, c=1.0, eps0=1.0,
                 mu0=1.0, n0=1.0, n_steps=1, diag_stride=1):
        self.nx, self.ny, self.Lx, self.Ly, self.dt = nx, ny, Lx, Ly, dt
        self.bdf_order, self.conserving = bdf_order, conserving
        self.c, self.eps0, self.mu0, self.n0 = c, eps0, mu0, n0
        self.n_steps, self.diag_stride = n_steps, diag_stride

    def params(self):
        return np.array([self.Lx, self.Ly, self.dt, self.c, self.eps0, self.mu0, self.n0])

    def iparams(self):
        return np.array([self.nx, self.ny, self.bdf_order, int(self.conserving), self.n_steps,
                         self.diag_stride], dtype=np.int32)


def simulate(lib_fn, prob, parts, want_fields=True):
    """Run lib_fn (o2_simulate or ref_p2_simulate) on a copy of parts.
    parts: dict x, y (np), P, v, vprev (np,3), q, m (np).  Returns (parts_out,
    diag (n_steps+1, 13), fields (8, nx, ny) or None, seconds)."""
    out = {k: np.ascontiguousarray(parts[k], dtype=np.float64).copy() for k in parts}
    np_ = out["x"].shape[0]
    diag = np.full((prob.n_steps + 1, 13), np.nan)
    fields = np.zeros((8, prob.nx * prob.ny)) if want_fields else None
    secs = np.zeros(1)
    rc = lib_fn(ptr(prob.params()), ptr(prob.iparams()), ctypes.c_long(np_), ptr(out["x"]),
                ptr(out["y"]), ptr(out["P"]), ptr(out["v"]), ptr(out["vprev"]), ptr(out["q"]),
                ptr(out["m"]), ptr(diag), ptr(fields), ptr(secs))
    if rc != 0:
        raise RuntimeError("simulate failed")
    if fields is not None:
        fields = fields.reshape(8, prob.nx, prob.ny)
    return out, diag, fields, float(secs[0])


def init_weibel(lib_fn, nx, ny, Lx, Ly, ppc, c=1.0, n0=1.0, vx=0.5, vy_max=0.01, sine=0.002,
                mode=1, seed=12345):
    nsub = max(1, int(round(np.sqrt(ppc))))
    cap = 2 * nx * ny * nsub * nsub
    a = {k: np.zeros(cap) for k in ("x", "y", "q", "m")}
    for k in ("P", "v", "vprev"):
        a[k] = np.zeros((cap, 3))
    n = lib_fn(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_double(Lx), ctypes.c_double(Ly),
               ctypes.c_int(ppc), ctypes.c_double(c), ctypes.c_double(n0), ctypes.c_double(vx),
               ctypes.c_double(vy_max), ctypes.c_double(sine), ctypes.c_int(mode),
               ctypes.c_uint(seed), ctypes.c_long(cap), ptr(a["x"]), ptr(a["y"]), ptr(a["P"]),
               ptr(a["v"]), ptr(a["vprev"]), ptr(a["q"]), ptr(a["m"]))
    assert n == cap, (n, cap)
    return a
