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


def generate_bimaxwellian(nx, ny, Lx, Ly, ppc, uth, udrift=(0.0, 0.0, 0.0), c=1.0, n0=1.0, seed=1):
    """The benchmark workloads' seeded plasma from the oracle's restatement
    (o_generate_bimaxwellian): the same dict of x, y, P, v, v_prev, q, m as
    the product's generator, without loading the product library."""
    n = nx * ny * ppc
    out = {"x": np.empty(n), "y": np.empty(n), "P": np.empty((n, 3)), "v": np.empty((n, 3)),
           "v_prev": np.empty((n, 3)), "q": np.empty(n), "m": np.empty(n)}
    uth = np.ascontiguousarray(uth, dtype=np.float64)
    ud = np.ascontiguousarray(udrift, dtype=np.float64)
    rc = oracle().o_generate_bimaxwellian(int(nx), int(ny), ctypes.c_double(Lx), ctypes.c_double(Ly), int(ppc),
                                          ctypes.c_double(c), ctypes.c_double(n0), ptr(uth), ptr(ud),
                                          ctypes.c_uint64(seed),
                                          *[ptr(out[k]) for k in ("x", "y", "P", "v", "v_prev", "q", "m")])
    if rc != 0:
        raise ValueError("o_generate_bimaxwellian: bad argument")
    return out


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


# ---------------------------------------------------------------------------
# Project3 (implicit GM-HC-CN) runs: dparams / iparams layout of
# oracle/ref/ref_p3_harness.cpp and oracle/p3_oracle.c.
REF_P3_SO = os.path.join(ROOT, "oracle", "_ref", "libref_p3.so")
P3_NDIAG = 23
P3_NINFO = 8
P3_NSTEPDIAG = 17
P3_DIAG_NAMES = ["gauss_rms", "gauss_max", "divE_rms", "sigma1_rho_rms", "gauss_normalization_rms",
                 "gauss_relative", "gauge_rms", "gauge_max", "psi_over_kappa2_rms", "divA_rms",
                 "gauge_normalization_rms", "gauge_relative", "field_energy", "kinetic_energy",
                 "total_energy", "rho_mode", "E_mode_re", "E_mode_im", "E_mode_abs", "Bz_y_mode_re",
                 "Bz_y_mode_im", "Bz_y_mode_abs", "mean_rho"]


def ref_p3():
    return _load(REF_P3_SO)


class P3Problem:
    def __init__(self, nx, ny, Lx, Ly, dt, nz=1, Lz=1.0, kappa=1.0, sigma1=1.0, sigma2=1.0, n0=1.0,
                 order=2, nq=8, split=True, nyquist=True, nl_rtol=1e-11, nl_atol=1e-13,
                 nl_maxit=80, and_mem=4, and_start=2, and_damp=0.5, and_reg=1e-12,
                 and_growth=1.2, loc_rtol=1e-12, loc_atol=1e-14, loc_maxit=64, loc_damp=1.0,
                 solver="anderson", n_steps=1, mode=1):
        self.__dict__.update(locals())
        del self.__dict__["self"]

    def dparams(self):
        return np.array([self.Lx, self.Ly, self.Lz, self.dt, self.kappa, self.sigma1, self.sigma2,
                         self.n0, self.nl_rtol, self.nl_atol, self.and_damp, self.and_reg,
                         self.and_growth, self.loc_rtol, self.loc_atol, self.loc_damp])

    def iparams(self):
        return np.array([self.nx, self.ny, self.nz, self.order, self.nq, int(self.split),
                         int(self.nyquist), self.nl_maxit, self.and_mem, self.and_start,
                         self.loc_maxit, 1 if self.solver == "picard" else 0, self.n_steps,
                         self.mode], dtype=np.int32)


def p3_run(fn, prob, x, v, q, m, want_fields=True, want_step_diag=False):
    """Run fn (ref_p3_run) on copies: x, v (np, 3).  Returns dict with x,
    v, P, v_prev, vbar, diag (n_steps+1, 22), info (n_steps, 8), fields
    (12, nx, ny), step_diag (n_steps, 17) and seconds (of the step loop,
    step diagnostics included when requested)."""
    n = len(q)
    out = {"x": np.ascontiguousarray(x, dtype=np.float64).copy(),
           "v": np.ascontiguousarray(v, dtype=np.float64).copy(),
           "P": np.zeros((n, 3)), "v_prev": np.zeros((n, 3)), "vbar": np.zeros((n, 3))}
    diag = np.full((prob.n_steps + 1, P3_NDIAG), np.nan)
    info = np.full((max(prob.n_steps, 1), P3_NINFO), np.nan)
    N = prob.nx * prob.ny * prob.nz
    fields = np.zeros((12, N)) if want_fields else None
    secs = np.zeros(1)
    sdiag = np.full((max(prob.n_steps, 1), P3_NSTEPDIAG), np.nan) if want_step_diag else None
    rc = fn(ptr(prob.dparams()), ptr(prob.iparams()), ctypes.c_long(n), ptr(out["x"]), ptr(out["v"]),
            ptr(out["P"]), ptr(out["v_prev"]), ptr(out["vbar"]),
            ptr(np.ascontiguousarray(q, dtype=np.float64)), ptr(np.ascontiguousarray(m, dtype=np.float64)),
            ptr(diag), ptr(info), ptr(fields), ptr(secs), ptr(sdiag))
    if rc != 0:
        raise RuntimeError("p3 run failed")
    out.update(diag=diag, info=info[:prob.n_steps], seconds=float(secs[0]))
    if sdiag is not None:
        out["step_diag"] = sdiag[:prob.n_steps]
    if fields is not None:
        out["fields"] = fields.reshape(12, prob.nx, prob.ny * prob.nz)
    return out


# Instability cases of the reference's initialize_state (ref_p3_case_state /
# ref_p3_case_run): the case keys of upic_p3_case.
P3_CASE_DEFAULTS = dict(v0=0.3, perturbation=0.02, two_stream_density_alpha=-1.0, tsi_transverse_seed=0.0,
                        weibel_B0=-1.0, particles_per_cell_pair=4, two_stream_eigenmode=1,
                        two_stream_finite_grid_theory=1, tsi_transverse_mode=1, weibel_eigenmode=1,
                        weibel_finite_grid_theory=1, landau_alpha=-1.0, thermal_velocity=1.0)


def p3_case_arrays(case, keys):
    k = dict(P3_CASE_DEFAULTS)
    k.update({a: b for a, b in keys.items() if a in k})
    cd = np.array([k["v0"], k["perturbation"], k["two_stream_density_alpha"], k["tsi_transverse_seed"],
                   k["weibel_B0"], k["landau_alpha"], k["thermal_velocity"]], dtype=np.float64)
    ci = np.array([{"two_stream": 0, "weibel": 1, "landau": 2}[case], k["particles_per_cell_pair"],
                   k["two_stream_eigenmode"],
                   k["two_stream_finite_grid_theory"], k["tsi_transverse_mode"], k["weibel_eigenmode"],
                   k["weibel_finite_grid_theory"]], dtype=np.int32)
    return cd, ci


def p3_case_state(lib, prob, case, keys, cap=2_000_000):
    """The reference's start state of an instability case: dict of x, v, P,
    v_prev (np, 3), q, m (np), A, U (3, nx, ny), growth_rate."""
    cd, ci = p3_case_arrays(case, keys)
    N = prob.nx * prob.ny * prob.nz
    out = {k: np.zeros((cap, 3)) for k in ("x", "v", "P", "v_prev")}
    out.update(q=np.zeros(cap), m=np.zeros(cap), A=np.zeros(3 * N), U=np.zeros(3 * N))
    g = np.zeros(1)
    lib.ref_p3_case_state.restype = ctypes.c_long
    n = lib.ref_p3_case_state(ptr(prob.dparams()), ptr(prob.iparams()), ptr(cd), ptr(ci), ctypes.c_long(cap),
                              ptr(out["x"]), ptr(out["v"]), ptr(out["P"]), ptr(out["v_prev"]), ptr(out["q"]),
                              ptr(out["m"]), ptr(out["A"]), ptr(out["U"]), ptr(g))
    if n < 0:
        raise RuntimeError("ref_p3_case_state failed")
    for k in ("x", "v", "P", "v_prev", "q", "m"):
        out[k] = out[k][:n]
    out["A"] = out["A"].reshape(3, prob.nx, prob.ny * prob.nz)
    out["U"] = out["U"].reshape(3, prob.nx, prob.ny * prob.nz)
    out["growth_rate"] = float(g[0])
    return out


def p3_case_run(lib, prob, case, keys):
    """An instability case run by the reference from its own start state:
    dict of diag (n_steps+1, 23), info (n_steps, 8), fields (12, nx, ny), seconds."""
    cd, ci = p3_case_arrays(case, keys)
    N = prob.nx * prob.ny * prob.nz
    diag = np.full((prob.n_steps + 1, P3_NDIAG), np.nan)
    info = np.full((max(prob.n_steps, 1), P3_NINFO), np.nan)
    fields = np.zeros((12, N))
    secs = np.zeros(1)
    rc = lib.ref_p3_case_run(ptr(prob.dparams()), ptr(prob.iparams()), ptr(cd), ptr(ci), ptr(diag), ptr(info),
                             ptr(fields), ptr(secs))
    if rc != 0:
        raise RuntimeError("ref_p3_case_run failed")
    return {"diag": diag, "info": info[:prob.n_steps], "fields": fields.reshape(12, prob.nx, prob.ny * prob.nz),
            "seconds": float(secs[0])}


def p3_particles(rng, nx, ny, ppc, Lx, Ly, uth=(0.02, 0.2, 0.0), n0=1.0, Lz=1.0):
    """Random electrons in [-L/2, L/2) (Project3's coordinates), normalized
    momentum u = gamma v Maxwellian with spreads uth, q/m = -1, neutralizing n0."""
    n = nx * ny * ppc
    x = np.zeros((n, 3))
    x[:, 0] = rng.uniform(-Lx / 2, Lx / 2, n)
    x[:, 1] = rng.uniform(-Ly / 2, Ly / 2, n)
    u = rng.normal(size=(n, 3)) * np.asarray(uth)
    gam = np.sqrt(1 + (u * u).sum(1))
    v = u / gam[:, None]
    q = np.full(n, -n0 * Lx * Ly * Lz / n)
    return x, v, q, np.abs(q)


# Project1 (non-relativistic implicit Picard) runs: dparams / iparams layout
# of oracle/ref/ref_p1_harness.cpp.
REF_P1_SO = os.path.join(ROOT, "oracle", "_ref", "libref_p1.so")
P1_NDIAG = 11
P1_NINFO = 6
P1_DIAG_NAMES = ["gauss_rms", "gauss_max", "gauge_rms", "field_energy", "kinetic_energy", "total_energy",
                 "rho_mode", "E_mode_re", "E_mode_im", "E_mode_abs", "mean_rho"]


def ref_p1():
    return _load(REF_P1_SO)


class P1Problem:
    def __init__(self, nx, ny, Lx, Ly, dt, nz=1, Lz=1.0, c=1.0, eps0=1.0, mu0=1.0, n0=1.0, order=2, nq=16,
                 split=True, picard_tol=1e-11, picard_maxit=16, sweep=True, n_steps=1, mode=1, ppc=4,
                 case="two_stream", v0=0.3, perturbation=0.02, landau_alpha=-1.0, vth=1.0):
        self.__dict__.update(locals())
        del self.__dict__["self"]

    def dparams(self):
        return np.array([self.Lx, self.Ly, self.Lz, self.dt, self.c, self.eps0, self.mu0, self.n0,
                         self.picard_tol, self.v0, self.perturbation, self.landau_alpha, self.vth])

    def iparams(self):
        return np.array([self.nx, self.ny, self.nz, self.order, self.nq, int(self.split), self.picard_maxit,
                         int(self.sweep), self.n_steps, self.mode, self.ppc,
                         1 if self.case.startswith("landau") else 0], dtype=np.int32)


def p1_init(lib, prob, cap=10_000_000):
    """Particles of the reference's own initial condition: x, v (np, 3), q, m."""
    x = np.zeros((cap, 3))
    v = np.zeros((cap, 3))
    q = np.zeros(cap)
    m = np.zeros(cap)
    lib.ref_p1_init.restype = ctypes.c_long
    n = lib.ref_p1_init(ptr(prob.dparams()), ptr(prob.iparams()), ctypes.c_long(cap), ptr(x), ptr(v), ptr(q),
                        ptr(m))
    if n < 0:
        raise RuntimeError("p1 init failed")
    return x[:n].copy(), v[:n].copy(), q[:n].copy(), m[:n].copy()


def p1_run(fn, prob, x, v, q, m, want_fields=True):
    """Run fn (ref_p1_run) on copies: x, v (np, 3).  Returns dict with x, v,
    P, v_prev, diag (n_steps+1, 11), info (n_steps, 6), step_diag (n_steps,
    17), fields (12, nx, ny*nz) and seconds."""
    n = len(q)
    out = {"x": np.ascontiguousarray(x, dtype=np.float64).copy(),
           "v": np.ascontiguousarray(v, dtype=np.float64).copy(),
           "P": np.zeros((n, 3)), "v_prev": np.zeros((n, 3))}
    diag = np.full((prob.n_steps + 1, P1_NDIAG), np.nan)
    info = np.full((max(prob.n_steps, 1), P1_NINFO), np.nan)
    sdiag = np.full((max(prob.n_steps, 1), 17), np.nan)
    N = prob.nx * prob.ny * prob.nz
    fields = np.zeros((12, N)) if want_fields else None
    secs = np.zeros(1)
    rc = fn(ptr(prob.dparams()), ptr(prob.iparams()), ctypes.c_long(n), ptr(out["x"]), ptr(out["v"]),
            ptr(out["P"]), ptr(out["v_prev"]), ptr(np.ascontiguousarray(q, dtype=np.float64)),
            ptr(np.ascontiguousarray(m, dtype=np.float64)), ptr(diag), ptr(info), ptr(sdiag), ptr(fields),
            ptr(secs))
    if rc != 0:
        raise RuntimeError("p1 run failed")
    out.update(diag=diag, info=info[:prob.n_steps], step_diag=sdiag[:prob.n_steps], seconds=float(secs[0]))
    if fields is not None:
        out["fields"] = fields.reshape(12, prob.nx, prob.ny * prob.nz)
    return out
