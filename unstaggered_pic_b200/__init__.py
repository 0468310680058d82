"""B200-native unstaggered generalized-momentum PIC step.

Python mirror of the C ABI in include/upic.h.  The numerical work runs in
libupic.so (hand-written CUDA for sm_100a); this module only marshals host
arrays.  Names follow the reference solver (sgong11/Unstaggered_PIC,
Project2/spectral_pic_part3.cpp): particles carry x, y, canonical momentum P,
velocity v, previous velocity v_prev, charge q and mass m; grids are nx*ny
doubles with node id = i*ny + j.
"""
import ctypes
import os

import numpy as np

from ._native import UPIC_ERR, UpicConfig, c_dp, lib

__all__ = ["UpicError", "Config", "ImplicitConfig", "NonrelConfig", "Simulation", "Ensemble", "autotune_explicit",
           "generate_bimaxwellian", "p3_initial_state", "P3_CASES", "MAP_LOG_COLUMNS", "FAILED_LOG_COLUMNS", "PROBE_COLUMNS",
           "convergence_method_name",
           "DIAG_COLUMNS", "IMPLICIT_DIAG_COLUMNS", "NONREL_DIAG_COLUMNS", "SOLVE_INFO_COLUMNS",
           "STEP_DIAG_COLUMNS", "METHODS",
           "FIELDS"]

METHODS = {"bdf1": 1, "bdf2": 2, "cn_orbit": 3, "cn_orbit_nonrel": 4}
CHARGE_UPDATES = {"conserving": 0, "naive": 1}
# FP64 throughout, or the mixed form of the explicit step (FP32 particles with
# cell-relative offsets, FP64 field solve and diagnostics)
PRECISIONS = {"fp64": 0, "mixed": 1}
# first guess of the implicit step's outer current iteration
PREDICTORS = {"previous": 0, "extrapolated": 1, "learned": 2}
NONLINEAR_SOLVERS = {"anderson_quasi_newton": 0, "anderson": 0, "picard": 1}
FIELDS = {"phi": 0, "Ax": 1, "Ay": 2, "Az": 3, "rho": 4, "Jx": 5, "Jy": 6, "Jz": 7,
          "psi": 8, "Ux": 9, "Uy": 10, "Uz": 11, "Ex": 12, "Ey": 13, "Ez": 14, "Bx": 15, "By": 16, "Bz": 17}
# Diagnostics columns of the reference's _diagnostics.csv (spectral_pic_part3.cpp:1117-1119).
DIAG_COLUMNS = ["gauge_rms", "gauss_rms", "continuity_rms", "Bz_l2", "B_l2", "E_l2", "rho_l2",
                "J_l2", "field_energy", "kinetic_energy", "total_energy", "max_speed",
                "mean_gamma"]
# Diagnostics of the implicit method (Diagnostics, ec_pic_nyquist_projected.cpp:3469-3519).
IMPLICIT_DIAG_COLUMNS = [
    "gauss_rms", "gauss_max", "divE_rms", "sigma1_rho_rms", "gauss_normalization_rms",
    "gauss_relative", "gauge_rms", "gauge_max", "psi_over_kappa2_rms", "divA_rms",
    "gauge_normalization_rms", "gauge_relative", "field_energy", "kinetic_energy", "total_energy",
    "rho_mode", "E_mode_re", "E_mode_im", "E_mode_abs", "Bz_y_mode_re", "Bz_y_mode_im",
    "Bz_y_mode_abs", "mean_rho"]
# Diagnostics of the non-relativistic method (Diagnostics, Project1/ec_pic_serial_demo.cpp:1037-1055),
# taken from the implicit row by name.
NONREL_DIAG_COLUMNS = ["gauss_rms", "gauss_max", "gauge_rms", "field_energy", "kinetic_energy",
                       "total_energy", "rho_mode", "E_mode_re", "E_mode_im", "E_mode_abs", "mean_rho"]
# Step diagnostics of the implicit method (StepDiagnostics, ec_pic_nyquist_projected.cpp:4303-4321),
# the column order of its _step_diagnostics.csv.
STEP_DIAG_COLUMNS = ["A_chain_abs_rms", "A_chain_rel_rms", "A_chain_max_norm", "A_chain_mean_norm",
                     "A_chain_work_defect", "delta_K", "delta_W", "delta_total_energy", "particle_work",
                     "grid_work", "deposit_gather_work_residual", "particle_energy_residual",
                     "field_energy_residual", "crossing_particles", "total_crossings", "avg_path_segments",
                     "max_path_segments"]
# Per-step outer-solve report (NonlinearSolveInfo, ec_pic_nyquist_projected.cpp:5493-5533).
SOLVE_INFO_COLUMNS = ["iterations", "converged", "final_rms_residual", "final_max_particle_residual",
                      "local_particle_iterations_max", "local_particle_iterations_mean",
                      "anderson_steps", "picard_fallback_steps", "picard_current_error",
                      "picard_velocity_error", "crossing_particles", "avg_path_segments",
                      "max_path_segments", "selective_fallback_used", "selective_refinement_restarts",
                      "selective_refined_particles", "selective_total_particle_substeps",
                      # first guess of the outer current iteration (not in the reference)
                      "predictor_used", "guess_error", "extrapolation_error", "learned_error", "learned_loss",
                      # the rest of NonlinearSolveInfo
                      "anderson_restarts", "nonlinear_absolute_rms_residual", "observed_convergence_rate",
                      "estimated_map_contraction", "backtracked_steps", "minimum_update_alpha",
                      "convergence_method", "uniform_substeps_used", "direct_attempt_iterations",
                      "selective_work_ratio", "selective_n1", "selective_n2", "selective_n4", "selective_n8",
                      "selective_n16", "selective_n32", "selective_n64"]
# Map evaluations of the last step_implicit call (upic_map_log): the columns
# of _particle_inner_history.csv after time_n, dt, with the step of the call.
MAP_LOG_COLUMNS = ["step", "map_evaluation", "particles_converged", "failed_particles",
                   "max_scaled_particle_residual", "local_iterations_mean", "local_iterations_max"]
# Failed-particle records of the last step_implicit call
# (upic_failed_particle_log): the columns of _failed_particle_diagnostics.csv
# after time_before, with the step of the call; failure_reason as a code
# (FAILURE_REASONS).
FAILED_LOG_COLUMNS = (["step", "layout_refinement_restart", "map_evaluation", "event_exhausted",
                       "failed_particles_in_event", "particle_index", "assigned_substeps",
                       "failed_substep_zero_based", "theta0", "theta1", "h", "local_iterations", "failure_reason",
                       "first_scaled_residual", "final_scaled_residual", "final_absolute_residual", "q", "m"] +
                      [f"{v}_{c}" for v in ("x0", "P0", "initial_guess", "last_guess", "last_map") for c in "xyz"])
FAILURE_REASONS = ["none", "nonfinite_map", "superluminal_map", "nonfinite_iterate", "superluminal_iterate",
                   "maximum_iterations", "too_many_knot_crossings"]
# Point probe columns (upic_probe_fields).
PROBE_COLUMNS = (["phi_h", "psi_h", "rho_h", "Ax_h", "Ay_h", "Az_h", "Ux_h", "Uy_h", "Uz_h", "Jx_h", "Jy_h", "Jz_h",
                  "Ex_grid_gather", "Ey_grid_gather", "Ez_grid_gather", "Bx_grid_gather", "By_grid_gather",
                  "Bz_grid_gather", "dphi_dx", "dphi_dy", "dphi_dz"] +
                 [f"dA{c}_d{d}" for c in "xyz" for d in "xyz"])


class UpicError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{UPIC_ERR.get(code, code)}: {msg}")
        self.code = code


def _p(a):
    return None if a is None else a.ctypes.data_as(c_dp)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


class Config:
    """Run configuration with the reference deck's keys and defaults
    (Config, spectral_pic_part3.cpp:174-231)."""

    def __init__(self, nx=32, ny=32, Lx=2 * np.pi, Ly=2 * np.pi, dt=0.05, method="bdf1",
                 charge_update="conserving", c=1.0, eps0=1.0, mu0=1.0, n0=1.0,
                 sort_interval=0, tile=0, guard=-1, precision="fp64"):
        self.nx, self.ny, self.Lx, self.Ly, self.dt = nx, ny, Lx, Ly, dt
        self.method, self.charge_update = method, charge_update
        self.c, self.eps0, self.mu0, self.n0 = c, eps0, mu0, n0
        self.sort_interval, self.tile, self.guard = sort_interval, tile, guard
        self.precision = precision

    def to_c(self):
        cfg = UpicConfig()
        lib().upic_config_default(ctypes.byref(cfg))
        cfg.nx, cfg.ny = int(self.nx), int(self.ny)
        cfg.Lx, cfg.Ly, cfg.dt = float(self.Lx), float(self.Ly), float(self.dt)
        cfg.method = METHODS[self.method] if isinstance(self.method, str) else int(self.method)
        cu = self.charge_update
        cfg.charge_update = CHARGE_UPDATES[cu] if isinstance(cu, str) else int(cu)
        cfg.c, cfg.eps0, cfg.mu0, cfg.n0 = float(self.c), float(self.eps0), float(self.mu0), float(self.n0)
        cfg.sort_interval, cfg.tile, cfg.guard = int(self.sort_interval), int(self.tile), int(self.guard)
        pr = self.precision
        cfg.precision = PRECISIONS[pr] if isinstance(pr, str) else int(pr)
        return cfg


class ImplicitConfig:
    """Deck of the implicit orbit-averaged GM-HC-CN method with the keys and
    defaults of the reference Config (ec_pic_nyquist_projected.cpp:837-1005),
    2D (nz = 1; Lz sets the cell volume).  Positions live in [-L/2, L/2)."""

    def __init__(self, nx=4, ny=4, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, dt=0.00625, kappa=1.0,
                 sigma1=1.0, sigma2=1.0, n0=1.0, spline_order=2, orbit_quad_order=16,
                 split_orbit_at_knots=True, nyquist_projection=False,
                 nonlinear_solver="anderson_quasi_newton", nonlinear_rtol=1.0e-12,
                 nonlinear_atol=1.0e-13, nonlinear_max_iter=32, anderson_memory=4, anderson_start=2,
                 anderson_damping=0.7, anderson_regularization=1.0e-12, anderson_growth_limit=1.2,
                 uniform_local_rtol=1.0e-11, uniform_local_atol=1.0e-13, uniform_local_max_iter=24,
                 uniform_local_damping=1.0, perturbation_mode=1, tile=0, guard=-1, current_predictor="previous",
                 local_warm_start=False, selective_particle_fallback=False, selective_particle_max_substeps=64,
                 learned_train_steps=200, learned_train_iters=4, learned_rate=1.0e-3, learned_seed=20261203):
        self.method = "cn_orbit"
        self.learned_train_steps, self.learned_train_iters = learned_train_steps, learned_train_iters
        self.learned_rate, self.learned_seed = learned_rate, learned_seed
        self.current_predictor, self.local_warm_start = current_predictor, local_warm_start
        self.selective_particle_fallback = selective_particle_fallback
        self.selective_particle_max_substeps = selective_particle_max_substeps
        self.nx, self.ny, self.Lx, self.Ly, self.Lz, self.dt = nx, ny, Lx, Ly, Lz, dt
        self.kappa, self.sigma1, self.sigma2, self.n0 = kappa, sigma1, sigma2, n0
        self.spline_order, self.orbit_quad_order = spline_order, orbit_quad_order
        self.split_orbit_at_knots, self.nyquist_projection = split_orbit_at_knots, nyquist_projection
        self.nonlinear_solver = nonlinear_solver
        self.nonlinear_rtol, self.nonlinear_atol = nonlinear_rtol, nonlinear_atol
        self.nonlinear_max_iter = nonlinear_max_iter
        self.anderson_memory, self.anderson_start = anderson_memory, anderson_start
        self.anderson_damping, self.anderson_regularization = anderson_damping, anderson_regularization
        self.anderson_growth_limit = anderson_growth_limit
        self.uniform_local_rtol, self.uniform_local_atol = uniform_local_rtol, uniform_local_atol
        self.uniform_local_max_iter, self.uniform_local_damping = uniform_local_max_iter, uniform_local_damping
        self.perturbation_mode, self.tile, self.guard = perturbation_mode, tile, guard

    def to_c(self):
        cfg = UpicConfig()
        lib().upic_config_default(ctypes.byref(cfg))
        cfg.nx, cfg.ny = int(self.nx), int(self.ny)
        cfg.Lx, cfg.Ly, cfg.Lz, cfg.dt = float(self.Lx), float(self.Ly), float(self.Lz), float(self.dt)
        cfg.method = METHODS["cn_orbit"]
        cfg.n0 = float(self.n0)
        cfg.kappa, cfg.sigma1, cfg.sigma2 = float(self.kappa), float(self.sigma1), float(self.sigma2)
        cfg.spline_order, cfg.orbit_quad_order = int(self.spline_order), int(self.orbit_quad_order)
        cfg.split_orbit_at_knots = int(bool(self.split_orbit_at_knots))
        cfg.nyquist_projection = int(bool(self.nyquist_projection))
        ns = self.nonlinear_solver
        cfg.nonlinear_solver = NONLINEAR_SOLVERS[ns] if isinstance(ns, str) else int(ns)
        cfg.nonlinear_rtol, cfg.nonlinear_atol = float(self.nonlinear_rtol), float(self.nonlinear_atol)
        cfg.nonlinear_max_iter = int(self.nonlinear_max_iter)
        cfg.anderson_memory, cfg.anderson_start = int(self.anderson_memory), int(self.anderson_start)
        cfg.anderson_damping = float(self.anderson_damping)
        cfg.anderson_regularization = float(self.anderson_regularization)
        cfg.anderson_growth_limit = float(self.anderson_growth_limit)
        cfg.local_rtol, cfg.local_atol = float(self.uniform_local_rtol), float(self.uniform_local_atol)
        cfg.local_max_iter = int(self.uniform_local_max_iter)
        cfg.local_damping = float(self.uniform_local_damping)
        cfg.perturbation_mode = int(self.perturbation_mode)
        cfg.tile, cfg.guard = int(self.tile), int(self.guard)
        cp = self.current_predictor
        cfg.current_predictor = PREDICTORS[cp] if isinstance(cp, str) else int(cp)
        cfg.local_warm_start = int(bool(self.local_warm_start))
        cfg.selective_particle_fallback = int(bool(self.selective_particle_fallback))
        cfg.selective_particle_max_substeps = int(self.selective_particle_max_substeps)
        cfg.learned_train_steps, cfg.learned_train_iters = int(self.learned_train_steps), int(self.learned_train_iters)
        cfg.learned_rate, cfg.learned_seed = float(self.learned_rate), int(self.learned_seed)
        return cfg


class NonrelConfig:
    """Deck of the non-relativistic implicit orbit-averaged method with
    Picard iteration on the particle velocities, with the keys and defaults
    of the reference Config (Project1/ec_pic_serial_demo.cpp:232-301), 2D
    (nz = 1; Lz sets the cell volume).  Positions live in [-L/2, L/2)."""

    def __init__(self, nx=4, ny=4, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, dt=0.00625, c=1.0, eps0=1.0,
                 mu0=1.0, n0=1.0, spline_order=2, orbit_quad_order=16, split_orbit_at_knots=True,
                 picard_tol=1.0e-11, picard_max_iter=16, final_consistency_sweep=True, perturbation_mode=1,
                 tile=0, guard=-1):
        self.method = "cn_orbit_nonrel"
        self.nx, self.ny, self.Lx, self.Ly, self.Lz, self.dt = nx, ny, Lx, Ly, Lz, dt
        self.c, self.eps0, self.mu0, self.n0 = c, eps0, mu0, n0
        self.spline_order, self.orbit_quad_order = spline_order, orbit_quad_order
        self.split_orbit_at_knots = split_orbit_at_knots
        self.picard_tol, self.picard_max_iter = picard_tol, picard_max_iter
        self.final_consistency_sweep = final_consistency_sweep
        self.perturbation_mode, self.tile, self.guard = perturbation_mode, tile, guard

    def to_c(self):
        cfg = UpicConfig()
        lib().upic_config_default(ctypes.byref(cfg))
        cfg.nx, cfg.ny = int(self.nx), int(self.ny)
        cfg.Lx, cfg.Ly, cfg.Lz, cfg.dt = float(self.Lx), float(self.Ly), float(self.Lz), float(self.dt)
        cfg.method = METHODS["cn_orbit_nonrel"]
        cfg.c, cfg.eps0, cfg.mu0, cfg.n0 = float(self.c), float(self.eps0), float(self.mu0), float(self.n0)
        cfg.spline_order, cfg.orbit_quad_order = int(self.spline_order), int(self.orbit_quad_order)
        cfg.split_orbit_at_knots = int(bool(self.split_orbit_at_knots))
        cfg.picard_tol, cfg.picard_max_iter = float(self.picard_tol), int(self.picard_max_iter)
        cfg.final_consistency_sweep = int(bool(self.final_consistency_sweep))
        cfg.perturbation_mode = int(self.perturbation_mode)
        cfg.tile, cfg.guard = int(self.tile), int(self.guard)
        return cfg


class Simulation:
    """One device context: particles + field state of the explicit BDF/IAEM
    step (Config) or of the implicit orbit-averaged GM-HC-CN step
    (ImplicitConfig)."""

    def __init__(self, config):
        self.config = config
        self._ctx = ctypes.c_void_p()
        cfg = config.to_c()
        rc = lib().upic_create(ctypes.byref(cfg), ctypes.byref(self._ctx))
        if rc != 0:
            raise UpicError(rc, lib().upic_last_error(None).decode())
        self.np = 0
        self.N = config.nx * config.ny
        self.implicit = cfg.method in (METHODS["cn_orbit"], METHODS["cn_orbit_nonrel"])

    def _check(self, rc):
        if rc != 0:
            raise UpicError(rc, lib().upic_last_error(self._ctx).decode())

    def close(self):
        if self._ctx:
            lib().upic_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._ctx

    def set_stream(self, stream_ptr):
        self._check(lib().upic_set_stream(self._ctx, ctypes.c_void_p(stream_ptr)))

    def set_particles(self, x, y, P, v, v_prev, q, m):
        n = len(x)
        arrs = [_f64(x), _f64(y), _f64(P, (n, 3)), _f64(v, (n, 3)), _f64(v_prev, (n, 3)), _f64(q),
                _f64(m)]
        self._check(lib().upic_set_particles(self._ctx, n, *[_p(a) for a in arrs]))
        self.np = n

    def get_particles(self, out=None):
        """Particle state in load order.  out: optional dict of preallocated
        float64 arrays x, y (n,) and P, v, v_prev (n, 3), e.g. views of
        pinned host memory, filled in place."""
        n = self.np
        if out is None:
            out = {"x": np.empty(n), "y": np.empty(n), "P": np.empty((n, 3)), "v": np.empty((n, 3)),
                   "v_prev": np.empty((n, 3))}
        else:
            for k, shape in (("x", (n,)), ("y", (n,)), ("P", (n, 3)), ("v", (n, 3)), ("v_prev", (n, 3))):
                a = out[k]
                if a.dtype != np.float64 or a.shape != shape or not a.flags.c_contiguous:
                    raise ValueError(f"out[{k!r}] must be a C-contiguous float64 array of shape {shape}")
        self._check(lib().upic_get_particles(self._ctx, n, _p(out["x"]), _p(out["y"]), _p(out["P"]),
                                             _p(out["v"]), _p(out["v_prev"])))
        return out

    def set_background(self, rho_bg):
        """Fixed background charge (nx, ny) in place of the uniform n0
        (explicit methods); None restores n0."""
        arr = None if rho_bg is None else _f64(rho_bg).ravel()
        self._check(lib().upic_set_background(self._ctx, _p(arr)))

    def save_state(self, path):
        """Checkpoint everything the next step reads to a binary file."""
        self._check(lib().upic_save_state(self._ctx, str(path).encode()))

    def load_state(self, path):
        """Restore a checkpoint written by a context of the same configuration;
        the run then continues as the saved one would have."""
        self._check(lib().upic_load_state(self._ctx, str(path).encode()))
        n = ctypes.c_long()
        self._check(lib().upic_particle_count(self._ctx, ctypes.byref(n)))
        self.np = n.value

    def init_fields(self, diagnostics=True):
        ncol = len(IMPLICIT_DIAG_COLUMNS) if self.implicit else len(DIAG_COLUMNS)
        row = np.empty(ncol) if diagnostics else None
        self._check(lib().upic_init_fields(self._ctx, _p(row)))
        return row

    def step_implicit(self, nsteps=1, diagnostics=True, step_diagnostics=False):
        """nsteps implicit steps; returns (diag rows, solve-info rows), and
        the step-diagnostics rows (STEP_DIAG_COLUMNS) as a third item when
        step_diagnostics is set."""
        diag = np.empty((nsteps, len(IMPLICIT_DIAG_COLUMNS))) if diagnostics else None
        info = np.empty((nsteps, len(SOLVE_INFO_COLUMNS)))
        sd = np.empty((nsteps, len(STEP_DIAG_COLUMNS))) if step_diagnostics else None
        self._check(lib().upic_step_implicit(self._ctx, int(nsteps), _p(diag), _p(info), _p(sd)))
        return (diag, info, sd) if step_diagnostics else (diag, info)

    def step(self, nsteps=1, diag_stride=1):
        diag = np.empty((nsteps, 13)) if diag_stride > 0 else None
        self._check(lib().upic_step(self._ctx, int(nsteps), int(diag_stride), _p(diag)))
        return diag

    def profile_enable(self, on=True):
        self._check(lib().upic_profile_enable(self._ctx, int(bool(on))))

    def profile_read(self):
        """(summed push-kernel ms, push launches, library kernel launches)."""
        ms = ctypes.c_double()
        n = ctypes.c_long()
        k = ctypes.c_long()
        self._check(lib().upic_profile_read(self._ctx, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(k)))
        return ms.value, n.value, k.value

    def steps_taken(self):
        s = ctypes.c_long()
        self._check(lib().upic_step_count(self._ctx, ctypes.byref(s)))
        return s.value

    def field(self, name):
        out = np.empty(self.N)
        self._check(lib().upic_get_field(self._ctx, FIELDS[name], _p(out)))
        return out.reshape(self.config.nx, self.config.ny)

    def set_initial_potential(self, A, U):
        """Initial A and U (3 x nx x ny) for the next init_fields of an
        implicit-method run (upic_set_initial_potential); None, None clears."""
        if A is None and U is None:
            self._check(lib().upic_set_initial_potential(self._ctx, None, None))
            return
        a, u = _f64(A, (3 * self.N,)), _f64(U, (3 * self.N,))
        self._check(lib().upic_set_initial_potential(self._ctx, _p(a), _p(u)))

    def push_iaem(self, x, y, P, v, v_prev, q, m, phi, A):
        """IAEM momentum push of the explicit method on the given fields
        (upic_push_iaem): returns the new P, v and v_prev (n x 3)."""
        xa, ya = _f64(x).ravel(), _f64(y).ravel()
        n = xa.size
        Pa, va, wa = (np.array(_f64(a, (n, 3)), copy=True) for a in (P, v, v_prev))
        qa, ma = _f64(q).ravel(), _f64(m).ravel()
        self._check(lib().upic_push_iaem(self._ctx, n, _p(xa), _p(ya), _p(Pa), _p(va), _p(wa), _p(qa), _p(ma),
                                         _p(_f64(phi, (self.N,))), _p(_f64(A, (3 * self.N,)))))
        return Pa, va, wa

    def push_gmhc(self, x, y, P, v, q, m, grad_phi_mid, An, Anp1):
        """One GM-HC-CN particle push in the given fields (upic_push_gmhc):
        returns x1, y1, P_end, v_end, vbar (NaN where the local solve failed)
        and the (iterations, failure reason) report per particle."""
        xa, ya = _f64(x).ravel(), _f64(y).ravel()
        n = xa.size
        Pa, va = _f64(P, (n, 3)), _f64(v, (n, 3))
        qa, ma = _f64(q).ravel(), _f64(m).ravel()
        g = _f64(grad_phi_mid, (2 * self.N,))
        a0, a1 = _f64(An, (3 * self.N,)), _f64(Anp1, (3 * self.N,))
        out = {"x1": np.empty(n), "y1": np.empty(n), "P_end": np.empty((n, 3)), "v_end": np.empty((n, 3)),
               "vbar": np.empty((n, 3))}
        rep = np.empty((n, 2), dtype=np.int32)
        self._check(lib().upic_push_gmhc(self._ctx, n, _p(xa), _p(ya), _p(Pa), _p(va), _p(qa), _p(ma), _p(g),
                                         _p(a0), _p(a1), *[_p(out[k]) for k in ("x1", "y1", "P_end", "v_end", "vbar")],
                                         rep.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        out["report"] = rep
        return out

    def fft_solve_cn(self, phi, psi, rho, A, U, J):
        """The field half of one implicit map evaluation on the given fields
        (upic_fft_solve_cn): dict of phi, psi, rho (nx x ny), A, U (3 x nx x ny)
        and grad_phi_mid (2 x nx x ny) of the new level."""
        nx, ny = self.config.nx, self.config.ny
        ins = [_f64(f, (k * self.N,)) for f, k in ((phi, 1), (psi, 1), (rho, 1), (A, 3), (U, 3), (J, 3))]
        out = {"phi": np.empty((nx, ny)), "psi": np.empty((nx, ny)), "rho": np.empty((nx, ny)),
               "A": np.empty((3, nx, ny)), "U": np.empty((3, nx, ny)), "grad_phi_mid": np.empty((2, nx, ny))}
        self._check(lib().upic_fft_solve_cn(self._ctx, *[_p(a) for a in ins],
                                            *[_p(out[k]) for k in ("phi", "psi", "rho", "A", "U", "grad_phi_mid")]))
        return out

    def map_log(self):
        """Map evaluations of the last step_implicit call, one row each in
        MAP_LOG_COLUMNS order (upic_map_log)."""
        n = ctypes.c_int()
        self._check(lib().upic_map_log(self._ctx, 0, None, ctypes.byref(n)))
        rows = np.empty((n.value, len(MAP_LOG_COLUMNS)))
        self._check(lib().upic_map_log(self._ctx, n.value, _p(rows), ctypes.byref(n)))
        return rows

    def failed_particle_log(self):
        """Failed-particle records of the last step_implicit call (selective
        fallback), one row per failed particle in FAILED_LOG_COLUMNS order
        (upic_failed_particle_log)."""
        n = ctypes.c_int()
        self._check(lib().upic_failed_particle_log(self._ctx, 0, None, ctypes.byref(n)))
        rows = np.empty((n.value, len(FAILED_LOG_COLUMNS)))
        self._check(lib().upic_failed_particle_log(self._ctx, n.value, _p(rows), ctypes.byref(n)))
        return rows

    def probe_fields(self, x, y):
        """Shape gathers and shape gradients of the accepted fields at the
        points (x, y), one row each in PROBE_COLUMNS order (upic_probe_fields)."""
        xa = _f64(x).ravel()
        ya = _f64(y).ravel()
        if ya.size != xa.size:
            raise ValueError("x and y differ in length")
        out = np.empty((xa.size, len(PROBE_COLUMNS)))
        self._check(lib().upic_probe_fields(self._ctx, xa.size, _p(xa), _p(ya), _p(out)))
        return out

    def write_field_snapshot(self, path, step, time, append=False):
        """Project3's field grid snapshot CSV rows of the accepted state
        (upic_write_field_snapshot)."""
        self._check(lib().upic_write_field_snapshot(self._ctx, os.fsencode(path), int(bool(append)), int(step),
                                                    float(time)))

    # ---- kernel-level entry points (include/upic.h) -----------------------
    def deposit_current(self, x, y, v, q):
        n = len(x)
        J = np.empty(3 * self.N)
        arrs = [_f64(x), _f64(y), _f64(v, (n, 3)), _f64(q)]
        self._check(lib().upic_deposit_current(self._ctx, n, *[_p(a) for a in arrs], _p(J)))
        return J.reshape(3, self.config.nx, self.config.ny)

    def deposit_charge(self, x, y, q):
        n = len(x)
        rho = np.empty(self.N)
        arrs = [_f64(x), _f64(y), _f64(q)]
        self._check(lib().upic_deposit_charge(self._ctx, n, *[_p(a) for a in arrs], _p(rho)))
        return rho.reshape(self.config.nx, self.config.ny)

    def gather(self, f, x, y):
        n = len(x)
        out = np.empty(n)
        self._check(lib().upic_gather(self._ctx, _p(_f64(f).ravel()), n, _p(_f64(x)), _p(_f64(y)),
                                      _p(out)))
        return out

    def fft2d(self, re, im, inverse=False):
        re = _f64(re).ravel().copy()
        im = _f64(im).ravel().copy()
        self._check(lib().upic_fft2d(self._ctx, _p(re), _p(im), int(bool(inverse))))
        shape = (self.config.nx, self.config.ny)
        return re.reshape(shape), im.reshape(shape)

    def spectral_derivative(self, f, direction):
        out = np.empty(self.N)
        self._check(lib().upic_spectral_derivative(self._ctx, _p(_f64(f).ravel()), int(direction),
                                                   _p(out)))
        return out.reshape(self.config.nx, self.config.ny)

    def poisson(self, rho):
        out = np.empty(self.N)
        self._check(lib().upic_poisson(self._ctx, _p(_f64(rho).ravel()), _p(out)))
        return out.reshape(self.config.nx, self.config.ny)

    def orbit_deposit(self, x, y, dx, vbar, q):
        """Orbit-averaged current of orbits (x, y) + s dx (implicit context)."""
        n = len(x)
        J = np.empty(3 * self.N)
        arrs = [_f64(x), _f64(y), _f64(dx, (n, 3)), _f64(vbar, (n, 3)), _f64(q)]
        self._check(lib().upic_orbit_deposit(self._ctx, n, *[_p(a) for a in arrs], _p(J)))
        return J.reshape(3, self.config.nx, self.config.ny)

    def orbit_gather(self, x, y, dx, mesh, An, Anp1):
        """Orbit averages of mesh (3 fields) and of the A gradient (implicit context):
        returns gathered (n, 3) and grad (n, 3, 3) [component][direction]."""
        n = len(x)
        gat = np.empty((n, 3))
        grad = np.empty((n, 3, 3))
        arrs = [_f64(x), _f64(y), _f64(dx, (n, 3)), _f64(mesh).ravel(), _f64(An).ravel(), _f64(Anp1).ravel()]
        self._check(lib().upic_orbit_gather(self._ctx, n, *[_p(a) for a in arrs], _p(gat), _p(grad)))
        return gat, grad

    def guess_conv(self, x, w, bias=None, mask=None, mode="relu", sign=1):
        """One periodic 3x3 conv of the learned predictor's network on the
        tensor cores.  x, mask: (nx, ny, 32) bf16 bit patterns (uint16); w:
        (32, 288) uint16; bias: 32 float32.  mode relu / mask return uint16
        (nx, ny, 32), linear returns float32 (nx, ny, 32)."""
        nx, ny = x.shape[0], x.shape[1]
        modes = {"relu": 0, "linear": 1, "mask": 2}
        x = np.ascontiguousarray(x, dtype=np.uint16)
        w = np.ascontiguousarray(w, dtype=np.uint16)
        b = None if bias is None else np.ascontiguousarray(bias, dtype=np.float32)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint16)
        out = np.empty((nx, ny, 32), dtype=np.float32 if mode == "linear" else np.uint16)
        vp = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        self._check(lib().upic_guess_conv(self._ctx, nx, ny, vp(x), vp(w), vp(b), vp(m), modes[mode], int(sign),
                                          vp(out)))
        return out

    def guess_wgrad(self, dz, x):
        """Weight (32, 288) and bias (32) gradients of one conv, float32."""
        nx, ny = x.shape[0], x.shape[1]
        dz = np.ascontiguousarray(dz, dtype=np.uint16)
        x = np.ascontiguousarray(x, dtype=np.uint16)
        g = np.empty(32 * 288 + 32, dtype=np.float32)
        self._check(lib().upic_guess_wgrad(self._ctx, nx, ny, dz.ctypes.data_as(ctypes.c_void_p),
                                           x.ctypes.data_as(ctypes.c_void_p), g.ctypes.data_as(ctypes.c_void_p)))
        return g[:32 * 288].reshape(32, 288), g[32 * 288:]

    def solve_bdf(self, source, hist):
        out = np.empty(self.N)
        h = _f64(hist).ravel()
        self._check(lib().upic_solve_bdf(self._ctx, _p(_f64(source).ravel()), _p(h), _p(out)))
        return out.reshape(self.config.nx, self.config.ny)


class Ensemble:
    """Independent explicit-method runs (loaded and started Simulations,
    each with its own grid, particles, tiling and re-sort interval) advanced
    together: `period` steps of all runs are recorded into one CUDA graph and
    replayed (upic_ensemble_*).  The Simulations stay usable afterwards."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s._ctx.value for s in self.sims])
        self._e = ctypes.c_void_p()
        rc = lib().upic_ensemble_create(arr, len(self.sims), ctypes.byref(self._e))
        if rc != 0:
            raise UpicError(rc, lib().upic_last_error(None).decode())
        p = ctypes.c_int()
        lib().upic_ensemble_period(self._e, ctypes.byref(p))
        self.period = p.value

    def step(self, nsteps):
        rc = lib().upic_ensemble_step(self._e, int(nsteps))
        if rc != 0:
            raise UpicError(rc, lib().upic_last_error(self.sims[0]._ctx).decode())

    def close(self):
        if self._e:
            lib().upic_ensemble_destroy(self._e)
            self._e = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def autotune_explicit(make_config, particles, tiles=(4, 8, 16), sort_intervals=(2, 4, 8), steps=8, warmup=3):
    """Pick the deposit tile edge and re-sort interval of an explicit run by
    timing each candidate on the run's own particles: make_config(tile,
    sort_interval) returns a Config; particles is the dict of
    generate_bimaxwellian.  Returns (tile, sort_interval, {candidate: ms per
    step}), steps timed by the host clock around upic_step (which returns
    when its work is complete)."""
    import time
    times = {}
    for tile in tiles:
        for si in sort_intervals:
            with Simulation(make_config(tile, si)) as sim:
                p = particles
                sim.set_particles(p["x"], p["y"], p["P"], p["v"], p["v_prev"], p["q"], p["m"])
                sim.init_fields(False)
                sim.step(warmup, 0)
                t0 = time.perf_counter()
                sim.step(steps, 0)
                times[(tile, si)] = 1e3 * (time.perf_counter() - t0) / steps
    best = min(times, key=times.get)
    return best[0], best[1], times


P3_CASES = {"two_stream": 0, "weibel": 1, "landau": 2}


def convergence_method_name(code):
    """The reference's convergence_method string of a solve-report code
    (upic_convergence_method_name)."""
    name = lib().upic_convergence_method_name(int(code))
    if name is None:
        raise ValueError(f"unknown convergence method code {code}")
    return name.decode()


def p3_initial_state(case, **keys):
    """Project3's cold-instability start (upic_p3_initial_state): case
    "two_stream" or "weibel" with Config keys (nx, ny, Lx, Ly, Lz, kappa,
    sigma1, n0, spline_order, perturbation_mode, particles_per_cell_pair, v0,
    perturbation, two_stream_*, tsi_transverse_*, weibel_*; the reference's
    defaults otherwise).  Returns a dict of x, y, v, q, m (particles in
    [-L/2, L/2)), A, U (3 x nx x ny) and growth_rate."""
    from ._native import UpicP3Case
    c = UpicP3Case()
    lib().upic_p3_case_default(ctypes.byref(c))
    c.kind = P3_CASES[case]
    for k, v in keys.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, int(v) if isinstance(getattr(c, k), int) else float(v))
    n = lib().upic_p3_case_particles(ctypes.byref(c))
    if n < 0:
        raise UpicError(-1, "invalid instability case")
    N = c.nx * c.ny
    out = {"x": np.empty(n), "y": np.empty(n), "v": np.empty((n, 3)), "q": np.empty(n), "m": np.empty(n),
           "A": np.empty((3, c.nx, c.ny)), "U": np.empty((3, c.nx, c.ny))}
    rate = np.zeros(1)
    rc = lib().upic_p3_initial_state(ctypes.byref(c), n, *[_p(out[k]) for k in ("x", "y", "v", "q", "m", "A", "U")],
                                     _p(rate))
    if rc != 0:
        raise UpicError(rc, "p3_initial_state failed")
    out["growth_rate"] = float(rate[0])
    assert out["A"].size == 3 * N
    return out


def generate_bimaxwellian(nx, ny, Lx, Ly, ppc, uth, udrift=(0.0, 0.0, 0.0), c=1.0, n0=1.0, seed=1):
    """Seeded synthetic plasma (upic_generate_bimaxwellian): returns a dict of
    x, y, P, v, v_prev, q, m in the reference's particle layout."""
    n = nx * ny * ppc
    out = {"x": np.empty(n), "y": np.empty(n), "P": np.empty((n, 3)), "v": np.empty((n, 3)),
           "v_prev": np.empty((n, 3)), "q": np.empty(n), "m": np.empty(n)}
    uth = _f64(uth)
    ud = _f64(udrift)
    rc = lib().upic_generate_bimaxwellian(int(nx), int(ny), float(Lx), float(Ly), int(ppc), float(c),
                                          float(n0), _p(uth), _p(ud), ctypes.c_uint64(seed),
                                          *[_p(out[k]) for k in ("x", "y", "P", "v", "v_prev", "q",
                                                                 "m")])
    if rc != 0:
        raise UpicError(rc, "generate_bimaxwellian failed")
    return out
