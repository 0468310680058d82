"""ctypes binding of libupic.so (include/upic.h).

The library is the product: there is no CPU fallback.  Loading fails loudly
when libupic.so has not been built (python -m unstaggered_pic_b200.build).
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libupic.so")

c_dp = ctypes.POINTER(ctypes.c_double)
c_ip = ctypes.POINTER(ctypes.c_int)

UPIC_ERR = {
    -1: "UPIC_ERR_CONFIG", -2: "UPIC_ERR_ARGUMENT", -3: "UPIC_ERR_CUDA", -4: "UPIC_ERR_STATE",
    -5: "UPIC_ERR_NONFINITE", -6: "UPIC_ERR_NONCONVERGED", -7: "UPIC_ERR_LOCAL_PARTICLE",
    -8: "UPIC_ERR_SUPERLUMINAL", -9: "UPIC_ERR_NOMEM", -10: "UPIC_ERR_TOO_LARGE",
}

# Exported C symbols with (restype, argtypes); the ABI test checks each one.
SYMBOLS = {
    "upic_abi_version": (ctypes.c_int, []),
    "upic_config_default": (ctypes.c_int, [ctypes.c_void_p]),
    "upic_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "upic_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "upic_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "upic_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "upic_set_particles": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 7),
    "upic_get_particles": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 5),
    "upic_init_fields": (ctypes.c_int, [ctypes.c_void_p, c_dp]),
    "upic_set_background": (ctypes.c_int, [ctypes.c_void_p, c_dp]),
    "upic_save_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "upic_load_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "upic_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    "upic_step_implicit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp, c_dp, c_dp]),
    "upic_step_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]),
    "upic_particle_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]),
    "upic_profile_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "upic_profile_read": (ctypes.c_int, [ctypes.c_void_p, c_dp, ctypes.POINTER(ctypes.c_long),
                                         ctypes.POINTER(ctypes.c_long)]),
    "upic_get_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp]),
    "upic_write_field_snapshot": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_long,
                                                 ctypes.c_double]),
    "upic_deposit_current": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 5),
    "upic_deposit_charge": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 4),
    "upic_gather": (ctypes.c_int, [ctypes.c_void_p, c_dp, ctypes.c_long, c_dp, c_dp, c_dp]),
    "upic_fft2d": (ctypes.c_int, [ctypes.c_void_p, c_dp, c_dp, ctypes.c_int]),
    "upic_spectral_derivative": (ctypes.c_int, [ctypes.c_void_p, c_dp, ctypes.c_int, c_dp]),
    "upic_poisson": (ctypes.c_int, [ctypes.c_void_p, c_dp, c_dp]),
    "upic_solve_bdf": (ctypes.c_int, [ctypes.c_void_p, c_dp, c_dp, c_dp]),
    "upic_orbit_deposit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 6),
    "upic_orbit_gather": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 8),
    "upic_guess_conv": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4
                        + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "upic_guess_wgrad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 3),
    "upic_ensemble_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "upic_ensemble_period": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "upic_ensemble_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "upic_ensemble_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "upic_deposit_current_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                    ctypes.c_double, ctypes.c_long, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p]),
    "upic_p3_case_default": (ctypes.c_int, [ctypes.c_void_p]),
    "upic_p3_case_particles": (ctypes.c_long, [ctypes.c_void_p]),
    "upic_p3_initial_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 8),
    "upic_set_initial_potential": (ctypes.c_int, [ctypes.c_void_p, c_dp, c_dp]),
    "upic_convergence_method_name": (ctypes.c_char_p, [ctypes.c_int]),
    "upic_set_time_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "upic_push_gmhc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 14 + [c_ip]),
    "upic_fft_solve_cn": (ctypes.c_int, [ctypes.c_void_p] + [c_dp] * 12),
    "upic_push_iaem": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long] + [c_dp] * 9),
    "upic_map_log": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp, c_ip]),
    "upic_failed_particle_log": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp, c_ip]),
    "upic_probe_fields": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long, c_dp, c_dp, c_dp]),
    "upic_generate_bimaxwellian": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_double, c_dp, c_dp, ctypes.c_uint64]
                                   + [c_dp] * 7),
}


class UpicP3Case(ctypes.Structure):
    """Mirror of struct upic_p3_case (include/upic.h)."""
    _fields_ = [
        ("kind", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
        ("kappa", ctypes.c_double), ("sigma1", ctypes.c_double), ("n0", ctypes.c_double),
        ("spline_order", ctypes.c_int), ("perturbation_mode", ctypes.c_int),
        ("particles_per_cell_pair", ctypes.c_int),
        ("v0", ctypes.c_double), ("perturbation", ctypes.c_double),
        ("two_stream_density_alpha", ctypes.c_double), ("two_stream_eigenmode", ctypes.c_int),
        ("two_stream_finite_grid_theory", ctypes.c_int),
        ("tsi_transverse_seed", ctypes.c_double), ("tsi_transverse_mode", ctypes.c_int),
        ("weibel_B0", ctypes.c_double), ("weibel_eigenmode", ctypes.c_int),
        ("weibel_finite_grid_theory", ctypes.c_int),
        ("landau_alpha", ctypes.c_double), ("thermal_velocity", ctypes.c_double),
    ]


class UpicConfig(ctypes.Structure):
    """Mirror of struct upic_config (include/upic.h)."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("method", ctypes.c_int), ("charge_update", ctypes.c_int),
        ("c", ctypes.c_double), ("eps0", ctypes.c_double), ("mu0", ctypes.c_double),
        ("n0", ctypes.c_double),
        ("precision", ctypes.c_int), ("sort_interval", ctypes.c_int),
        ("tile", ctypes.c_int), ("guard", ctypes.c_int),
        ("reserved", ctypes.c_int * 8),
        ("Lz", ctypes.c_double),
        ("kappa", ctypes.c_double), ("sigma1", ctypes.c_double), ("sigma2", ctypes.c_double),
        ("spline_order", ctypes.c_int), ("orbit_quad_order", ctypes.c_int),
        ("split_orbit_at_knots", ctypes.c_int), ("nyquist_projection", ctypes.c_int),
        ("nonlinear_solver", ctypes.c_int), ("nonlinear_max_iter", ctypes.c_int),
        ("anderson_memory", ctypes.c_int), ("anderson_start", ctypes.c_int),
        ("local_max_iter", ctypes.c_int),
        ("nonlinear_rtol", ctypes.c_double), ("nonlinear_atol", ctypes.c_double),
        ("anderson_damping", ctypes.c_double), ("anderson_regularization", ctypes.c_double),
        ("anderson_growth_limit", ctypes.c_double),
        ("local_rtol", ctypes.c_double), ("local_atol", ctypes.c_double),
        ("local_damping", ctypes.c_double),
        ("perturbation_mode", ctypes.c_int),
        ("picard_tol", ctypes.c_double), ("picard_max_iter", ctypes.c_int),
        ("final_consistency_sweep", ctypes.c_int),
        ("current_predictor", ctypes.c_int),
        ("local_warm_start", ctypes.c_int),
        ("selective_particle_fallback", ctypes.c_int), ("selective_particle_max_substeps", ctypes.c_int),
        ("learned_train_steps", ctypes.c_int), ("learned_train_iters", ctypes.c_int),
        ("learned_rate", ctypes.c_double), ("learned_seed", ctypes.c_ulonglong),
    ]


_lib = None


def lib():
    """Load libupic.so once; raise if it is missing (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the CUDA library with "
            "`python -m unstaggered_pic_b200.build` (no CPU fallback exists)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SYMBOLS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L
