/*
 * upic.h -- C ABI of the B200-native unstaggered generalized-momentum PIC step.
 *
 * The reference (sgong11/Unstaggered_PIC) exposes this step only as
 * single-file C++ solvers driven by `prog deck.txt`; its step functions are
 * `static` inside one translation unit.  This header is the drop-in boundary
 * a host driver (or an FFI binding: ctypes, cgo, JNI) calls instead.  Every
 * entry point names the reference function(s) it replaces, as
 * Project<N>/<file>:<line>.
 *
 * Conventions (those of the reference):
 *   - grids are nx*ny doubles, node id = i*ny + j (x index i is the slow one),
 *     Project2/spectral_pic_part3.cpp:313-317;
 *   - explicit methods place particles in [0,Lx)x[0,Ly) with node i at x=i*dx
 *     (spectral_pic_part3.cpp:537-552);
 *   - per-particle 3-vectors (P, v, v_prev) are interleaved x,y,z triples,
 *     the memory layout of the reference's std::vector<Vec3>;
 *   - all arithmetic is FP64 unless the context is created with
 *     UPIC_PRECISION_MIXED.
 *
 * Errors: every call returns 0 on success or a negative UPIC_ERR_* code;
 * upic_last_error() returns the message.  No exception crosses the ABI.
 * A context belongs to one host thread.  Work is ordered on the context's
 * CUDA stream (upic_set_stream) and every call that returns host data
 * synchronizes that stream.
 */
#ifndef UPIC_H
#define UPIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UPIC_ABI_VERSION 2

/* Error codes. */
enum {
    UPIC_OK = 0,
    UPIC_ERR_CONFIG = -1,         /* bad deck / config (reference throws in read_config) */
    UPIC_ERR_ARGUMENT = -2,       /* bad pointer, size or enum */
    UPIC_ERR_CUDA = -3,           /* a CUDA runtime call failed */
    UPIC_ERR_STATE = -4,          /* call out of order (e.g. step before particles) */
    UPIC_ERR_NONFINITE = -5,      /* non-finite particle or field value detected */
    UPIC_ERR_NONCONVERGED = -6,   /* outer nonlinear solve failed (NonlinearSolveFailure) */
    UPIC_ERR_LOCAL_PARTICLE = -7, /* per-particle local solve failed */
    UPIC_ERR_SUPERLUMINAL = -8,   /* |v| >= c in a relativistic iterate */
    UPIC_ERR_NOMEM = -9,          /* device allocation failed */
    UPIC_ERR_TOO_LARGE = -10      /* size exceeds a fixed capacity (UPIC_NOALLOC_MAX_NODES) */
};

/* Methods.  BDF1/BDF2: explicit spectral GM step with IAEM push,
 * Project2/spectral_pic_part3.cpp:1094-1189.  CN_ORBIT: implicit
 * energy-conserving orbit-averaged GM-HC-CN step (relativistic
 * Higuera-Cary rotation, Crank-Nicolson potentials, outer Anderson/Picard
 * iteration on the mesh current), Project3/ec_pic_nyquist_projected.cpp
 * nonlinear_step_orbit:6477.  CN_ORBIT_NONREL: the non-relativistic
 * orbit-averaged CN step with Picard iteration on the particle velocities,
 * Project1/ec_pic_serial_demo.cpp picard_step_orbit:1509 (c, eps0, mu0 as in
 * the explicit methods; no Nyquist projection, Nyquist wave numbers kept).
 * The implicit methods run in 2D (nz = 1). */
enum { UPIC_METHOD_BDF1 = 1, UPIC_METHOD_BDF2 = 2, UPIC_METHOD_CN_ORBIT = 3, UPIC_METHOD_CN_ORBIT_NONREL = 4 };

/* First guess of the implicit step's outer current iteration.  PREVIOUS:
 * the last accepted current, as the reference does
 * (nonlinear_step_uniform_subcycled, ec_pic_nyquist_projected.cpp:5887).
 * EXTRAPOLATED: 2 J^n - J^{n-1} (the previous current on the first step
 * after upic_init_fields); not in the reference.  LEARNED (CN_ORBIT only):
 * the extrapolation plus the correction predicted by a small conv net
 * (4 layers of 3x3 periodic convolutions, 32 channels, BF16 on the tensor
 * cores) from the last three steps' J, A and phi, trained online on the
 * accepted currents of the first learned_train_steps steps; a step uses it
 * only when on the step before the learned prediction was closer to the
 * accepted current than the extrapolation, else the extrapolation.  The
 * iteration still runs to the same tolerances, so only the iteration count
 * changes. */
enum { UPIC_PREDICTOR_PREVIOUS = 0, UPIC_PREDICTOR_EXTRAPOLATED = 1, UPIC_PREDICTOR_LEARNED = 2 };

/* Outer nonlinear solver of the implicit method (Config::nonlinear_solver,
 * ec_pic_nyquist_projected.cpp:891). */
enum { UPIC_SOLVER_ANDERSON = 0, UPIC_SOLVER_PICARD = 1 };

/* Charge source: continuity-consistent (conserving) or redeposited (naive),
 * spectral_pic_part3.cpp:1147-1152. */
enum { UPIC_CHARGE_CONSERVING = 0, UPIC_CHARGE_NAIVE = 1 };

enum { UPIC_PRECISION_FP64 = 0, UPIC_PRECISION_MIXED = 1 };

/* Field selectors for upic_get_field.  E and B are derived on request from
 * the resident state: explicit methods E = -grad phi - dA/dt with the step's
 * BDF derivative and B = curl A (compute_diagnostics,
 * Project2/spectral_pic_part3.cpp:918-944); implicit methods E = -grad phi - U
 * and B = curl A (compute_E, spectral_curl,
 * Project3/ec_pic_nyquist_projected.cpp:3338, :1780). */
enum {
    UPIC_FIELD_PHI = 0,
    UPIC_FIELD_AX = 1,
    UPIC_FIELD_AY = 2,
    UPIC_FIELD_AZ = 3,
    UPIC_FIELD_RHO = 4,
    UPIC_FIELD_JX = 5,
    UPIC_FIELD_JY = 6,
    UPIC_FIELD_JZ = 7,
    UPIC_FIELD_PSI = 8,
    UPIC_FIELD_UX = 9,
    UPIC_FIELD_UY = 10,
    UPIC_FIELD_UZ = 11,
    UPIC_FIELD_EX = 12,
    UPIC_FIELD_EY = 13,
    UPIC_FIELD_EZ = 14,
    UPIC_FIELD_BX = 15,
    UPIC_FIELD_BY = 16,
    UPIC_FIELD_BZ = 17,
    UPIC_FIELD_COUNT = 18
};

/* Diagnostics row, the column order of the reference's _diagnostics.csv after
 * step,time,requested_method,active_method,charge_update
 * (spectral_pic_part3.cpp:886-900, 1117-1119). */
enum {
    UPIC_DIAG_GAUGE_RMS = 0,
    UPIC_DIAG_GAUSS_RMS,
    UPIC_DIAG_CONTINUITY_RMS,
    UPIC_DIAG_BZ_L2,
    UPIC_DIAG_B_L2,
    UPIC_DIAG_E_L2,
    UPIC_DIAG_RHO_L2,
    UPIC_DIAG_J_L2,
    UPIC_DIAG_FIELD_ENERGY,
    UPIC_DIAG_KINETIC_ENERGY,
    UPIC_DIAG_TOTAL_ENERGY,
    UPIC_DIAG_MAX_SPEED,
    UPIC_DIAG_MEAN_GAMMA,
    UPIC_DIAG_COUNT
};

/* Run configuration; mirrors the reference deck keys of
 * spectral_pic_part3.cpp:174-231 (Config).  Fill with upic_config_default(). */
typedef struct upic_config {
    int nx, ny;              /* powers of two (radix-2 FFT), read_config:281 */
    double Lx, Ly;
    double dt;
    int method;              /* UPIC_METHOD_* */
    int charge_update;       /* UPIC_CHARGE_* */
    double c, eps0, mu0;     /* normalized constants */
    double n0;               /* fixed uniform ion background density */
    int precision;           /* UPIC_PRECISION_* */
    int sort_interval;       /* steps between particle re-sorts; 0 = automatic */
    int tile;                /* deposit tile edge in cells; 0 = automatic */
    int guard;               /* deposit window guard in cells; -1 = automatic */
    int reserved[8];
    /* Implicit method (UPIC_METHOD_CN_ORBIT): the Project3 deck keys
     * (Config, ec_pic_nyquist_projected.cpp:837-1005).  Positions are in
     * [-L/2, L/2) with node i at -L/2 + i*dx, as in Project3. */
    double Lz;                     /* cell volume dV = dx*dy*Lz (nz = 1) */
    double kappa, sigma1, sigma2;  /* nondimensional light speed and sources */
    int spline_order;              /* 1..4 */
    int orbit_quad_order;          /* Gauss-Legendre points per orbit segment */
    int split_orbit_at_knots;
    int nyquist_projection;
    int nonlinear_solver;          /* UPIC_SOLVER_* */
    int nonlinear_max_iter;
    int anderson_memory;           /* 1..4 */
    int anderson_start;
    int local_max_iter;            /* particle_local_max_iter */
    double nonlinear_rtol, nonlinear_atol;
    double anderson_damping, anderson_regularization, anderson_growth_limit;
    double local_rtol, local_atol, local_damping;  /* particle_local_* */
    int perturbation_mode;         /* x (and y) Fourier mode of the diagnostics */
    /* Non-relativistic implicit method (UPIC_METHOD_CN_ORBIT_NONREL): the
     * Project1 deck keys (Config, ec_pic_serial_demo.cpp:232-301). */
    double picard_tol;
    int picard_max_iter;
    int final_consistency_sweep;
    /* First outer-iteration guess of the implicit GM-HC-CN step's mesh
     * current (UPIC_PREDICTOR_*). */
    int current_predictor;
    /* Implicit GM-HC-CN step: with 1, each particle's local fixed point starts
     * from its orbit velocity of the previous current-map evaluation of the
     * same step instead of from v^n (the reference's start,
     * solve_local_particle_substep, ec_pic_nyquist_projected.cpp:4930).  The
     * local and outer tolerances are unchanged; results agree with the
     * reference to those tolerances, not bit for bit.  Default 0. */
    int local_warm_start;
    /* Implicit GM-HC-CN step: selective particle sub-cycling fallback
     * (Config::selective_particle_fallback / selective_particle_max_substeps,
     * nonlinear_step_selective_particle_fallback, ec_pic_nyquist_projected.cpp
     * :6328).  When a particle's local solve fails over the full dt, failing
     * particles are advanced in 2, 4, ... up to max_substeps (a power of two
     * <= 64) chained substeps and the outer current solve restarts. */
    int selective_particle_fallback;
    int selective_particle_max_substeps;
    /* UPIC_PREDICTOR_LEARNED: training steps (accepted steps whose current
     * trains the net, from the third step on; default 200), Adam iterations
     * per training step (default 4), Adam learning rate (default 1e-3),
     * weight-initialisation seed. */
    int learned_train_steps;
    int learned_train_iters;
    double learned_rate;
    unsigned long long learned_seed;
} upic_config;

typedef struct upic_ctx upic_ctx;

/* Diagnostics row of the implicit method: the Diagnostics struct of
 * ec_pic_nyquist_projected.cpp:3469-3519 (columns of its _diagnostics.csv). */
enum {
    UPIC_P3_GAUSS_RMS = 0, UPIC_P3_GAUSS_MAX, UPIC_P3_DIVE_RMS, UPIC_P3_SIGMA1_RHO_RMS,
    UPIC_P3_GAUSS_NORM_RMS, UPIC_P3_GAUSS_RELATIVE, UPIC_P3_GAUGE_RMS, UPIC_P3_GAUGE_MAX,
    UPIC_P3_PSI_OVER_KAPPA2_RMS, UPIC_P3_DIVA_RMS, UPIC_P3_GAUGE_NORM_RMS, UPIC_P3_GAUGE_RELATIVE,
    UPIC_P3_FIELD_ENERGY, UPIC_P3_KINETIC_ENERGY, UPIC_P3_TOTAL_ENERGY, UPIC_P3_RHO_MODE,
    UPIC_P3_E_MODE_RE, UPIC_P3_E_MODE_IM, UPIC_P3_E_MODE_ABS, UPIC_P3_BZ_Y_MODE_RE,
    UPIC_P3_BZ_Y_MODE_IM, UPIC_P3_BZ_Y_MODE_ABS, UPIC_P3_MEAN_RHO, UPIC_P3_DIAG_COUNT
};
/* UPIC_METHOD_CN_ORBIT_NONREL fills the same row with Project1's
 * definitions (compute_diagnostics, ec_pic_serial_demo.cpp:1057): Gauss law
 * div E - rho/eps0, gauge psi/c^2 + div A, field energy eps0/2 E^2 + B^2/(2
 * mu0), kinetic energy sum m v^2/2; Project1's columns are gauss_rms,
 * gauss_max, gauge_rms, field/kinetic/total energy, rho_mode, E_mode_*,
 * mean_rho. */

/* Per-step solve report of the implicit method (NonlinearSolveInfo,
 * ec_pic_nyquist_projected.cpp:5493-5533). */
enum {
    UPIC_INFO_ITERATIONS = 0, UPIC_INFO_CONVERGED, UPIC_INFO_FINAL_RMS_RESIDUAL,
    UPIC_INFO_FINAL_MAX_PARTICLE_RESIDUAL, UPIC_INFO_LOCAL_ITER_MAX, UPIC_INFO_LOCAL_ITER_MEAN,
    UPIC_INFO_ANDERSON_STEPS, UPIC_INFO_PICARD_STEPS,
    /* Picard errors of the last iteration (picard_step_orbit,
     * ec_pic_serial_demo.cpp:1509-1530; NaN for CN_ORBIT) and the path
     * statistics of the accepted orbits (crossing particles, average and
     * maximum segments per orbit), the _diagnostics.csv columns of both. */
    UPIC_INFO_CURRENT_ERROR, UPIC_INFO_VELOCITY_ERROR, UPIC_INFO_CROSSING_PARTICLES,
    UPIC_INFO_AVG_PATH_SEGMENTS, UPIC_INFO_MAX_PATH_SEGMENTS,
    /* selective sub-cycling (NonlinearSolveInfo::selective_*): fallback used,
     * refinement restarts, refined particles, total particle substeps */
    UPIC_INFO_SELECTIVE_FALLBACK_USED, UPIC_INFO_SELECTIVE_RESTARTS, UPIC_INFO_SELECTIVE_REFINED,
    UPIC_INFO_SELECTIVE_SUBSTEPS,
    /* first guess of the outer current iteration (CN_ORBIT): the predictor
     * used (UPIC_PREDICTOR_*), and the relative rms distances |J - J^{n+1}| /
     * |J^{n+1}| from the accepted current of the guess used, of the
     * extrapolation 2 J^n - J^{n-1} and of the learned prediction (NaN when
     * not formed), and the learned predictor's training loss on this step
     * (mean squared error in units of the rms second difference of J; NaN
     * when it did not train) */
    UPIC_INFO_PREDICTOR_USED, UPIC_INFO_GUESS_ERROR, UPIC_INFO_EXTRAPOLATION_ERROR, UPIC_INFO_LEARNED_ERROR,
    UPIC_INFO_LEARNED_LOSS,
    /* the rest of NonlinearSolveInfo (CN_ORBIT; NaN for CN_ORBIT_NONREL):
     * Anderson restarts (history cleared by the growth limit, a failed or
     * non-finite candidate, or a failed Anderson line search), the final
     * absolute rms residual, the observed convergence rate (final / first
     * relative rms residual)^(1/(iterations-1)) (observed_nonlinear_
     * convergence_rate :5534; inf with fewer than 2 iterations), the secant
     * map contraction rms(G(x_k) - G(x_{k-1})) / rms(x_k - x_{k-1}) of the
     * last iterate pair with rms(x_k - x_{k-1}) > 64 eps (:5990-5996; inf
     * when none), updates accepted with alpha < 1 and the smallest such
     * alpha (1 when none), the method code of the last accepted update
     * (UPIC_METHOD_CODE_*, upic_convergence_method_name), the largest
     * substep count of the particle layout, the outer iterations of the
     * failed direct attempt before a selective fallback, the selective
     * work ratio (particle substeps / particles) and the particles at 1,
     * 2, 4, ..., 64 substeps */
    UPIC_INFO_ANDERSON_RESTARTS, UPIC_INFO_FINAL_ABS_RMS_RESIDUAL, UPIC_INFO_OBSERVED_RATE,
    UPIC_INFO_MAP_CONTRACTION, UPIC_INFO_BACKTRACKED_STEPS, UPIC_INFO_MIN_UPDATE_ALPHA,
    UPIC_INFO_CONVERGENCE_METHOD, UPIC_INFO_SUBSTEPS_USED, UPIC_INFO_DIRECT_ATTEMPT_ITERATIONS,
    UPIC_INFO_SELECTIVE_WORK_RATIO, UPIC_INFO_SELECTIVE_N1, UPIC_INFO_SELECTIVE_N2, UPIC_INFO_SELECTIVE_N4,
    UPIC_INFO_SELECTIVE_N8, UPIC_INFO_SELECTIVE_N16, UPIC_INFO_SELECTIVE_N32, UPIC_INFO_SELECTIVE_N64,
    UPIC_INFO_COUNT
};

/* Method code of UPIC_INFO_CONVERGENCE_METHOD: base + 8 * form.  Bases
 * (the update_method strings of nonlinear_step_uniform_subcycled :5878):
 * none, picard, picard_fallback (converged before any update),
 * current_anderson, current_anderson_backtracked, current_picard,
 * current_picard_backtracked.  Forms (the prefix nonlinear_step_orbit
 * :6477 and the selective fallback :6328 put in front): plain, the
 * direct full-dt solve ("nested_full_dt_"), the selective fallback
 * ("selective_"). */
enum {
    UPIC_METHOD_CODE_NONE = 0, UPIC_METHOD_CODE_PICARD, UPIC_METHOD_CODE_PICARD_FALLBACK,
    UPIC_METHOD_CODE_ANDERSON, UPIC_METHOD_CODE_ANDERSON_BACKTRACKED, UPIC_METHOD_CODE_CURRENT_PICARD,
    UPIC_METHOD_CODE_CURRENT_PICARD_BACKTRACKED,
    UPIC_METHOD_FORM_DIRECT = 8, UPIC_METHOD_FORM_SELECTIVE = 16
};

/* Step diagnostics of the implicit method: StepDiagnostics of
 * compute_step_diagnostics, ec_pic_nyquist_projected.cpp:4501 (:4303-4321),
 * in the column order of its _step_diagnostics.csv (:8462-8473). */
enum {
    UPIC_SD_A_CHAIN_ABS_RMS = 0, UPIC_SD_A_CHAIN_REL_RMS, UPIC_SD_A_CHAIN_MAX_NORM,
    UPIC_SD_A_CHAIN_MEAN_NORM, UPIC_SD_A_CHAIN_WORK_DEFECT, UPIC_SD_DELTA_K, UPIC_SD_DELTA_W,
    UPIC_SD_DELTA_TOTAL_ENERGY, UPIC_SD_PARTICLE_WORK, UPIC_SD_GRID_WORK,
    UPIC_SD_DEPOSIT_GATHER_WORK_RESIDUAL, UPIC_SD_PARTICLE_ENERGY_RESIDUAL,
    UPIC_SD_FIELD_ENERGY_RESIDUAL, UPIC_SD_CROSSING_PARTICLES, UPIC_SD_TOTAL_CROSSINGS,
    UPIC_SD_AVERAGE_PATH_SEGMENTS, UPIC_SD_MAX_PATH_SEGMENTS, UPIC_SD_COUNT
};

/* ABI version of the loaded library (UPIC_ABI_VERSION). */
int upic_abi_version(void);

/* Defaults of the reference Config (spectral_pic_part3.cpp:174-231). */
int upic_config_default(upic_config* cfg);

/* Validate cfg (read_config:281-293) and allocate a context on the current
 * CUDA device.  Replaces make_grid (spectral_pic_part3.cpp:332). */
int upic_create(const upic_config* cfg, upic_ctx** out);
int upic_destroy(upic_ctx* ctx);

/* Message of the last error on ctx (or of the last failed upic_create when
 * ctx is NULL).  The pointer stays valid until the next call on ctx. */
const char* upic_last_error(const upic_ctx* ctx);

/* Order the context's work on a caller-provided cudaStream_t (NULL restores
 * the context's own stream). */
int upic_set_stream(upic_ctx* ctx, void* cuda_stream);

/* Load the mobile electrons (ParticleSet::electrons,
 * spectral_pic_part3.cpp:586-622): positions x,y; canonical momentum P,
 * velocity v and previous velocity v_prev as xyz triples; per-particle
 * charge q and mass m.  Copies host -> device. */
int upic_set_particles(upic_ctx* ctx, long np, const double* x, const double* y,
                       const double* P, const double* v, const double* v_prev,
                       const double* q, const double* m);

/* Copy the particle state back in the order it was given. */
int upic_get_particles(upic_ctx* ctx, long np, double* x, double* y, double* P, double* v,
                       double* v_prev);

/* Fixed background charge density (explicit methods): rho_bg, nx*ny doubles,
 * replaces the uniform ion density n0 in rho0 and in every naive charge
 * re-deposit -- the reference's ParticleSet::fixed_ion_rho, which the cloud
 * example fills from stationary ions (spectral_pic_part3.cpp:618-621,
 * 720-724, deposit_total_charge_naive :739).  NULL restores n0.  Call it
 * before upic_init_fields. */
int upic_set_background(upic_ctx* ctx, const double* rho_bg);

/* Checkpoint / restart -- no counterpart in the reference, which writes CSV
 * field snapshots only (ec_pic_nyquist_projected.cpp write_field_grid_snapshot
 * :8160) and cannot resume a run.  upic_save_state writes everything the next
 * step of the context reads (particles in their current order, field
 * spectra and histories, deposit accumulators, step counters) to a binary
 * file; upic_load_state restores it into a context created with the same
 * configuration (UPIC_ERR_CONFIG otherwise), after which the run continues
 * bit for bit as the saved one would have.  The file holds device-order
 * state of this library version; it is not a portable exchange format. */
int upic_save_state(upic_ctx* ctx, const char* path);
int upic_load_state(upic_ctx* ctx, const char* path);

/* Start-up fields: rho0 = n0 + deposited electron charge, J0 = deposited
 * current, phi0 from Poisson, A0 = 0, all BDF histories filled with copies
 * (spectral_pic_part3.cpp:1100-1111).  If diag_row is not NULL it receives
 * the step-0 diagnostics row (BDF1 derivatives, :1121-1131).
 * Implicit method: rho = deposited charge + n0 (zero mean), phi from
 * Poisson, psi = A = U = 0, J deposited, P = m gamma v, v_prev from a
 * backward Lorentz step (ec_pic_nyquist_projected.cpp:4061-4123, 3423);
 * diag_row then has UPIC_P3_DIAG_COUNT entries. */
int upic_init_fields(upic_ctx* ctx, double* diag_row);

/* Advance nsteps implicit steps (nonlinear_step_orbit,
 * ec_pic_nyquist_projected.cpp:6477, then compute_diagnostics :3521 and, the
 * run loop's per-step record, compute_step_diagnostics :4501 at :8835).
 * diag (optional): nsteps x UPIC_P3_DIAG_COUNT; info (optional): nsteps x
 * UPIC_INFO_COUNT; step_diag (optional, one extra orbit pass per step):
 * nsteps x UPIC_SD_COUNT.  A step that does not converge returns
 * UPIC_ERR_NONCONVERGED, one whose per-particle solve fails returns
 * UPIC_ERR_LOCAL_PARTICLE; the state then stays at the last accepted step. */
int upic_step_implicit(upic_ctx* ctx, int nsteps, double* diag, double* info, double* step_diag);

/* Advance nsteps steps of the explicit BDF/IAEM method (loop body of
 * run_simulation, spectral_pic_part3.cpp:1133-1189).  diag (optional):
 * nsteps x UPIC_DIAG_COUNT rows; diagnostics are computed on steps where
 * (global step % diag_stride == 0) or on the last step of this call, and
 * other rows are filled with NaN.  diag_stride <= 0 disables diagnostics. */
int upic_step(upic_ctx* ctx, int nsteps, int diag_stride, double* diag);

/* Profiling of the dominant kernel: with on != 0, CUDA events are recorded
 * on the context's stream around every particle push kernel of upic_step
 * (gather + push + next-step deposit).  on = 0 disables and clears.  No
 * reference counterpart (the reference only times whole runs with a wall
 * clock, Project3/ec_pic_nyquist_projected.cpp:145-197). */
int upic_profile_enable(upic_ctx* ctx, int on);

/* Summed device time (ms) and count of the push kernels recorded since
 * upic_profile_enable, and the number of kernels this library has launched
 * since it was loaded (all contexts). */
int upic_profile_read(upic_ctx* ctx, double* push_ms, long* push_launches, long* kernel_launches);

/* Number of steps taken since upic_init_fields. */
int upic_step_count(const upic_ctx* ctx, long* steps);
/* Number of particles the context holds (upic_set_particles or a restored state). */
int upic_particle_count(const upic_ctx* ctx, long* np);

/* Fields of the current time level (phi, A, rho, J; implicit method also
 * psi = d phi/dt and U = dA/dt), nx*ny doubles. */
int upic_get_field(upic_ctx* ctx, int which, double* host);

/* Field snapshot of the implicit methods' accepted state in the columns of
 * Project3's _field_grid_snapshots.csv (write_field_grid_header :8137-8140,
 * write_field_grid_snapshot :8160): step,time,spline_order,ix,iy,iz,x,y,z,
 * phi,psi,rho,Ax,Ay,Az,Ux,Uy,Uz,Jx,Jy,Jz,Ex,Ey,Ez,Bx,By,Bz, one row per node
 * (x-major; x = -Lx/2 + ix*dx as in Project3's box, iz = 0, z = -Lz/2),
 * values at 17 significant digits.  append = 0 creates the file with the
 * header, append != 0 adds rows to it.  UPIC_ERR_STATE for explicit
 * methods, whose state has no psi or U. */
int upic_write_field_snapshot(upic_ctx* ctx, const char* path, int append, long step, double time);

/* Time step of the next implicit steps (CN_ORBIT, CN_ORBIT_NONREL): the
 * reference's run loop shortens the last step to the remaining time,
 * dt_try = min(dt, n_steps*dt - time) (main, ec_pic_nyquist_projected.cpp
 * :8702).  0 < dt <= the dt the context was created with (its deposit
 * window covers kappa*dt of travel); UPIC_ERR_STATE for explicit methods,
 * whose BDF coefficients are fixed at creation. */
int upic_set_time_step(upic_ctx* ctx, double dt);

/* The reference's string for a UPIC_INFO_CONVERGENCE_METHOD code
 * ("nested_full_dt_current_anderson", ...); NULL for an unknown code. */
const char* upic_convergence_method_name(int code);

/* Map evaluations of the last upic_step_implicit call (CN_ORBIT), the rows
 * of Project3's _particle_inner_history.csv after its time_n,dt columns
 * (nonlinear_step_uniform_subcycled :5918-5945): step of the call (0 ..
 * nsteps-1), map_evaluation (1, 2, ... within one outer solve; a selective
 * fallback restarts the count), particles_converged (1 when every local
 * particle solve converged, else 0), failed_particles,
 * max_scaled_particle_residual (inf when non-finite),
 * local_iterations_mean (NaN when particles failed), local_iterations_max.
 * *nrows receives the number of rows; min(capacity, *nrows) rows of
 * UPIC_MAPLOG_COUNT doubles are copied to rows. */
enum {
    UPIC_MAPLOG_STEP = 0, UPIC_MAPLOG_EVALUATION, UPIC_MAPLOG_CONVERGED, UPIC_MAPLOG_FAILED,
    UPIC_MAPLOG_MAX_SCALED_RESIDUAL, UPIC_MAPLOG_ITER_MEAN, UPIC_MAPLOG_ITER_MAX, UPIC_MAPLOG_COUNT
};
int upic_map_log(upic_ctx* ctx, int capacity, double* rows, int* nrows);

/* Failed-particle records of the last upic_step_implicit call (CN_ORBIT with
 * selective_particle_fallback): one row per particle whose local solve
 * failed in a map evaluation of the selective layout (the
 * FailedParticleDiagnostic list of evaluate_selective_current_map_at_layout,
 * ec_pic_nyquist_projected.cpp:5331-5350, sorted by particle index), with
 * the columns of Project3's _failed_particle_diagnostics.csv after its
 * time_before column (write_failed_particle_diagnostics :6234): step of the
 * call, layout_refinement_restart, map_evaluation, event_exhausted (1 when
 * the event left a particle at the substep limit), failed_particles_in_event,
 * particle_index (load order), assigned_substeps, failed_substep (0-based),
 * theta0, theta1, h, local_iterations, failure_reason (0-5 as the
 * reference's LocalParticleFailureReason; 6 = more knot crossings than the
 * orbit quadrature holds), first_scaled_residual, final_scaled_residual,
 * final_absolute_residual, q, m, x0 (3; z = 0), P0 (3), initial_guess (3),
 * last_guess (3), last_map (3).  Every failed particle of an event is
 * listed; the reference's file keeps the worst selective_failure_diagnostic_
 * limit of them (and the worst exhausted one), which the writer selects.
 * *nrows receives the number of rows; min(capacity, *nrows) rows of
 * UPIC_FAILLOG_COUNT doubles are copied to rows. */
enum {
    UPIC_FAILLOG_STEP = 0, UPIC_FAILLOG_RESTART, UPIC_FAILLOG_EVALUATION, UPIC_FAILLOG_EXHAUSTED,
    UPIC_FAILLOG_IN_EVENT, UPIC_FAILLOG_PARTICLE, UPIC_FAILLOG_SUBSTEPS, UPIC_FAILLOG_FAILED_SUBSTEP,
    UPIC_FAILLOG_THETA0, UPIC_FAILLOG_THETA1, UPIC_FAILLOG_H, UPIC_FAILLOG_ITERATIONS, UPIC_FAILLOG_REASON,
    UPIC_FAILLOG_FIRST_SCALED, UPIC_FAILLOG_FINAL_SCALED, UPIC_FAILLOG_FINAL_ABSOLUTE, UPIC_FAILLOG_Q,
    UPIC_FAILLOG_M, UPIC_FAILLOG_X0, UPIC_FAILLOG_P0 = UPIC_FAILLOG_X0 + 3,
    UPIC_FAILLOG_INITIAL_GUESS = UPIC_FAILLOG_P0 + 3, UPIC_FAILLOG_LAST_GUESS = UPIC_FAILLOG_INITIAL_GUESS + 3,
    UPIC_FAILLOG_LAST_MAP = UPIC_FAILLOG_LAST_GUESS + 3, UPIC_FAILLOG_COUNT = UPIC_FAILLOG_LAST_MAP + 3
};
int upic_failed_particle_log(upic_ctx* ctx, int capacity, double* rows, int* nrows);

/* Point probes of the implicit method's accepted fields with the particle
 * shape (evaluate_reconstructed_field_probe, ec_pic_nyquist_projected.cpp
 * :7924-7945): for each point (x[p], y[p]) the B-spline gathers of phi,
 * psi, rho, A, U, J, of the grid fields E = -grad phi - U and B = curl A
 * (compute_E :3338, spectral_curl :1780), the shape gradient grad(S phi)
 * (gather_shape_gradient_scalar_at) and grad(S A) (gradA[c][d] =
 * dA_c/dx_d); z derivatives are 0 on the 2D grid.  out: np x
 * UPIC_PROBE_COUNT doubles.  CN_ORBIT contexts. */
enum {
    UPIC_PROBE_PHI = 0, UPIC_PROBE_PSI = 1, UPIC_PROBE_RHO = 2, UPIC_PROBE_A = 3, UPIC_PROBE_U = 6,
    UPIC_PROBE_J = 9, UPIC_PROBE_E = 12, UPIC_PROBE_B = 15, UPIC_PROBE_GRAD_PHI = 18, UPIC_PROBE_GRAD_A = 21,
    UPIC_PROBE_COUNT = 30
};
int upic_probe_fields(upic_ctx* ctx, long np, const double* x, const double* y, double* out);

/* ---- Kernel-level entry points (host arrays in and out).  Each runs the
 * same device kernels as upic_step on the context's grid. ------------- */

/* J (3 x nx*ny) = sum_p q v S(x_p)/dA: deposit_current,
 * spectral_pic_part3.cpp:747-755 (scatter_scalar :554). */
int upic_deposit_current(upic_ctx* ctx, long np, const double* x, const double* y,
                         const double* v, const double* q, double* J);

/* rho = n0 + sum_p q S(x_p)/dA: deposit_total_charge_naive,
 * spectral_pic_part3.cpp:739-745. */
int upic_deposit_charge(upic_ctx* ctx, long np, const double* x, const double* y,
                        const double* q, double* rho);

/* out[p] = sum f S(x_p): gather_scalar, spectral_pic_part3.cpp:564-574. */
int upic_gather(upic_ctx* ctx, const double* f, long np, const double* x, const double* y,
                double* out);

/* In-place complex 2D FFT (rows then columns), inverse scaled by 1/N:
 * fft2d, spectral_pic_part3.cpp:406-424. */
int upic_fft2d(upic_ctx* ctx, double* re, double* im, int inverse);

/* Pseudo-spectral d/dx (dir 0) or d/dy (dir 1) with the Nyquist wave number
 * zeroed: spectral_derivative, spectral_pic_part3.cpp:440-447. */
int upic_spectral_derivative(upic_ctx* ctx, const double* f, int dir, double* out);

/* IAEM momentum push of the explicit method on the caller's fields
 * (push_particles_momentum_and_velocity, spectral_pic_part3.cpp:1057-1090):
 * for particles at (x, y) -- already advanced, x^{n+1} = x^n + dt v^n
 * (:1050) -- quadratic gathers of A, grad phi and grad A (spectral
 * derivatives of phi and A, nx*ny and 3 x nx*ny), P += q dt (-grad phi +
 * (grad A) . (2 v - v_prev)), v from the canonical momentum
 * (velocity_from_canonical :602), v_prev = the old v.  P, v, v_prev (xyz
 * triples) are updated in place.  Explicit-method contexts; the run state
 * is not touched. */
int upic_push_iaem(upic_ctx* ctx, long np, const double* x, const double* y, double* P, double* v, double* v_prev,
                   const double* q, const double* m, const double* phi, const double* A);

/* phi = Poisson(rho), zero-mean: solve_initial_phi_from_poisson,
 * spectral_pic_part3.cpp:819-827. */
int upic_poisson(upic_ctx* ctx, const double* rho, double* phi);

/* One BDF Helmholtz solve (solve_bdf_wave_scalar, spectral_pic_part3.cpp:829-848):
 * hist holds u^n, u^{n-1}, ... (2 fields for BDF1, 4 for BDF2). */
int upic_solve_bdf(upic_ctx* ctx, const double* source, const double* hist, double* out);

/* Kernel-level orbit integrals of the implicit method (context created with
 * UPIC_METHOD_CN_ORBIT; its grid, spline order, Gauss rule, knot splitting
 * and Nyquist projection apply).  Orbits are x0 + s*dx, s in [0,1], with x0
 * = (x[p], y[p]) and dx, vbar as xyz triples (2D: their z components are not
 * used).
 * J (3 x nx*ny) = sum_p q vbar <S(x0 + s dx)>_s / dV, Nyquist-projected:
 * path_average_deposit_current, Project3/ec_pic_nyquist_projected.cpp:2784. */
int upic_orbit_deposit(upic_ctx* ctx, long np, const double* x, const double* y, const double* dx,
                       const double* vbar, const double* q, double* J);

/* gathered[3p+c] = <mesh_c S>_s and grad[9p+3c+d] = <((1-s) An_c + s Anp1_c)
 * dS/dx_d>_s (d = z column 0 in 2D), mesh/An/Anp1 3 x nx*ny planar:
 * path_average_gather_and_gradient, ec_pic_nyquist_projected.cpp:3016. */
int upic_orbit_gather(upic_ctx* ctx, long np, const double* x, const double* y, const double* dx,
                      const double* mesh, const double* An, const double* Anp1, double* gathered,
                      double* grad);

/* One GM-HC-CN particle push of the implicit method (CN_ORBIT context: its
 * grid, spline order, Gauss rule, knot splitting, local tolerances and dt)
 * in the caller's fields: per particle the damped local fixed point on the
 * orbit velocity, each iterate through the kick-rotate-kick map with the
 * orbit averages of grad phi_mid and of D_A (solve_local_particle_substep,
 * Project3/ec_pic_nyquist_projected.cpp:4930; evaluate_local_particle_substep
 * :4843 with h = dt, theta0 = 0, theta1 = 1).  grad_phi_mid: 2 x nx*ny (x, y
 * derivatives of phi at the mid level); An, Anp1: 3 x nx*ny (A^n, A^{n+1}).
 * Per particle: x, y in [-L/2, L/2), P (canonical momentum) and v (the
 * first guess) as xyz triples, q, m.  Out: the end position x1, y1, P_end
 * and v_end (triples) and the accepted orbit velocity vbar (triple), NaN
 * where the local solve failed; report[2p] = local iterations,
 * report[2p+1] = 0 or the failure reason (1 non-finite map, 2 superluminal
 * map, 3 non-finite iterate, 4 superluminal iterate, 5 maximum iterations,
 * 6 too many knot crossings).  The context's run state is not touched. */
int upic_push_gmhc(upic_ctx* ctx, long np, const double* x, const double* y, const double* P, const double* v,
                   const double* q, const double* m, const double* grad_phi_mid, const double* An,
                   const double* Anp1, double* x1, double* y1, double* P_end, double* v_end, double* vbar,
                   int* report);

/* The field half of one implicit map evaluation (CN_ORBIT context) on the
 * caller's fields (nx*ny each, vectors 3 x nx*ny): the current J projected
 * onto the Nyquist-free modes when the context projects, the continuity
 * update rho1 = rho - dt div J (zero mean, projected;
 * continuity_charge_update :3288), the Crank-Nicolson step of (phi, psi)
 * with the mid-level charge and of (A, U) with J (cn_potential_update
 * :3249 through cn_fft_wave_step_from_spectra :3131; phi1 and psi1 with
 * zero mean), and optionally grad_phi_mid = (grad phi + grad phi1) / 2
 * (2 x nx*ny; :5278-5285).  The context's run state is not touched. */
int upic_fft_solve_cn(upic_ctx* ctx, const double* phi, const double* psi, const double* rho, const double* A,
                      const double* U, const double* J, double* phi1, double* psi1, double* rho1, double* A1,
                      double* U1, double* grad_phi_mid);

/* Ensembles of independent runs (no counterpart in the reference, whose
 * runs are one process each).  Each run is a context
 * created, loaded and started as usual (upic_create, upic_set_particles,
 * upic_init_fields) with its own grid, particle count, tiling and re-sort
 * interval; upic_ensemble_step advances every run by nsteps with the same
 * result as upic_step(run, nsteps, 0, NULL) on each, but records `period`
 * steps of all runs (period: the least common multiple of 5 and twice every
 * run's sort_interval, upic_ensemble_period) into one CUDA graph, each run's
 * kernels on its own stream, and replays it: one launch advances all runs
 * by `period` steps.  Steps beyond a multiple of the period run with
 * ordinary launches.  No diagnostics rows are produced (call upic_step on a
 * run for those).  The runs stay owned by the caller, must outlive the
 * ensemble and must not be used by other calls while upic_ensemble_step
 * runs; the call returns when every run's work is complete.  Calls on a run
 * between ensemble steps are allowed (stepping it, or reloading or
 * restarting it with upic_set_particles, upic_init_fields, upic_load_state,
 * upic_set_stream or upic_set_background): the next ensemble step records a
 * new graph whenever the recorded one no longer matches a run's state.  Errors are reported on the first run's context
 * (upic_last_error(runs[0])), or on NULL for upic_ensemble_create.
 * An ensemble of implicit-method runs (all CN_ORBIT or CN_ORBIT_NONREL;
 * methods of the two kinds cannot be mixed) cannot be recorded, since each
 * step's iteration count is decided on the host: upic_ensemble_step then
 * advances every run with upic_step_implicit(run, nsteps, NULL, NULL, NULL)
 * on a pool of host threads, each run on its own stream, and the period is
 * 1. */
typedef struct upic_ensemble upic_ensemble;
int upic_ensemble_create(upic_ctx* const* runs, int nruns, upic_ensemble** ens);
int upic_ensemble_period(const upic_ensemble* ens, int* period);
int upic_ensemble_step(upic_ensemble* ens, int nsteps);
int upic_ensemble_destroy(upic_ensemble* ens);

/* Kernel-level pieces of the learned predictor's network (any context; no
 * counterpart in the reference).  Activations are nx*ny x 32 bf16 (raw
 * uint16 bits), pixel p = ix*ny + iy; w is 32 x 288 bf16, row = output
 * channel, column = tap*32 + input channel, tap = (dx+1)*3 + (dy+1).
 * upic_guess_conv: out[p][n] = sum_{t,c} x[wrap(p + sign*d_t)][c] w[n][t*32+c]
 * (+ bias[n] when bias != NULL) on the tensor cores; mode 0: ReLU, bf16 out
 * (nx*ny x 32 uint16); 1: linear, fp32 out (nx*ny x 32 float); 2: times
 * (mask[p][n] > 0), bf16 out.  sign is +1 or -1.
 * upic_guess_wgrad: grad[n*288 + t*32 + c] = sum_p dz[p][n] x[wrap(p + d_t)][c]
 * and grad[9216 + n] = sum_p dz[p][n] (fp32, 9248 floats). */
int upic_guess_conv(upic_ctx* ctx, int nx, int ny, const uint16_t* x, const uint16_t* w, const float* bias,
                    const uint16_t* mask, int mode, int sign, void* out);
int upic_guess_wgrad(upic_ctx* ctx, int nx, int ny, const uint16_t* dz, const uint16_t* x, float* grad);

/* Largest grid (nx*ny nodes) upic_deposit_current_noalloc accepts: its
 * scratch is a fixed 6*UPIC_NOALLOC_MAX_NODES+3 uint64 array (3 MiB). */
#define UPIC_NOALLOC_MAX_NODES 65536

/* Current deposit that allocates nothing -- no counterpart in the reference.
 * Same result as upic_deposit_current (J = sum_p q v S(x_p)/dA, quadratic
 * B-spline, x in [0,Lx)), for callers that may not call cudaMalloc: hosts
 * that reserve all device memory up front through their own allocator, or
 * loops that cannot risk the device synchronization an allocation may
 * cause.  x, y (np), v (3*np xyz triples), q (np) and J (3*nx*ny) are DEVICE
 * pointers owned by the caller; work is queued on `stream` (a cudaStream_t,
 * NULL = default stream), and the call returns once that work has finished
 * (it reads back one status word), so J is complete on return.
 * Scratch lives in one fixed __device__ array per GPU (3 MiB, held by every
 * GPU that loads the library until exit).  The first call on a device
 * resolves that array's device address and keeps it for the life of the
 * process, so make the first call on each device before any stream capture,
 * and do not call it again after a cudaDeviceReset of that device.  Every
 * call uses the same array and clears it first: calls that overlap on the
 * GPU (different streams, or host threads sharing a device) race and must
 * be serialized by the caller.
 * Returns UPIC_ERR_TOO_LARGE when nx*ny > UPIC_NOALLOC_MAX_NODES,
 * UPIC_ERR_NONFINITE (with J set to NaN) when a position, velocity or charge
 * is not finite, and UPIC_ERR_CUDA, without launching, when a CUDA error
 * from the caller's earlier work is pending (that error is left in place). */
int upic_deposit_current_noalloc(int nx, int ny, double Lx, double Ly, long np, const double* x,
                                 const double* y, const double* v, const double* q, double* J,
                                 void* stream);

/* ---- Project3's cold-instability initial states (2D, nz = 1) ------------
 * initialize_two_stream_3d_linear_x (Project3/ec_pic_nyquist_projected.cpp
 * :3689) and initialize_weibel_filamentation_3d (:3961): two cold electron
 * streams at +-v0 along x on the same quiet-start positions (cell-centred,
 * particles_per_cell_pair per cell along x), seeded with the growing
 * cold-fluid eigenmode (the Config keys of the same names, defaults as the
 * reference's Config).  upic_p3_initial_state fills x, y (in [-L/2, L/2)),
 * v (xyz triples), q, m (upic_p3_case_particles entries) and the initial
 * A, U (3 x nx*ny each; zero for the two-stream case), and the cold-fluid
 * growth rate of the seeded mode (cold_two_stream_growth_rate :4160,
 * cold_weibel_growth_rate :4197) when growth_rate is not NULL.  Host code;
 * the arrays are the reference's bit for bit.  Start a run from them with
 * upic_set_particles (P and v_prev are recomputed), upic_set_initial_potential
 * and upic_init_fields.  UPIC_P3_LANDAU is Project3's retained Landau
 * example (initialize_landau_damping_1d3d :3853): particles_per_cell_pair
 * quiet-start velocities (thermal_velocity times Acklam's inverse normal
 * CDF at (j + 1/2)/nv) along x at every cell centre, charges q0 (1 + alpha
 * cos(k x)) with alpha = landau_alpha (perturbation when negative), A = U
 * = 0, growth rate 0; UPIC_ERR_CONFIG for fewer than 2 velocities or
 * |alpha| >= 1. */
enum { UPIC_P3_TWO_STREAM = 0, UPIC_P3_WEIBEL = 1, UPIC_P3_LANDAU = 2 };
typedef struct upic_p3_case {
    int kind;                       /* UPIC_P3_TWO_STREAM or UPIC_P3_WEIBEL */
    int nx, ny;
    double Lx, Ly, Lz;
    double kappa, sigma1, n0;
    int spline_order;
    int perturbation_mode;          /* mode along x (two-stream) or y (Weibel) */
    int particles_per_cell_pair;
    double v0;                      /* stream speed, |v0| < kappa */
    double perturbation;            /* legacy two-stream velocity seed; Weibel B0 when weibel_B0 < 0 */
    double two_stream_density_alpha;/* density eigenmode amplitude; < 0: legacy velocity seed */
    int two_stream_eigenmode;
    int two_stream_finite_grid_theory;
    double tsi_transverse_seed;     /* common v_x seed amplitude along y */
    int tsi_transverse_mode;
    double weibel_B0;               /* B_z seed amplitude; < 0: perturbation */
    int weibel_eigenmode;
    int weibel_finite_grid_theory;
    double landau_alpha;            /* Landau density amplitude; < 0: perturbation */
    double thermal_velocity;        /* Landau Maxwellian thermal speed */
} upic_p3_case;
int upic_p3_case_default(upic_p3_case* c);
long upic_p3_case_particles(const upic_p3_case* c);
int upic_p3_initial_state(const upic_p3_case* c, long capacity, double* x, double* y, double* v, double* q,
                          double* m, double* A, double* U, double* growth_rate);

/* Initial vector potential A and its time derivative U (3 x nx*ny each,
 * host arrays, reference index order) for the next upic_init_fields of an
 * implicit-method context, which then uses them instead of A = U = 0: they
 * are Nyquist-projected with the rest of the start state, the canonical
 * momenta become P = m gamma v + q A(x), and the history velocities see
 * E = -grad phi - U and B = curl A (project_initial_state :3398,
 * initialize_relativistic_history_velocity :3423).  NULL, NULL clears them.
 * UPIC_ERR_STATE for explicit methods. */
int upic_set_initial_potential(upic_ctx* ctx, const double* A, const double* U);

/* Seeded synthetic plasma generator (splitmix64 + Box-Muller, independent of
 * any C++ library's distributions): np_per_cell electrons per cell at uniform
 * random positions in [0,Lx)x[0,Ly) with a drifting bi-Maxwellian in
 * normalized momentum u = gamma v / c (thermal spreads uth[3], drift
 * udrift[3]); P = m gamma v, v_prev = v, q = -n0*Lx*Ly/Np, m = |q|.
 * Deterministic for a given seed, independent of thread count. */
int upic_generate_bimaxwellian(int nx, int ny, double Lx, double Ly, int np_per_cell,
                               double c, double n0, const double* uth, const double* udrift,
                               uint64_t seed, double* x, double* y, double* P, double* v,
                               double* v_prev, double* q, double* m);

#ifdef __cplusplus
}
#endif
#endif /* UPIC_H */
