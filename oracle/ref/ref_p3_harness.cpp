// Test infrastructure only: a C-ABI harness around the reference's implicit
// energy-conserving GM-HC-CN solver (Project3/ec_pic_nyquist_projected.cpp).
//
// Same pattern as the reference's own regression harness
// (Project3/tests/test_solver.cpp:3-5): the solver translation unit is
// included with `main` renamed, and the `static` functions run unmodified on
// injected particles and fields.  Built by oracle/Makefile into
// oracle/_ref/libref_p3.so (serial: no -fopenmp).

#include <new>

#define main upic_ref_p3_cli_main
#include "ec_pic_nyquist_projected.cpp"
#undef main

#include <chrono>
#include <cstring>

namespace {

// dparams / iparams layout shared with oracle/p3_oracle.c and the tests.
enum {
    D_LX, D_LY, D_LZ, D_DT, D_KAPPA, D_SIGMA1, D_SIGMA2, D_N0, D_NL_RTOL, D_NL_ATOL,
    D_AND_DAMP, D_AND_REG, D_AND_GROWTH, D_LOC_RTOL, D_LOC_ATOL, D_LOC_DAMP, D_COUNT
};
enum {
    I_NX, I_NY, I_NZ, I_ORDER, I_NQ, I_SPLIT, I_NYQ, I_NL_MAXIT, I_AND_MEM, I_AND_START,
    I_LOC_MAXIT, I_SOLVER, I_NSTEPS, I_MODE, I_COUNT
};
constexpr int kDiag = 23;
// selective particle sub-cycling fallback of the next ref_p3_run
// (ref_p3_set_fallback) and its per-step report (ref_p3_selective_info)
bool g_fallback = false;
int g_fallback_max = 64;
std::vector<double> g_selective;  // per step: used, restarts, refined, total substeps

constexpr int kInfo = 8;
constexpr int kStepDiag = 17;

Config make_cfg(const double* d, const int* ip) {
    Config c;
    c.nx = ip[I_NX]; c.ny = ip[I_NY]; c.nz = ip[I_NZ];
    c.Lx = d[D_LX]; c.Ly = d[D_LY]; c.Lz = d[D_LZ];
    c.dt = d[D_DT];
    c.kappa = d[D_KAPPA]; c.sigma1 = d[D_SIGMA1]; c.sigma2 = d[D_SIGMA2];
    c.n0 = d[D_N0];
    c.spline_order = ip[I_ORDER];
    c.orbit_quad_order = ip[I_NQ];
    c.split_orbit_at_knots = ip[I_SPLIT] != 0;
    c.nyquist_projection = ip[I_NYQ] != 0;
    c.nonlinear_solver = ip[I_SOLVER] == 1 ? "picard" : "anderson_quasi_newton";
    c.nonlinear_rtol = d[D_NL_RTOL];
    c.nonlinear_atol = d[D_NL_ATOL];
    c.nonlinear_max_iter = ip[I_NL_MAXIT];
    c.anderson_memory = ip[I_AND_MEM];
    c.anderson_start = ip[I_AND_START];
    c.anderson_damping = d[D_AND_DAMP];
    c.anderson_regularization = d[D_AND_REG];
    c.anderson_growth_limit = d[D_AND_GROWTH];
    c.uniform_local_rtol = d[D_LOC_RTOL];
    c.uniform_local_atol = d[D_LOC_ATOL];
    c.uniform_local_max_iter = ip[I_LOC_MAXIT];
    c.uniform_local_damping = d[D_LOC_DAMP];
    c.uniform_particle_subcycling = false;
    c.selective_particle_fallback = g_fallback;
    c.selective_particle_max_substeps = g_fallback_max;
    c.adaptive_dt = false;
    c.run_unit_tests = false;
    c.output_prefix = "/tmp/upic_ref_p3";
    return c;
}

void store_diag(const Diagnostics& d, double* o) {
    const double v[kDiag] = {d.gauss_rms, d.gauss_max, d.divE_rms, d.sigma1_rho_rms,
                             d.gauss_normalization_rms, d.gauss_relative, d.gauge_rms,
                             d.gauge_max, d.psi_over_kappa2_rms, d.divA_rms,
                             d.gauge_normalization_rms, d.gauge_relative, d.field_energy,
                             d.kinetic_energy, d.total_energy, d.rho_mode, d.E_mode_re,
                             d.E_mode_im, d.E_mode_abs, d.Bz_y_mode_re, d.Bz_y_mode_im,
                             d.Bz_y_mode_abs, d.mean_rho};
    std::memcpy(o, v, sizeof(v));
}

void store_step_diag(const StepDiagnostics& d, double* o) {
    const double v[kStepDiag] = {d.A_chain_abs_rms, d.A_chain_rel_rms, d.A_chain_max_norm,
                                 d.A_chain_mean_norm, d.A_chain_work_defect, d.delta_K, d.delta_W,
                                 d.delta_total_energy, d.particle_work, d.grid_work,
                                 d.deposit_gather_work_residual, d.particle_energy_residual,
                                 d.field_energy_residual, (double)d.crossing_particles,
                                 (double)d.total_crossings, d.average_path_segments,
                                 (double)d.max_path_segments};
    std::memcpy(o, v, sizeof(v));
}

void copy_vec3(const std::vector<Vec3>& a, double* out) {
    for (std::size_t p = 0; p < a.size(); ++p)
        for (int d = 0; d < 3; ++d) out[3 * p + d] = a[p][d];
}

}  // namespace

extern "C" {

// Enable the reference's selective particle sub-cycling fallback
// (nonlinear_step_selective_particle_fallback, :6328) for later runs.
int ref_p3_set_fallback(int enable, int max_substeps) {
    g_fallback = enable != 0;
    g_fallback_max = max_substeps;
    return 0;
}

// Per step of the last ref_p3_run: selective_fallback_used,
// selective_refinement_restarts, selective_refined_particles,
// selective_total_particle_substeps (NonlinearSolveInfo).
int ref_p3_selective_info(double* out, int nsteps) {
    for (int k = 0; k < 4 * nsteps && k < (int)g_selective.size(); ++k) out[k] = g_selective[k];
    return 0;
}

// Gauss-Legendre nodes and weights on [0,1] (gauss_legendre_01, :2479).
int ref_p3_gauss_legendre(int n, double* s, double* w) {
    Quadrature q = gauss_legendre_01(n);
    for (int i = 0; i < n; ++i) { s[i] = q.s[i]; w[i] = q.w[i]; }
    return 0;
}

// Orbit-averaged current deposit (path_average_deposit_current, :2784).
int ref_p3_orbit_deposit(const double* d, const int* ip, long np, const double* x0,
                         const double* dx, const double* vbar, const double* q, double* J) {
    Config c = make_cfg(d, ip);
    Grid g = make_grid(c);
    Quadrature quad = gauss_legendre_01(c.orbit_quad_order);
    std::vector<Vec3> X(np), DX(np), V(np);
    std::vector<Real> Q(q, q + np);
    for (long p = 0; p < np; ++p)
        for (int k = 0; k < 3; ++k) {
            X[p][k] = x0[3 * p + k];
            DX[p][k] = dx[3 * p + k];
            V[p][k] = vbar[3 * p + k];
        }
    VecField Jf = path_average_deposit_current(X, DX, V, Q, g, c.spline_order, quad,
                                               c.split_orbit_at_knots, nullptr);
    for (int k = 0; k < 3; ++k) std::memcpy(J + (std::size_t)k * g.N, Jf[k].data(), sizeof(double) * g.N);
    return 0;
}

// Fused orbit gather + D_A (path_average_gather_and_gradient, :3016):
// gathered (3 per particle) and gradient (9 per particle, [comp][dir]).
int ref_p3_orbit_gather(const double* d, const int* ip, long np, const double* x0,
                        const double* dx, const double* mesh, const double* An,
                        const double* Anp1, double* gathered, double* grad) {
    Config c = make_cfg(d, ip);
    Grid g = make_grid(c);
    Quadrature quad = gauss_legendre_01(c.orbit_quad_order);
    std::vector<Vec3> X(np), DX(np);
    for (long p = 0; p < np; ++p)
        for (int k = 0; k < 3; ++k) {
            X[p][k] = x0[3 * p + k];
            DX[p][k] = dx[3 * p + k];
        }
    VecField M, A0, A1;
    for (int k = 0; k < 3; ++k) {
        M[k].assign(mesh + (std::size_t)k * g.N, mesh + (std::size_t)(k + 1) * g.N);
        A0[k].assign(An + (std::size_t)k * g.N, An + (std::size_t)(k + 1) * g.N);
        A1[k].assign(Anp1 + (std::size_t)k * g.N, Anp1 + (std::size_t)(k + 1) * g.N);
    }
    OrbitGatherGradient o = path_average_gather_and_gradient(X, DX, M, A0, A1, g, c.spline_order,
                                                             quad, c.split_orbit_at_knots);
    for (long p = 0; p < np; ++p) {
        for (int k = 0; k < 3; ++k) gathered[3 * p + k] = o.gathered[p][k];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) grad[9 * p + 3 * a + b] = o.gradient[p][a][b];
    }
    return 0;
}

// One GM-HC local particle solve per particle (solve_local_particle_substep
// :4930 with h = dt, theta0 = 0, theta1 = 1) in the given fields:
// grad_phi_mid 3 x N, An (st.A) and Anp1 (A_end) 3 x N.  x0, P0, v (first
// guess): 3*np; out: x1, P_end, v_end, vbar 3*np each (NaN on failure),
// report: iterations, failure reason (LocalParticleFailureReason) per
// particle.
int ref_p3_push_gmhc(const double* d, const int* ip, long np, const double* x0, const double* P0,
                     const double* v, const double* q, const double* m, const double* gpm, const double* An,
                     const double* Anp1, double* x1, double* P_end, double* v_end, double* vbar, int* report) {
    Config c = make_cfg(d, ip);
    Grid g = make_grid(c);
    Quadrature quad = gauss_legendre_01(c.orbit_quad_order);
    State st;
    VecField Ae, G;
    for (int k = 0; k < 3; ++k) {
        st.A[k].assign(An + (std::size_t)k * g.N, An + (std::size_t)(k + 1) * g.N);
        Ae[k].assign(Anp1 + (std::size_t)k * g.N, Anp1 + (std::size_t)(k + 1) * g.N);
        G[k].assign(gpm + (std::size_t)k * g.N, gpm + (std::size_t)(k + 1) * g.N);
    }
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (long p = 0; p < np; ++p) {
        const Vec3 X{x0[3 * p], x0[3 * p + 1], x0[3 * p + 2]};
        const Vec3 P{P0[3 * p], P0[3 * p + 1], P0[3 * p + 2]};
        const Vec3 V{v[3 * p], v[3 * p + 1], v[3 * p + 2]};
        Vec3 vb{0.0, 0.0, 0.0};
        LocalParticleStep mapped;
        LocalParticleSolveReport rep;
        const bool ok = solve_local_particle_substep(V, X, P, q[p], m[p], c.dt, 0.0, 1.0, st, Ae, G, g, c, quad,
                                                     vb, mapped, rep);
        const Vec3 xe = wrap_pos(add3(X, mul3(c.dt, vb)), g.L);
        for (int k = 0; k < 3; ++k) {
            x1[3 * p + k] = ok ? xe[k] : nan;
            P_end[3 * p + k] = ok ? mapped.P_end[k] : nan;
            v_end[3 * p + k] = ok ? mapped.v_end[k] : nan;
            vbar[3 * p + k] = ok ? vb[k] : nan;
        }
        report[2 * p] = rep.iterations;
        report[2 * p + 1] = (int)rep.failure_reason;
    }
    return 0;
}

// The field half of a map evaluation (:5265-5285) on the given fields:
// J_field projected, rho_end (continuity_charge_update :3288), rho_mid,
// cn_potential_update (:3249) from the state's spectra, grad_phi_mid.
// in: phi, psi, rho (N each), A, U, J (3N each); out: phi1, psi1, rho1
// (N), A1, U1 (3N), gpm (3N, z zero).
int ref_p3_fft_solve_cn(const double* d, const int* ip, const double* phi, const double* psi, const double* rho,
                        const double* A, const double* U, const double* J, double* phi1, double* psi1,
                        double* rho1, double* A1, double* U1, double* gpm) {
    Config c = make_cfg(d, ip);
    Grid g = make_grid(c);
    State st;
    st.phi.assign(phi, phi + g.N);
    st.psi.assign(psi, psi + g.N);
    st.rho.assign(rho, rho + g.N);
    VecField Jf;
    for (int k = 0; k < 3; ++k) {
        st.A[k].assign(A + (std::size_t)k * g.N, A + (std::size_t)(k + 1) * g.N);
        st.U[k].assign(U + (std::size_t)k * g.N, U + (std::size_t)(k + 1) * g.N);
        Jf[k].assign(J + (std::size_t)k * g.N, J + (std::size_t)(k + 1) * g.N);
    }
    const WaveSpectralState cache = make_wave_spectral_state(st.phi, st.psi, st.A, st.U, g);
    const VecField grad_phi_n = spectral_gradient_scalar(st.phi, g);
    project_nyquist(Jf, g);
    const Field rho_end = continuity_charge_update(st.rho, Jf, c.dt, g);
    Field rho_mid(g.N);
    for (int id = 0; id < g.N; ++id) rho_mid[id] = 0.5 * (st.rho[id] + rho_end[id]);
    Field phi_end, psi_end;
    VecField A_end, U_end;
    cn_potential_update(st, rho_mid, Jf, c.dt, g, c.kappa, c.sigma1, c.sigma2, phi_end, psi_end, A_end, U_end,
                        &cache);
    const VecField grad_phi_end = spectral_gradient_scalar(phi_end, g);
    std::memcpy(phi1, phi_end.data(), sizeof(double) * g.N);
    std::memcpy(psi1, psi_end.data(), sizeof(double) * g.N);
    std::memcpy(rho1, rho_end.data(), sizeof(double) * g.N);
    for (int k = 0; k < 3; ++k) {
        std::memcpy(A1 + (std::size_t)k * g.N, A_end[k].data(), sizeof(double) * g.N);
        std::memcpy(U1 + (std::size_t)k * g.N, U_end[k].data(), sizeof(double) * g.N);
        for (int id = 0; id < g.N; ++id)
            gpm[(std::size_t)k * g.N + id] = 0.5 * (grad_phi_n[k][id] + grad_phi_end[k][id]);
    }
    return 0;
}

// Config of an instability case: case_d = {v0, perturbation,
// two_stream_density_alpha, tsi_transverse_seed, weibel_B0}, case_i = {kind
// (0 two-stream, 1 Weibel), particles_per_cell_pair, two_stream_eigenmode,
// two_stream_finite_grid_theory, tsi_transverse_mode, weibel_eigenmode,
// weibel_finite_grid_theory}; the mode is iparams' I_MODE.
Config make_case_cfg(const double* d, const int* ip, const double* cd, const int* ci) {
    Config c = make_cfg(d, ip);
    c.test_case = ci[0] == 2 ? "landau" : (ci[0] == 1 ? "cold_relativistic_weibel" : "cold_relativistic_two_stream");
    c.perturbation_mode = ip[I_MODE];
    c.particles_per_cell_pair = ci[1];
    c.two_stream_eigenmode = ci[2] != 0;
    c.two_stream_finite_grid_theory = ci[3] != 0;
    c.tsi_transverse_mode = ci[4];
    c.weibel_eigenmode = ci[5] != 0;
    c.weibel_finite_grid_theory = ci[6] != 0;
    c.v0 = cd[0];
    c.perturbation = cd[1];
    c.two_stream_density_alpha = cd[2];
    c.tsi_transverse_seed = cd[3];
    c.weibel_B0 = cd[4];
    c.landau_alpha = cd[5];
    c.thermal_velocity = cd[6];
    return c;
}

// Injected start-up state (the tail of initialize_weibel_filamentation_3d,
// :4061-4123, with the caller's particles, A = U = 0) followed by n_steps of
// nonlinear_step_orbit (:6477) and compute_diagnostics (:3521) per step.
//   x, v: 3*np in/out (positions in [-L/2, L/2)); P, v_prev, vbar: 3*np out
//   diag: (n_steps+1) x 22; info: n_steps x 8 {iterations, converged,
//   final_rms_residual, final_max_particle_residual, local_iter_max,
//   local_iter_mean, anderson_steps, picard_steps}; fields (optional): phi,
//   psi, rho, A(3), U(3), J(3) = 12 x N after the last step; step_diag
//   (optional): n_steps x 17, compute_step_diagnostics (:4501) of each step
//   as the run loop calls it (:8835), StepDiagnostics members in the column
//   order of _step_diagnostics.csv (:8462-8473).
int ref_p3_run(const double* d, const int* ip, long np, double* x, double* v, double* P,
               double* v_prev, double* vbar, const double* q, const double* m, double* diag,
               double* info, double* fields, double* seconds, double* step_diag) {
    try {
        Config c = make_cfg(d, ip);
        Grid g = make_grid(c);
        Quadrature quad = gauss_legendre_01(c.orbit_quad_order);
        State st;
        st.x.resize(np); st.v.resize(np); st.v_prev.resize(np); st.vbar_last.resize(np);
        st.P.resize(np); st.q.assign(q, q + np); st.m.assign(m, m + np);
        for (long p = 0; p < np; ++p)
            for (int k = 0; k < 3; ++k) {
                st.x[p][k] = x[3 * p + k];
                st.v[p][k] = v[3 * p + k];
            }
        for (auto& xx : st.x) xx = wrap_pos(xx, g.L);
        Field rho_e = deposit_scalar_to_mesh(st.x, st.q, g, c.spline_order, true);
        st.rho.assign(g.N, 0.0);
        for (int id = 0; id < g.N; ++id) st.rho[id] = rho_e[id] + c.n0;
        subtract_mean(st.rho);
        st.phi = solve_periodic_poisson_for_phi(st.rho, g, c.sigma1);
        st.psi.assign(g.N, 0.0);
        st.A = zero_vecfield(g.N);
        st.U = zero_vecfield(g.N);
        st.J = deposit_current_to_mesh(st.x, st.v, st.q, g, c.spline_order);
        for (long p = 0; p < np; ++p) {
            const Vec3 pm = momentum_from_v(st.v[p], st.m[p], c.kappa);
            const Vec3 A0p = gather_vector_at(st.A, st.x[p], g, c.spline_order);
            st.P[p] = add3(pm, mul3(st.q[p], A0p));
        }
        project_initial_state(st, g, c);
        initialize_relativistic_history_velocity(st, g, c);
        const int mode = ip[I_MODE];
        if (diag) store_diag(compute_diagnostics(st, g, c.sigma1, c.sigma2, c.kappa, mode), diag);
        const auto t0 = std::chrono::steady_clock::now();
        g_selective.assign(4 * (std::size_t)std::max(ip[I_NSTEPS], 0), 0.0);
        for (int s = 1; s <= ip[I_NSTEPS]; ++s) {
            std::vector<NonlinearHistoryEntry> hist;
            NonlinearSolveInfo si;
            const State s0 = step_diag ? st : State{};
            st = nonlinear_step_orbit(st, g, c, quad, hist, &si, (s - 1) * c.dt);
            if (step_diag)
                store_step_diag(compute_step_diagnostics(s0, st, g, c.dt, c.spline_order, quad, c.sigma1,
                                                         c.sigma2, c.kappa, c.split_orbit_at_knots),
                                step_diag + (std::size_t)kStepDiag * (s - 1));
            if (diag) store_diag(compute_diagnostics(st, g, c.sigma1, c.sigma2, c.kappa, mode),
                                 diag + (std::size_t)kDiag * s);
            if (info) {
                double* o = info + (std::size_t)kInfo * (s - 1);
                o[0] = si.iterations; o[1] = si.converged; o[2] = si.final_rms_residual;
                o[3] = si.final_max_particle_residual; o[4] = si.local_particle_iterations_max;
                o[5] = si.local_particle_iterations_mean; o[6] = si.anderson_steps;
                o[7] = si.picard_fallback_steps;
            }
            double* sl = g_selective.data() + 4 * (std::size_t)(s - 1);
            sl[0] = si.selective_fallback_used ? 1.0 : 0.0;
            sl[1] = si.selective_refinement_restarts;
            sl[2] = (double)si.selective_refined_particles;
            sl[3] = (double)si.selective_total_particle_substeps;
        }
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        copy_vec3(st.x, x);
        copy_vec3(st.v, v);
        copy_vec3(st.P, P);
        copy_vec3(st.v_prev, v_prev);
        copy_vec3(st.vbar_last, vbar);
        if (fields) {
            const Field* f[12] = {&st.phi, &st.psi, &st.rho, &st.A[0], &st.A[1], &st.A[2],
                                  &st.U[0], &st.U[1], &st.U[2], &st.J[0], &st.J[1], &st.J[2]};
            for (int k = 0; k < 12; ++k)
                std::memcpy(fields + (std::size_t)k * g.N, f[k]->data(), sizeof(double) * g.N);
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_p3_run: %s\n", e.what());
        return -1;
    }
}

// The reference's own start state of an instability case (initialize_state
// :4125, after project_initial_state and the history velocities): x, v, P,
// v_prev (3*np), q, m (np), A, U (3 x N), growth (1): the case's cold-fluid
// rate (selected_theory_growth_rate).  Returns np, or -1 (error, message on
// stderr) or -2 (cap too small).
long ref_p3_case_state(const double* d, const int* ip, const double* cd, const int* ci, long cap, double* x,
                       double* v, double* P, double* v_prev, double* q, double* m, double* A, double* U,
                       double* growth) {
    try {
        Config c = make_case_cfg(d, ip, cd, ci);
        Grid g = make_grid(c);
        State st = initialize_state(c, g);
        const long np = (long)st.x.size();
        if (np > cap) return -2;
        copy_vec3(st.x, x);
        copy_vec3(st.v, v);
        copy_vec3(st.P, P);
        copy_vec3(st.v_prev, v_prev);
        std::memcpy(q, st.q.data(), sizeof(double) * np);
        std::memcpy(m, st.m.data(), sizeof(double) * np);
        for (int k = 0; k < 3; ++k) {
            std::memcpy(A + (std::size_t)k * g.N, st.A[k].data(), sizeof(double) * g.N);
            std::memcpy(U + (std::size_t)k * g.N, st.U[k].data(), sizeof(double) * g.N);
        }
        if (growth) *growth = selected_theory_growth_rate(c, g);
        return np;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_p3_case_state: %s\n", e.what());
        return -1;
    }
}

// An instability case run from the reference's own start state: n_steps of
// nonlinear_step_orbit (:6477) with compute_diagnostics (:3521) per step;
// diag (n_steps+1) x 23, info n_steps x 8, fields 12 x N after the last step
// (the layouts of ref_p3_run).
int ref_p3_case_run(const double* d, const int* ip, const double* cd, const int* ci, double* diag, double* info,
                    double* fields, double* seconds) {
    try {
        Config c = make_case_cfg(d, ip, cd, ci);
        Grid g = make_grid(c);
        Quadrature quad = gauss_legendre_01(c.orbit_quad_order);
        State st = initialize_state(c, g);
        const int mode = ip[I_MODE];
        if (diag) store_diag(compute_diagnostics(st, g, c.sigma1, c.sigma2, c.kappa, mode), diag);
        const auto t0 = std::chrono::steady_clock::now();
        for (int s = 1; s <= ip[I_NSTEPS]; ++s) {
            std::vector<NonlinearHistoryEntry> hist;
            NonlinearSolveInfo si;
            st = nonlinear_step_orbit(st, g, c, quad, hist, &si, (s - 1) * c.dt);
            if (diag) store_diag(compute_diagnostics(st, g, c.sigma1, c.sigma2, c.kappa, mode),
                                 diag + (std::size_t)kDiag * s);
            if (info) {
                double* o = info + (std::size_t)kInfo * (s - 1);
                o[0] = si.iterations; o[1] = si.converged; o[2] = si.final_rms_residual;
                o[3] = si.final_max_particle_residual; o[4] = si.local_particle_iterations_max;
                o[5] = si.local_particle_iterations_mean; o[6] = si.anderson_steps;
                o[7] = si.picard_fallback_steps;
            }
        }
        if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (fields) {
            const Field* f[12] = {&st.phi, &st.psi, &st.rho, &st.A[0], &st.A[1], &st.A[2],
                                  &st.U[0], &st.U[1], &st.U[2], &st.J[0], &st.J[1], &st.J[2]};
            for (int k = 0; k < 12; ++k)
                std::memcpy(fields + (std::size_t)k * g.N, f[k]->data(), sizeof(double) * g.N);
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_p3_case_run: %s\n", e.what());
        return -1;
    }
}

// The reference's own command-line program on a deck file (main :8336):
// returns its exit code; output files go where the deck's output_prefix says.
int ref_p3_run_deck(const char* deck) {
    char prog[] = "ec_pic_nyquist_projected";
    std::string d(deck);
    std::vector<char> arg(d.begin(), d.end());
    arg.push_back('\0');
    char* argv[] = {prog, arg.data(), nullptr};
    return upic_ref_p3_cli_main(2, argv);
}

}  // extern "C"
