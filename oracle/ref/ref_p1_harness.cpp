// Test infrastructure only: a C-ABI harness around the reference's
// non-relativistic implicit orbit-averaged Picard solver
// (Project1/ec_pic_serial_demo.cpp).  The solver translation unit is included
// with `main` renamed (the pattern of Project3/tests/test_solver.cpp:3-5) and
// its `static` functions run unmodified.  Built by oracle/Makefile into
// oracle/_ref/libref_p1.so.

#include <new>

#define main upic_ref_p1_cli_main
#include "ec_pic_serial_demo.cpp"
#undef main

#include <chrono>
#include <cstring>

namespace {

// dparams / iparams layout shared with the tests (oracle_lib.P1Problem).
enum {
    D_LX, D_LY, D_LZ, D_DT, D_C, D_EPS0, D_MU0, D_N0, D_PICARD_TOL, D_V0, D_PERT, D_LANDAU_ALPHA,
    D_VTH, D_COUNT
};
enum {
    I_NX, I_NY, I_NZ, I_ORDER, I_NQ, I_SPLIT, I_PICARD_MAXIT, I_SWEEP, I_NSTEPS, I_MODE, I_PPC, I_CASE,
    I_COUNT
};
constexpr int kDiag = 11;
constexpr int kInfo = 6;
constexpr int kStepDiag = 17;

Config make_cfg(const double* d, const int* ip) {
    Config c;
    c.nx = ip[I_NX]; c.ny = ip[I_NY]; c.nz = ip[I_NZ];
    c.Lx = d[D_LX]; c.Ly = d[D_LY]; c.Lz = d[D_LZ];
    c.dt = d[D_DT];
    c.c = d[D_C]; c.eps0 = d[D_EPS0]; c.mu0 = d[D_MU0]; c.n0 = d[D_N0];
    c.spline_order = ip[I_ORDER];
    c.orbit_quad_order = ip[I_NQ];
    c.split_orbit_at_knots = ip[I_SPLIT] != 0;
    c.picard_tol = d[D_PICARD_TOL];
    c.picard_max_iter = ip[I_PICARD_MAXIT];
    c.final_consistency_sweep = ip[I_SWEEP] != 0;
    c.n_steps = ip[I_NSTEPS];
    c.perturbation_mode = ip[I_MODE];
    c.particles_per_cell_pair = ip[I_PPC];
    c.test_case = ip[I_CASE] == 1 ? "landau_weak" : "two_stream";
    c.v0 = d[D_V0];
    c.perturbation = d[D_PERT];
    c.landau_alpha = d[D_LANDAU_ALPHA];
    c.thermal_velocity = d[D_VTH];
    c.run_unit_tests = false;
    return c;
}

void store_diag(const Diagnostics& d, double* o) {
    const double v[kDiag] = {d.gauss_rms, d.gauss_max, d.gauge_rms, d.field_energy, d.kinetic_energy,
                             d.total_energy, d.rho_mode, d.E_mode_re, d.E_mode_im, d.E_mode_abs, d.mean_rho};
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

}  // namespace

extern "C" {

// Particles of the reference's own initial condition (initialize_state
// :1306; two_stream :1151 or Landau :1214): x, v as xyz triples, q, m.
// Returns the particle count; arrays must hold `cap` particles.
long ref_p1_init(const double* d, const int* ip, long cap, double* x, double* v, double* q, double* m) {
    try {
        Config c = make_cfg(d, ip);
        Grid g = make_grid(c);
        State st = initialize_state(c, g);
        const long np = (long)st.x.size();
        if (np > cap) return -np;
        for (long p = 0; p < np; ++p) {
            for (int k = 0; k < 3; ++k) {
                x[3 * p + k] = st.x[p][k];
                v[3 * p + k] = st.v[p][k];
            }
            q[p] = st.q[p];
            m[p] = st.m[p];
        }
        return np;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_p1_init: %s\n", e.what());
        return -1;
    }
}

// Injected particles, the start-up of the reference's initializers (the
// common tail of :1188-1211 and :1283-1303), then n_steps of picard_step_orbit
// (:1509) with compute_diagnostics (:1057), compute_step_diagnostics (:1384)
// and the path statistics of the main loop (:1846-1853) per step.
//   x, v: 3*np in/out; P, v_prev: 3*np out; diag: (n_steps+1) x 11;
//   info: n_steps x 6 {picard iterations, current error, velocity error,
//   crossing particles, avg path segments, max path segments};
//   step_diag: n_steps x 17; fields: phi, psi, rho, A(3), U(3), J(3) = 12 x N.
int ref_p1_run(const double* d, const int* ip, long np, double* x, double* v, double* P, double* v_prev,
               const double* q, const double* m, double* diag, double* info, double* step_diag,
               double* fields, double* seconds) {
    try {
        Config c = make_cfg(d, ip);
        Grid g = make_grid(c);
        Quadrature quad = gauss_legendre_01(c.orbit_quad_order);
        State st;
        st.x.resize(np); st.v.resize(np); st.v_prev.resize(np); st.P.resize(np);
        st.q.assign(q, q + np); st.m.assign(m, m + np);
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
        st.J = deposit_current_to_mesh(st.x, st.v, st.q, g, c.spline_order);
        st.phi = solve_periodic_poisson_for_phi(st.rho, g, c.eps0);
        st.psi.assign(g.N, 0.0);
        st.A = zero_vecfield(g.N);
        st.U = zero_vecfield(g.N);
        for (long p = 0; p < np; ++p) st.P[p] = mul3(st.m[p], st.v[p]);
        {
            State tmp = st;
            const VecField E0 = compute_E(tmp, g);
            const auto E0p = gather_vector_all(st.x, E0, g, c.spline_order);
            for (long p = 0; p < np; ++p) {
                const Vec3 acc = mul3(st.q[p] / st.m[p], E0p[p]);
                st.v_prev[p] = sub3(st.v[p], mul3(c.dt, acc));
            }
        }
        if (diag) store_diag(compute_diagnostics(st, g, c.eps0, c.mu0, c.c, c.perturbation_mode), diag);
        const auto t0 = std::chrono::steady_clock::now();
        for (int n = 0; n < c.n_steps; ++n) {
            State s0 = st;
            std::vector<PicardHistoryEntry> hist;
            st = picard_step_orbit(s0, g, c, quad, hist);
            if (step_diag)
                store_step_diag(compute_step_diagnostics(s0, st, g, c.dt, c.spline_order, quad, c.eps0, c.mu0,
                                                         c.split_orbit_at_knots),
                                step_diag + (std::size_t)kStepDiag * n);
            if (diag)
                store_diag(compute_diagnostics(st, g, c.eps0, c.mu0, c.c, c.perturbation_mode),
                           diag + (std::size_t)kDiag * (n + 1));
            if (info) {
                std::vector<Vec3> dxp(np);
                for (long p = 0; p < np; ++p) dxp[p] = mul3(c.dt, mul3(0.5, add3(st.v[p], s0.v[p])));
                const PathStats ps = compute_path_stats(s0.x, dxp, g, c.spline_order, c.split_orbit_at_knots);
                double* o = info + (std::size_t)kInfo * n;
                o[0] = (double)hist.size();
                o[1] = hist.empty() ? NAN : hist.back().current_error;
                o[2] = hist.empty() ? NAN : hist.back().velocity_error;
                o[3] = (double)ps.crossing_particles;
                o[4] = ps.n_particles ? (double)ps.total_segments / (double)ps.n_particles : 0.0;
                o[5] = (double)ps.max_segments;
            }
        }
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        for (long p = 0; p < np; ++p)
            for (int k = 0; k < 3; ++k) {
                x[3 * p + k] = st.x[p][k];
                v[3 * p + k] = st.v[p][k];
                P[3 * p + k] = st.P[p][k];
                v_prev[3 * p + k] = st.v_prev[p][k];
            }
        if (fields) {
            const Field* f[12] = {&st.phi, &st.psi, &st.rho, &st.A[0], &st.A[1], &st.A[2],
                                  &st.U[0], &st.U[1], &st.U[2], &st.J[0], &st.J[1], &st.J[2]};
            for (int k = 0; k < 12; ++k) std::memcpy(fields + (std::size_t)k * g.N, f[k]->data(), sizeof(double) * g.N);
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_p1_run: %s\n", e.what());
        return -1;
    }
}

// The reference's own command-line program on a deck file (main :1768):
// returns its exit code; output files go where the deck's output_prefix says.
int ref_p1_run_deck(const char* deck) {
    char prog[] = "ec_pic_serial_demo";
    std::string d(deck);
    std::vector<char> arg(d.begin(), d.end());
    arg.push_back('\0');
    char* argv[] = {prog, arg.data(), nullptr};
    return upic_ref_p1_cli_main(2, argv);
}

}  // extern "C"
