// Test infrastructure only: a C-ABI harness around the reference's explicit
// spectral BDF/IAEM solver (Project2/spectral_pic_part3.cpp).
//
// The reference is a single translation unit whose functions are `static`.
// This harness textually includes it with `main` renamed (the pattern of
// Project3/tests/test_solver.cpp:3-5), so the reference's own functions run
// unmodified on injected particle arrays.  Nothing here re-implements the
// reference: every numerical call below is the reference's code.
//
// Built by oracle/Makefile into oracle/_ref/libref_p2.so.  Only tests/,
// __graft_entry__.smoke() and bench.py (CPU baseline / reference arm) load it.

#define main upic_ref_p2_cli_main
#include "spectral_pic_part3.cpp"
#undef main

#include <chrono>
#include <cstring>

namespace {

struct HarnessCfg {
    Config cfg;
    Grid g;
};

// Build a reference Config/Grid from plain scalars (weibel example semantics:
// uniform fixed ion background n0, quadratic shape, BDF1/BDF2).
HarnessCfg make_cfg(int nx, int ny, double Lx, double Ly, double dt, int bdf_order,
                    int conserving, double c, double eps0, double mu0, double n0) {
    HarnessCfg h;
    h.cfg.nx = nx;
    h.cfg.ny = ny;
    h.cfg.Lx = Lx;
    h.cfg.Ly = Ly;
    h.cfg.dt = dt;
    h.cfg.method = bdf_order == 2 ? "bdf2" : "bdf1";
    h.cfg.charge_update = conserving ? "conserving" : "naive";
    h.cfg.c = c;
    h.cfg.eps0 = eps0;
    h.cfg.mu0 = mu0;
    h.cfg.n0 = n0;
    h.cfg.run_unit_tests = false;
    h.g = make_grid(h.cfg);
    return h;
}

void load_particles(std::vector<Particle>& out, long np, const double* x, const double* y,
                    const double* P, const double* v, const double* vprev,
                    const double* q, const double* m) {
    out.resize(static_cast<std::size_t>(np));
    for (long p = 0; p < np; ++p) {
        Particle& e = out[static_cast<std::size_t>(p)];
        e.x = x[p];
        e.y = y[p];
        e.P = Vec3{P[3 * p], P[3 * p + 1], P[3 * p + 2]};
        e.v = Vec3{v[3 * p], v[3 * p + 1], v[3 * p + 2]};
        e.v_prev = Vec3{vprev[3 * p], vprev[3 * p + 1], vprev[3 * p + 2]};
        e.q = q[p];
        e.m = m[p];
    }
}

void store_particles(const std::vector<Particle>& in, double* x, double* y, double* P,
                     double* v, double* vprev) {
    for (std::size_t p = 0; p < in.size(); ++p) {
        const Particle& e = in[p];
        x[p] = e.x;
        y[p] = e.y;
        for (int d = 0; d < 3; ++d) {
            P[3 * p + d] = e.P[d];
            v[3 * p + d] = e.v[d];
            vprev[3 * p + d] = e.v_prev[d];
        }
    }
}

void store_diag(const Diagnostics& d, double* out) {
    const double vals[13] = {d.gauge_rms, d.gauss_rms, d.continuity_rms, d.Bz_l2, d.B_l2,
                             d.E_l2, d.rho_l2, d.J_l2, d.field_energy, d.kinetic_energy,
                             d.total_energy, d.max_speed, d.mean_gamma};
    std::memcpy(out, vals, sizeof(vals));
}

}  // namespace

extern "C" {

// Full CLI run of a deck (the reference's own main).  Returns its exit code.
int ref_p2_run_deck(const char* deck_path) {
    char prog[] = "spectral_pic_part3";
    char* argv[] = {prog, const_cast<char*>(deck_path), nullptr};
    return upic_ref_p2_cli_main(2, argv);
}

// In-place 2D FFT (reference fft2d), data laid out id = i*ny + j.
int ref_p2_fft2d(int nx, int ny, double* re, double* im, int inverse) {
    try {
        HarnessCfg h = make_cfg(nx, ny, 1.0, 1.0, 0.1, 1, 1, 1.0, 1.0, 1.0, 1.0);
        CField d(static_cast<std::size_t>(h.g.N));
        for (int id = 0; id < h.g.N; ++id) d[id] = Complex(re[id], im[id]);
        fft2d(d, h.g, inverse != 0);
        for (int id = 0; id < h.g.N; ++id) {
            re[id] = d[id].real();
            im[id] = d[id].imag();
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// J = deposit_current(electrons) (Project2/spectral_pic_part3.cpp:747).
int ref_p2_deposit_current(int nx, int ny, double Lx, double Ly, long np, const double* x,
                           const double* y, const double* v, const double* q, double* J) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, 0.1, 1, 1, 1.0, 1.0, 1.0, 1.0);
    std::vector<Particle> e(static_cast<std::size_t>(np));
    for (long p = 0; p < np; ++p) {
        e[p].x = x[p];
        e[p].y = y[p];
        e[p].v = Vec3{v[3 * p], v[3 * p + 1], v[3 * p + 2]};
        e[p].q = q[p];
    }
    auto Jf = deposit_current(e, h.g);
    for (int c = 0; c < 3; ++c)
        std::memcpy(J + static_cast<std::size_t>(c) * h.g.N, Jf[c].data(), sizeof(double) * h.g.N);
    return 0;
}

// rho = ion background + scatter of electron charge (spectral_pic_part3.cpp:739).
int ref_p2_deposit_charge(int nx, int ny, double Lx, double Ly, double n0, long np,
                          const double* x, const double* y, const double* q, double* rho) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, 0.1, 1, 1, 1.0, 1.0, 1.0, n0);
    ParticleSet ps;
    ps.fixed_ion_rho.assign(static_cast<std::size_t>(h.g.N), n0);
    ps.electrons.resize(static_cast<std::size_t>(np));
    for (long p = 0; p < np; ++p) {
        ps.electrons[p].x = x[p];
        ps.electrons[p].y = y[p];
        ps.electrons[p].q = q[p];
    }
    Field r = deposit_total_charge_naive(ps.electrons, ps, h.g);
    std::memcpy(rho, r.data(), sizeof(double) * h.g.N);
    return 0;
}

// out[p] = gather_scalar(f, x_p, y_p) (spectral_pic_part3.cpp:564).
int ref_p2_gather(int nx, int ny, double Lx, double Ly, const double* f, long np,
                  const double* x, const double* y, double* out) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, 0.1, 1, 1, 1.0, 1.0, 1.0, 1.0);
    Field ff(f, f + h.g.N);
    for (long p = 0; p < np; ++p) out[p] = gather_scalar(ff, h.g, x[p], y[p]);
    return 0;
}

// IAEM momentum push (push_particles_momentum_and_velocity :1057) of the
// given particles in the fields phi (N) and A (3N), with the reference's
// spectral gradients (spectral_gradient_scalar / spectral_gradient_vector);
// P, v, v_prev (3*np) updated in place.
int ref_p2_push_iaem(int nx, int ny, double Lx, double Ly, double dt, double c, long np, const double* x,
                     const double* y, double* P, double* v, double* v_prev, const double* q, const double* m,
                     const double* phi, const double* A) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, dt, 1, 1, c, 1.0, 1.0, 1.0);
    std::vector<Particle> e;
    load_particles(e, np, x, y, P, v, v_prev, q, m);
    std::array<Field, 3> An;
    for (int k = 0; k < 3; ++k) An[k].assign(A + (std::size_t)k * h.g.N, A + (std::size_t)(k + 1) * h.g.N);
    const Field ph(phi, phi + h.g.N);
    const auto grad_phi = spectral_gradient_scalar(ph, h.g);
    const auto grad_A = spectral_gradient_vector(An, h.g);
    push_particles_momentum_and_velocity(e, An, grad_phi, grad_A, h.cfg, h.g);
    for (long p = 0; p < np; ++p) {
        const Particle& pe = e[static_cast<std::size_t>(p)];
        const Vec3* src[3] = {&pe.P, &pe.v, &pe.v_prev};
        double* dst[3] = {P, v, v_prev};
        for (int k = 0; k < 3; ++k) {
            dst[k][3 * p] = src[k]->x;
            dst[k][3 * p + 1] = src[k]->y;
            dst[k][3 * p + 2] = src[k]->z;
        }
    }
    return 0;
}

// Spectral derivative d/dx (dir=0) or d/dy (dir=1) (spectral_pic_part3.cpp:440).
int ref_p2_spectral_derivative(int nx, int ny, double Lx, double Ly, const double* f, int dir,
                               double* out) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, 0.1, 1, 1, 1.0, 1.0, 1.0, 1.0);
    Field ff(f, f + h.g.N);
    Field r = spectral_derivative(ff, h.g, dir);
    std::memcpy(out, r.data(), sizeof(double) * h.g.N);
    return 0;
}

// Poisson start-up (spectral_pic_part3.cpp:819).
int ref_p2_poisson(int nx, int ny, double Lx, double Ly, double eps0, const double* rho,
                   double* phi) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, 0.1, 1, 1, 1.0, eps0, 1.0, 1.0);
    Field r(rho, rho + h.g.N);
    Field p = solve_initial_phi_from_poisson(r, h.cfg, h.g);
    std::memcpy(phi, p.data(), sizeof(double) * h.g.N);
    return 0;
}

// Run the reference step loop (run_simulation, spectral_pic_part3.cpp:1094-1189)
// on injected electrons with a uniform fixed ion background n0.
//
//   params = {Lx, Ly, dt, c, eps0, mu0, n0}
//   iparams = {nx, ny, bdf_order(1|2), conserving(1|0), n_steps, diag_stride}
//   diag_out: (n_steps+1) rows x 13 columns (Diagnostics field order), rows
//             written for step 0 and every step where diagnostics run; other
//             rows are left untouched.
//   fields_out (optional, may be NULL): final phi, A_x, A_y, A_z, rho, J_x, J_y, J_z
//             (8 x nx*ny) after the last step.
//   seconds_out (optional): wall seconds of the step loop, diagnostics included.
int ref_p2_simulate(const double* params, const int* iparams, long np, double* x, double* y,
                    double* P, double* v, double* vprev, const double* q, const double* m,
                    double* diag_out, double* fields_out, double* seconds_out) {
    try {
        HarnessCfg h = make_cfg(iparams[0], iparams[1], params[0], params[1], params[2], iparams[2],
                                iparams[3], params[3], params[4], params[5], params[6]);
        h.cfg.n_steps = iparams[4];
        h.cfg.diagnostic_stride = iparams[5];
        const Config& cfg = h.cfg;
        const Grid& g = h.g;
        ParticleSet ps;
        load_particles(ps.electrons, np, x, y, P, v, vprev, q, m);
        ps.fixed_ion_rho.assign(static_cast<std::size_t>(g.N), cfg.n0);

        Field rho0 = deposit_total_charge_naive(ps.electrons, ps, g);
        std::array<Field, 3> J0 = deposit_current(ps.electrons, g);
        Field phi0 = solve_initial_phi_from_poisson(rho0, cfg, g);
        std::array<Field, 3> A0{zero_field(g), zero_field(g), zero_field(g)};
        FieldState state;
        state.phi.initialize(phi0, 5);
        for (int comp = 0; comp < 3; ++comp) state.A[comp].initialize(A0[comp], 5);
        state.rho.initialize(rho0, 5);
        state.J = J0;

        BDFCoeffs bdf0{"bdf1", {1.0, -1.0}};
        if (diag_out) {
            Diagnostics d0 = compute_diagnostics(
                ps.electrons, state, state.phi.current(),
                {state.A[0].current(), state.A[1].current(), state.A[2].current()},
                state.rho.current(), state.J, bdf0, cfg, g);
            store_diag(d0, diag_out);
        }
        const auto t0 = std::chrono::steady_clock::now();
        for (int step = 1; step <= cfg.n_steps; ++step) {
            const BDFCoeffs bdf = bdf_coefficients_for_step(cfg, step);
            advance_particles_positions(ps.electrons, cfg, g);
            std::array<Field, 3> J_new = deposit_current(ps.electrons, g);
            Field rho_new;
            if (cfg.charge_update == "conserving")
                rho_new = update_charge_from_continuity(state.rho, J_new, bdf, cfg, g);
            else
                rho_new = deposit_total_charge_naive(ps.electrons, ps, g);
            Field phi_source(g.N, 0.0);
            for (int id = 0; id < g.N; ++id) phi_source[id] = rho_new[id] / cfg.eps0;
            Field phi_new = solve_bdf_wave_scalar(phi_source, state.phi, bdf, cfg, g);
            std::array<Field, 3> A_new{zero_field(g), zero_field(g), zero_field(g)};
            for (int comp = 0; comp < 3; ++comp) {
                Field A_source(g.N, 0.0);
                for (int id = 0; id < g.N; ++id) A_source[id] = cfg.mu0 * J_new[comp][id];
                A_new[comp] = solve_bdf_wave_scalar(A_source, state.A[comp], bdf, cfg, g);
            }
            const auto grad_phi = spectral_gradient_scalar(phi_new, g);
            const auto grad_A = spectral_gradient_vector(A_new, g);
            push_particles_momentum_and_velocity(ps.electrons, A_new, grad_phi, grad_A, cfg, g);
            if (diag_out && (step % std::max(1, cfg.diagnostic_stride) == 0 || step == cfg.n_steps)) {
                Diagnostics d = compute_diagnostics(ps.electrons, state, phi_new, A_new, rho_new,
                                                    J_new, bdf, cfg, g);
                store_diag(d, diag_out + 13 * static_cast<std::size_t>(step));
            }
            if (fields_out && step == cfg.n_steps) {
                const Field* src[8] = {&phi_new, &A_new[0], &A_new[1], &A_new[2],
                                       &rho_new, &J_new[0], &J_new[1], &J_new[2]};
                for (int f = 0; f < 8; ++f)
                    std::memcpy(fields_out + static_cast<std::size_t>(f) * g.N, src[f]->data(),
                                sizeof(double) * g.N);
            }
            state.phi.push_new(std::move(phi_new));
            for (int comp = 0; comp < 3; ++comp) state.A[comp].push_new(std::move(A_new[comp]));
            state.rho.push_new(std::move(rho_new));
            state.J = std::move(J_new);
        }
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds_out) *seconds_out = std::chrono::duration<double>(t1 - t0).count();
        store_particles(ps.electrons, x, y, P, v, vprev);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_p2_simulate: %s\n", e.what());
        return -1;
    }
}

// Reference Weibel initializer (spectral_pic_part3.cpp:624): fills arrays of
// size np_capacity; returns the electron count, or -1 if it does not fit.
long ref_p2_init_weibel(int nx, int ny, double Lx, double Ly, int ppc, double c, double n0,
                        double vx, double vy_max, double sine, int mode, unsigned seed,
                        long np_capacity, double* x, double* y, double* P, double* v,
                        double* vprev, double* q, double* m) {
    HarnessCfg h = make_cfg(nx, ny, Lx, Ly, 0.1, 1, 1, c, 1.0, 1.0, n0);
    h.cfg.particles_per_cell = ppc;
    h.cfg.weibel_vx = vx;
    h.cfg.weibel_vy_max = vy_max;
    h.cfg.weibel_sine_perturb = sine;
    h.cfg.perturbation_mode = mode;
    h.cfg.seed = seed;
    ParticleSet ps;
    initialize_weibel_particles(h.cfg, h.g, ps);
    const long n = static_cast<long>(ps.electrons.size());
    if (n > np_capacity) return -1;
    store_particles(ps.electrons, x, y, P, v, vprev);
    for (long p = 0; p < n; ++p) {
        q[p] = ps.electrons[p].q;
        m[p] = ps.electrons[p].m;
    }
    return n;
}

}  // extern "C"
