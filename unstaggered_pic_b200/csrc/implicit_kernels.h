// Launch interface of the implicit orbit-averaged GM-HC-CN kernels
// (implicit.cu), used by api_implicit.cu.
#pragma once

#include <cuda_runtime.h>

#include "kernels.h"

namespace upic {

// Gather record of the implicit map, per node: grad phi_mid (x, y), A^n (3),
// A^{n+1} trial (3).
constexpr int kIRec = 8;
constexpr int kIRecGpm = 0;
constexpr int kIRecAn = 2;
constexpr int kIRecAe = 5;
constexpr int kMaxQuad = 32;
// Knot crossings per particle orbit that the device kernel can hold
// (breakpoints of both axes plus the two ends).
constexpr int kMaxBreaks = 40;

// Failure reasons of the per-particle local fixed point
// (LocalParticleFailureReason, Project3/ec_pic_nyquist_projected.cpp:204-211).
enum LocalFailure {
    kLocalOk = 0,
    kLocalNonfiniteMap = 1,
    kLocalSuperluminalMap = 2,
    kLocalNonfiniteIterate = 3,
    kLocalSuperluminalIterate = 4,
    kLocalMaxIter = 5,
    kLocalTooManyCrossings = 6
};

struct MapStats {
    unsigned long long iter_total;
    int iter_max;
    int failures;
    // smallest (original particle index << 8 | LocalFailure) over failing
    // particles, ~0 when none failed
    unsigned long long first_fail_key;
    unsigned long long worst_scaled_bits;  // max final scaled residual (bit pattern)
};

struct ImplicitMapArgs {
    // current state (sorted order)
    const double *x, *y, *Px, *Py, *Pz, *vx, *vy, *vz;
    const double *q, *m;
    double q0, m0;
    const int* id;
    // trial end state, written by the final (consistency) evaluation
    double *ox, *oy, *oPx, *oPy, *oPz, *ovx, *ovy, *ovz, *obx, *oby, *obz;
    long np;
    int write_state;
    // grid (Project3 coordinates: x in [-L/2, L/2), node i at x = -L/2 + i dx)
    double Lx, Ly, inv_dx, inv_dy, inv_dV;
    double dt, kappa;
    const double* rec;  // kIRec doubles per node
    int split;
    double loc_rtol, loc_atol, loc_damp;
    int loc_maxit;
    // deposit of the orbit-averaged current
    const Chunk* chunks;
    const int* nchunks;
    unsigned long long* acc;  // [comp][hi,lo][N]
    double scale[3];
    MapStats* stats;
    // Gauss rules on [0, 1] (device, 4 x kMaxQuad doubles: nodes and
    // weights of the deck's nq-point rule, then of the mnq-point rule used
    // for segment moments)
    const double* qtab;
    int nq, mnq;
    // Picard deposit (picard = true): guess velocities, orbit vbar = (guess + v) / 2;
    // a particle with a component of vbar above vb_limit (or not finite) is
    // counted as a failure, since its deposit could leave the fixed-point range
    const double *gx, *gy, *gz;
    double vb_limit;
    // local fixed point of the relativistic map: start guesses (null: v^n)
    // and where to keep each particle's converged orbit velocity (null: not kept)
    const double *warm_x, *warm_y, *warm_z;
    double *keep_x, *keep_y, *keep_z;
    // selective particle sub-cycling (ec_pic_nyquist_projected.cpp:5235,
    // :6328): nsub[p] substeps of dt / nsub[p] per particle (null: all 1).
    // The map kernel skips particles with nsub > 1; the refined kernel
    // advances the compact list refined[0..nref).  Failing particles are
    // appended to failed[] (count in *nfailed) when failed is not null.
    const int* nsub;
    const int* refined;
    int nref;
    int grid_nx, grid_ny;  // grid of the refined kernel (the map kernel takes it from its tile geometry)
    // sub-orbit records of the refined particles (x0, y0, vbar from roff[i]),
    // written by the final evaluation (write_state), or null
    const int* roff;
    double* sub_rec;
    int* failed;
    int* nfailed;
    // orbit velocities handed from the local-solve launch to the deposit
    // launch of a split map evaluation (NaN for a particle that deposits
    // nothing), or null: one fused launch
    double *vbar_x, *vbar_y, *vbar_z;
};
// The refined particles of a sub-cycled map evaluation: chained local
// solves over [k/n, (k+1)/n] of the step with time-interpolated fields, each
// sub-orbit deposited with weight q/n (point quadrature, fixed-point grid adds).
cudaError_t launch_refined_map(int order, bool uniform, const ImplicitMapArgs& a, cudaStream_t st);
// Records of the failed particles failed[0..nf) of the map evaluation whose
// arguments are a (kFailRec doubles each, in failed order), for a grid of
// tg's size: each particle's failing local solve run again with its report.
constexpr int kFailRec = 28;
cudaError_t launch_failure_report(int order, bool uniform, bool split, const TileGeom& tg, const ImplicitMapArgs& a,
                                  const int* failed, int nf, double* out, cudaStream_t st);
// nsub[p] = 1 for p < n
cudaError_t launch_fill_int(int n, int value, int* out, cudaStream_t st);

// split: knot splitting of the orbit (ImplicitMapArgs::split); picard: the
// non-relativistic Picard deposit instead of the local GM-HC solve.  Both
// select the kernel instance.
cudaError_t launch_implicit_map(int order, bool uniform, bool split, const TileGeom& tg,
                                const ImplicitMapArgs& a, int grid, cudaStream_t st, bool picard = false);
int implicit_map_smem_bytes(const TileGeom& tg, int order);
cudaError_t implicit_configure_smem(const TileGeom& tg, int order, bool split, bool picard = false);
int implicit_map_occupancy(const TileGeom& tg, int order, bool split, bool picard = false);

// Point deposit of rho (q S / dV, slot 3) and J (q v S / dV, slots 0..2) at
// the particle positions (deposit_scalar_to_mesh :2117, deposit_current_to_mesh
// :2182), for the start-up state.
struct PointDepositArgs {
    const double *x, *y, *vx, *vy, *vz, *q;
    double q0;
    long np;
    int nx, ny;
    double Lx, Ly, inv_dx, inv_dy, inv_dV;
    unsigned long long* acc;
    double scale[4];
};
cudaError_t launch_point_deposit(int order, const PointDepositArgs& a, cudaStream_t st);

// Kernel-level orbit integrals (path_average_deposit_current :2784,
// path_average_gather_and_gradient :3016) over orbits x0 + s dx, s in [0,1],
// 2D (the third components of dx are not used; the z column of grad is 0).
struct OrbitArgs {
    const double *x, *y, *dx, *vbar, *q;   // dx, vbar: xyz triples; q null = q0
    double q0;
    long np;
    int nx, ny;
    double Lx, Ly, inv_dx, inv_dy, inv_dV;
    int split, nq;
    const double* qtab;                    // Gauss rule (nodes, then weights at +kMaxQuad)
    unsigned long long* acc;               // deposit: [comp][hi,lo][N]
    double scale[3];
    const double *mesh, *An, *Ae;          // gather: 3 x N planar fields
    double *gathered, *grad;               // gather: 3 and 9 ([comp][dir]) per particle
    int* err;                              // set to 1 when an orbit crosses too many knots
};
cudaError_t launch_orbit_deposit(int order, const OrbitArgs& a, cudaStream_t st);
cudaError_t launch_orbit_gather(int order, const OrbitArgs& a, cudaStream_t st);

// Step diagnostics (compute_subcycled_step_diagnostics :4340, one level per
// particle): A-chain residual R = (A^{n+1}(x1) - A^n(x0)) - dt (<U_mid> +
// D_A vbar), particle work dt q vbar.<E_mid>, knot-crossing counts.
struct StepDiagArgs {
    const double *x, *y;              // orbit starts (state n, sorted order)
    const double *bx, *by, *bz;       // accepted orbit velocities (same order)
    const double* q;                  // per particle, or null (q0)
    double q0;
    long np;
    int nx, ny;
    double Lx, Ly, inv_dx, inv_dy, dt;
    int split, nq;
    const double* qtab;
    const double* rec;                // 12 doubles per node: An, Ae, U_mid, E_mid
    double* partials;                 // grid x 16 (then the refined kernel's blocks)
    unsigned long long* counts;       // segments, crossings, crossing particles, max segments
    // sub-cycled particles of the step: nsub per particle (null: none), the
    // refined list, their sub-orbit records (x0, y0, vbar; 5 doubles) from
    // roff[i], and the most blocks the refined kernel may use
    const int* nsub;
    const int* refined;
    int nref;
    const int* roff;
    const double* sub;
    int refined_grid_max;
};
// Spectra (12 x N) of A^n, A^{n+1}, U_mid, E_mid from the two states' spectra.
cudaError_t launch_step_diag_spectra(int N, const double* kx, const double* ky, const double2* s0,
                                     const double2* s1, double2* out12, cudaStream_t st);
// out13: double-double sums R.R, A_delta.A_delta, rhs.rhs, |R|, -q vbar.R,
// dt q vbar.<E_mid> ([0..11]) and max |R| ([12]).
cudaError_t launch_step_diag(int order, const StepDiagArgs& a, int grid, double* out13, cudaStream_t st);
// out2: double-double sum of J . E_mid over nodes and components.
cudaError_t launch_grid_work(int N, const double* J, const double* rec12, double* partials, int grid,
                             double* out2, cudaStream_t st);

// Gather of planar 3-vector fields at particle positions (gather_vector_at :2267).
cudaError_t launch_gather3(int order, int nx, int ny, double Lx, double Ly, const double* f3,
                           long np, const double* x, const double* y, double* out3,
                           cudaStream_t st);

// GM-HC-CN push of a particle list in the node records a.rec (grad phi_mid,
// A^n, A^{n+1}): in7 = x, y, Px, Py, Pz, q, m (planar, stride np), guess3 =
// first guesses (planar); out = x1, y1, P_end (3), v_end (3), vbar (3)
// (planar; NaN where the local solve failed); rep = iterations, reason per
// particle (solve_local_particle_substep :4930).
cudaError_t launch_gmhc_push(int order, const ImplicitMapArgs& a, int nx, int ny, long np, const double* in7,
                             const double* guess3, double* out, int* rep, cudaStream_t st);

// Point probes of 18 planar fields (phi, psi, rho, A, U, J, E, B): their
// shape gathers, grad(S phi) and grad(S A), 30 values per point
// (evaluate_reconstructed_field_probe :7924).
cudaError_t launch_probe(int order, int nx, int ny, double Lx, double Ly, const double* F18, long np,
                         const double* x, const double* y, double* out30, cudaStream_t st);

// P += q A(x) with A a planar 3-vector field (the canonical momentum of a
// start state with a non-zero A, :4113-4117); q per particle or q0.
cudaError_t launch_add_qA(int order, int nx, int ny, double Lx, double Ly, const double* A3, long np,
                          const double* x, const double* y, const double* q, double q0, double* Px, double* Py,
                          double* Pz, cudaStream_t st);

// k-space map step: J_field spectra -> rho_end, rho_mid, CN (phi, psi), (A, U)
// and the spectra of grad phi_mid and A_end (continuity_charge_update :3288,
// cn_potential_update :3249, cn_fft_wave_step_from_spectra :3131).
struct CnArgs {
    int nx, ny, N;
    const double *kx, *ky, *k2;
    const unsigned char* excl;  // Nyquist-plane mask (projection on) or null
    const double2* Jhat;        // 3 x N (J_field)
    const double2* st;          // state spectra: phi, psi, rho, A(3), U(3) (9 x N)
    double2* out;               // end spectra: phi, psi, rho, A(3), U(3) (9 x N)
    double2* gspec;             // grad phi_mid (2), A_end (3): 5 x N
    double dt, kappa, sigma1, sigma2;
};
cudaError_t launch_cn_kspace(const CnArgs& a, cudaStream_t st);

// Spectra of E (3), B (3), div E, div A, psi, rho (10 x N) from the state
// spectra phi, psi, rho, A(3), U(3).
cudaError_t launch_diag_spectra(int N, const double* kx, const double* ky, const double2* st_spec, double2* out,
                                cudaStream_t st);
// P = m gamma(v) v (start-up canonical momentum with A = 0).
cudaError_t launch_momentum_from_v(long np, const double* vx, const double* vy, const double* vz, const double* m,
                                   double m0, double kappa, double* Px, double* Py, double* Pz, cudaStream_t st);

// Project every even-grid Nyquist plane out of real fields (project_nyquist
// :2044): alternating-mean subtraction along x lines then y lines.
cudaError_t launch_project_nyquist(double* f, int ncomp, int nx, int ny, cudaStream_t st);

// Zero the k = 0 mode and the excluded Nyquist modes of spectra.
cudaError_t launch_kspace_mask(double2* f, int ncomp, int N, const unsigned char* excl, int zero_mean,
                               cudaStream_t st);

// Outer-iteration vector algebra on node currents (3 x N planar).
struct NormSums {
    double r2[2], map2[2], guess2[2];  // double-double sums
    double max_rel, max_scaled;
};
cudaError_t launch_residual_norms(int N, const double* map, const double* guess, double floor_rel,
                                  double atol, double rtol, double* partials, int grid,
                                  NormSums* out, cudaStream_t st);
// Gram dots of the Anderson history: dr_i = r[i+1]-r[i] for i < m; sums
// dr_i.dr_j (i>=j, packed) and dr_i.r[m], in double-double.
cudaError_t launch_anderson_dots(int N3, const double* const* r, int m, double* partials, int grid,
                                 double* out, cudaStream_t st);
// out = x[m] + beta r[m] - sum_j gamma_j (dx_j + beta dr_j)
cudaError_t launch_anderson_candidate(int N3, const double* const* x, const double* const* r, int m,
                                      double beta, const double* gamma, double* out, cudaStream_t st);
// *flag |= 1 when any of v[0..n) is not finite (finite_node_vector :5051);
// the caller clears *flag.
cudaError_t launch_nonfinite_flag(int n, const double* v, int* flag, cudaStream_t st);
// out = 2 v - w (Picard predictor, ec_pic_serial_demo.cpp:1514)
cudaError_t launch_extrapolate(int n, const double* v, const double* w, double* out, cudaStream_t st);
// out = (a + b) / 2
cudaError_t launch_half_sum(int n, const double* a, const double* b, double* out, cudaStream_t st);
// out = a + s (b - a)
cudaError_t launch_lerp(int n, const double* a, const double* b, double s, double* out, cudaStream_t st);
// out = a + s b
cudaError_t launch_axpy(int n, const double* a, const double* b, double s, double* out, cudaStream_t st);

// Diagnostics of the implicit method (compute_diagnostics :3521): real fields
// planar in `f` (phi, psi, rho, A(3), U(3) real; E(3), B(3), divE, divA
// appended by the caller), particle kinetic energy.
struct ImplicitDiagArgs {
    int N;
    const double* psi;
    const double* rho;
    const double* E;     // 3 x N
    const double* B;     // 3 x N
    const double* divE;
    const double* divA;
    double sigma1, kappa;
    double* partials;    // grid x 32
    int grid;
};
// sums: [0..1] gauss^2, [2..3] divE^2, [4..5] rho^2, [6..7] gauge^2, [8..9] psi^2,
// [10..11] divA^2, [12..13] E^2, [14..15] B^2, [16..17] rho; [18] gauss max, [19] gauge max
cudaError_t launch_implicit_diag(const ImplicitDiagArgs& a, double* out20, cudaStream_t st);
// kinetic energy over particles (double-double): out[0..1]; relativistic
// m kappa^2 (gamma - 1), or m v^2 / 2 with nonrel
cudaError_t launch_kinetic(long np, const double* vx, const double* vy, const double* vz,
                           const double* m, double m0, double kappa, double* partials, int grid,
                           double* out, cudaStream_t st, bool nonrel = false);

// Non-relativistic Picard push (picard_push_kernel, Project1
// evaluate_picard_map_orbit :1455): trial state and the double-double sums
// |v_next - v_guess|^2 (r2), |v_next|^2 (map2), |v_guess|^2 (guess2).
struct PicardPushArgs {
    const double *x, *y, *Px, *Py, *Pz, *vx, *vy, *vz;   // state n (sorted order)
    const double *gx, *gy, *gz;                          // velocity guess
    const double *q, *m;
    double q0, m0;
    long np;
    double *ox, *oy, *oPx, *oPy, *oPz, *ovx, *ovy, *ovz;  // trial end state
    int nx, ny;
    double Lx, Ly, inv_dx, inv_dy, dt;
    const double* rec;
    int split, nq, mnq;
    const double* qtab;
    double* partials;  // grid x 8
    int* err;          // += particles whose orbit crosses too many knots
};
cudaError_t launch_picard_push(int order, bool uniform, bool split, const PicardPushArgs& a, int grid,
                              NormSums* out, cudaStream_t st);
// P = m v, v_prev = v - dt (q/m) E(x) (Project1 start-up).
cudaError_t launch_picard_startup(int order, int nx, int ny, double Lx, double Ly, const double* E3, long np,
                                  const double* x, const double* y, const double* vx, const double* vy,
                                  const double* vz, const double* q, double q0, const double* m, double m0,
                                  double dt, double* Px, double* Py, double* Pz, double* wx, double* wy, double* wz,
                                  cudaStream_t st);
struct PathStatsArgs {
    const double *x, *y;                  // orbit starts
    const double *bx, *by;                // orbit velocity, or null: (v1 + v0) / 2
    const double *v1x, *v1y, *v0x, *v0y;
    long np;
    int nx, ny;
    double Lx, Ly, dt;
    int split;
    unsigned long long* counts;           // segments, crossings, crossing particles, max segments
};
cudaError_t launch_path_stats(int order, const PathStatsArgs& a, cudaStream_t st);

// Lorentz backward start-up of v_prev (initialize_relativistic_history_velocity :3423)
cudaError_t launch_history_velocity(int order, int nx, int ny, double Lx, double Ly, const double* E3,
                                    const double* B3, long np, const double* x, const double* y,
                                    const double* vx, const double* vy, const double* vz,
                                    const double* q, double q0, const double* m, double m0,
                                    double kappa, double dt, double* wx, double* wy, double* wz,
                                    cudaStream_t st);

}  // namespace upic
