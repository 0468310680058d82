// Project3's cold-instability initial states on the 2D grid (nz = 1), the
// start of its manuscript runs (host code).
//
//   two-stream: initialize_two_stream_3d_linear_x
//               (Project3/ec_pic_nyquist_projected.cpp:3689)
//   Weibel:     initialize_weibel_filamentation_3d (:3961)
//   Landau:     initialize_landau_damping_1d3d (:3853), the retained
//               electrostatic teaching example
//
// Both put two cold counter-streaming electron populations (+-v0 along x) on
// the same quiet-start positions -- cell-centred lines, particles_per_cell_pair
// per cell along x -- and seed the growing cold-fluid eigenmode of the
// instability: velocity perturbations and stream weights from the linear
// eigenvector (the B-spline scatter/gather factor S(k) included when the
// finite-grid theory is on), and for Weibel the matching A_x and U_x = Gamma
// A_x on the mesh.  The rest of the reference's start-up (rho, phi, J,
// canonical momenta, Nyquist projection, history velocities) is
// upic_init_fields on a context that received these particles and, through
// upic_set_initial_potential, these fields.  The arithmetic follows the
// reference's expressions term for term with the same C library calls, so
// the arrays are the reference's bit for bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/upic.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

// wrap1 (:704): x into [-L/2, L/2)
double wrap_centered(double x, double L) {
    double y = std::fmod(x + 0.5 * L, L);
    if (y < 0.0) y += L;
    return y - 0.5 * L;
}

// cell_centered_grid(n, L, true) (:3599): node i of n cell centres of [-L/2, L/2)
double cell_center(int i, int n, double L) {
    const double dx = L / static_cast<double>(n);
    double x = (static_cast<double>(i) + 0.5) * dx;
    x -= 0.5 * L;
    return x;
}

// sinc_unormalized (:1138) and bspline_mode_factor_1d (:1157): the Fourier
// amplitude of a degree-r centred B-spline, sinc(k dx / 2)^(r+1)
double mode_factor(int degree, double k, double dx) {
    const double a = 0.5 * k * dx;
    const double s = (std::abs(a) < 1.0e-12) ? 1.0 : std::sin(a) / a;
    return std::pow(s, static_cast<double>(degree + 1));
}

// gamma_from_v (:623); false when |v| >= kappa
bool gamma_of(double vx, double vy, double vz, double kappa, double& g) {
    const double beta2 = (vx * vx + vy * vy + vz * vz) / (kappa * kappa);
    if (beta2 >= 1.0) return false;
    g = 1.0 / std::sqrt(std::max(1.0e-300, 1.0 - beta2));
    return true;
}

bool speed_ok(double vx, double vy, double vz, double kappa) {
    return std::sqrt(vx * vx + vy * vy + vz * vz) < kappa;
}

// Cold symmetric two-stream growth rate with omega_p^2 |S(k)|^2
// (cold_two_stream_growth_rate :4160).
double two_stream_rate(const upic_p3_case& c) {
    const double k = 2.0 * kPi * static_cast<double>(std::max(1, c.perturbation_mode)) / c.Lx;
    double g0;
    if (!gamma_of(c.v0, 0.0, 0.0, c.kappa, g0)) return 0.0;
    const double S = c.two_stream_finite_grid_theory ? mode_factor(c.spline_order, k, c.Lx / c.nx) : 1.0;
    const double wp2 = (c.sigma1 * c.n0) * S * S;
    const double a = wp2 / (2.0 * g0 * g0 * g0);
    const double b = k * k * c.v0 * c.v0;
    const double y = b + a - std::sqrt(a * a + 4.0 * a * b);
    return (y < 0.0) ? std::sqrt(-y) : 0.0;
}

// Cold filamentation (Weibel) growth rate for k along y (cold_weibel_growth_rate :4197).
double weibel_rate(const upic_p3_case& c) {
    const double k = 2.0 * kPi * static_cast<double>(std::max(1, c.perturbation_mode)) / c.Ly;
    double g0;
    if (!gamma_of(c.v0, 0.0, 0.0, c.kappa, g0)) return 0.0;
    const double S = c.weibel_finite_grid_theory ? mode_factor(c.spline_order, k, c.Ly / c.ny) : 1.0;
    const double wp2 = (c.sigma1 * c.n0) * S * S;
    const double A = c.kappa * c.kappa * k * k + wp2 / (g0 * g0 * g0);
    const double C = k * k * wp2 * c.v0 * c.v0 / g0;
    const double g2 = 0.5 * (std::sqrt(A * A + 4.0 * C) - A);
    return (g2 > 0.0) ? std::sqrt(g2) : 0.0;
}

bool valid(const upic_p3_case* c) {
    return c && (c->kind == UPIC_P3_TWO_STREAM || c->kind == UPIC_P3_WEIBEL || c->kind == UPIC_P3_LANDAU) &&
           c->nx > 0 && c->ny > 0 &&
           c->Lx > 0.0 && c->Ly > 0.0 && c->Lz > 0.0 && c->kappa > 0.0 && c->spline_order >= 1 &&
           c->spline_order <= 4;
}

int two_stream(const upic_p3_case& c, double* x, double* y, double* v, double* q, double* m, double* A,
               double* U, double* rate) {
    const int nxl = c.nx * c.particles_per_cell_pair;
    const long nbase = (long)nxl * c.ny;
    const long np = 2 * nbase;
    const double kx = 2.0 * kPi * static_cast<double>(c.perturbation_mode) / c.Lx;
    if (!(kx > 0.0)) return UPIC_ERR_CONFIG;
    double g0;
    if (!gamma_of(c.v0, 0.0, 0.0, c.kappa, g0)) return UPIC_ERR_SUPERLUMINAL;
    const double g03 = g0 * g0 * g0;
    const double alpha = (c.two_stream_density_alpha >= 0.0) ? c.two_stream_density_alpha : 0.0;
    if (std::abs(alpha) >= 0.25) return UPIC_ERR_CONFIG;
    const bool eig = c.two_stream_eigenmode && c.two_stream_density_alpha >= 0.0;
    const double S = c.two_stream_finite_grid_theory ? mode_factor(c.spline_order, kx, c.Lx / c.nx) : 1.0;
    const double gl = two_stream_rate(c);
    // grid E amplitude of the density mode rho = alpha n0 cos(k x), felt by
    // the particles as S E
    const double Eg = (eig && alpha > 0.0) ? (alpha * c.sigma1 * c.n0 / kx) : 0.0;
    const double Ep = S * Eg;
    const double den = kx * kx * c.v0 * c.v0 + gl * gl;
    const double vc = (den > 0.0) ? (Ep * kx * c.v0 / (g03 * den)) : 0.0;
    const double vs = (den > 0.0) ? (Ep * gl / (g03 * den)) : 0.0;
    const double nc = (den > 0.0) ? (-kx * Ep * (kx * kx * c.v0 * c.v0 - gl * gl) / (g03 * den * den)) : 0.0;
    const double ns = (den > 0.0) ? (2.0 * kx * kx * c.v0 * gl * Ep / (g03 * den * den)) : 0.0;
    long p = 0;
    for (int j = 0; j < c.ny; ++j) {
        const double yb = cell_center(j, c.ny, c.Ly);
        for (int i = 0; i < nxl; ++i, ++p) {
            const double xb = cell_center(i, nxl, c.Lx);
            const double ph = kx * xb;
            const double cp = std::cos(ph), sp = std::sin(ph);
            x[p] = x[nbase + p] = wrap_centered(xb, c.Lx);
            y[p] = y[nbase + p] = wrap_centered(yb, c.Ly);
            double vp, vm;
            if (eig) {
                vp = +c.v0 + (+vc * cp - vs * sp);
                vm = -c.v0 + (-vc * cp - vs * sp);
            } else {
                const double sv = c.perturbation * std::sin(kx * xb);
                vp = +c.v0 + sv;
                vm = -c.v0 + sv;
            }
            v[3 * p] = vp;
            v[3 * p + 1] = v[3 * p + 2] = 0.0;
            v[3 * (nbase + p)] = vm;
            v[3 * (nbase + p) + 1] = v[3 * (nbase + p) + 2] = 0.0;
        }
    }
    // a common transverse v_x seed (a J_x perturbation along y, not an eigenmode)
    if (c.tsi_transverse_seed != 0.0)
        for (long k = 0; k < np; ++k)
            v[3 * k] += c.tsi_transverse_seed * std::cos(2.0 * kPi * c.tsi_transverse_mode * y[k] / c.Ly);
    for (long k = 0; k < np; ++k)
        if (!speed_ok(v[3 * k], v[3 * k + 1], v[3 * k + 2], c.kappa)) return UPIC_ERR_SUPERLUMINAL;
    const double qm = -c.n0 * (c.Lx * c.Ly * c.Lz) / static_cast<double>(np);
    p = 0;
    for (int j = 0; j < c.ny; ++j)
        for (int i = 0; i < nxl; ++i, ++p) {
            double wp = 1.0, wm = 1.0;
            if (eig) {
                const double ph = kx * cell_center(i, nxl, c.Lx);
                const double cp = std::cos(ph), sp = std::sin(ph);
                wp = 1.0 + nc * cp + ns * sp;
                wm = 1.0 + nc * cp - ns * sp;
            } else if (c.two_stream_density_alpha >= 0.0) {
                const double w = 1.0 + alpha * std::cos(kx * cell_center(i, nxl, c.Lx));
                wp = wm = w;
            }
            if (!(wp > 0.0) || !(wm > 0.0)) return UPIC_ERR_CONFIG;
            q[p] = qm * wp;
            q[nbase + p] = qm * wm;
            m[p] = std::abs(q[p]);
            m[nbase + p] = std::abs(q[nbase + p]);
        }
    const long N = (long)c.nx * c.ny;
    for (long k = 0; k < 3 * N; ++k) A[k] = U[k] = 0.0;
    if (rate) *rate = gl;
    return UPIC_OK;
}

int weibel(const upic_p3_case& c, double* x, double* y, double* v, double* q, double* m, double* A, double* U,
           double* rate) {
    const int per = std::max(1, c.particles_per_cell_pair);
    const int nxl = c.nx * per;
    const long nbase = (long)nxl * c.ny;
    const long np = 2 * nbase;
    if (std::abs(c.v0) >= c.kappa) return UPIC_ERR_SUPERLUMINAL;
    const int mode = std::max(1, c.perturbation_mode);
    const double ky = 2.0 * kPi * static_cast<double>(mode) / c.Ly;
    const double B0 = (c.weibel_B0 >= 0.0) ? c.weibel_B0 : c.perturbation;
    const double G = weibel_rate(c);
    if (c.weibel_eigenmode && !(G > 0.0)) return UPIC_ERR_CONFIG;  // the mode is not unstable
    double g0;
    if (!gamma_of(c.v0, 0.0, 0.0, c.kappa, g0)) return UPIC_ERR_SUPERLUMINAL;
    const double S = c.weibel_finite_grid_theory ? mode_factor(c.spline_order, ky, c.Ly / c.ny) : 1.0;
    // growing-mode relations relative to the mesh B_z amplitude B0 (q/m = -1)
    const bool eig = c.weibel_eigenmode && G > 0.0;
    const double dvx = eig ? (S * B0 / (ky * g0 * g0 * g0)) : 0.0;
    const double dvy = eig ? (S * c.v0 * B0 / (g0 * G)) : 0.0;
    const double dn = eig ? (S * c.v0 * ky * B0 / (g0 * G * G)) : 0.0;
    if (std::abs(dn) >= 0.25) return UPIC_ERR_CONFIG;
    long p = 0;
    for (int j = 0; j < c.ny; ++j) {
        const double yb = cell_center(j, c.ny, c.Ly);
        const double ph = ky * yb;
        const double cp = std::cos(ph), sp = std::sin(ph);
        for (int i = 0; i < nxl; ++i, ++p) {
            const double xb = cell_center(i, nxl, c.Lx);
            x[p] = x[nbase + p] = wrap_centered(xb, c.Lx);
            y[p] = y[nbase + p] = wrap_centered(yb, c.Ly);
            v[3 * p] = +c.v0 + dvx * cp;
            v[3 * p + 1] = +dvy * sp;
            v[3 * p + 2] = 0.0;
            v[3 * (nbase + p)] = -c.v0 + dvx * cp;
            v[3 * (nbase + p) + 1] = -dvy * sp;
            v[3 * (nbase + p) + 2] = 0.0;
        }
    }
    for (long k = 0; k < np; ++k)
        if (!speed_ok(v[3 * k], v[3 * k + 1], v[3 * k + 2], c.kappa)) return UPIC_ERR_SUPERLUMINAL;
    const double qm = -c.n0 * (c.Lx * c.Ly * c.Lz) / static_cast<double>(np);
    p = 0;
    for (int j = 0; j < c.ny; ++j) {
        const double cp = std::cos(ky * cell_center(j, c.ny, c.Ly));
        const double wp = 1.0 - dn * cp, wm = 1.0 + dn * cp;
        if (!(wp > 0.0) || !(wm > 0.0)) return UPIC_ERR_CONFIG;
        for (int i = 0; i < nxl; ++i, ++p) {
            q[p] = qm * wp;
            q[nbase + p] = qm * wm;
            m[p] = std::abs(q[p]);
            m[nbase + p] = std::abs(q[nbase + p]);
        }
    }
    // A_x = (B0 / k) cos(k y) (B_z = B0 sin(k y)), U_x = Gamma A_x
    const long N = (long)c.nx * c.ny;
    for (long k = 0; k < 3 * N; ++k) A[k] = U[k] = 0.0;
    const double hy = c.Ly / c.ny;
    for (int i = 0; i < c.nx; ++i)
        for (int j = 0; j < c.ny; ++j) {
            const double yj = -0.5 * c.Ly + static_cast<double>(j) * hy;
            const double ax = (B0 / ky) * std::cos(ky * yj);
            A[(long)i * c.ny + j] = ax;
            U[(long)i * c.ny + j] = c.weibel_eigenmode ? (G * ax) : 0.0;
        }
    if (rate) *rate = G;
    return UPIC_OK;
}

// Acklam's rational approximation of the inverse standard normal CDF (P. J.
// Acklam, "An algorithm for computing the inverse normal cumulative
// distribution function", 2003): a central rational function for
// 0.02425 <= p <= 0.97575 and a tail form in sqrt(-2 log p) outside, the
// quiet-start sampler of normal_quantile (:3623); 0 < p < 1.
double acklam_quantile(double p) {
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    const double lo = 0.02425, hi = 1.0 - lo;
    if (p < lo || p > hi) {
        const double t = std::sqrt(-2.0 * std::log(p < lo ? p : 1.0 - p));
        const double v = (((((c[0] * t + c[1]) * t + c[2]) * t + c[3]) * t + c[4]) * t + c[5]) /
                         ((((d[0] * t + d[1]) * t + d[2]) * t + d[3]) * t + 1.0);
        return p < lo ? v : -v;
    }
    const double q = p - 0.5, r = q * q;
    return (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
           (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
}

double landau_alpha(const upic_p3_case& c) { return c.landau_alpha >= 0.0 ? c.landau_alpha : c.perturbation; }

// initialize_landau_damping_1d3d (:3853) on the 2D grid: rows y outer, x
// inner, nv velocities per cell centre; q = q0 (1 + alpha cos(k x)), m = |q|.
int landau(const upic_p3_case& c, double* x, double* y, double* v, double* q, double* m, double* A, double* U,
           double* rate) {
    const int nv = c.particles_per_cell_pair;
    const double alpha = landau_alpha(c);
    if (nv < 2 || !(std::abs(alpha) < 1.0)) return UPIC_ERR_CONFIG;
    std::vector<double> vq(nv);
    for (int j = 0; j < nv; ++j) vq[j] = c.thermal_velocity * acklam_quantile((j + 0.5) / (double)nv);
    const long np = (long)c.nx * c.ny * nv;
    const double kx = 2.0 * kPi * static_cast<double>(c.perturbation_mode) / c.Lx;
    const double q0 = -c.n0 * (c.Lx * c.Ly * c.Lz) / static_cast<double>(np);
    long p = 0;
    for (int j = 0; j < c.ny; ++j) {
        const double yc = cell_center(j, c.ny, c.Ly);
        for (int i = 0; i < c.nx; ++i) {
            const double xc = cell_center(i, c.nx, c.Lx);
            const double w = 1.0 + alpha * std::cos(kx * xc);
            for (int jv = 0; jv < nv; ++jv, ++p) {
                x[p] = wrap_centered(xc, c.Lx);
                y[p] = wrap_centered(yc, c.Ly);
                v[3 * p] = vq[jv];
                v[3 * p + 1] = 0.0;
                v[3 * p + 2] = 0.0;
                q[p] = q0 * w;
                m[p] = std::abs(q[p]);
            }
        }
    }
    const long N = (long)c.nx * c.ny;
    std::fill(A, A + 3 * N, 0.0);
    std::fill(U, U + 3 * N, 0.0);
    if (rate) *rate = 0.0;
    return UPIC_OK;
}

}  // namespace

extern "C" int upic_p3_case_default(upic_p3_case* c) {
    if (!c) return UPIC_ERR_ARGUMENT;
    *c = upic_p3_case{};
    c->kind = UPIC_P3_TWO_STREAM;
    c->nx = c->ny = 16;
    c->Lx = c->Ly = c->Lz = 2.0 * kPi;
    c->kappa = 1.0;
    c->sigma1 = 1.0;
    c->n0 = 1.0;
    c->spline_order = 2;
    c->perturbation_mode = 1;
    c->particles_per_cell_pair = 4;
    c->v0 = 0.3;
    c->perturbation = 0.02;
    c->two_stream_density_alpha = -1.0;
    c->two_stream_eigenmode = 1;
    c->two_stream_finite_grid_theory = 1;
    c->tsi_transverse_seed = 0.0;
    c->tsi_transverse_mode = 1;
    c->weibel_B0 = -1.0;
    c->weibel_eigenmode = 1;
    c->weibel_finite_grid_theory = 1;
    c->landau_alpha = -1.0;
    c->thermal_velocity = 1.0;
    return UPIC_OK;
}

extern "C" long upic_p3_case_particles(const upic_p3_case* c) {
    if (!valid(c)) return -1;
    const int per = c->kind == UPIC_P3_WEIBEL ? std::max(1, c->particles_per_cell_pair) : c->particles_per_cell_pair;
    if (per <= 0) return -1;
    if (c->kind == UPIC_P3_LANDAU) return (long)c->nx * c->ny * per;
    return 2L * c->nx * per * c->ny;
}

extern "C" int upic_p3_initial_state(const upic_p3_case* c, long capacity, double* x, double* y, double* v,
                                     double* q, double* m, double* A, double* U, double* growth_rate) {
    const long np = upic_p3_case_particles(c);
    if (np < 0) return UPIC_ERR_CONFIG;
    if (capacity < np || (np > 0 && (!x || !y || !v || !q || !m)) || !A || !U) return UPIC_ERR_ARGUMENT;
    if (c->kind == UPIC_P3_LANDAU) return landau(*c, x, y, v, q, m, A, U, growth_rate);
    return c->kind == UPIC_P3_WEIBEL ? weibel(*c, x, y, v, q, m, A, U, growth_rate)
                                     : two_stream(*c, x, y, v, q, m, A, U, growth_rate);
}
