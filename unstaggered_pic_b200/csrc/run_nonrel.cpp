// upic_run --nonrel: deck-driven drop-in for the reference's non-relativistic
// implicit solver CLI (Project1/ec_pic_serial_demo.cpp `main:1768-1882`):
// reads the same `key = value` deck (read_config :319-367), builds the same
// two-stream or Landau particles (initialize_state :1306), advances the
// Picard step through the C ABI (UPIC_METHOD_CN_ORBIT_NONREL) on the GPU and
// writes <output_prefix>_diagnostics.csv, _step_diagnostics.csv,
// _particle_sample.csv, _config_echo.txt and _unit_tests.txt in its formats.
//
// Runs are 2D or 1D (nz = 1).  The start-up checks of run_unit_tests
// (:1556-1713) run as 2D versions of the reference's four tests, with its
// seeds, sizes, messages and thresholds.
//
// Exit codes as the reference: 0 ok, 1 error (message on stderr), 2 usage,
// 3 unit-test failure.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/upic.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

// Deck keys and defaults of the reference's Config (:232-301).
struct NonrelDeck {
    int nx = 4, ny = 4, nz = 4;
    double Lx = 2.0 * kPi, Ly = 2.0 * kPi, Lz = 2.0 * kPi;
    int n_steps = 6;
    double dt = 0.00625;
    std::string test_case = "two_stream";
    int particles_per_cell_pair = 4;
    int spline_order = 2;
    int orbit_quad_order = 16;
    bool split_orbit_at_knots = true;
    double picard_tol = 1.0e-11;
    int picard_max_iter = 16;
    bool final_consistency_sweep = true;
    bool run_unit_tests = true;
    double c = 1.0, eps0 = 1.0, mu0 = 1.0;
    double n0 = 1.0, v0 = 0.3, perturbation = 0.02, landau_alpha = -1.0, thermal_velocity = 1.0;
    int perturbation_mode = 1;
    double theory_omega = 0.0, theory_gamma = 0.0;
    unsigned int seed = 12345;
    std::string output_prefix = "orbit_smoke";
};

std::string trim(const std::string& s) {
    const auto a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const auto b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::string lowercase(std::string s) {
    for (char& ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

bool parse_bool(const std::string& v) {
    const std::string t = lowercase(trim(v));
    return t == "1" || t == "true" || t == "yes" || t == "on";
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// read_config (:319-367): keys are case sensitive, values trimmed, `#`
// starts a comment, unknown keys warn.
NonrelDeck read_deck(const std::string& path) {
    NonrelDeck d;
    std::ifstream in(path);
    if (!in) throw std::runtime_error("could not open input file: " + path);
    std::string line;
    while (std::getline(in, line)) {
        const auto sharp = line.find('#');
        if (sharp != std::string::npos) line = line.substr(0, sharp);
        const auto eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = trim(line.substr(0, eq));
        const std::string val = trim(line.substr(eq + 1));
        if (key.empty()) continue;
        std::istringstream ss(val);
        if (key == "nx") ss >> d.nx;
        else if (key == "ny") ss >> d.ny;
        else if (key == "nz") ss >> d.nz;
        else if (key == "Lx") ss >> d.Lx;
        else if (key == "Ly") ss >> d.Ly;
        else if (key == "Lz") ss >> d.Lz;
        else if (key == "n_steps") ss >> d.n_steps;
        else if (key == "dt") ss >> d.dt;
        else if (key == "test_case" || key == "initial_condition" || key == "example") d.test_case = lowercase(val);
        else if (key == "particles_per_cell_pair" || key == "particles_per_cell" ||
                 key == "velocity_samples_per_cell") ss >> d.particles_per_cell_pair;
        else if (key == "spline_order") ss >> d.spline_order;
        else if (key == "orbit_quad_order") ss >> d.orbit_quad_order;
        else if (key == "split_orbit_at_knots") d.split_orbit_at_knots = parse_bool(val);
        else if (key == "picard_tol") ss >> d.picard_tol;
        else if (key == "picard_max_iter") ss >> d.picard_max_iter;
        else if (key == "final_consistency_sweep") d.final_consistency_sweep = parse_bool(val);
        else if (key == "run_unit_tests") d.run_unit_tests = parse_bool(val);
        else if (key == "c") ss >> d.c;
        else if (key == "eps0") ss >> d.eps0;
        else if (key == "mu0") ss >> d.mu0;
        else if (key == "n0") ss >> d.n0;
        else if (key == "v0") ss >> d.v0;
        else if (key == "perturbation") ss >> d.perturbation;
        else if (key == "landau_alpha" || key == "landau_density_perturbation") ss >> d.landau_alpha;
        else if (key == "thermal_velocity" || key == "vth") ss >> d.thermal_velocity;
        else if (key == "perturbation_mode") ss >> d.perturbation_mode;
        else if (key == "theory_omega" || key == "landau_theory_omega") ss >> d.theory_omega;
        else if (key == "theory_gamma" || key == "landau_theory_gamma") ss >> d.theory_gamma;
        else if (key == "seed") ss >> d.seed;
        else if (key == "output_prefix") d.output_prefix = val;
        else std::cerr << "warning: unknown input key ignored: " << key << "\n";
    }
    return d;
}

bool is_landau(const NonrelDeck& d) {
    const std::string& t = d.test_case;
    return t == "landau" || t == "landau_weak" || t == "landau_strong" || t == "weak_landau" ||
           t == "strong_landau";
}

bool is_two_stream(const NonrelDeck& d) {
    const std::string& t = d.test_case;
    return t == "two_stream" || t == "two-stream" || t == "twostream";
}

double landau_amplitude(const NonrelDeck& d) { return d.landau_alpha >= 0.0 ? d.landau_alpha : d.perturbation; }

// Periodic wrap into [-L/2, L/2) (wrap1 :160).
double wrap_centered(double x, double L) {
    double y = std::fmod(x + 0.5 * L, L);
    if (y < 0.0) y += L;
    return y - 0.5 * L;
}

// Cell centres of an n-cell axis, shifted to [-L/2, L/2) when centered
// (cell_centered_grid :1091).
std::vector<double> cell_centres(int n, double L, bool centered) {
    std::vector<double> x(n);
    const double h = L / (double)n;
    for (int i = 0; i < n; ++i) {
        x[i] = ((double)i + 0.5) * h;
        if (centered) x[i] -= 0.5 * L;
    }
    return x;
}

// Inverse standard-normal CDF by P. J. Acklam's rational approximation
// (the published algorithm: a central rational function in p - 1/2 and two
// tail rational functions in sqrt(-2 log p), switching at p = 0.02425),
// which normal_quantile (:1103) uses for the Landau quiet start.
double inverse_normal_cdf(double p) {
    if (!(p > 0.0 && p < 1.0)) throw std::runtime_error("normal_quantile requires 0<p<1");
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    const double p_low = 0.02425;
    auto tail = [&](double t) {
        const double num = ((((c[0] * t + c[1]) * t + c[2]) * t + c[3]) * t + c[4]) * t + c[5];
        const double den = (((d[0] * t + d[1]) * t + d[2]) * t + d[3]) * t + 1.0;
        return num / den;
    };
    if (p < p_low) return tail(std::sqrt(-2.0 * std::log(p)));
    if (p > 1.0 - p_low) return -tail(std::sqrt(-2.0 * std::log(1.0 - p)));
    const double u = p - 0.5, r = u * u;
    const double num = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * u;
    const double den = ((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0;
    return num / den;
}

// Particles in the ABI layout: positions, v as xyz triples, q, m (z is the
// nz = 1 plane's centre, 0, and stays there: these loads have vz = 0).
struct Loaded {
    std::vector<double> x, y, v, q, m;
    long size() const { return (long)x.size(); }
};

// Cold counter-streaming beams along x with a sine velocity seed
// (initialize_two_stream_3d_linear_x :1151): nx*ppc beam positions per line,
// every (y, z) cell line, beam +v0 first, then -v0.
Loaded two_stream(const NonrelDeck& d) {
    const std::vector<double> xl = cell_centres(d.nx * d.particles_per_cell_pair, d.Lx, true);
    const std::vector<double> yl = cell_centres(d.ny, d.Ly, true);
    const std::vector<double> zl = cell_centres(d.nz, d.Lz, true);
    std::vector<double> bx, by;
    for (double y : yl)
        for (size_t iz = 0; iz < zl.size(); ++iz)
            for (double x : xl) {
                bx.push_back(x);
                by.push_back(y);
            }
    const size_t nb = bx.size(), np = 2 * nb;
    Loaded L;
    L.x.resize(np);
    L.y.resize(np);
    L.v.assign(3 * np, 0.0);
    const double k = 2.0 * kPi * (double)d.perturbation_mode / d.Lx;
    for (size_t p = 0; p < nb; ++p) {
        const double seed_v = d.perturbation * std::sin(k * bx[p]);
        for (size_t beam = 0; beam < 2; ++beam) {
            const size_t i = beam * nb + p;
            L.x[i] = wrap_centered(bx[p], d.Lx);
            L.y[i] = wrap_centered(by[p], d.Ly);
            L.v[3 * i] = (beam == 0 ? +d.v0 : -d.v0) + seed_v;
        }
    }
    const double volume = d.Lx * d.Ly * d.Lz;
    const double qm = -d.n0 * volume / (double)np;
    L.q.assign(np, qm);
    L.m.assign(np, std::fabs(qm));
    return L;
}

// Landau quiet start (initialize_landau_damping_1d3d :1214): per cell the nv
// velocities v_th * Phi^-1((j + 1/2)/nv), macro-charge q0 (1 + alpha cos kx),
// m = |q|.
Loaded landau(const NonrelDeck& d) {
    const int nv = d.particles_per_cell_pair;
    if (nv < 2) throw std::runtime_error("Landau examples need at least two velocity samples per cell");
    const double alpha = landau_amplitude(d);
    if (std::fabs(alpha) >= 1.0)
        throw std::runtime_error(
            "Landau density amplitude must satisfy |alpha| < 1 so all macro weights stay positive");
    const std::vector<double> xl = cell_centres(d.nx, d.Lx, true);
    const std::vector<double> yl = cell_centres(d.ny, d.Ly, true);
    const std::vector<double> zl = cell_centres(d.nz, d.Lz, true);
    std::vector<double> vq(nv);
    for (int j = 0; j < nv; ++j) vq[j] = d.thermal_velocity * inverse_normal_cdf(((double)j + 0.5) / (double)nv);
    const size_t np = (size_t)d.nx * d.ny * d.nz * nv;
    const double k = 2.0 * kPi * (double)d.perturbation_mode / d.Lx;
    const double q0 = -d.n0 * (d.Lx * d.Ly * d.Lz) / (double)np;
    Loaded L;
    L.x.reserve(np);
    for (double y : yl)
        for (size_t iz = 0; iz < zl.size(); ++iz)
            for (double x : xl) {
                const double weight = 1.0 + alpha * std::cos(k * x);
                for (int j = 0; j < nv; ++j) {
                    L.x.push_back(wrap_centered(x, d.Lx));
                    L.y.push_back(wrap_centered(y, d.Ly));
                    L.v.push_back(vq[j]);
                    L.v.push_back(0.0);
                    L.v.push_back(0.0);
                    L.q.push_back(q0 * weight);
                    L.m.push_back(std::fabs(q0 * weight));
                }
            }
    return L;
}

Loaded initial_particles(const NonrelDeck& d) {
    if (is_two_stream(d)) return two_stream(d);
    if (is_landau(d)) return landau(d);
    throw std::runtime_error("unknown test_case/initial_condition: " + d.test_case);
}

void check(int rc, const upic_ctx* ctx) {
    if (rc != UPIC_OK) throw std::runtime_error(upic_last_error(ctx));
}

upic_config abi_config(const NonrelDeck& d) {
    upic_config uc;
    upic_config_default(&uc);
    uc.method = UPIC_METHOD_CN_ORBIT_NONREL;
    uc.nx = d.nx;
    uc.ny = d.ny;
    uc.Lx = d.Lx;
    uc.Ly = d.Ly;
    uc.Lz = d.Lz;
    uc.dt = d.dt;
    uc.c = d.c;
    uc.eps0 = d.eps0;
    uc.mu0 = d.mu0;
    uc.n0 = d.n0;
    uc.spline_order = d.spline_order;
    uc.orbit_quad_order = d.orbit_quad_order;
    uc.split_orbit_at_knots = d.split_orbit_at_knots ? 1 : 0;
    uc.picard_tol = d.picard_tol;
    uc.picard_max_iter = d.picard_max_iter;
    uc.final_consistency_sweep = d.final_consistency_sweep ? 1 : 0;
    uc.perturbation_mode = d.perturbation_mode;
    return uc;
}

// A context that is destroyed on scope exit.
struct Ctx {
    upic_ctx* c = nullptr;
    explicit Ctx(const upic_config& uc) {
        if (upic_create(&uc, &c) != UPIC_OK) throw std::runtime_error(upic_last_error(nullptr));
    }
    ~Ctx() { upic_destroy(c); }
    Ctx(const Ctx&) = delete;
    Ctx& operator=(const Ctx&) = delete;
};

void load(Ctx& ctx, const Loaded& L) {
    const long n = L.size();
    std::vector<double> P(3 * n, 0.0);
    check(upic_set_particles(ctx.c, n, L.x.data(), L.y.data(), P.data(), L.v.data(), L.v.data(), L.q.data(),
                             L.m.data()), ctx.c);
}

double rms(const std::vector<double>& a) {
    long double s = 0.0L;
    for (double v : a) s += (long double)v * (long double)v;
    return std::sqrt((double)(s / (long double)std::max<size_t>(1, a.size())));
}

// R = A^{n+1}(x1) - A^n(x0) - dt (<U_mid> + D_A vbar) per orbit
// (compute_RA_orbit_residual :1330) from the library's orbit gathers: the
// point values are orbit averages over zero-length orbits.
struct RA {
    std::vector<double> R, dA, rhs;
};

RA ra_residual(Ctx& ctx, const std::vector<double>& x0, const std::vector<double>& y0,
               const std::vector<double>& vbar, const std::vector<double>& A0, const std::vector<double>& A1,
               const std::vector<double>& U, double dt, double Lx, double Ly) {
    const long n = (long)x0.size();
    std::vector<double> dx(3 * n), zero(3 * n, 0.0), x1(n), y1(n);
    for (long p = 0; p < n; ++p) {
        for (int k = 0; k < 3; ++k) dx[3 * p + k] = dt * vbar[3 * p + k];
        x1[p] = wrap_centered(x0[p] + dx[3 * p], Lx);
        y1[p] = wrap_centered(y0[p] + dx[3 * p + 1], Ly);
    }
    std::vector<double> Ub(3 * n), D(9 * n), A0p(3 * n), A1p(3 * n), scratch(9 * n);
    check(upic_orbit_gather(ctx.c, n, x0.data(), y0.data(), dx.data(), U.data(), A0.data(), A1.data(), Ub.data(),
                            D.data()), ctx.c);
    check(upic_orbit_gather(ctx.c, n, x0.data(), y0.data(), zero.data(), A0.data(), A0.data(), A0.data(),
                            A0p.data(), scratch.data()), ctx.c);
    check(upic_orbit_gather(ctx.c, n, x1.data(), y1.data(), zero.data(), A1.data(), A1.data(), A1.data(),
                            A1p.data(), scratch.data()), ctx.c);
    RA r;
    r.R.resize(3 * n);
    r.dA.resize(3 * n);
    r.rhs.resize(3 * n);
    for (long p = 0; p < n; ++p)
        for (int a = 0; a < 3; ++a) {
            const double* g = &D[9 * p + 3 * a];
            const double Dv = g[0] * vbar[3 * p] + g[1] * vbar[3 * p + 1] + g[2] * vbar[3 * p + 2];
            r.dA[3 * p + a] = A1p[3 * p + a] - A0p[3 * p + a];
            r.rhs[3 * p + a] = dt * (Ub[3 * p + a] + Dv);
            r.R[3 * p + a] = r.dA[3 * p + a] - r.rhs[3 * p + a];
        }
    return r;
}

// Distinct knot-crossing times of one orbit in x and y
// (path_breakpoints_for_particle :782); returns the segment count.
int segments(double x0, double y0, double dxx, double dxy, int nx, int ny, double Lx, double Ly, int order) {
    std::vector<double> b;
    const double off = 0.5 * (double)(order - 1);
    const double xs[2] = {x0, y0}, ds[2] = {dxx, dxy}, Ls[2] = {Lx, Ly};
    const int ns[2] = {nx, ny};
    for (int k = 0; k < 2; ++k) {
        const double h = Ls[k] / ns[k];
        const double u0 = (wrap_centered(xs[k], Ls[k]) + 0.5 * Ls[k]) / h;
        const double du = ds[k] / h;
        if (std::fabs(du) < 1.0e-300) continue;
        const double a0 = u0 - off, a1 = a0 + du;
        const long long first = (long long)std::floor(std::min(a0, a1)) + 1;
        const long long last = (long long)std::ceil(std::max(a0, a1)) - 1;
        for (long long m = first; m <= last; ++m) {
            const double s = ((double)m - a0) / du;
            if (s > 1.0e-13 && s < 1.0 - 1.0e-13) b.push_back(s);
        }
    }
    std::sort(b.begin(), b.end());
    int distinct = 0;
    double last_s = -1.0;
    for (double s : b)
        if (distinct == 0 || std::fabs(s - last_s) > 1.0e-12) {
            ++distinct;
            last_s = s;
        }
    return distinct + 1;
}

void random_fields(std::mt19937_64& rng, std::normal_distribution<double>& normal, int N, double dt,
                   std::vector<double>& A0, std::vector<double>& U, std::vector<double>& A1) {
    A0.assign(3 * N, 0.0);
    U.assign(3 * N, 0.0);
    A1.assign(3 * N, 0.0);
    for (int m = 0; m < 3; ++m)
        for (int id = 0; id < N; ++id) {
            A0[m * N + id] = normal(rng);
            U[m * N + id] = normal(rng);
            A1[m * N + id] = A0[m * N + id] + dt * U[m * N + id];
        }
}

NonrelDeck unit_deck(int n, double dt, int order, int nq) {
    NonrelDeck t;
    t.nx = t.ny = n;
    t.nz = 1;
    t.Lx = t.Ly = t.Lz = 2.0 * kPi;
    t.dt = dt;
    t.spline_order = order;
    t.orbit_quad_order = nq;
    return t;
}

// The four start-up tests of the reference (:1556-1713) in 2D.
bool unit_tests(std::ostream& os) {
    bool ok = true;
    os << std::scientific << std::setprecision(6);
    {   // test_RA_orbit_chain_rule (:1556)
        const NonrelDeck t = unit_deck(8, 0.01, 2, 20);
        Ctx ctx(abi_config(t));
        std::mt19937_64 rng(11);
        std::normal_distribution<double> normal(0.0, 1.0);
        std::uniform_int_distribution<int> cell(0, t.nx - 1);
        const int np = 128;
        const double h = t.Lx / t.nx;
        std::vector<double> x0(np), y0(np), vb(3 * np);
        for (int p = 0; p < np; ++p) {
            const int ix = cell(rng), iy = cell(rng);
            (void)cell(rng);  // the z cell of the 3D test
            x0[p] = -0.5 * t.Lx + (ix + 0.31) * h;
            y0[p] = -0.5 * t.Ly + (iy + 0.37) * h;
            for (int k = 0; k < 3; ++k) vb[3 * p + k] = 0.03 * normal(rng);
        }
        std::vector<double> A0, U, A1;
        random_fields(rng, normal, t.nx * t.ny, t.dt, A0, U, A1);
        const RA r = ra_residual(ctx, x0, y0, vb, A0, A1, U, t.dt, t.Lx, t.Ly);
        const double abs_rms = rms(r.R), rel_rms = abs_rms / (0.5 * (rms(r.dA) + rms(r.rhs)) + 1.0e-300);
        os << "R_A,p chain-rule unit test: abs_rms=" << abs_rms << " rel_rms=" << rel_rms << "\n";
        if (!(abs_rms < 5.0e-12 && rel_rms < 5.0e-10)) {
            os << "FAILED: R_A,p residual is too large\n";
            ok = false;
        }
    }
    {   // test_RA_orbit_chain_rule_with_crossings (:1604)
        NonrelDeck t = unit_deck(8, 1.0, 1, 16);
        const int np = 96;
        const double h = t.Lx / t.nx;
        std::vector<double> x0(np), y0(np), vb(3 * np);
        for (int p = 0; p < np; ++p) {
            const int ix = p % t.nx, iy = (p / t.nx) % t.ny;
            const double sx = (p % 2 == 0) ? 0.49 : -0.49;
            const double sy = ((p / 2) % 2 == 0) ? 0.45 : -0.45;
            const double sz = ((p / 4) % 2 == 0) ? 0.42 : -0.42;
            x0[p] = -0.5 * t.Lx + (ix + 0.5 + sx) * h;
            y0[p] = -0.5 * t.Ly + (iy + 0.5 + sy) * h;
            vb[3 * p] = 0.35 * h * (sx > 0.0 ? 1.0 : -1.0);
            vb[3 * p + 1] = 0.25 * h * (sy > 0.0 ? 1.0 : -1.0);
            vb[3 * p + 2] = 0.20 * h * (sz > 0.0 ? 1.0 : -1.0);
        }
        std::mt19937_64 rng(17);
        std::normal_distribution<double> normal(0.0, 1.0);
        std::vector<double> A0, U, A1;
        random_fields(rng, normal, t.nx * t.ny, t.dt, A0, U, A1);
        double split_abs, unsplit_abs;
        {
            Ctx ctx(abi_config(t));
            split_abs = rms(ra_residual(ctx, x0, y0, vb, A0, A1, U, t.dt, t.Lx, t.Ly).R);
        }
        t.split_orbit_at_knots = false;
        {
            Ctx ctx(abi_config(t));
            unsplit_abs = rms(ra_residual(ctx, x0, y0, vb, A0, A1, U, t.dt, t.Lx, t.Ly).R);
        }
        long crossing = 0;
        int max_seg = 1;
        for (int p = 0; p < np; ++p) {
            // the reference passes vbar itself as the path (dt = 1)
            const int ns = segments(x0[p], y0[p], vb[3 * p], vb[3 * p + 1], t.nx, t.ny, t.Lx, t.Ly, 1);
            crossing += ns > 1;
            max_seg = std::max(max_seg, ns);
        }
        os << "R_A,p crossing unit test: split_abs_rms=" << split_abs << " unsplit_abs_rms=" << unsplit_abs
           << " crossing_particles=" << crossing << " max_segments=" << max_seg << "\n";
        if (!(split_abs < 5.0e-12 && unsplit_abs > 1.0e-10 && crossing > 0)) {
            os << "FAILED: split-path crossing test did not behave as expected\n";
            ok = false;
        }
    }
    {   // test_initial_gauss_law (:1660)
        NonrelDeck t = unit_deck(8, 0.00625, 2, 16);
        t.particles_per_cell_pair = 2;
        Ctx ctx(abi_config(t));
        load(ctx, two_stream(t));
        double row[UPIC_P3_DIAG_COUNT];
        check(upic_init_fields(ctx.c, row), ctx.c);
        os << "Initial Gauss-law unit test: gauss_rms=" << row[UPIC_P3_GAUSS_RMS] << "\n";
        if (!(row[UPIC_P3_GAUSS_RMS] < 5.0e-11)) {
            os << "FAILED: initial Gauss residual is too large\n";
            ok = false;
        }
    }
    {   // test_one_step_gauss_law_and_RA (:1680)
        NonrelDeck t = unit_deck(4, 0.00625, 2, 16);
        t.particles_per_cell_pair = 2;
        Ctx ctx(abi_config(t));
        load(ctx, two_stream(t));
        check(upic_init_fields(ctx.c, nullptr), ctx.c);
        double row[UPIC_P3_DIAG_COUNT], info[UPIC_INFO_COUNT], sd[UPIC_SD_COUNT];
        check(upic_step_implicit(ctx.c, 1, row, info, sd), ctx.c);
        os << "One-step Gauss-law unit test: gauss_rms=" << row[UPIC_P3_GAUSS_RMS] << "\n"
           << "One-step R_A,p unit test: A_chain_abs_rms=" << sd[UPIC_SD_A_CHAIN_ABS_RMS] << "\n"
           << "One-step deposit/gather work residual=" << sd[UPIC_SD_DEPOSIT_GATHER_WORK_RESIDUAL] << "\n";
        if (!(row[UPIC_P3_GAUSS_RMS] < 5.0e-10 && sd[UPIC_SD_A_CHAIN_ABS_RMS] < 5.0e-10)) {
            os << "FAILED: one-step Gauss or R_A,p test failed\n";
            ok = false;
        }
    }
    return ok;
}

// The Diagnostics columns of compute_diagnostics (:1057) in the library row.
const int kDiagCols[11] = {UPIC_P3_GAUSS_RMS,    UPIC_P3_GAUSS_MAX,      UPIC_P3_GAUGE_RMS, UPIC_P3_FIELD_ENERGY,
                           UPIC_P3_KINETIC_ENERGY, UPIC_P3_TOTAL_ENERGY, UPIC_P3_RHO_MODE,  UPIC_P3_E_MODE_RE,
                           UPIC_P3_E_MODE_IM,    UPIC_P3_E_MODE_ABS,     UPIC_P3_MEAN_RHO};

}  // namespace

int run_nonrel(const std::string& path) {
    const NonrelDeck d = read_deck(path);
    if (!pow2(d.nx) || !pow2(d.ny) || !pow2(d.nz))
        throw std::runtime_error("the in-file radix-2 FFT requires nx, ny, nz to be powers of two");
    if (d.nz != 1) throw std::runtime_error("this build runs 2D and 1D decks only (nz = 1)");

    std::cout << "B200 orbit-discrete-gradient Picard CN potential PIC (UPIC_METHOD_CN_ORBIT_NONREL)\n";
    std::cout << "test_case = " << d.test_case << "\n";
    std::cout << "grid = " << d.nx << " x " << d.ny << " x " << d.nz << ", dt = " << d.dt
              << ", steps = " << d.n_steps << "\n";

    std::ofstream unit_log(d.output_prefix + "_unit_tests.txt");
    if (d.run_unit_tests) {
        std::ostringstream log;
        const bool ok = unit_tests(log);
        std::cout << log.str();
        unit_log << log.str();
        if (!ok) {
            std::cerr << "one or more unit tests failed\n";
            return 3;
        }
        std::cout << "Unit tests passed.\n";
    }

    const Loaded L = initial_particles(d);
    const long np = L.size();
    {   // write_config_echo (:1730)
        std::ofstream out(d.output_prefix + "_config_echo.txt");
        const double dV = (d.Lx / d.nx) * (d.Ly / d.ny) * (d.Lz / d.nz);
        out << "test_case=" << d.test_case << "\n" << "nx=" << d.nx << "\n" << "ny=" << d.ny << "\n"
            << "nz=" << d.nz << "\n" << std::setprecision(17) << "Lx=" << d.Lx << "\n" << "Ly=" << d.Ly << "\n"
            << "Lz=" << d.Lz << "\n" << "n_steps=" << d.n_steps << "\n" << "dt=" << d.dt << "\n"
            << "particles=" << np << "\n"
            << "particles_per_cell_pair_or_velocity_samples=" << d.particles_per_cell_pair << "\n"
            << "spline_order=" << d.spline_order << "\n" << "orbit_quad_order=" << d.orbit_quad_order << "\n"
            << "split_orbit_at_knots=" << (d.split_orbit_at_knots ? "true" : "false") << "\n"
            << "picard_tol=" << d.picard_tol << "\n" << "picard_max_iter=" << d.picard_max_iter << "\n"
            << "final_consistency_sweep=" << (d.final_consistency_sweep ? "true" : "false") << "\n"
            << "c=" << d.c << "\n" << "eps0=" << d.eps0 << "\n" << "mu0=" << d.mu0 << "\n" << "n0=" << d.n0 << "\n"
            << "v0=" << d.v0 << "\n" << "perturbation=" << d.perturbation << "\n"
            << "landau_alpha=" << landau_amplitude(d) << "\n" << "thermal_velocity=" << d.thermal_velocity << "\n"
            << "perturbation_mode=" << d.perturbation_mode << "\n" << "theory_omega=" << d.theory_omega << "\n"
            << "theory_gamma=" << d.theory_gamma << "\n" << "dV=" << dV << "\n";
    }

    Ctx ctx(abi_config(d));
    load(ctx, L);
    double row[UPIC_P3_DIAG_COUNT], info[UPIC_INFO_COUNT], sd[UPIC_SD_COUNT];
    check(upic_init_fields(ctx.c, row), ctx.c);
    const double theory_E0 = row[UPIC_P3_E_MODE_ABS];
    const bool theory = (std::fabs(d.theory_gamma) > 0.0 || std::fabs(d.theory_omega) > 0.0) && theory_E0 > 0.0;

    std::ofstream diag(d.output_prefix + "_diagnostics.csv");
    diag << "step,time,gauss_rms,gauss_max,gauge_rms,field_energy,kinetic_energy,total_energy,"
         << "rho_mode,E_mode_re,E_mode_im,E_mode_abs,theory_E_abs,E_over_theory,mean_rho,"
         << "picard_iterations,picard_current_error,picard_velocity_error,"
         << "crossing_particles,avg_path_segments,max_path_segments\n";
    std::ofstream stepcsv(d.output_prefix + "_step_diagnostics.csv");
    stepcsv << "step,time,A_chain_abs_rms,A_chain_rel_rms,A_chain_max_norm,A_chain_mean_norm,A_chain_work_defect,"
               "delta_K,delta_W,delta_total_energy,particle_work,grid_work,deposit_gather_work_residual,"
               "particle_energy_residual,field_energy_residual,crossing_particles,total_crossings,"
               "avg_path_segments,max_path_segments\n";
    // one _diagnostics.csv row (the write_diag lambda of main)
    auto write_diag = [&](int step, double time, const double* r, int iters, double cur, double vel, long cross,
                          double avg, long maxseg) {
        double th = kNaN, ratio = kNaN;
        if (theory) {
            th = theory_E0 * std::exp(d.theory_gamma * time);
            ratio = r[UPIC_P3_E_MODE_ABS] / (th + 1.0e-300);
        }
        diag << step << "," << std::setprecision(17) << time;
        for (int k = 0; k < 10; ++k) diag << "," << r[kDiagCols[k]];
        diag << "," << th << "," << ratio << "," << r[UPIC_P3_MEAN_RHO] << "," << iters << "," << cur << ","
             << vel << "," << cross << "," << avg << "," << maxseg << "\n";
    };
    write_diag(0, 0.0, row, 0, kNaN, kNaN, 0, 0.0, 1);

    for (int n = 0; n < d.n_steps; ++n) {
        check(upic_step_implicit(ctx.c, 1, row, info, sd), ctx.c);
        const double time = (n + 1) * d.dt;
        const int iters = (int)info[UPIC_INFO_ITERATIONS];
        write_diag(n + 1, time, row, iters, info[UPIC_INFO_CURRENT_ERROR], info[UPIC_INFO_VELOCITY_ERROR],
                   (long)info[UPIC_INFO_CROSSING_PARTICLES], info[UPIC_INFO_AVG_PATH_SEGMENTS],
                   (long)info[UPIC_INFO_MAX_PATH_SEGMENTS]);
        stepcsv << (n + 1) << "," << std::setprecision(17) << time;
        for (int k = 0; k < UPIC_SD_COUNT; ++k) {
            const bool integer = k == UPIC_SD_CROSSING_PARTICLES || k == UPIC_SD_TOTAL_CROSSINGS ||
                                 k == UPIC_SD_MAX_PATH_SEGMENTS;
            if (integer) stepcsv << "," << (long)sd[k];
            else stepcsv << "," << sd[k];
        }
        stepcsv << "\n";
        if ((n + 1) % std::max(1, d.n_steps / 5) == 0 || n == d.n_steps - 1) {
            std::cout << std::scientific << std::setprecision(3) << "step " << std::setw(5) << (n + 1) << "/"
                      << d.n_steps << " Gauss=" << row[UPIC_P3_GAUSS_RMS] << " R_A=" << sd[UPIC_SD_A_CHAIN_ABS_RMS]
                      << " dE=" << sd[UPIC_SD_DELTA_TOTAL_ENERGY]
                      << " crossings=" << (long)sd[UPIC_SD_TOTAL_CROSSINGS] << " Picard=" << iters << "\n";
        }
    }

    {   // write_particle_sample (:1716), at most 20000 evenly spaced particles
        std::vector<double> x(np), y(np), P(3 * np), v(3 * np), vp(3 * np);
        check(upic_get_particles(ctx.c, np, x.data(), y.data(), P.data(), v.data(), vp.data()), ctx.c);
        std::ofstream out(d.output_prefix + "_particle_sample.csv");
        out << "particle,x,y,z,vx,vy,vz,q,m\n";
        const size_t nw = std::min<size_t>(20000, (size_t)np);
        for (size_t r = 0; r < nw; ++r) {
            const size_t p = nw == 1 ? 0 : r * ((size_t)np - 1) / (nw - 1);
            out << p << "," << std::setprecision(17) << x[p] << "," << y[p] << "," << 0.0 << "," << v[3 * p] << ","
                << v[3 * p + 1] << "," << v[3 * p + 2] << "," << L.q[p] << "," << L.m[p] << "\n";
        }
    }
    std::cout << std::scientific << std::setprecision(6) << "Final Gauss RMS = " << row[UPIC_P3_GAUSS_RMS] << "\n"
              << "Final gauge RMS = " << row[UPIC_P3_GAUGE_RMS] << "\n"
              << "Final total energy = " << row[UPIC_P3_TOTAL_ENERGY] << "\n";
    return 0;
}
