// upic_run --p3: deck-driven drop-in for the reference's relativistic
// implicit solver CLI (Project3/ec_pic_nyquist_projected.cpp `main:8336`):
// reads the same `key = value` deck (read_config :1178-1433, with its aliases,
// validation and warnings), builds the same two-stream, Weibel or Landau
// start (initialize_state :4125 through upic_p3_initial_state), advances the
// GM-HC-CN step through the C ABI (UPIC_METHOD_CN_ORBIT) on the GPU with the
// reference's fixed-step loop (the last step shortened to the remaining
// time), and writes its output files in its formats:
//
//   _diagnostics.csv, _step_diagnostics.csv, _adaptive_diagnostics.csv,
//   _particle_inner_history.csv, _config_echo.txt, _unit_tests.txt,
//   _particle_sample.csv, _failed_particle_diagnostics.csv,
//   _field_line_probe.csv, _field_knot_jumps.csv, _field_grid_snapshots.csv,
//   _velocity_moments.csv, _field_spectrum.csv, _particles_t<time>.csv.
//
// Runs are 2D or 1D (nz = 1).  run_unit_tests runs 2D versions of six of the
// reference's start-up tests (orbit adjointness, initial and one-step Gauss
// law, multistep energy, instability set-up, two-stream eigenmode growth)
// with its sizes, messages and thresholds.  Failed-particle diagnostics keep
// the header only: the library reports a failing particle set by count and
// first index, not per particle.
//
// Exit codes as the reference: 0 ok, 1 error (message on stderr), 2 usage,
// 3 unit-test failure.
#include <algorithm>
#include <array>
#include <cctype>
#include <cfloat>
#include <chrono>
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
constexpr double kInf = std::numeric_limits<double>::infinity();

using Clock = std::chrono::steady_clock;

// Deck keys and defaults of the reference's Config (:837-1005).
struct P3Deck {
    int nx = 4, ny = 4, nz = 4;
    double Lx = 2.0 * kPi, Ly = 2.0 * kPi, Lz = 2.0 * kPi;
    int n_steps = 6;
    double dt = 0.00625;
    bool adaptive_dt = false;
    double adaptive_dt_min = 0.0, adaptive_dt_shrink = 0.5, adaptive_dt_growth = 2.0;
    int adaptive_dt_growth_interval = 4, adaptive_max_attempts = 4;
    std::string test_case = "cold_relativistic_two_stream";
    int particles_per_cell_pair = 4;
    int spline_order = 2;
    int orbit_quad_order = 16;
    bool split_orbit_at_knots = true;
    bool nyquist_projection = false;
    std::string nonlinear_solver = "anderson_quasi_newton";
    double nonlinear_rtol = 1.0e-12, nonlinear_atol = 1.0e-13;
    int nonlinear_max_iter = 32, anderson_memory = 4, anderson_start = 2;
    double anderson_damping = 0.7, anderson_regularization = 1.0e-12, anderson_growth_limit = 1.2;
    bool uniform_particle_subcycling = false, uniform_refine_on_failure = false;
    int uniform_initial_substeps = 1, uniform_substeps = 10, uniform_max_substeps = 20;
    double uniform_subcycling_start_time = 0.0;
    double uniform_local_rtol = 1.0e-11, uniform_local_atol = 1.0e-13;
    int uniform_local_max_iter = 24;
    double uniform_local_damping = 1.0;
    bool selective_particle_fallback = false;
    int selective_particle_max_substeps = 64, selective_particle_dynamic_chunk = 4;
    bool selective_failure_diagnostics = true;
    int selective_failure_diagnostic_limit = 16;
    bool field_diagnostics = true;
    double field_diagnostics_interval = 10.0;
    int field_probe_points_per_cell = 32;
    std::string field_probe_axis = "auto";
    bool field_grid_snapshots = false;
    std::vector<double> particle_snapshot_times;
    bool run_unit_tests = true;
    double kappa = 1.0, sigma1 = 1.0, sigma2 = 1.0;
    double n0 = 1.0, v0 = 0.3, perturbation = 0.02, two_stream_density_alpha = -1.0;
    bool two_stream_eigenmode = true, two_stream_finite_grid_theory = true;
    double weibel_B0 = -1.0;
    bool weibel_eigenmode = true, weibel_finite_grid_theory = true;
    double landau_alpha = -1.0, thermal_velocity = 1.0;
    int perturbation_mode = 1;
    double theory_omega = 0.0, theory_gamma = 0.0;
    bool transverse_diagnostics = false;
    double transverse_spectrum_interval = 1.0, tsi_transverse_seed = 0.0;
    int tsi_transverse_mode = 1;
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

bool is_two_stream(const std::string& tc) {
    static const char* names[] = {"two_stream", "two-stream", "twostream", "relativistic_two_stream",
                                  "relativistic-two-stream", "cold_relativistic_two_stream",
                                  "cold-relativistic-two-stream", "cold_two_stream", "cold-two-stream"};
    for (const char* n : names)
        if (tc == n) return true;
    return false;
}

bool is_weibel(const std::string& tc) {
    static const char* names[] = {"weibel", "relativistic_weibel", "relativistic-weibel", "cold_relativistic_weibel",
                                  "cold-relativistic-weibel", "filamentation", "cold_filamentation",
                                  "cold-filamentation"};
    for (const char* n : names)
        if (tc == n) return true;
    return false;
}

bool is_landau(const std::string& tc) {
    return tc == "landau" || tc == "landau_weak" || tc == "landau_strong" || tc == "weak_landau" ||
           tc == "strong_landau";
}

double effective_dt_min(const P3Deck& d) { return d.adaptive_dt_min > 0.0 ? d.adaptive_dt_min : d.dt / 16.0; }
double weibel_seed(const P3Deck& d) { return d.weibel_B0 >= 0.0 ? d.weibel_B0 : d.perturbation; }
double landau_amplitude(const P3Deck& d) { return d.landau_alpha >= 0.0 ? d.landau_alpha : d.perturbation; }

// read_config (:1178-1433): keys, aliases, warnings and checks in its order.
P3Deck read_deck(const std::string& path) {
    P3Deck d;
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
        auto is = [&](std::initializer_list<const char*> names) {
            for (const char* n : names)
                if (key == n) return true;
            return false;
        };
        if (is({"nx"})) ss >> d.nx;
        else if (is({"ny"})) ss >> d.ny;
        else if (is({"nz"})) ss >> d.nz;
        else if (is({"Lx"})) ss >> d.Lx;
        else if (is({"Ly"})) ss >> d.Ly;
        else if (is({"Lz"})) ss >> d.Lz;
        else if (is({"n_steps"})) ss >> d.n_steps;
        else if (is({"dt"})) ss >> d.dt;
        else if (is({"test_case", "initial_condition", "example"})) d.test_case = lowercase(val);
        else if (is({"particles_per_cell_pair", "particles_per_cell", "velocity_samples_per_cell"}))
            ss >> d.particles_per_cell_pair;
        else if (is({"spline_order"})) ss >> d.spline_order;
        else if (is({"orbit_quad_order"})) ss >> d.orbit_quad_order;
        else if (is({"split_orbit_at_knots"})) d.split_orbit_at_knots = parse_bool(val);
        else if (is({"nonlinear_solver"})) d.nonlinear_solver = lowercase(val);
        else if (is({"nonlinear_rtol", "nonlinear_tol", "picard_tol"})) ss >> d.nonlinear_rtol;
        else if (is({"nonlinear_atol"})) ss >> d.nonlinear_atol;
        else if (is({"nyquist_projection"})) d.nyquist_projection = parse_bool(val);
        else if (is({"nonlinear_max_iter", "picard_max_iter"})) ss >> d.nonlinear_max_iter;
        else if (is({"anderson_memory"})) ss >> d.anderson_memory;
        else if (is({"anderson_start"})) ss >> d.anderson_start;
        else if (is({"anderson_damping"})) ss >> d.anderson_damping;
        else if (is({"anderson_regularization"})) ss >> d.anderson_regularization;
        else if (is({"anderson_growth_limit"})) ss >> d.anderson_growth_limit;
        else if (is({"uniform_particle_subcycling", "uniform_subcycling"}))
            d.uniform_particle_subcycling = parse_bool(val);
        else if (is({"uniform_refine_on_failure", "particle_refine_on_failure"}))
            d.uniform_refine_on_failure = parse_bool(val);
        else if (is({"uniform_initial_substeps", "particle_initial_substeps"})) ss >> d.uniform_initial_substeps;
        else if (is({"uniform_substeps", "particle_substeps"})) ss >> d.uniform_substeps;
        else if (is({"uniform_max_substeps", "particle_max_substeps"})) ss >> d.uniform_max_substeps;
        else if (is({"uniform_subcycling_start_time", "particle_subcycling_start_time"}))
            ss >> d.uniform_subcycling_start_time;
        else if (is({"uniform_local_rtol", "particle_local_rtol"})) ss >> d.uniform_local_rtol;
        else if (is({"uniform_local_atol", "particle_local_atol"})) ss >> d.uniform_local_atol;
        else if (is({"uniform_local_max_iter", "particle_local_max_iter"})) ss >> d.uniform_local_max_iter;
        else if (is({"uniform_local_damping", "particle_local_damping"})) ss >> d.uniform_local_damping;
        else if (is({"selective_particle_fallback", "selective_subcycle_fallback"}))
            d.selective_particle_fallback = parse_bool(val);
        else if (is({"selective_particle_max_substeps", "selective_max_substeps"}))
            ss >> d.selective_particle_max_substeps;
        else if (is({"selective_particle_dynamic_chunk", "selective_dynamic_chunk"}))
            ss >> d.selective_particle_dynamic_chunk;
        else if (is({"selective_failure_diagnostics", "failed_particle_diagnostics"}))
            d.selective_failure_diagnostics = parse_bool(val);
        else if (is({"selective_failure_diagnostic_limit", "failed_particle_diagnostic_limit"}))
            ss >> d.selective_failure_diagnostic_limit;
        else if (is({"field_diagnostics", "write_field_diagnostics"})) d.field_diagnostics = parse_bool(val);
        else if (is({"field_diagnostics_interval", "field_output_interval"})) ss >> d.field_diagnostics_interval;
        else if (is({"field_probe_points_per_cell", "field_samples_per_cell"})) ss >> d.field_probe_points_per_cell;
        else if (is({"field_probe_axis"})) d.field_probe_axis = lowercase(val);
        else if (is({"field_grid_snapshots", "write_full_field_snapshots"})) d.field_grid_snapshots = parse_bool(val);
        else if (is({"particle_snapshot_times"})) {
            std::string times = val;
            std::replace(times.begin(), times.end(), ',', ' ');
            std::istringstream values(times);
            d.particle_snapshot_times.clear();
            double t;
            while (values >> t) {
                if (!std::isfinite(t) || t < 0.0)
                    throw std::runtime_error("particle_snapshot_times must be finite and nonnegative");
                d.particle_snapshot_times.push_back(t);
            }
            if (!values.eof()) throw std::runtime_error("invalid particle_snapshot_times list");
            std::sort(d.particle_snapshot_times.begin(), d.particle_snapshot_times.end());
            d.particle_snapshot_times.erase(
                std::unique(d.particle_snapshot_times.begin(), d.particle_snapshot_times.end()),
                d.particle_snapshot_times.end());
        } else if (is({"adaptive_dt", "adaptive_time_step", "adaptive_timestep", "adaptive_reject_on_unconverged"}))
            d.adaptive_dt = parse_bool(val);
        else if (is({"adaptive_dt_min", "dt_min"})) ss >> d.adaptive_dt_min;
        else if (is({"adaptive_dt_shrink", "dt_shrink"})) ss >> d.adaptive_dt_shrink;
        else if (is({"adaptive_dt_growth", "dt_growth"})) ss >> d.adaptive_dt_growth;
        else if (is({"adaptive_dt_growth_interval", "dt_growth_interval"})) ss >> d.adaptive_dt_growth_interval;
        else if (is({"adaptive_max_attempts", "max_step_attempts"})) ss >> d.adaptive_max_attempts;
        else if (is({"picard_relaxation", "picard_omega", "relaxed_picard_omega", "picard_relaxation_min",
                     "picard_omega_min", "picard_relaxation_shrink", "picard_relaxation_growth",
                     "picard_adaptive_relaxation", "adaptive_picard_relaxation", "picard_current_in_convergence",
                     "picard_converge_current", "final_consistency_sweep", "picard_require_converged",
                     "reject_unconverged_picard"}))
            std::cerr << "warning: obsolete Picard control ignored: " << key << "\n";
        else if (is({"adaptive_dt_max", "dt_max", "adaptive_max_accepted_steps", "max_accepted_steps",
                     "adaptive_energy_rtol", "energy_accept_rtol", "adaptive_finish_exactly"}))
            std::cerr << "warning: unsupported adaptive time-step control ignored: " << key << "\n";
        else if (is({"run_unit_tests"})) d.run_unit_tests = parse_bool(val);
        else if (is({"kappa"})) ss >> d.kappa;
        else if (is({"c"})) {
            ss >> d.kappa;
            std::cerr << "warning: c is deprecated; use kappa in the nondimensional paper notation\n";
        } else if (is({"sigma1"})) ss >> d.sigma1;
        else if (is({"sigma2"})) ss >> d.sigma2;
        else if (is({"eps0"})) {
            double eps0 = 1.0;
            ss >> eps0;
            d.sigma1 = 1.0 / eps0;
            std::cerr << "warning: eps0 is deprecated; use sigma1=1/eps0 in the nondimensional paper notation\n";
        } else if (is({"mu0"})) {
            ss >> d.sigma2;
            std::cerr << "warning: mu0 is deprecated; use sigma2 in the nondimensional paper notation\n";
        } else if (is({"n0", "rho0", "background_density"})) ss >> d.n0;
        else if (is({"v0"})) ss >> d.v0;
        else if (is({"perturbation"})) ss >> d.perturbation;
        else if (is({"two_stream_density_alpha", "density_perturbation", "alpha_x"})) ss >> d.two_stream_density_alpha;
        else if (is({"two_stream_eigenmode", "initialize_two_stream_eigenmode"}))
            d.two_stream_eigenmode = parse_bool(val);
        else if (is({"two_stream_finite_grid_theory"})) d.two_stream_finite_grid_theory = parse_bool(val);
        else if (is({"weibel_finite_grid_theory"})) d.weibel_finite_grid_theory = parse_bool(val);
        else if (is({"finite_grid_theory"})) {
            d.two_stream_finite_grid_theory = parse_bool(val);
            d.weibel_finite_grid_theory = parse_bool(val);
        } else if (is({"weibel_B0", "magnetic_perturbation", "initial_B0"})) ss >> d.weibel_B0;
        else if (is({"weibel_eigenmode", "initialize_weibel_eigenmode"})) d.weibel_eigenmode = parse_bool(val);
        else if (is({"landau_alpha", "landau_density_perturbation"})) ss >> d.landau_alpha;
        else if (is({"thermal_velocity", "vth"})) ss >> d.thermal_velocity;
        else if (is({"perturbation_mode"})) ss >> d.perturbation_mode;
        else if (is({"theory_omega", "landau_theory_omega"})) ss >> d.theory_omega;
        else if (is({"theory_gamma", "landau_theory_gamma"})) ss >> d.theory_gamma;
        else if (is({"transverse_diagnostics"})) d.transverse_diagnostics = parse_bool(val);
        else if (is({"transverse_spectrum_interval"})) ss >> d.transverse_spectrum_interval;
        else if (is({"tsi_transverse_seed"})) ss >> d.tsi_transverse_seed;
        else if (is({"tsi_transverse_mode"})) ss >> d.tsi_transverse_mode;
        else if (is({"seed"})) ss >> d.seed;
        else if (is({"output_prefix"})) d.output_prefix = val;
        else std::cerr << "warning: unknown input key ignored: " << key << "\n";
    }
    if (!std::isfinite(d.transverse_spectrum_interval) || !(d.transverse_spectrum_interval > 0.0) ||
        !std::isfinite(d.tsi_transverse_seed) || d.tsi_transverse_mode < 1)
        throw std::runtime_error("invalid transverse diagnostic interval or seed controls");
    if (d.tsi_transverse_seed != 0.0 &&
        (!is_two_stream(lowercase(d.test_case)) || d.ny < 3 || d.tsi_transverse_mode >= d.ny / 2))
        throw std::runtime_error("TSI transverse seed requires a two-stream case and 0<mode<ny/2");
    if (!(d.kappa > 0.0) || !(d.sigma1 > 0.0) || !(d.sigma2 > 0.0))
        throw std::runtime_error("nondimensional coefficients require kappa>0, sigma1>0, sigma2>0");
    if (!(d.dt > 0.0) || d.n_steps < 0) throw std::runtime_error("time stepping requires dt>0 and n_steps>=0");
    const double dt_min = effective_dt_min(d);
    if (!(dt_min > 0.0) || dt_min > d.dt || !(d.adaptive_dt_shrink > 0.0) || !(d.adaptive_dt_shrink < 1.0) ||
        !(d.adaptive_dt_growth > 1.0) || d.adaptive_dt_growth_interval < 1 || d.adaptive_max_attempts < 1)
        throw std::runtime_error(
            "adaptive controls require 0<dt_min<=dt, 0<dt_shrink<1, "
            "dt_growth>1, dt_growth_interval>=1, and adaptive_max_attempts>=1");
    if (d.nonlinear_solver != "picard" && d.nonlinear_solver != "anderson_quasi_newton")
        throw std::runtime_error("nonlinear_solver must be picard or anderson_quasi_newton");
    if (!(d.nonlinear_rtol > 0.0) || !(d.nonlinear_atol > 0.0) || d.nonlinear_max_iter <= 0)
        throw std::runtime_error("nonlinear controls require nonlinear_rtol>0, "
                                 "nonlinear_atol>0, and nonlinear_max_iter>0");
    if (d.anderson_memory < 1 || d.anderson_start < 0)
        throw std::runtime_error("Anderson controls require anderson_memory>=1 and anderson_start>=0");
    if (!(d.anderson_damping > 0.0) || !(d.anderson_damping <= 1.0))
        throw std::runtime_error("anderson_damping must satisfy 0 < damping <= 1");
    if (!(d.anderson_regularization >= 0.0) || !(d.anderson_growth_limit > 1.0))
        throw std::runtime_error("Anderson controls require regularization>=0 and growth_limit>1");
    if (d.uniform_initial_substeps < 1 || d.uniform_initial_substeps > d.uniform_substeps || d.uniform_substeps < 1 ||
        d.uniform_max_substeps < d.uniform_substeps || !(d.uniform_subcycling_start_time >= 0.0) ||
        !(d.uniform_local_rtol > 0.0) || !(d.uniform_local_atol > 0.0) || d.uniform_local_max_iter < 1 ||
        !(d.uniform_local_damping > 0.0) || !(d.uniform_local_damping <= 1.0))
        throw std::runtime_error(
            "uniform particle subcycling requires 1<=initial_substeps<=substeps<=max_substeps, "
            "start_time>=0, positive local "
            "rtol/atol/max_iter, and 0<local_damping<=1");
    if (d.selective_particle_max_substeps < 1 || d.selective_particle_max_substeps > 64 ||
        !pow2(d.selective_particle_max_substeps) || d.selective_particle_dynamic_chunk < 1 ||
        d.selective_failure_diagnostic_limit < 1)
        throw std::runtime_error(
            "selective particle fallback requires a power-of-two "
            "max_substeps in [1,64], dynamic_chunk>=1, and "
            "failure_diagnostic_limit>=1");
    if (d.selective_particle_fallback && d.uniform_particle_subcycling)
        throw std::runtime_error(
            "selective_particle_fallback and uniform_particle_subcycling "
            "cannot both be enabled");
    if (d.selective_particle_fallback && d.adaptive_dt)
        throw std::runtime_error(
            "selective_particle_fallback requires adaptive_dt=false so the "
            "macro dt remains fixed when the dt/max_substeps particle floor "
            "is exhausted");
    if (!(d.field_diagnostics_interval >= 0.0) || d.field_probe_points_per_cell < 2 ||
        (d.field_probe_axis != "auto" && d.field_probe_axis != "x" && d.field_probe_axis != "y" &&
         d.field_probe_axis != "z"))
        throw std::runtime_error(
            "field diagnostics require interval>=0, points_per_cell>=2, "
            "and field_probe_axis=auto, x, y, or z");
    const double compat = d.kappa * d.kappa * d.sigma2;
    const double rel = std::abs(d.sigma1 - compat) / std::max(1.0, std::abs(d.sigma1));
    if (rel > 1.0e-10) {
        std::ostringstream msg;
        msg << "Maxwell-compatible nondimensionalization requires sigma1 = kappa^2*sigma2; got sigma1=" << d.sigma1
            << ", kappa^2*sigma2=" << compat;
        throw std::runtime_error(msg.str());
    }
    return d;
}

void check(int rc, const upic_ctx* ctx) {
    if (rc != UPIC_OK) throw std::runtime_error(upic_last_error(ctx));
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

upic_config abi_config(const P3Deck& d) {
    upic_config uc;
    upic_config_default(&uc);
    uc.method = UPIC_METHOD_CN_ORBIT;
    uc.nx = d.nx;
    uc.ny = d.ny;
    uc.Lx = d.Lx;
    uc.Ly = d.Ly;
    uc.Lz = d.Lz;
    uc.dt = d.dt;
    uc.kappa = d.kappa;
    uc.sigma1 = d.sigma1;
    uc.sigma2 = d.sigma2;
    uc.n0 = d.n0;
    uc.spline_order = d.spline_order;
    uc.orbit_quad_order = d.orbit_quad_order;
    uc.split_orbit_at_knots = d.split_orbit_at_knots ? 1 : 0;
    uc.nyquist_projection = d.nyquist_projection ? 1 : 0;
    uc.nonlinear_solver = d.nonlinear_solver == "picard" ? UPIC_SOLVER_PICARD : UPIC_SOLVER_ANDERSON;
    uc.nonlinear_max_iter = d.nonlinear_max_iter;
    uc.anderson_memory = d.anderson_memory;
    uc.anderson_start = d.anderson_start;
    uc.local_max_iter = d.uniform_local_max_iter;
    uc.nonlinear_rtol = d.nonlinear_rtol;
    uc.nonlinear_atol = d.nonlinear_atol;
    uc.anderson_damping = d.anderson_damping;
    uc.anderson_regularization = d.anderson_regularization;
    uc.anderson_growth_limit = d.anderson_growth_limit;
    uc.local_rtol = d.uniform_local_rtol;
    uc.local_atol = d.uniform_local_atol;
    uc.local_damping = d.uniform_local_damping;
    uc.perturbation_mode = d.perturbation_mode;
    uc.selective_particle_fallback = d.selective_particle_fallback ? 1 : 0;
    uc.selective_particle_max_substeps = d.selective_particle_max_substeps;
    return uc;
}

// The deck's start (initialize_state :4125) from upic_p3_initial_state.
struct Start {
    std::vector<double> x, y, v, q, m, A, U;
    double growth = 0.0;
    long size() const { return (long)x.size(); }
};

upic_p3_case case_of(const P3Deck& d) {
    upic_p3_case c;
    upic_p3_case_default(&c);
    const std::string tc = lowercase(d.test_case);
    c.kind = is_two_stream(tc) ? UPIC_P3_TWO_STREAM : (is_weibel(tc) ? UPIC_P3_WEIBEL : UPIC_P3_LANDAU);
    c.nx = d.nx;
    c.ny = d.ny;
    c.Lx = d.Lx;
    c.Ly = d.Ly;
    c.Lz = d.Lz;
    c.kappa = d.kappa;
    c.sigma1 = d.sigma1;
    c.n0 = d.n0;
    c.spline_order = d.spline_order;
    c.perturbation_mode = d.perturbation_mode;
    c.particles_per_cell_pair = d.particles_per_cell_pair;
    c.v0 = d.v0;
    c.perturbation = d.perturbation;
    c.two_stream_density_alpha = d.two_stream_density_alpha;
    c.two_stream_eigenmode = d.two_stream_eigenmode ? 1 : 0;
    c.two_stream_finite_grid_theory = d.two_stream_finite_grid_theory ? 1 : 0;
    c.tsi_transverse_seed = d.tsi_transverse_seed;
    c.tsi_transverse_mode = d.tsi_transverse_mode;
    c.weibel_B0 = d.weibel_B0;
    c.weibel_eigenmode = d.weibel_eigenmode ? 1 : 0;
    c.weibel_finite_grid_theory = d.weibel_finite_grid_theory ? 1 : 0;
    c.landau_alpha = d.landau_alpha;
    c.thermal_velocity = d.thermal_velocity;
    return c;
}

Start initial_state(const P3Deck& d) {
    const std::string tc = lowercase(d.test_case);
    if (!is_two_stream(tc) && !is_weibel(tc) && !is_landau(tc))
        throw std::runtime_error("unknown test_case/initial_condition: " + d.test_case);
    if (is_landau(tc)) {
        if (d.particles_per_cell_pair < 2)
            throw std::runtime_error("Landau examples need at least two velocity samples per cell");
        if (std::abs(landau_amplitude(d)) >= 1.0)
            throw std::runtime_error(
                "Landau density amplitude must satisfy |alpha| < 1 so all macro weights stay positive");
    }
    const upic_p3_case c = case_of(d);
    const long np = upic_p3_case_particles(&c);
    if (np <= 0) throw std::runtime_error("the initial condition has no particles (particles_per_cell_pair)");
    Start s;
    s.x.resize(np);
    s.y.resize(np);
    s.v.resize(3 * np);
    s.q.resize(np);
    s.m.resize(np);
    const long N = (long)d.nx * d.ny;
    s.A.resize(3 * N);
    s.U.resize(3 * N);
    if (upic_p3_initial_state(&c, np, s.x.data(), s.y.data(), s.v.data(), s.q.data(), s.m.data(), s.A.data(),
                              s.U.data(), &s.growth) != UPIC_OK)
        throw std::runtime_error("the initial condition is invalid (stream speed, perturbation or seed mode)");
    for (long p = 0; p < np; ++p) {
        const double* v = &s.v[3 * p];
        if (!(std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) < d.kappa))
            throw std::runtime_error("relativistic initial velocity must satisfy |v| < kappa");
    }
    return s;
}

// A run on the library: particles loaded, potential set, fields started.
void start(Ctx& ctx, const Start& s, double* diag_row) {
    const long n = s.size();
    std::vector<double> P(3 * n, 0.0);
    check(upic_set_particles(ctx.c, n, s.x.data(), s.y.data(), P.data(), s.v.data(), s.v.data(), s.q.data(),
                             s.m.data()),
          ctx.c);
    check(upic_set_initial_potential(ctx.c, s.A.data(), s.U.data()), ctx.c);
    check(upic_init_fields(ctx.c, diag_row), ctx.c);
}

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

std::string wall_duration(double s) {
    const long ms = (long)std::llround(s * 1000.0);
    std::ostringstream o;
    o << std::setfill('0') << std::setw(2) << ms / 3600000 << ":" << std::setw(2) << (ms / 60000) % 60 << ":"
      << std::setw(2) << (ms / 1000) % 60 << "." << std::setw(3) << ms % 1000;
    return o.str();
}

// ---- start-up checks (run_unit_tests) ---------------------------------------
// 2D versions of the reference's tests with its sizes, seeds, messages and
// thresholds; nz = 1, so the z extents only set the cell volume.

P3Deck test_deck() {
    P3Deck d;
    d.run_unit_tests = false;
    d.field_diagnostics = false;
    return d;
}

// test_orbit_deposit_gather_adjointness (:6952): particle power q vbar.<E>
// against mesh power J.E dV for random orbits on an 8x8 grid.
bool test_adjoint(std::ostream& os) {
    P3Deck d = test_deck();
    d.nx = d.ny = 8;
    d.nz = 1;
    d.dt = 0.20;
    d.spline_order = 2;
    d.orbit_quad_order = 18;
    Ctx ctx(abi_config(d));
    std::mt19937_64 rng(23);
    std::uniform_real_distribution<double> uni(-0.5, 0.5);
    std::normal_distribution<double> normal(0.0, 1.0);
    const long np = 64;
    std::vector<double> x(np), y(np), dx(3 * np), vb(3 * np), q(np);
    for (long p = 0; p < np; ++p) {
        x[p] = d.Lx * uni(rng);
        y[p] = d.Ly * uni(rng);
        (void)uni(rng);
        vb[3 * p] = 0.35 * normal(rng);
        vb[3 * p + 1] = 0.20 * normal(rng);
        vb[3 * p + 2] = 0.15 * normal(rng);
        for (int c = 0; c < 3; ++c) dx[3 * p + c] = d.dt * vb[3 * p + c];
        q[p] = 0.1 * normal(rng);
    }
    const long N = (long)d.nx * d.ny;
    std::vector<double> E(3 * N), J(3 * N), gat(3 * np), grad(9 * np);
    for (double& e : E) e = normal(rng);
    // start a context state for the kernel-level calls (one cold particle)
    {
        std::vector<double> one{0.0}, v3{0.0, 0.0, 0.0}, P3{0.0, 0.0, 0.0}, qq{-1.0}, mm{1.0};
        check(upic_set_particles(ctx.c, 1, one.data(), one.data(), P3.data(), v3.data(), v3.data(), qq.data(),
                                 mm.data()),
              ctx.c);
        check(upic_init_fields(ctx.c, nullptr), ctx.c);
    }
    check(upic_orbit_gather(ctx.c, np, x.data(), y.data(), dx.data(), E.data(), E.data(), E.data(), gat.data(),
                            grad.data()),
          ctx.c);
    check(upic_orbit_deposit(ctx.c, np, x.data(), y.data(), dx.data(), vb.data(), q.data(), J.data()), ctx.c);
    long double particle = 0.0L, mesh = 0.0L;
    for (long p = 0; p < np; ++p)
        particle += (long double)q[p] *
                    (vb[3 * p] * gat[3 * p] + vb[3 * p + 1] * gat[3 * p + 1] + vb[3 * p + 2] * gat[3 * p + 2]);
    for (long k = 0; k < 3 * N; ++k) mesh += (long double)J[k] * E[k];
    const double dV = (d.Lx / d.nx) * (d.Ly / d.ny) * (d.Lz / d.nz);
    const double residual = (double)(particle - mesh * dV);
    const double scale = std::abs((double)particle) + std::abs((double)(mesh * dV)) + 1.0;
    os << std::scientific << std::setprecision(6) << "Orbit deposit/gather adjoint unit test: residual=" << residual
       << " rel=" << std::abs(residual) / scale << "\n";
    if (!(std::abs(residual) / scale < 5.0e-14)) {
        os << "FAILED: orbit scatter/gather work identity failed\n";
        return false;
    }
    return true;
}

P3Deck two_stream_test_deck(int n, int ppc) {
    P3Deck d = test_deck();
    d.test_case = "cold_relativistic_two_stream";
    d.nx = d.ny = n;
    d.nz = 1;
    d.dt = 0.00625;
    d.spline_order = 2;
    d.particles_per_cell_pair = ppc;
    return d;
}

// test_initial_gauss_law (:7150)
bool test_initial_gauss(std::ostream& os) {
    const P3Deck d = two_stream_test_deck(8, 2);
    Ctx ctx(abi_config(d));
    double row[UPIC_P3_DIAG_COUNT];
    start(ctx, initial_state(d), row);
    os << std::scientific << std::setprecision(6) << "Initial Gauss-law unit test: gauss_rms=" << row[UPIC_P3_GAUSS_RMS]
       << "\n";
    if (!(row[UPIC_P3_GAUSS_RMS] < 5.0e-11)) {
        os << "FAILED: initial Gauss residual is too large\n";
        return false;
    }
    return true;
}

// test_one_step_gauss_law_and_RA (:7185)
bool test_one_step(std::ostream& os) {
    P3Deck d = two_stream_test_deck(4, 2);
    d.orbit_quad_order = 16;
    d.nonlinear_rtol = 1.0e-11;
    d.nonlinear_max_iter = 16;
    Ctx ctx(abi_config(d));
    double row[UPIC_P3_DIAG_COUNT], info[UPIC_INFO_COUNT], sd[UPIC_SD_COUNT];
    start(ctx, initial_state(d), row);
    check(upic_step_implicit(ctx.c, 1, row, info, sd), ctx.c);
    os << std::scientific << std::setprecision(6) << "One-step Gauss-law unit test: gauss_rms=" << row[UPIC_P3_GAUSS_RMS]
       << "\n"
       << "One-step R_A,p unit test: A_chain_abs_rms=" << sd[UPIC_SD_A_CHAIN_ABS_RMS] << "\n"
       << "One-step deposit/gather work residual=" << sd[UPIC_SD_DEPOSIT_GATHER_WORK_RESIDUAL] << "\n"
       << "One-step particle-energy residual=" << sd[UPIC_SD_PARTICLE_ENERGY_RESIDUAL] << "\n"
       << "One-step field-energy residual=" << sd[UPIC_SD_FIELD_ENERGY_RESIDUAL] << "\n"
       << "One-step total-energy residual=" << sd[UPIC_SD_DELTA_TOTAL_ENERGY] << "\n";
    if (!(row[UPIC_P3_GAUSS_RMS] < 5.0e-10 && sd[UPIC_SD_A_CHAIN_ABS_RMS] < 5.0e-10 &&
          std::abs(sd[UPIC_SD_DEPOSIT_GATHER_WORK_RESIDUAL]) < 5.0e-13 &&
          std::abs(sd[UPIC_SD_PARTICLE_ENERGY_RESIDUAL]) < 5.0e-10 &&
          std::abs(sd[UPIC_SD_FIELD_ENERGY_RESIDUAL]) < 5.0e-10 && std::abs(sd[UPIC_SD_DELTA_TOTAL_ENERGY]) < 5.0e-10)) {
        os << "FAILED: one-step Gauss, R_A,p, work, or energy-balance test failed\n";
        return false;
    }
    return true;
}

// test_small_multistep_energy_conservation (:7238)
bool test_multistep(std::ostream& os) {
    P3Deck d = two_stream_test_deck(4, 2);
    d.orbit_quad_order = 16;
    d.nonlinear_rtol = 1.0e-11;
    d.nonlinear_max_iter = 16;
    d.two_stream_density_alpha = 0.01;
    d.perturbation = 0.0;
    Ctx ctx(abi_config(d));
    double row[UPIC_P3_DIAG_COUNT], info[UPIC_INFO_COUNT], sd[UPIC_SD_COUNT];
    start(ctx, initial_state(d), row);
    const double E0 = row[UPIC_P3_TOTAL_ENERGY];
    double drift = 0.0, dE = 0.0, chain = 0.0, pres = 0.0, fres = 0.0;
    for (int n = 0; n < 4; ++n) {
        check(upic_step_implicit(ctx.c, 1, row, info, sd), ctx.c);
        drift = std::max(drift, std::abs((row[UPIC_P3_TOTAL_ENERGY] - E0) / E0));
        dE = std::max(dE, std::abs(sd[UPIC_SD_DELTA_TOTAL_ENERGY]));
        chain = std::max(chain, sd[UPIC_SD_A_CHAIN_ABS_RMS]);
        pres = std::max(pres, std::abs(sd[UPIC_SD_PARTICLE_ENERGY_RESIDUAL]));
        fres = std::max(fres, std::abs(sd[UPIC_SD_FIELD_ENERGY_RESIDUAL]));
    }
    os << std::scientific << std::setprecision(6) << "Small multistep energy unit test: max_rel_drift=" << drift
       << " max_step_dE=" << dE << " max_A_chain=" << chain << " max_particle_res=" << pres
       << " max_field_res=" << fres << "\n";
    if (!(drift < 5.0e-11 && dE < 5.0e-10 && chain < 5.0e-10 && pres < 5.0e-10 && fres < 5.0e-10)) {
        os << "FAILED: small multistep energy-conservation regression failed\n";
        return false;
    }
    return true;
}

// test_instability_initialization_and_theory (:7307)
bool test_instability_setup(std::ostream& os) {
    P3Deck ts = two_stream_test_deck(4, 2);
    ts.Lx = 8.0 * kPi;
    ts.spline_order = 1;
    ts.v0 = 0.9;
    ts.perturbation = 0.0;
    ts.two_stream_density_alpha = 0.01;
    double rts[UPIC_P3_DIAG_COUNT], rwb[UPIC_P3_DIAG_COUNT];
    const Start sts = initial_state(ts);
    {
        Ctx ctx(abi_config(ts));
        start(ctx, sts, rts);
    }
    P3Deck wb = test_deck();
    wb.test_case = "cold_relativistic_weibel";
    wb.nx = wb.ny = 4;
    wb.nz = 1;
    wb.spline_order = 1;
    wb.particles_per_cell_pair = 1;
    wb.v0 = 0.9;
    wb.weibel_B0 = 1.0e-4;
    const Start swb = initial_state(wb);
    const long N = (long)wb.nx * wb.ny;
    std::vector<double> J(3 * N);
    {
        Ctx ctx(abi_config(wb));
        start(ctx, swb, rwb);
        for (int c = 0; c < 3; ++c) check(upic_get_field(ctx.c, UPIC_FIELD_JX + c, J.data() + c * N), ctx.c);
    }
    double ms = 0.0;
    for (int c = 0; c < 3; ++c) {
        long double s = 0.0L;
        for (long k = 0; k < N; ++k) s += (long double)J[c * N + k] * J[c * N + k];
        const double r = std::sqrt((double)(s / (long double)N));
        ms += r * r;
    }
    const double J_rms = std::sqrt(ms / 3.0);
    os << std::scientific << std::setprecision(6) << "Instability IC/theory unit test: ts_gamma=" << sts.growth
       << " ts_gauss=" << rts[UPIC_P3_GAUSS_RMS] << " wb_gamma=" << swb.growth
       << " wb_Bz_mode=" << rwb[UPIC_P3_BZ_Y_MODE_ABS] << " wb_J_rms=" << J_rms << "\n";
    if (!(sts.growth > 0.0 && rts[UPIC_P3_GAUSS_RMS] < 5.0e-10 && swb.growth > 0.0 &&
          rwb[UPIC_P3_BZ_Y_MODE_ABS] > 1.0e-6 && J_rms > 1.0e-8 && rwb[UPIC_P3_GAUSS_RMS] < 5.0e-10)) {
        os << "FAILED: instability initialization or cold-theory reference failed\n";
        return false;
    }
    return true;
}

// test_two_stream_eigenmode_growth (:7372): the fitted |E_x(k)| growth of a
// 16x1 eigenmode run against the finite-grid cold-fluid rate.
bool test_eigenmode_growth(std::ostream& os) {
    P3Deck d = test_deck();
    d.test_case = "cold_relativistic_two_stream";
    d.nx = 16;
    d.ny = 1;
    d.nz = 1;
    d.Lx = 8.0 * kPi;
    d.dt = 0.05;
    d.spline_order = 1;
    d.orbit_quad_order = 6;
    d.particles_per_cell_pair = 4;
    d.nonlinear_rtol = 1.0e-10;
    d.nonlinear_max_iter = 20;
    d.v0 = 0.9;
    d.perturbation = 0.0;
    d.two_stream_density_alpha = 1.0e-3;
    const Start s = initial_state(d);
    Ctx ctx(abi_config(d));
    double row[UPIC_P3_DIAG_COUNT];
    start(ctx, s, row);
    const double gamma_ref = s.growth, E0 = row[UPIC_P3_E_MODE_ABS], W0 = row[UPIC_P3_TOTAL_ENERGY];
    if (!(E0 > 0.0 && gamma_ref > 0.0)) {
        os << "FAILED: two-stream eigenmode growth test has zero seed or nonpositive theory rate\n";
        return false;
    }
    long double S0 = 0, S1 = 0, S2 = 0, Sy = 0, Sty = 0;
    auto add = [&](double t, double amp) {
        const double yv = std::log(std::max(amp, 1.0e-300));
        S0 += 1.0L;
        S1 += t;
        S2 += (long double)t * t;
        Sy += yv;
        Sty += (long double)t * yv;
    };
    add(0.0, E0);
    const int steps = 80;
    std::vector<double> diag((size_t)steps * UPIC_P3_DIAG_COUNT);
    check(upic_step_implicit(ctx.c, steps, diag.data(), nullptr, nullptr), ctx.c);
    double mode_err = 0.0, energy = 0.0;
    for (int n = 0; n < steps; ++n) {
        const double* r = &diag[(size_t)n * UPIC_P3_DIAG_COUNT];
        const double t = (n + 1) * d.dt;
        add(t, r[UPIC_P3_E_MODE_ABS]);
        mode_err = std::max(mode_err, std::abs(r[UPIC_P3_E_MODE_ABS] / (E0 * std::exp(gamma_ref * t)) - 1.0));
        energy = std::max(energy, std::abs((r[UPIC_P3_TOTAL_ENERGY] - W0) / W0));
    }
    const double gamma_fit = (double)((S0 * Sty - S1 * Sy) / (S0 * S2 - S1 * S1));
    const double err = std::abs(gamma_fit - gamma_ref) / gamma_ref;
    os << std::scientific << std::setprecision(6) << "Two-stream eigenmode growth unit test: gamma_fit=" << gamma_fit
       << " gamma_ref=" << gamma_ref << " rel_growth_error=" << err << " max_mode_over_theory_error=" << mode_err
       << " max_rel_energy=" << energy << "\n";
    if (!(err < 5.0e-3 && mode_err < 5.0e-3 && energy < 5.0e-10)) {
        os << "FAILED: two-stream eigenmode growth no longer matches cold-fluid theory\n";
        return false;
    }
    return true;
}

bool unit_tests(std::ostream& os) {
    bool ok = true;
    ok = test_adjoint(os) && ok;
    ok = test_initial_gauss(os) && ok;
    ok = test_one_step(os) && ok;
    ok = test_multistep(os) && ok;
    ok = test_instability_setup(os) && ok;
    ok = test_eigenmode_growth(os) && ok;
    return ok;
}

// ---- output ------------------------------------------------------------------

// The NonlinearSolveInfo columns of one row.
// _failed_particle_diagnostics.csv rows of one step (write_failed_particle_diagnostics
// :6234): per failure event (layout restart, map evaluation) the
// selective_failure_diagnostic_limit particles of largest final scaled
// residual (non-finite first, the reference's sort), and in an exhausted
// event also the worst particle at the substep limit, in particle order.
void write_failed_particles(upic_ctx* c, const P3Deck& d, double time_before) {
    static const char* reasons[] = {"none", "nonfinite_map", "superluminal_map", "nonfinite_iterate",
                                    "superluminal_iterate", "maximum_iterations", "too_many_knot_crossings"};
    int n = 0;
    check(upic_failed_particle_log(c, 0, nullptr, &n), c);
    if (n == 0) return;
    std::vector<double> rows((size_t)n * UPIC_FAILLOG_COUNT);
    check(upic_failed_particle_log(c, n, rows.data(), &n), c);
    std::ofstream out(d.output_prefix + "_failed_particle_diagnostics.csv", std::ios::app);
    auto at = [&](int i, int col) { return rows[(size_t)i * UPIC_FAILLOG_COUNT + col]; };
    for (int b = 0; b < n;) {
        int e = b;
        while (e < n && at(e, UPIC_FAILLOG_RESTART) == at(b, UPIC_FAILLOG_RESTART) &&
               at(e, UPIC_FAILLOG_EVALUATION) == at(b, UPIC_FAILLOG_EVALUATION) &&
               at(e, UPIC_FAILLOG_STEP) == at(b, UPIC_FAILLOG_STEP))
            ++e;
        const int m = e - b;
        std::vector<int> order(m);
        for (int i = 0; i < m; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](int i, int j) {
            const double x = at(b + i, UPIC_FAILLOG_FINAL_SCALED), y = at(b + j, UPIC_FAILLOG_FINAL_SCALED);
            if (!std::isfinite(x)) return (bool)std::isfinite(y);
            if (!std::isfinite(y)) return false;
            return x > y;
        });
        std::vector<char> selected(m, 0);
        const int limit = std::min(m, d.selective_failure_diagnostic_limit);
        for (int i = 0; i < limit; ++i) selected[order[i]] = 1;
        const bool exhausted = at(b, UPIC_FAILLOG_EXHAUSTED) != 0.0;
        if (exhausted) {
            int worst = -1;
            for (int i = 0; i < m; ++i) {
                if (at(b + i, UPIC_FAILLOG_SUBSTEPS) < d.selective_particle_max_substeps) continue;
                if (worst < 0) {
                    worst = i;
                    continue;
                }
                const double cand = at(b + i, UPIC_FAILLOG_FINAL_SCALED), cur = at(b + worst, UPIC_FAILLOG_FINAL_SCALED);
                if ((!std::isfinite(cand) && std::isfinite(cur)) ||
                    (std::isfinite(cand) && std::isfinite(cur) && cand > cur))
                    worst = i;
            }
            if (worst >= 0) selected[worst] = 1;
        }
        out << std::setprecision(17);
        for (int i = 0; i < m; ++i) {
            if (!selected[i]) continue;
            const int r = b + i;
            const int reason = (int)at(r, UPIC_FAILLOG_REASON);
            out << time_before << "," << (long)at(r, UPIC_FAILLOG_RESTART) << "," << (long)at(r, UPIC_FAILLOG_EVALUATION)
                << "," << (exhausted ? 1 : 0) << "," << (long)at(r, UPIC_FAILLOG_IN_EVENT) << ","
                << (long)at(r, UPIC_FAILLOG_PARTICLE) << "," << (long)at(r, UPIC_FAILLOG_SUBSTEPS) << ","
                << (long)at(r, UPIC_FAILLOG_FAILED_SUBSTEP) << "," << at(r, UPIC_FAILLOG_THETA0) << ","
                << at(r, UPIC_FAILLOG_THETA1) << "," << at(r, UPIC_FAILLOG_H) << ","
                << (long)at(r, UPIC_FAILLOG_ITERATIONS) << "," << (reason >= 0 && reason < 7 ? reasons[reason] : "unknown");
            for (int col = UPIC_FAILLOG_FIRST_SCALED; col < UPIC_FAILLOG_COUNT; ++col) out << "," << at(r, col);
            out << "\n";
        }
        b = e;
    }
}

struct Solve {
    double iterations = 0, converged = 1, rms = kNaN, max_particle = kNaN, abs_rms = kNaN;
    double restarts = 0, anderson = 0, picard = 0;
    std::string method = "initial_state";
    double rate = kInf, contraction = kInf, backtracked = 0, min_alpha = 1.0;
    double local_mean = 0, local_max = 0, substeps = 0, fallback = 0, direct = 0, layout_restarts = 0;
    double refined = 0, total_substeps = 0, work_ratio = 1.0;
    double levels[7] = {0, 0, 0, 0, 0, 0, 0};
};

Solve solve_of(const double* in) {
    Solve s;
    s.iterations = in[UPIC_INFO_ITERATIONS];
    s.converged = in[UPIC_INFO_CONVERGED];
    s.rms = in[UPIC_INFO_FINAL_RMS_RESIDUAL];
    s.max_particle = in[UPIC_INFO_FINAL_MAX_PARTICLE_RESIDUAL];
    s.abs_rms = in[UPIC_INFO_FINAL_ABS_RMS_RESIDUAL];
    s.restarts = in[UPIC_INFO_ANDERSON_RESTARTS];
    s.anderson = in[UPIC_INFO_ANDERSON_STEPS];
    s.picard = in[UPIC_INFO_PICARD_STEPS];
    const char* name = upic_convergence_method_name((int)in[UPIC_INFO_CONVERGENCE_METHOD]);
    s.method = name ? name : "none";
    s.rate = in[UPIC_INFO_OBSERVED_RATE];
    s.contraction = in[UPIC_INFO_MAP_CONTRACTION];
    s.backtracked = in[UPIC_INFO_BACKTRACKED_STEPS];
    s.min_alpha = in[UPIC_INFO_MIN_UPDATE_ALPHA];
    s.local_mean = in[UPIC_INFO_LOCAL_ITER_MEAN];
    s.local_max = in[UPIC_INFO_LOCAL_ITER_MAX];
    s.substeps = in[UPIC_INFO_SUBSTEPS_USED];
    s.fallback = in[UPIC_INFO_SELECTIVE_FALLBACK_USED];
    s.direct = in[UPIC_INFO_DIRECT_ATTEMPT_ITERATIONS];
    s.layout_restarts = in[UPIC_INFO_SELECTIVE_RESTARTS];
    s.refined = in[UPIC_INFO_SELECTIVE_REFINED];
    s.total_substeps = in[UPIC_INFO_SELECTIVE_SUBSTEPS];
    s.work_ratio = in[UPIC_INFO_SELECTIVE_WORK_RATIO];
    for (int k = 0; k < 7; ++k) s.levels[k] = in[UPIC_INFO_SELECTIVE_N1 + k];
    return s;
}

// The local-solve and selective columns shared by the three step records.
void write_local_columns(std::ostream& o, const Solve& s) {
    o << s.local_mean << "," << s.local_max << "," << s.substeps << "," << s.fallback << "," << s.direct << ","
      << s.layout_restarts << "," << s.refined << "," << s.total_substeps << "," << s.work_ratio;
    for (double l : s.levels) o << "," << l;
}

struct Probe {
    double phi, psi, rho, A[3], U[3], J[3], Eg[3], Es[3], Bg[3], Bs[3], gA[3][3];
};

Probe probe_of(const double* r) {
    Probe p;
    p.phi = r[UPIC_PROBE_PHI];
    p.psi = r[UPIC_PROBE_PSI];
    p.rho = r[UPIC_PROBE_RHO];
    for (int c = 0; c < 3; ++c) {
        p.A[c] = r[UPIC_PROBE_A + c];
        p.U[c] = r[UPIC_PROBE_U + c];
        p.J[c] = r[UPIC_PROBE_J + c];
        p.Eg[c] = r[UPIC_PROBE_E + c];
        p.Bg[c] = r[UPIC_PROBE_B + c];
        p.Es[c] = -(r[UPIC_PROBE_GRAD_PHI + c] + p.U[c]);
        for (int e = 0; e < 3; ++e) p.gA[c][e] = r[UPIC_PROBE_GRAD_A + 3 * c + e];
    }
    // curl_from_shape_gradient (:7881)
    p.Bs[0] = p.gA[2][1] - p.gA[1][2];
    p.Bs[1] = p.gA[0][2] - p.gA[2][0];
    p.Bs[2] = p.gA[1][0] - p.gA[0][1];
    return p;
}

double norm_diff(const double* a, const double* b) {
    const double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return std::sqrt(x * x + y * y + z * z);
}

double matrix_diff(const double a[3][3], const double b[3][3]) {
    long double s = 0.0L;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const long double e = (long double)a[i][j] - (long double)b[i][j];
            s += e * e;
        }
    return std::sqrt((double)s);
}

const char* axis_label(int a) { return a == 0 ? "x" : (a == 1 ? "y" : "z"); }

// write_field_line_and_knot_snapshot (:8043): line probes along the probe
// axis through the origin and two-sided probes at every spline knot on it.
void field_line_and_knots(std::ostream& line, std::ostream& jumps, upic_ctx* ctx, const P3Deck& d, int axis,
                          int step, double time) {
    const int n_axis = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
    const double L = axis == 0 ? d.Lx : (axis == 1 ? d.Ly : d.Lz);
    const double h = L / n_axis;
    const int ns = n_axis * d.field_probe_points_per_cell;
    std::vector<double> pos(3 * (size_t)ns, 0.0);
    for (int s = 0; s < ns; ++s) pos[3 * (size_t)s + axis] = -0.5 * L + (s + 0.5) * L / ns;
    const double offset = 0.5 * (d.spline_order - 1);
    const double eps = 1.0e-8 * h;
    std::vector<double> kpos(6 * (size_t)n_axis, 0.0), kcoord(n_axis);
    for (int k = 0; k < n_axis; ++k) {
        double u = std::fmod(k + offset, (double)n_axis);
        if (u < 0.0) u += n_axis;
        kcoord[k] = -0.5 * L + u * h;
        kpos[6 * (size_t)k + axis] = kcoord[k] - eps;
        kpos[6 * (size_t)k + 3 + axis] = kcoord[k] + eps;
    }
    // one probe call for the line and both sides of every knot (x, y only:
    // the 2D fields do not depend on z)
    const long np = ns + 2L * n_axis;
    std::vector<double> px(np), py(np), out((size_t)np * UPIC_PROBE_COUNT);
    for (int s = 0; s < ns; ++s) {
        px[s] = pos[3 * (size_t)s];
        py[s] = pos[3 * (size_t)s + 1];
    }
    for (int k = 0; k < 2 * n_axis; ++k) {
        px[ns + k] = kpos[3 * (size_t)k];
        py[ns + k] = kpos[3 * (size_t)k + 1];
    }
    check(upic_probe_fields(ctx, np, px.data(), py.data(), out.data()), ctx);
    for (int s = 0; s < ns; ++s) {
        const Probe p = probe_of(&out[(size_t)s * UPIC_PROBE_COUNT]);
        const double* x = &pos[3 * (size_t)s];
        line << step << "," << time << "," << d.spline_order << "," << axis_label(axis) << "," << s << ","
             << x[axis] << "," << x[0] << "," << x[1] << "," << x[2] << "," << p.phi << "," << p.psi << "," << p.rho;
        for (const double* f : {p.A, p.U, p.J, p.Eg, p.Es, p.Bg, p.Bs})
            for (int c = 0; c < 3; ++c) line << "," << f[c];
        for (int c = 0; c < 3; ++c)
            for (int e = 0; e < 3; ++e) line << "," << p.gA[c][e];
        line << "," << norm_diff(p.Es, p.Eg) << "," << norm_diff(p.Bs, p.Bg) << "\n";
    }
    for (int k = 0; k < n_axis; ++k) {
        const Probe l = probe_of(&out[(size_t)(ns + 2 * k) * UPIC_PROBE_COUNT]);
        const Probe r = probe_of(&out[(size_t)(ns + 2 * k + 1) * UPIC_PROBE_COUNT]);
        jumps << step << "," << time << "," << d.spline_order << "," << axis_label(axis) << "," << k << ","
              << kcoord[k] << "," << eps << "," << norm_diff(r.A, l.A) << "," << norm_diff(r.Eg, l.Eg) << ","
              << norm_diff(r.Es, l.Es) << "," << norm_diff(r.Bg, l.Bg) << "," << norm_diff(r.Bs, l.Bs) << ","
              << matrix_diff(r.gA, l.gA);
        for (const double* f : {l.Bs, r.Bs, l.Es, r.Es})
            for (int c = 0; c < 3; ++c) jumps << "," << f[c];
        jumps << "\n";
    }
}

// write_transverse_moments (:7702): mass-weighted velocity moments.
void velocity_moments(std::ostream& o, const std::vector<double>& v, const std::vector<double>& m, int step,
                      double time) {
    const size_t np = m.size();
    long double mass = 0.0L, mean[3] = {0, 0, 0}, sq[3] = {0, 0, 0}, var[3] = {0, 0, 0};
    for (size_t p = 0; p < np; ++p) {
        mass += m[p];
        for (int c = 0; c < 3; ++c) {
            mean[c] += m[p] * (long double)v[3 * p + c];
            sq[c] += m[p] * (long double)v[3 * p + c] * v[3 * p + c];
        }
    }
    if (!(mass > 0.0L)) throw std::runtime_error("nonpositive mass in velocity moments");
    for (int c = 0; c < 3; ++c) mean[c] /= mass;
    for (size_t p = 0; p < np; ++p)
        for (int c = 0; c < 3; ++c) {
            const long double dv = v[3 * p + c] - mean[c];
            var[c] += m[p] * dv * dv;
        }
    o << step << ',' << std::setprecision(17) << time << ',' << np << ',' << mass;
    for (int c = 0; c < 3; ++c) o << ',' << mean[c];
    for (int c = 0; c < 3; ++c) o << ',' << std::sqrt(sq[c] / mass);
    for (int c = 0; c < 3; ++c) o << ',' << var[c] / mass;
    o << '\n';
}

// write_transverse_spectrum (:7747): |FFT|^2 / N^2 of E and B folded onto
// (|m_x|, |m_y|, |m_z|) bins.
void field_spectrum(std::ostream& o, upic_ctx* ctx, const P3Deck& d, int step, double time) {
    const int nx = d.nx, ny = d.ny, N = nx * ny;
    const int sx = nx / 2 + 1, sy = ny / 2 + 1;
    std::vector<std::array<double, 6>> power((size_t)sx * sy, std::array<double, 6>{});
    const double scale = 1.0 / ((double)N * N);
    std::vector<double> re(N), im(N);
    for (int f = 0; f < 6; ++f) {
        check(upic_get_field(ctx, UPIC_FIELD_EX + f, re.data()), ctx);
        std::fill(im.begin(), im.end(), 0.0);
        check(upic_fft2d(ctx, re.data(), im.data(), 0), ctx);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const int a = std::min(i, nx - i), b = std::min(j, ny - j);
                const double h2 = re[i * ny + j] * re[i * ny + j] + im[i * ny + j] * im[i * ny + j];
                power[(size_t)a * sy + b][f] += h2 * scale;
            }
    }
    for (int a = 0; a < sx; ++a)
        for (int b = 0; b < sy; ++b) {
            const char* kind = (a == 0 && b == 0) ? "zero" : (b == 0 ? "longitudinal" : (a == 0 ? "transverse" : "oblique"));
            o << step << ',' << std::setprecision(17) << time << ',' << a << ',' << b << ',' << 0 << ',' << kind;
            for (double p : power[(size_t)a * sy + b]) o << ',' << p;
            o << '\n';
        }
}

// The particles of the accepted state in the reference's order.
struct Particles {
    std::vector<double> x, y, v;
};

Particles particles_of(upic_ctx* ctx, long np) {
    Particles p;
    p.x.resize(np);
    p.y.resize(np);
    p.v.resize(3 * np);
    std::vector<double> P(3 * np), vp(3 * np);
    check(upic_get_particles(ctx, np, p.x.data(), p.y.data(), P.data(), p.v.data(), vp.data()), ctx);
    return p;
}

void config_echo(const std::string& path, const P3Deck& d, long np, double auto_rate) {
    std::ofstream out(path);
    const double dV = (d.Lx / d.nx) * (d.Ly / d.ny) * (d.Lz / d.nz);
    out << "test_case=" << d.test_case << "\n";
    out << "transverse_diagnostics=" << (d.transverse_diagnostics ? "true" : "false") << "\n";
    out << "transverse_spectrum_interval=" << std::setprecision(17) << d.transverse_spectrum_interval << "\n";
    out << "tsi_transverse_seed=" << d.tsi_transverse_seed << "\n";
    out << "tsi_transverse_mode=" << d.tsi_transverse_mode << "\n";
    out << "nyquist_projection=" << d.nyquist_projection << "\n";
    out << "nx=" << d.nx << "\n" << "ny=" << d.ny << "\n" << "nz=" << d.nz << "\n";
    out << "Lx=" << d.Lx << "\n" << "Ly=" << d.Ly << "\n" << "Lz=" << d.Lz << "\n";
    out << "n_steps=" << d.n_steps << "\n" << "dt=" << d.dt << "\n";
    out << "target_time=" << (static_cast<double>(d.n_steps) * d.dt) << "\n";
    out << "particles=" << np << "\n";
    out << "particles_per_cell_pair_or_velocity_samples=" << d.particles_per_cell_pair << "\n";
    out << "spline_order=" << d.spline_order << "\n" << "orbit_quad_order=" << d.orbit_quad_order << "\n";
    out << "split_orbit_at_knots=" << (d.split_orbit_at_knots ? "true" : "false") << "\n";
    out << "macro_time_step=" << (d.adaptive_dt ? "adaptive_rejection" : "fixed") << "\n";
    out << "adaptive_dt=" << (d.adaptive_dt ? "true" : "false") << "\n";
    out << "adaptive_dt_min=" << effective_dt_min(d) << "\n";
    out << "adaptive_dt_shrink=" << d.adaptive_dt_shrink << "\n";
    out << "adaptive_dt_growth=" << d.adaptive_dt_growth << "\n";
    out << "adaptive_dt_growth_interval=" << d.adaptive_dt_growth_interval << "\n";
    out << "adaptive_max_attempts=" << d.adaptive_max_attempts << "\n";
    out << "nonlinear_solver=" << d.nonlinear_solver << "\n";
    out << "nonlinear_rtol=" << d.nonlinear_rtol << "\n" << "nonlinear_atol=" << d.nonlinear_atol << "\n";
    out << "nonlinear_max_iter=" << d.nonlinear_max_iter << "\n";
    out << "anderson_memory=" << d.anderson_memory << "\n" << "anderson_start=" << d.anderson_start << "\n";
    out << "anderson_damping=" << d.anderson_damping << "\n";
    out << "anderson_regularization=" << d.anderson_regularization << "\n";
    out << "anderson_growth_limit=" << d.anderson_growth_limit << "\n";
    out << "uniform_particle_subcycling=" << (d.uniform_particle_subcycling ? "true" : "false") << "\n";
    out << "uniform_refine_on_failure=" << (d.uniform_refine_on_failure ? "true" : "false") << "\n";
    out << "uniform_initial_substeps=" << d.uniform_initial_substeps << "\n";
    out << "uniform_substeps=" << d.uniform_substeps << "\n";
    out << "uniform_max_substeps=" << d.uniform_max_substeps << "\n";
    out << "uniform_subcycling_start_time=" << d.uniform_subcycling_start_time << "\n";
    for (const char* prefix : {"particle", "uniform"}) {
        out << prefix << "_local_rtol=" << d.uniform_local_rtol << "\n";
        out << prefix << "_local_atol=" << d.uniform_local_atol << "\n";
        out << prefix << "_local_max_iter=" << d.uniform_local_max_iter << "\n";
    }
    out << "uniform_local_damping=" << d.uniform_local_damping << "\n";
    out << "selective_particle_fallback=" << (d.selective_particle_fallback ? "true" : "false") << "\n";
    out << "selective_particle_max_substeps=" << d.selective_particle_max_substeps << "\n";
    out << "selective_particle_dynamic_chunk=" << d.selective_particle_dynamic_chunk << "\n";
    out << "selective_failure_diagnostics=" << (d.selective_failure_diagnostics ? "true" : "false") << "\n";
    out << "selective_failure_diagnostic_limit=" << d.selective_failure_diagnostic_limit << "\n";
    out << "particle_snapshot_times=";
    for (double t : d.particle_snapshot_times) out << t << ' ';
    out << "\n";
    out << "field_diagnostics=" << (d.field_diagnostics ? "true" : "false") << "\n";
    out << "field_diagnostics_interval=" << d.field_diagnostics_interval << "\n";
    out << "field_probe_points_per_cell=" << d.field_probe_points_per_cell << "\n";
    out << "field_probe_axis=" << d.field_probe_axis << "\n";
    out << "field_grid_snapshots=" << (d.field_grid_snapshots ? "true" : "false") << "\n";
    out << "kappa=" << d.kappa << "\n" << "sigma1=" << d.sigma1 << "\n" << "sigma2=" << d.sigma2 << "\n";
    out << "sigma1_minus_kappa2_sigma2=" << (d.sigma1 - d.kappa * d.kappa * d.sigma2) << "\n";
    out << "rho0=" << d.n0 << "\n" << "v0=" << d.v0 << "\n" << "perturbation=" << d.perturbation << "\n";
    out << "two_stream_density_alpha=" << d.two_stream_density_alpha << "\n";
    out << "two_stream_eigenmode=" << (d.two_stream_eigenmode ? "true" : "false") << "\n";
    out << "two_stream_finite_grid_theory=" << (d.two_stream_finite_grid_theory ? "true" : "false") << "\n";
    out << "weibel_B0=" << weibel_seed(d) << "\n";
    out << "weibel_eigenmode=" << (d.weibel_eigenmode ? "true" : "false") << "\n";
    out << "weibel_finite_grid_theory=" << (d.weibel_finite_grid_theory ? "true" : "false") << "\n";
    out << "landau_alpha=" << landau_amplitude(d) << "\n";
    out << "thermal_velocity=" << d.thermal_velocity << "\n";
    out << "perturbation_mode=" << d.perturbation_mode << "\n";
    out << "theory_omega=" << d.theory_omega << "\n" << "theory_gamma=" << d.theory_gamma << "\n";
    out << "auto_theory_growth_rate=" << auto_rate << "\n";
    out << "dV=" << dV << "\n";
}

}  // namespace

int run_p3(const std::string& path) {
    const Clock::time_point t_start = Clock::now();
    const P3Deck d = read_deck(path);
    if (d.adaptive_dt || d.uniform_particle_subcycling)
        throw std::runtime_error("manuscript runs require adaptive_dt=false, uniform_particle_subcycling=false");
    {
        std::ofstream inner(d.output_prefix + "_particle_inner_history.csv");
        if (!inner) throw std::runtime_error("cannot open particle inner history");
        inner << "time_n,dt,map_evaluation,particles_converged,failed_particles,max_scaled_particle_residual,"
                 "local_iterations_mean,local_iterations_max\n";
    }
    std::cout << "Nested particle solve: frozen-field inner iterations, then outer current Anderson; "
              << (d.selective_particle_fallback ? "selective refinement on local failure\n"
                                                : "full dt, no temporal substeps\n");
    if (!pow2(d.nx) || !pow2(d.ny) || !pow2(d.nz))
        throw std::runtime_error("the in-file radix-2 FFT requires nx, ny, nz to be powers of two");
    if (d.nz != 1) throw std::runtime_error("this build runs 2D and 1D decks only (nz = 1)");
    std::cout << "B200 GM-HC-CN orbit-averaged PIC (UPIC_METHOD_CN_ORBIT)\n";
    std::cout << "test_case = " << d.test_case << "\n";
    std::cout << "grid = " << d.nx << " x " << d.ny << " x " << d.nz << ", dt = " << d.dt << ", steps = " << d.n_steps
              << "\n";
    if (d.selective_particle_fallback)
        std::cout << "direct-first selective particle fallback: fixed macro dt; failed particles refine through "
                     "powers of two to dt/"
                  << d.selective_particle_max_substeps << ", local_max_iter=" << d.uniform_local_max_iter << "\n";

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

    const Start S = initial_state(d);
    const long np = S.size();
    const std::string tc = lowercase(d.test_case);
    // selected_theory_growth_rate (:4228)
    const double theory_growth =
        std::abs(d.theory_gamma) > 0.0 ? d.theory_gamma : ((is_two_stream(tc) || is_weibel(tc)) ? S.growth : d.theory_gamma);
    config_echo(d.output_prefix + "_config_echo.txt", d, np, theory_growth);

    Ctx ctx(abi_config(d));
    double row[UPIC_P3_DIAG_COUNT], info[UPIC_INFO_COUNT], sd[UPIC_SD_COUNT];
    start(ctx, S, row);
    const bool use_B = is_weibel(tc);
    const double amp0 = use_B ? row[UPIC_P3_BZ_Y_MODE_ABS] : row[UPIC_P3_E_MODE_ABS];
    const bool has_theory = (std::abs(theory_growth) > 0.0 || std::abs(d.theory_omega) > 0.0) && amp0 > 0.0;
    if (std::abs(theory_growth) > 0.0) {
        std::cout << std::scientific << std::setprecision(6) << "linear theory growth/damping rate = " << theory_growth
                  << (use_B ? " using |B_z(k_y)|" : " using |E_x(k_x)|") << "\n";
    }

    std::ofstream diag(d.output_prefix + "_diagnostics.csv");
    diag << "step,time,gauss_rms,gauss_max,divE_rms,sigma1_rho_rms,gauss_normalization_rms,gauss_relative,"
            "gauge_rms,gauge_max,psi_over_kappa2_rms,divA_rms,gauge_normalization_rms,gauge_relative,"
            "field_energy,kinetic_energy,total_energy,"
            "rho_mode,E_mode_re,E_mode_im,E_mode_abs,Bz_y_mode_re,Bz_y_mode_im,Bz_y_mode_abs,"
            "theory_growth_rate,theory_mode_abs,mode_over_theory,mean_rho,"
            "nonlinear_iterations,nonlinear_converged,nonlinear_rms_residual,"
            "nonlinear_max_particle_residual,nonlinear_absolute_rms_residual,"
            "anderson_restarts,anderson_steps,picard_fallback_steps,convergence_method,"
            "observed_convergence_rate,estimated_map_contraction,backtracked_steps,minimum_update_alpha,"
            "local_particle_iterations_mean,local_particle_iterations_max,uniform_substeps_used,"
            "selective_fallback_used,direct_attempt_iterations,selective_refinement_restarts,"
            "selective_refined_particles,selective_total_particle_substeps,selective_work_ratio,"
            "selective_n1,selective_n2,selective_n4,selective_n8,selective_n16,selective_n32,selective_n64,"
            "crossing_particles,avg_path_segments,max_path_segments,dt,elapsed_wall_seconds\n";
    std::ofstream stepcsv(d.output_prefix + "_step_diagnostics.csv");
    stepcsv << "step,time,nonlinear_iterations,nonlinear_rms_residual,nonlinear_max_particle_residual,"
               "anderson_restarts,convergence_method,observed_convergence_rate,"
               "estimated_map_contraction,backtracked_steps,minimum_update_alpha,"
               "local_particle_iterations_mean,local_particle_iterations_max,uniform_substeps_used,"
               "selective_fallback_used,direct_attempt_iterations,selective_refinement_restarts,"
               "selective_refined_particles,selective_total_particle_substeps,selective_work_ratio,"
               "selective_n1,selective_n2,selective_n4,selective_n8,selective_n16,selective_n32,selective_n64,"
               "A_chain_abs_rms,A_chain_rel_rms,A_chain_max_norm,"
               "A_chain_mean_norm,A_chain_work_defect,delta_K,delta_W,delta_total_energy,particle_work,"
               "grid_work,deposit_gather_work_residual,particle_energy_residual,field_energy_residual,"
               "crossing_particles,total_crossings,avg_path_segments,max_path_segments,dt,elapsed_wall_seconds\n";
    std::ofstream adaptive(d.output_prefix + "_adaptive_diagnostics.csv");
    adaptive << "accepted_step,time_before,attempt,dt,outcome,nonlinear_iterations,"
                "nonlinear_rms_residual,nonlinear_max_particle_residual,"
                "observed_convergence_rate,estimated_map_contraction,"
                "backtracked_steps,minimum_update_alpha,"
                "local_particle_iterations_mean,local_particle_iterations_max,uniform_substeps_used,"
                "selective_fallback_used,direct_attempt_iterations,selective_refinement_restarts,"
                "selective_refined_particles,selective_total_particle_substeps,selective_work_ratio,"
                "selective_n1,selective_n2,selective_n4,selective_n8,selective_n16,selective_n32,selective_n64,"
                "elapsed_wall_seconds\n";
    if (d.selective_failure_diagnostics) {
        std::ofstream failed(d.output_prefix + "_failed_particle_diagnostics.csv");
        failed << "time_before,layout_refinement_restart,map_evaluation,event_exhausted,"
                  "failed_particles_in_event,particle_index,assigned_substeps,failed_substep_zero_based,"
                  "theta0,theta1,h,local_iterations,failure_reason,first_scaled_residual,"
                  "final_scaled_residual,final_absolute_residual,q,m,"
                  "x0_x,x0_y,x0_z,P0_x,P0_y,P0_z,"
                  "initial_guess_x,initial_guess_y,initial_guess_z,"
                  "last_guess_x,last_guess_y,last_guess_z,"
                  "last_map_x,last_map_y,last_map_z\n";
    }
    std::ofstream line_csv, jump_csv, grid_csv, moments_csv, spectrum_csv;
    const std::string axis_name = lowercase(d.field_probe_axis);
    const int axis = axis_name == "x" ? 0 : (axis_name == "y" ? 1 : (axis_name == "z" ? 2 : (use_B ? 1 : 0)));
    if (d.field_diagnostics) {
        line_csv.open(d.output_prefix + "_field_line_probe.csv");
        jump_csv.open(d.output_prefix + "_field_knot_jumps.csv");
        if (!line_csv || !jump_csv) throw std::runtime_error("could not open field reconstruction diagnostics files");
        line_csv << "step,time,spline_order,probe_axis,sample,coordinate,x,y,z,"
                    "phi_h,psi_h,rho_h,Ax_h,Ay_h,Az_h,Ux_h,Uy_h,Uz_h,Jx_h,Jy_h,Jz_h,"
                    "Ex_grid_gather,Ey_grid_gather,Ez_grid_gather,"
                    "Ex_shape_phi,Ey_shape_phi,Ez_shape_phi,"
                    "Bx_grid_gather,By_grid_gather,Bz_grid_gather,"
                    "Bx_shape_A,By_shape_A,Bz_shape_A,"
                    "dAx_dx,dAx_dy,dAx_dz,dAy_dx,dAy_dy,dAy_dz,dAz_dx,dAz_dy,dAz_dz,"
                    "E_representation_difference,B_representation_difference\n";
        jump_csv << "step,time,spline_order,probe_axis,knot,knot_coordinate,epsilon,"
                    "A_jump,E_grid_gather_jump,E_shape_phi_jump,"
                    "B_grid_gather_jump,B_shape_A_jump,gradA_jump,"
                    "Bx_shape_left,By_shape_left,Bz_shape_left,"
                    "Bx_shape_right,By_shape_right,Bz_shape_right,"
                    "Ex_shape_left,Ey_shape_left,Ez_shape_left,"
                    "Ex_shape_right,Ey_shape_right,Ez_shape_right\n";
        line_csv << std::setprecision(17);
        jump_csv << std::setprecision(17);
        std::cout << "field reconstruction diagnostics = " << d.output_prefix << "_field_line_probe.csv and "
                  << d.output_prefix << "_field_knot_jumps.csv (axis=" << axis_label(axis)
                  << ", samples_per_cell=" << d.field_probe_points_per_cell << ")\n";
    }
    const std::string grid_path = d.output_prefix + "_field_grid_snapshots.csv";
    const bool grid_snapshots = d.field_diagnostics && d.field_grid_snapshots;
    if (d.transverse_diagnostics) {
        moments_csv.open(d.output_prefix + "_velocity_moments.csv");
        spectrum_csv.open(d.output_prefix + "_field_spectrum.csv");
        if (!moments_csv || !spectrum_csv) throw std::runtime_error("cannot open transverse diagnostic files");
        moments_csv << "step,time,particles,total_mass,mean_vx,mean_vy,mean_vz,rms_vx,rms_vy,rms_vz,var_vx,var_vy,"
                       "var_vz\n";
        spectrum_csv << "step,time,abs_mx,abs_my,abs_mz,wavevector_class,Ex_power,Ey_power,Ez_power,Bx_power,"
                        "By_power,Bz_power\n";
    }
    diag << std::setprecision(17);
    stepcsv << std::setprecision(17);
    adaptive << std::setprecision(17);

    const double target = static_cast<double>(d.n_steps) * d.dt;
    const double teps = 128.0 * DBL_EPSILON * std::max(1.0, std::abs(target));
    double next_spectrum = 0.0;
    // the write_diag lambda of main (:8585)
    auto write_diag = [&](int step, double time, const Solve& s, long cross, double avg, long maxseg,
                          const double* r, double step_dt) {
        if (d.transverse_diagnostics) {
            const Particles p = particles_of(ctx.c, np);
            velocity_moments(moments_csv, p.v, S.m, step, time);
            const double eps = 128.0 * DBL_EPSILON * std::max(1.0, target);
            if (time + eps >= next_spectrum || time + eps >= target) {
                field_spectrum(spectrum_csv, ctx.c, d, step, time);
                next_spectrum =
                    (std::floor((time + eps) / d.transverse_spectrum_interval) + 1.0) * d.transverse_spectrum_interval;
                spectrum_csv.flush();
            }
            moments_csv.flush();
        }
        double th = kNaN, ratio = kNaN;
        if (has_theory) {
            th = amp0 * std::exp(theory_growth * time);
            ratio = (use_B ? r[UPIC_P3_BZ_Y_MODE_ABS] : r[UPIC_P3_E_MODE_ABS]) / (th + 1.0e-300);
        }
        diag << step << "," << time;
        for (int k = 0; k <= UPIC_P3_BZ_Y_MODE_ABS; ++k) diag << "," << r[k];
        diag << "," << theory_growth << "," << th << "," << ratio << "," << r[UPIC_P3_MEAN_RHO] << ","
             << s.iterations << "," << s.converged << "," << s.rms << "," << s.max_particle << "," << s.abs_rms << ","
             << s.restarts << "," << s.anderson << "," << s.picard << "," << s.method << "," << s.rate << ","
             << s.contraction << "," << s.backtracked << "," << s.min_alpha << ",";
        write_local_columns(diag, s);
        diag << "," << cross << "," << avg << "," << maxseg << "," << step_dt << "," << seconds_since(t_start) << "\n";
    };
    auto field_snapshot = [&](int step, double time) {
        field_line_and_knots(line_csv, jump_csv, ctx.c, d, axis, step, time);
        if (grid_snapshots) check(upic_write_field_snapshot(ctx.c, grid_path.c_str(), step > 0 || time > 0.0 ? 1 : 0,
                                                           step, time),
                                  ctx.c);
        line_csv.flush();
        jump_csv.flush();
    };
    size_t next_particle_snapshot = 0;
    double time = 0.0;
    auto particle_snapshots = [&](int step) {
        while (next_particle_snapshot < d.particle_snapshot_times.size() &&
               d.particle_snapshot_times[next_particle_snapshot] <= time + teps) {
            const double req = d.particle_snapshot_times[next_particle_snapshot++];
            std::ostringstream name;
            name << d.output_prefix << "_particles_t" << std::setprecision(17) << req << ".csv";
            const Particles p = particles_of(ctx.c, np);
            std::ofstream out(name.str());
            if (!out) throw std::runtime_error("could not open particle snapshot: " + name.str());
            out << "step,time,requested_time,particle,x,y,z,vx,vy,vz,q,m\n" << std::setprecision(17);
            for (long k = 0; k < np; ++k)
                out << step << ',' << time << ',' << req << ',' << k << ',' << p.x[k] << ',' << p.y[k] << ',' << 0.0
                    << ',' << p.v[3 * k] << ',' << p.v[3 * k + 1] << ',' << p.v[3 * k + 2] << ',' << S.q[k] << ','
                    << S.m[k] << '\n';
            out.close();
            if (!out) throw std::runtime_error("failed writing particle snapshot: " + name.str());
            std::cout << "particle snapshot = " << name.str() << " (accepted time " << std::setprecision(17) << time
                      << ", particles " << np << ")\n"
                      << std::setprecision(6);
        }
    };

    write_diag(0, 0.0, Solve{}, 0, 0.0, 1, row, 0.0);
    double last_field_time = -kInf;
    double next_field_time = d.field_diagnostics_interval > 0.0 ? d.field_diagnostics_interval : kInf;
    if (d.field_diagnostics) {
        field_snapshot(0, 0.0);
        last_field_time = 0.0;
    }
    for (double t : d.particle_snapshot_times)
        if (t > target + teps)
            std::cerr << "warning: particle snapshot time " << t << " exceeds end time " << target << "\n";
    particle_snapshots(0);
    std::cout << std::scientific << std::setprecision(3) << "fixed stepping: nominal dt=" << d.dt
              << ", dt_min=" << effective_dt_min(d) << ", target_time=" << target
              << ", nonlinear_solver=" << d.nonlinear_solver << "\n";

    const double progress_interval = target > 0.0 ? target / 5.0 : 0.0;
    double next_progress = progress_interval;
    double ctx_dt = d.dt;
    int accepted = 0;
    std::vector<double> maplog;
    while (time + teps < target) {
        const double dt_try = std::min(d.dt, target - time);
        if (dt_try != ctx_dt) {
            check(upic_set_time_step(ctx.c, dt_try), ctx.c);
            ctx_dt = dt_try;
        }
        const int rc = upic_step_implicit(ctx.c, 1, row, info, sd);
        const std::string err = rc ? upic_last_error(ctx.c) : "";
        {   // the step's map evaluations (particle_history, :5918-5945)
            int n = 0;
            check(upic_map_log(ctx.c, 0, nullptr, &n), ctx.c);
            maplog.resize((size_t)n * UPIC_MAPLOG_COUNT);
            check(upic_map_log(ctx.c, n, maplog.data(), &n), ctx.c);
            std::ofstream inner(d.output_prefix + "_particle_inner_history.csv", std::ios::app);
            inner << std::setprecision(17);
            for (int k = 0; k < n; ++k) {
                const double* m = &maplog[(size_t)k * UPIC_MAPLOG_COUNT];
                inner << time << "," << dt_try << "," << m[UPIC_MAPLOG_EVALUATION] << "," << m[UPIC_MAPLOG_CONVERGED]
                      << "," << m[UPIC_MAPLOG_FAILED] << "," << m[UPIC_MAPLOG_MAX_SCALED_RESIDUAL] << ","
                      << m[UPIC_MAPLOG_ITER_MEAN] << "," << m[UPIC_MAPLOG_ITER_MAX] << "\n";
            }
        }
        if (d.selective_failure_diagnostics) write_failed_particles(ctx.c, d, time);
        if (rc != UPIC_OK) {
            // the rejected attempt (:8741-8771); its solve report is not
            // returned by a failing step, so the counters keep their defaults
            Solve s;
            s.method = "none";
            s.rms = s.max_particle = kInf;
            adaptive << (accepted + 1) << "," << time << ",1," << dt_try << ",rejected," << 0 << "," << s.rms << ","
                     << s.max_particle << "," << kInf << "," << kInf << ",0,1,";
            Solve z;
            z.method = "none";
            write_local_columns(adaptive, z);
            adaptive << "," << seconds_since(t_start) << "\n";
            std::ostringstream msg;
            msg << "fixed step " << (accepted + 1) << " failed at t=" << std::defaultfloat << std::setprecision(6)
                << time << ": " << err;
            throw std::runtime_error(msg.str());
        }
        const Solve s = solve_of(info);
        adaptive << (accepted + 1) << "," << time << ",1," << dt_try << ",accepted," << s.iterations << "," << s.rms
                 << "," << s.max_particle << "," << s.rate << "," << s.contraction << "," << s.backtracked << ","
                 << s.min_alpha << ",";
        write_local_columns(adaptive, s);
        adaptive << "," << seconds_since(t_start) << "\n";
        adaptive.flush();
        time += dt_try;
        if (std::abs(time - target) <= teps) time = target;
        ++accepted;
        particle_snapshots(accepted);
        // path statistics of the step from its step diagnostics (:8827-8840)
        const long cross = (long)sd[UPIC_SD_CROSSING_PARTICLES];
        const long long segs = std::llround(sd[UPIC_SD_AVERAGE_PATH_SEGMENTS] * (double)np);
        const double avg = np ? (double)segs / (double)np : 0.0;
        write_diag(accepted, time, s, cross, avg, (long)sd[UPIC_SD_MAX_PATH_SEGMENTS], row, dt_try);
        stepcsv << accepted << "," << time << "," << s.iterations << "," << s.rms << "," << s.max_particle << ","
                << s.restarts << "," << s.method << "," << s.rate << "," << s.contraction << "," << s.backtracked << ","
                << s.min_alpha << ",";
        write_local_columns(stepcsv, s);
        for (int k = 0; k < UPIC_SD_COUNT; ++k) {
            const bool integer =
                k == UPIC_SD_CROSSING_PARTICLES || k == UPIC_SD_TOTAL_CROSSINGS || k == UPIC_SD_MAX_PATH_SEGMENTS;
            if (integer) stepcsv << "," << (long)sd[k];
            else stepcsv << "," << sd[k];
        }
        stepcsv << "," << dt_try << "," << seconds_since(t_start) << "\n";
        diag.flush();
        stepcsv.flush();
        const bool final_state = time + teps >= target;
        const bool interval_state = d.field_diagnostics_interval > 0.0 && time + teps >= next_field_time;
        if (d.field_diagnostics && (final_state || interval_state) && std::abs(time - last_field_time) > teps) {
            field_snapshot(accepted, time);
            last_field_time = time;
            while (next_field_time <= time + teps) next_field_time += d.field_diagnostics_interval;
        }
        if (progress_interval > 0.0 && (time + teps >= next_progress || time + teps >= target)) {
            std::cout << std::scientific << std::setprecision(3) << "accepted_step " << std::setw(5) << accepted
                      << " t=" << time << "/" << target << " dt=" << dt_try << " Gauss=" << row[UPIC_P3_GAUSS_RMS]
                      << " R_A=" << sd[UPIC_SD_A_CHAIN_ABS_RMS] << " R_work=" << sd[UPIC_SD_DEPOSIT_GATHER_WORK_RESIDUAL]
                      << " dE=" << sd[UPIC_SD_DELTA_TOTAL_ENERGY] << " Rnl=" << s.rms << " Rnl_max=" << s.max_particle
                      << " restarts=" << (long)s.restarts << " method=" << s.method << " rho=" << s.rate
                      << " Lsec=" << s.contraction << " bt=" << (long)s.backtracked
                      << " crossings=" << (long)sd[UPIC_SD_TOTAL_CROSSINGS] << " nonlinear_iters=" << (long)s.iterations
                      << " wall=" << wall_duration(seconds_since(t_start)) << "\n";
            while (next_progress <= time + teps && next_progress < target) next_progress += progress_interval;
        }
    }

    {   // write_particle_sample (:7791), at most 20000 evenly spaced particles
        const Particles p = particles_of(ctx.c, np);
        std::ofstream out(d.output_prefix + "_particle_sample.csv");
        out << "particle,x,y,z,vx,vy,vz,q,m\n";
        const size_t nw = std::min<size_t>(20000, (size_t)np);
        for (size_t r = 0; r < nw; ++r) {
            const size_t k = nw == 1 ? 0 : r * ((size_t)np - 1) / (nw - 1);
            out << k << "," << std::setprecision(17) << p.x[k] << "," << p.y[k] << "," << 0.0 << "," << p.v[3 * k]
                << "," << p.v[3 * k + 1] << "," << p.v[3 * k + 2] << "," << S.q[k] << "," << S.m[k] << "\n";
        }
    }
    const double wall = seconds_since(t_start);
    std::cout << std::scientific << std::setprecision(6) << "Final Gauss RMS = " << row[UPIC_P3_GAUSS_RMS] << "\n"
              << "Final relative Gauss residual = " << row[UPIC_P3_GAUSS_RELATIVE] << "\n"
              << "Final gauge RMS = " << row[UPIC_P3_GAUGE_RMS] << "\n"
              << "Final relative gauge residual = " << row[UPIC_P3_GAUGE_RELATIVE] << "\n"
              << "Final total energy = " << row[UPIC_P3_TOTAL_ENERGY] << "\n"
              << "Total wall time = " << wall_duration(wall) << " (" << wall << " s)\n";
    return 0;
}
