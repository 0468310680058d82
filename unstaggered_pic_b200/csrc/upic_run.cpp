// upic_run: deck-driven drop-in for the reference's explicit solver CLI
// (Project2/spectral_pic_part3.cpp `main:1198`): reads the same `key = value`
// deck, loads the same particles, advances the step through the C ABI
// (include/upic.h) on the GPU and writes the reference's output files
// <output_prefix>_diagnostics.csv, _particle_sample.csv and _config_echo.txt
// in its formats.
//
//     upic_run deck.txt              Project2 decks (spectral_pic_part3)
//     upic_run --nonrel deck.txt     Project1 decks (ec_pic_serial_demo), run_nonrel.cpp
//     upic_run --p3 deck.txt         Project3 decks (ec_pic_nyquist_projected), run_p3.cpp
//
// Exit codes as the reference: 0 ok, 1 error (message on stderr), 2 usage,
// 3 failed start-up unit tests (Project1 decks).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/upic.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

// Deck keys, defaults and validation of the reference's Config / read_config
// (spectral_pic_part3.cpp:174-231, 233-293).
struct Deck {
    std::string example = "weibel";
    std::string method = "bdf1";
    std::string charge_update = "conserving";
    int nx = 32, ny = 32;
    double Lx = 2.0 * kPi, Ly = 2.0 * kPi;
    int n_steps = 100;
    double dt = 0.05;
    int particles_per_cell = 4;
    int cloud_particles = 4096;
    double c = 1.0, eps0 = 1.0, mu0 = 1.0, n0 = 1.0;
    double electron_charge_sign = -1.0, ion_charge_sign = 1.0;
    double weibel_vx = 0.5, weibel_vy_max = 0.01, weibel_sine_perturb = 0.002;
    int perturbation_mode = 1;
    double cloud_sigma = 1.0, cloud_drift = 0.01, cloud_thermal = 0.005;
    unsigned int seed = 12345;
    int diagnostic_stride = 1;
    int particle_sample_count = 2000;
    std::string output_prefix = "run";
    bool run_unit_tests = true;
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

Deck read_deck(const std::string& path) {
    Deck d;
    std::ifstream in(path);
    if (!in) throw std::runtime_error("could not open input file: " + path);
    std::string line;
    while (std::getline(in, line)) {
        const auto sharp = line.find('#');
        if (sharp != std::string::npos) line = line.substr(0, sharp);
        const auto eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = lowercase(trim(line.substr(0, eq)));
        const std::string val = trim(line.substr(eq + 1));
        if (key.empty()) continue;
        std::istringstream ss(val);
        if (key == "example" || key == "test_case") d.example = lowercase(val);
        else if (key == "method") d.method = lowercase(val);
        else if (key == "charge_update") d.charge_update = lowercase(val);
        else if (key == "nx") ss >> d.nx;
        else if (key == "ny") ss >> d.ny;
        else if (key == "lx") ss >> d.Lx;
        else if (key == "ly") ss >> d.Ly;
        else if (key == "n_steps") ss >> d.n_steps;
        else if (key == "dt") ss >> d.dt;
        else if (key == "particles_per_cell") ss >> d.particles_per_cell;
        else if (key == "cloud_particles") ss >> d.cloud_particles;
        else if (key == "c") ss >> d.c;
        else if (key == "eps0") ss >> d.eps0;
        else if (key == "mu0") ss >> d.mu0;
        else if (key == "n0") ss >> d.n0;
        else if (key == "electron_charge_sign") ss >> d.electron_charge_sign;
        else if (key == "ion_charge_sign") ss >> d.ion_charge_sign;
        else if (key == "weibel_vx") ss >> d.weibel_vx;
        else if (key == "weibel_vy_max") ss >> d.weibel_vy_max;
        else if (key == "weibel_sine_perturb") ss >> d.weibel_sine_perturb;
        else if (key == "perturbation_mode") ss >> d.perturbation_mode;
        else if (key == "cloud_sigma") ss >> d.cloud_sigma;
        else if (key == "cloud_drift") ss >> d.cloud_drift;
        else if (key == "cloud_thermal") ss >> d.cloud_thermal;
        else if (key == "seed") ss >> d.seed;
        else if (key == "diagnostic_stride") ss >> d.diagnostic_stride;
        else if (key == "particle_sample_count") ss >> d.particle_sample_count;
        else if (key == "output_prefix") d.output_prefix = val;
        else if (key == "run_unit_tests") d.run_unit_tests = parse_bool(val);
        else std::cerr << "warning: unknown input key ignored: " << key << "\n";
    }
    if (!pow2(d.nx) || !pow2(d.ny))
        throw std::runtime_error("the internal radix-2 FFT requires nx and ny to be powers of two");
    if (d.method != "bdf1" && d.method != "bdf2")
        throw std::runtime_error("method must be bdf1 or bdf2 in this teaching code");
    if (d.charge_update != "conserving" && d.charge_update != "naive")
        throw std::runtime_error("charge_update must be conserving or naive");
    if (d.example != "weibel" && d.example != "cloud" && d.example != "drifting_cloud")
        throw std::runtime_error("example must be weibel or cloud");
    return d;
}

// Particles in the ABI's layout (P, v, v_prev as xyz triples).
struct Particles {
    std::vector<double> x, y, P, v, vp, q, m;
    long size() const { return (long)x.size(); }
    void push(double px, double py, const double* vel, double pq, double pm, double c) {
        x.push_back(px);
        y.push_back(py);
        // A = 0 at start-up: P = m gamma v (canonical_from_velocity with A = 0)
        const double v2 = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
        const double gam = 1.0 / std::sqrt(std::max(1.0e-14, 1.0 - v2 / (c * c)));
        for (int k = 0; k < 3; ++k) {
            P.push_back(pm * gam * vel[k]);
            v.push_back(vel[k]);
            vp.push_back(vel[k]);
        }
        q.push_back(pq);
        m.push_back(pm);
    }
};

// Weibel quiet start: nsub x nsub positions per cell, two counter-streaming
// beams in x, uniform random vy plus a sine seed, drawn in the reference's
// order from std::mt19937 (initialize_weibel_particles :624-667).
Particles weibel_particles(const Deck& d) {
    const int nsub = std::max(1, (int)std::round(std::sqrt((double)d.particles_per_cell)));
    const long total = 2L * d.nx * d.ny * nsub * nsub;
    const double dx = d.Lx / d.nx, dy = d.Ly / d.ny;
    const double w = d.n0 * (d.Lx * d.Ly) / (double)total;
    const double q = d.electron_charge_sign * w, m = w;
    std::mt19937 rng(d.seed);
    std::uniform_real_distribution<double> uy(-d.weibel_vy_max, d.weibel_vy_max);
    Particles p;
    for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < d.ny; ++j)
            for (int a = 0; a < nsub; ++a)
                for (int b = 0; b < nsub; ++b) {
                    const double x = ((double)i + ((double)a + 0.5) / nsub) * dx;
                    const double y = ((double)j + ((double)b + 0.5) / nsub) * dy;
                    const double sine = d.weibel_sine_perturb * d.c * std::sin(2.0 * kPi * d.perturbation_mode * x / d.Lx);
                    for (int beam = -1; beam <= 1; beam += 2) {
                        const double vel[3] = {(double)beam * d.weibel_vx * d.c, uy(rng) + sine, 0.0};
                        p.push(x, y, vel, q, m, d.c);
                    }
                }
    return p;
}

double wrap_periodic(double x, double L) {
    x -= std::floor(x / L) * L;
    if (x >= L) x -= L;
    if (x < 0.0) x += L;
    return x;
}

// Gaussian cloud of electrons over a matching stationary ion cloud, drawn in
// the reference's order from std::mt19937 and std::normal_distribution
// (initialize_cloud_particles :669-725).  Ions are returned separately: they
// only contribute their fixed charge.
Particles cloud_particles(const Deck& d, Particles& ions) {
    const int np = d.cloud_particles;
    const double w = d.n0 * (d.Lx * d.Ly) / (double)np;
    const double qe = d.electron_charge_sign * w, qi = d.ion_charge_sign * w;
    std::mt19937 rng(d.seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    Particles e;
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int n = 0; n < np; ++n) {
        const double xc = 0.5 * d.Lx + d.cloud_sigma * normal(rng);
        const double yc = 0.5 * d.Ly + d.cloud_sigma * normal(rng);
        const double x = wrap_periodic(xc, d.Lx), y = wrap_periodic(yc, d.Ly);
        double vel[3];
        vel[0] = d.cloud_drift * d.c + d.cloud_thermal * normal(rng);
        vel[1] = d.cloud_drift * d.c + d.cloud_thermal * normal(rng);
        vel[2] = 0.0;
        const double sp = std::sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
        const double vmax = 0.2 * d.c;
        if (sp > vmax)
            for (double& vk : vel) vk *= vmax / sp;
        e.push(x, y, vel, qe, w, d.c);
        ions.push(x, y, zero, qi, w, d.c);
    }
    return e;
}

void check(int rc, const upic_ctx* ctx) {
    if (rc != UPIC_OK) throw std::runtime_error(upic_last_error(ctx));
}

upic_config abi_config(const Deck& d, double n0) {
    upic_config uc;
    upic_config_default(&uc);
    uc.nx = d.nx;
    uc.ny = d.ny;
    uc.Lx = d.Lx;
    uc.Ly = d.Ly;
    uc.dt = d.dt;
    uc.method = d.method == "bdf2" ? UPIC_METHOD_BDF2 : UPIC_METHOD_BDF1;
    uc.charge_update = d.charge_update == "naive" ? UPIC_CHARGE_NAIVE : UPIC_CHARGE_CONSERVING;
    uc.c = d.c;
    uc.eps0 = d.eps0;
    uc.mu0 = d.mu0;
    uc.n0 = n0;
    return uc;
}

// The reference's start-up check of the spectral derivative on a 16x8 grid
// (run_unit_tests :1006-1044), through the library's derivative.
void unit_tests(const Deck& d) {
    Deck t = d;
    t.nx = 16;
    t.ny = 8;
    t.Lx = t.Ly = 2.0 * kPi;
    upic_config uc = abi_config(t, t.n0);
    upic_ctx* ctx = nullptr;
    if (upic_create(&uc, &ctx) != UPIC_OK) throw std::runtime_error(upic_last_error(nullptr));
    const int N = t.nx * t.ny;
    const double hx = t.Lx / t.nx, hy = t.Ly / t.ny;
    std::vector<double> f(N), fx(N), fy(N);
    for (int i = 0; i < t.nx; ++i)
        for (int j = 0; j < t.ny; ++j) f[i * t.ny + j] = std::sin(3.0 * i * hx) + 0.5 * std::cos(2.0 * j * hy);
    const int rc1 = upic_spectral_derivative(ctx, f.data(), 0, fx.data());
    const int rc2 = rc1 ? rc1 : upic_spectral_derivative(ctx, f.data(), 1, fy.data());
    if (rc2) {
        const std::string msg = upic_last_error(ctx);
        upic_destroy(ctx);
        throw std::runtime_error(msg);
    }
    upic_destroy(ctx);
    double errx = 0.0, erry = 0.0;
    for (int i = 0; i < t.nx; ++i)
        for (int j = 0; j < t.ny; ++j) {
            const int id = i * t.ny + j;
            errx = std::max(errx, std::fabs(fx[id] - 3.0 * std::cos(3.0 * i * hx)));
            erry = std::max(erry, std::fabs(fy[id] + std::sin(2.0 * j * hy)));
        }
    if (errx > 1.0e-10 || erry > 1.0e-10) {
        std::ostringstream msg;
        msg << "FFT derivative unit test failed: errx=" << errx << " erry=" << erry;
        throw std::runtime_error(msg.str());
    }
}

void write_row(std::ofstream& out, long step, double time, const Deck& d, const char* active, const double* r) {
    out << step << ',' << time << ',' << d.method << ',' << active << ',' << d.charge_update;
    for (int k = 0; k < UPIC_DIAG_COUNT; ++k) out << ',' << r[k];
    out << "\n";
}

void run(const Deck& d) {
    if (d.run_unit_tests) unit_tests(d);
    Particles ions;
    const bool cloud = d.example != "weibel";
    Particles e = cloud ? cloud_particles(d, ions) : weibel_particles(d);
    const int N = d.nx * d.ny;

    // stationary ions: their deposited charge is the fixed background
    std::vector<double> bg;
    if (cloud) {
        upic_config uc0 = abi_config(d, 0.0);
        upic_ctx* c0 = nullptr;
        if (upic_create(&uc0, &c0) != UPIC_OK) throw std::runtime_error(upic_last_error(nullptr));
        bg.assign(N, 0.0);
        const int rc = upic_deposit_charge(c0, ions.size(), ions.x.data(), ions.y.data(), ions.q.data(), bg.data());
        const std::string msg = rc ? upic_last_error(c0) : "";
        upic_destroy(c0);
        if (rc) throw std::runtime_error(msg);
    }

    upic_config uc = abi_config(d, d.n0);
    upic_ctx* ctx = nullptr;
    if (upic_create(&uc, &ctx) != UPIC_OK) throw std::runtime_error(upic_last_error(nullptr));
    try {
        check(upic_set_particles(ctx, e.size(), e.x.data(), e.y.data(), e.P.data(), e.v.data(), e.vp.data(),
                                 e.q.data(), e.m.data()), ctx);
        if (cloud) check(upic_set_background(ctx, bg.data()), ctx);

        {   // write_config_echo (:964-984)
            std::ofstream out(d.output_prefix + "_config_echo.txt");
            out << std::setprecision(17);
            out << "example = " << d.example << "\n" << "method = " << d.method << "\n"
                << "charge_update = " << d.charge_update << "\n" << "nx = " << d.nx << "\n"
                << "ny = " << d.ny << "\n" << "Lx = " << d.Lx << "\n" << "Ly = " << d.Ly << "\n"
                << "dt = " << d.dt << "\n" << "n_steps = " << d.n_steps << "\n" << "c = " << d.c << "\n"
                << "eps0 = " << d.eps0 << "\n" << "mu0 = " << d.mu0 << "\n" << "n0 = " << d.n0 << "\n"
                << "mobile_electrons = " << e.size() << "\n" << "static_ions = " << ions.size() << "\n"
                << "cell_area = " << (d.Lx / d.nx) * (d.Ly / d.ny) << "\n"
                << "output_prefix = " << d.output_prefix << "\n";
        }

        std::ofstream diag(d.output_prefix + "_diagnostics.csv");
        diag << std::setprecision(17);
        diag << "step,time,requested_method,active_method,charge_update,"
             << "gauge_rms,gauss_rms,continuity_rms,Bz_l2,B_l2,E_l2,rho_l2,J_l2,"
             << "field_energy,kinetic_energy,total_energy,max_speed,mean_gamma\n";
        double row0[UPIC_DIAG_COUNT];
        check(upic_init_fields(ctx, row0), ctx);
        write_row(diag, 0, 0.0, d, "initial", row0);

        // the step loop in blocks; rows of steps without diagnostics are NaN
        const int stride = std::max(1, d.diagnostic_stride);
        const int block = 1000;
        std::vector<double> rows((size_t)block * UPIC_DIAG_COUNT);
        const char* active = d.method == "bdf2" ? "bdf2" : "bdf1";
        for (int s0 = 0; s0 < d.n_steps; s0 += block) {
            const int k = std::min(block, d.n_steps - s0);
            // diagnostics on step % stride == 0 and on the run's last step
            check(upic_step(ctx, k, stride, rows.data()), ctx);
            for (int i = 0; i < k; ++i) {
                const int step = s0 + i + 1;
                if (step % stride == 0 || step == d.n_steps)
                    write_row(diag, step, step * d.dt, d, active, rows.data() + (size_t)i * UPIC_DIAG_COUNT);
            }
        }

        // write_particle_sample (:986-998), electrons in their load order
        std::vector<double> x(e.size()), y(e.size()), P(3 * e.size()), v(3 * e.size()), vp(3 * e.size());
        check(upic_get_particles(ctx, e.size(), x.data(), y.data(), P.data(), v.data(), vp.data()), ctx);
        std::ofstream ps(d.output_prefix + "_particle_sample.csv");
        ps << std::setprecision(17);
        ps << "id,x,y,x_centered,y_centered,vx,vy,vz,q,m,gamma\n";
        const long count = std::min<long>(d.particle_sample_count, e.size());
        for (long i = 0; i < count; ++i) {
            const double* vi = &v[3 * i];
            const double beta2 = (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]) / (d.c * d.c);
            const double gam = 1.0 / std::sqrt(std::max(1.0e-14, 1.0 - beta2));
            ps << i << ',' << x[i] << ',' << y[i] << ',' << x[i] - 0.5 * d.Lx << ',' << y[i] - 0.5 * d.Ly << ','
               << vi[0] << ',' << vi[1] << ',' << vi[2] << ',' << e.q[i] << ',' << e.m[i] << ',' << gam << "\n";
        }
    } catch (...) {
        upic_destroy(ctx);
        throw;
    }
    upic_destroy(ctx);
    std::cout << "wrote " << d.output_prefix << "_diagnostics.csv\n";
    std::cout << "wrote " << d.output_prefix << "_particle_sample.csv\n";
    std::cout << "wrote " << d.output_prefix << "_config_echo.txt\n";
}

}  // namespace

int run_nonrel(const std::string& path);
int run_p3(const std::string& path);

int main(int argc, char** argv) {
    try {
        const bool nonrel = argc == 3 && std::string(argv[1]) == "--nonrel";
        const bool p3 = argc == 3 && std::string(argv[1]) == "--p3";
        if ((argc != 2 && !nonrel && !p3) || (argc == 2 && std::string(argv[1]).rfind("--", 0) == 0)) {
            std::cerr << "usage: " << argv[0] << " [--nonrel | --p3] input_file.txt\n";
            return 2;
        }
        if (nonrel) return run_nonrel(argv[2]);
        if (p3) return run_p3(argv[2]);
        run(read_deck(argv[1]));
        return 0;
    } catch (const std::exception& ex) {
        std::cerr << "error: " << ex.what() << "\n";
        return 1;
    }
}
