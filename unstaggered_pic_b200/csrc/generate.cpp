// Seeded synthetic plasma generator (host).  The reference's own initializers
// draw from std::mt19937 and libstdc++ distributions
// (Project2/spectral_pic_part3.cpp:624-733); the plasmas of the benchmark
// workloads have no reference initializer, so they come from this generator,
// which depends on no library distribution: every particle owns a splitmix64
// stream seeded from (seed, particle index), positions are uniform in its
// cell, and normalized momenta u = gamma v / c are Box-Muller normals.  The
// result is therefore identical for any thread count.
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/upic.h"

namespace {

inline uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Uniform in [0, 1) with 53 random bits.
inline double uniform01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * 0x1.0p-53; }

// Pair of standard normals (Box-Muller on (0,1] x [0,1)).
inline void normal2(uint64_t& s, double& a, double& b) {
    const double u1 = 1.0 - uniform01(s);
    const double u2 = uniform01(s);
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double t = 6.283185307179586476925286766559 * u2;
    a = r * std::cos(t);
    b = r * std::sin(t);
}

}  // namespace

extern "C" int upic_generate_bimaxwellian(int nx, int ny, double Lx, double Ly, int ppc, double c,
                                          double n0, const double* uth, const double* udrift,
                                          uint64_t seed, double* x, double* y, double* P, double* v,
                                          double* v_prev, double* q, double* m) {
    if (nx <= 0 || ny <= 0 || ppc <= 0 || !(Lx > 0) || !(Ly > 0) || !(c > 0) || !uth || !udrift || !x ||
        !y || !P || !v || !v_prev || !q || !m)
        return UPIC_ERR_ARGUMENT;
    const long np = (long)nx * ny * ppc;
    const double dx = Lx / nx, dy = Ly / ny;
    const double macro = n0 * Lx * Ly / (double)np;
    const double qe = -macro, me = macro;
    auto work = [&](long p0, long p1) {
        for (long p = p0; p < p1; ++p) {
            const long cell = p / ppc;
            const int i = (int)(cell / ny), j = (int)(cell % ny);
            uint64_t s = seed ^ (0xd1b54a32d192ed03ull * (uint64_t)(p + 1));
            splitmix64(s);
            x[p] = ((double)i + uniform01(s)) * dx;
            y[p] = ((double)j + uniform01(s)) * dy;
            double g0, g1, g2, g3;
            normal2(s, g0, g1);
            normal2(s, g2, g3);
            (void)g3;
            const double u[3] = {udrift[0] + uth[0] * g0, udrift[1] + uth[1] * g1, udrift[2] + uth[2] * g2};
            const double gam = std::sqrt(1.0 + u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            for (int d = 0; d < 3; ++d) {
                const double vd = c * u[d] / gam;
                v[3 * p + d] = vd;
                v_prev[3 * p + d] = vd;
                P[3 * p + d] = me * c * u[d];
            }
            q[p] = qe;
            m[p] = me;
        }
    };
    unsigned nt = std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if (nt > 64) nt = 64;
    if (np < 65536) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
        const long a = np * t / nt, b = np * (t + 1) / nt;
        th.emplace_back(work, a, b);
    }
    for (auto& t : th) t.join();
    return UPIC_OK;
}
