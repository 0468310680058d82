/*
 * TEST INFRASTRUCTURE ONLY (CPU oracle).  Restatement of the seeded synthetic
 * plasma that the benchmark workloads use (the configurations' bi-Maxwellian
 * plasmas have no initializer in the reference; the product generates them
 * with upic_generate_bimaxwellian).  The published algorithm restated here:
 * one splitmix64 stream per particle (Steele, Lea and Flood, "Fast splittable
 * pseudorandom number generators", OOPSLA 2014: increment 0x9e3779b97f4a7c15,
 * mix constants 0xbf58476d1ce4e5b9 / 0x94d049bb133111eb, shifts 30/27/31),
 * seeded as seed XOR (0xd1b54a32d192ed03 * (p + 1)) and advanced once;
 * uniforms from the top 53 bits; normals by the Box-Muller transform on
 * (0,1] x [0,1).  Particle p sits in cell p / ppc (x-major, cell = i*ny + j)
 * at a uniform position inside it; u = udrift + uth * (g0, g1, g2) is the
 * normalized momentum, v = c u / gamma, P = m c u, v_prev = v,
 * q = -n0 Lx Ly / Np, m = |q|.  Serial: the stream of a particle depends on
 * its index only, so the result equals the product's for any thread count.
 * Lets bench.py's reference arm and the CPU tests build the workload's
 * particles without loading the product library.
 */
#include <math.h>
#include <stdint.h>
#include "oracle.h"

static uint64_t sm64(uint64_t* s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static double unif(uint64_t* s) { return (double)(sm64(s) >> 11) * 0x1.0p-53; }

static void box_muller(uint64_t* s, double* a, double* b) {
    const double u1 = 1.0 - unif(s);
    const double u2 = unif(s);
    const double r = sqrt(-2.0 * log(u1));
    const double t = 6.283185307179586476925286766559 * u2;
    *a = r * cos(t);
    *b = r * sin(t);
}

int o_generate_bimaxwellian(int nx, int ny, double Lx, double Ly, int ppc, double c, double n0,
                            const double* uth, const double* udrift, uint64_t seed, double* x,
                            double* y, double* P, double* v, double* v_prev, double* q, double* m) {
    if (nx <= 0 || ny <= 0 || ppc <= 0 || !(Lx > 0) || !(Ly > 0) || !(c > 0)) return -2;
    const long np = (long)nx * ny * ppc;
    const double dx = Lx / nx, dy = Ly / ny;
    const double w = n0 * Lx * Ly / (double)np;
    for (long p = 0; p < np; ++p) {
        const long cell = p / ppc;
        const int i = (int)(cell / ny), j = (int)(cell % ny);
        uint64_t s = seed ^ (0xd1b54a32d192ed03ull * (uint64_t)(p + 1));
        sm64(&s);
        x[p] = ((double)i + unif(&s)) * dx;
        y[p] = ((double)j + unif(&s)) * dy;
        double g[4];
        box_muller(&s, &g[0], &g[1]);
        box_muller(&s, &g[2], &g[3]);
        double u[3], u2 = 0.0;
        for (int d = 0; d < 3; ++d) {
            u[d] = udrift[d] + uth[d] * g[d];
            u2 += u[d] * u[d];
        }
        /* same association as the product: 1 + u0^2 + u1^2 + u2^2 left to right */
        const double gam = sqrt(1.0 + u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        (void)u2;
        for (int d = 0; d < 3; ++d) {
            const double vd = c * u[d] / gam;
            v[3 * p + d] = vd;
            v_prev[3 * p + d] = vd;
            P[3 * p + d] = w * c * u[d];
        }
        q[p] = -w;
        m[p] = w;
    }
    return 0;
}
