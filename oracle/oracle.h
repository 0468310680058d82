/*
 * CPU oracle for the unstaggered GM-PIC step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU baseline as the checker.
 * The product (libupic.so) never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle_ref.py checks these functions bit for bit
 * against the reference's own code (oracle/_ref/libref_p2.so, compiled from the
 * reference sources by oracle/Makefile), and tests/test_oracle_golden.py checks
 * full oracle runs of the reference's shipped decks against the published
 * numbers in Project2/docs/validation_summary.json.
 *
 * Conventions follow Project2/spectral_pic_part3.cpp: node id = i*ny + j
 * (x index i is the slow one), positions in [0, L), quadratic B-spline.
 */
#ifndef UPIC_ORACLE_H
#define UPIC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Grid wave numbers kx, ky, k2 (N = nx*ny each).  spectral_pic_part3.cpp:320-357 */
void o2_wavenumbers(int nx, int ny, double Lx, double Ly, double* kx, double* ky, double* k2);

/* In-place complex 2D FFT, rows (y) then columns (x).  spectral_pic_part3.cpp:372-424 */
int o2_fft2d(int nx, int ny, double* re, double* im, int inverse);

/* J (3 x N) = sum_p q v S(x_p)/dA.  spectral_pic_part3.cpp:747-755 */
void o2_deposit_current(int nx, int ny, double Lx, double Ly, long np, const double* x,
                        const double* y, const double* v, const double* q, double* J);

/* rho = n0 (fixed ions) + sum_p q S(x_p)/dA.  spectral_pic_part3.cpp:739-745 */
void o2_deposit_charge(int nx, int ny, double Lx, double Ly, double n0, long np,
                       const double* x, const double* y, const double* q, double* rho);

/* out[p] = sum f S(x_p).  spectral_pic_part3.cpp:564-574 */
void o2_gather(int nx, int ny, double Lx, double Ly, const double* f, long np,
               const double* x, const double* y, double* out);

/* d/dx (dir 0) or d/dy (dir 1), pseudo-spectral.  spectral_pic_part3.cpp:440-447 */
void o2_spectral_derivative(int nx, int ny, double Lx, double Ly, const double* f, int dir,
                            double* out);

/* phi from Poisson, zero-mean gauge.  spectral_pic_part3.cpp:819-827 */
void o2_poisson(int nx, int ny, double Lx, double Ly, double eps0, const double* rho,
                double* phi);

/* Full explicit BDF/IAEM run on injected electrons; same argument contract as
 * ref_p2_simulate in oracle/ref/ref_p2_harness.cpp.  spectral_pic_part3.cpp:1094-1189 */
int o2_simulate(const double* params, const int* iparams, long np, double* x, double* y,
                double* P, double* v, double* vprev, const double* q, const double* m,
                double* diag_out, double* fields_out, double* seconds_out);

/* Reference Weibel quiet start (spectral_pic_part3.cpp:624-669), including the
 * libstdc++ std::mt19937 / uniform_real_distribution draw sequence. */
long o2_init_weibel(int nx, int ny, double Lx, double Ly, int ppc, double c, double n0,
                    double vx, double vy_max, double sine, int mode, unsigned seed,
                    long np_capacity, double* x, double* y, double* P, double* v,
                    double* vprev, double* q, double* m);

/* Seeded bi-Maxwellian plasma of the benchmark workloads (splitmix64 streams
 * per particle + Box-Muller); the same arrays as upic_generate_bimaxwellian.
 * Returns 0, or -2 on a bad argument. */
int o_generate_bimaxwellian(int nx, int ny, double Lx, double Ly, int ppc, double c, double n0,
                            const double* uth, const double* udrift, uint64_t seed, double* x,
                            double* y, double* P, double* v, double* v_prev, double* q, double* m);

/* std::mt19937 restated (C++ [rand.eng.mers] parameters). */
typedef struct {
    uint32_t mt[624];
    int idx;
} o_mt19937;
void o_mt_seed(o_mt19937* g, uint32_t seed);
uint32_t o_mt_next(o_mt19937* g);
/* libstdc++ generate_canonical<double, 53>(mt19937): two 32-bit draws. */
double o_mt_canonical(o_mt19937* g);

#ifdef __cplusplus
}
#endif
#endif
