/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the explicit spectral BDF/IAEM
 * step of Project2/spectral_pic_part3.cpp (the reference).  Every function
 * restates one reference function, in the same floating-point operation order,
 * so that it reproduces the reference bit for bit (checked against the
 * reference's own compiled code by tests/test_oracle_ref.py).  Compiled with
 * -ffp-contract=off because the reference build (-O2, x86-64, no -mfma) does
 * not contract multiply-adds.
 *
 * Layout: node id = i*ny + j; fields of N = nx*ny doubles; particle vectors
 * (P, v, v_prev) are interleaved xyz triples, 3*np doubles.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "oracle.h"

static const double O_PI = 3.141592653589793238462643383279502884;

typedef struct {
    int nx, ny, N;
    double Lx, Ly, dx, dy, dA;
    double *kx, *ky, *k2;
} o2_grid;

/* spectral_pic_part3.cpp:320-330 (Nyquist wave number zeroed). */
static int mode_number(int i, int n) {
    if (n > 1 && i == n / 2) return 0;
    return (i < n / 2) ? i : i - n;
}

void o2_wavenumbers(int nx, int ny, double Lx, double Ly, double* kx, double* ky, double* k2) {
    for (int i = 0; i < nx; ++i) {
        const double kxi = 2.0 * O_PI * (double)mode_number(i, nx) / Lx;
        for (int j = 0; j < ny; ++j) {
            const double kyj = 2.0 * O_PI * (double)mode_number(j, ny) / Ly;
            const int id = i * ny + j;
            kx[id] = kxi;
            ky[id] = kyj;
            k2[id] = kxi * kxi + kyj * kyj;
        }
    }
}

/* spectral_pic_part3.cpp:332-357 */
static void grid_init(o2_grid* g, int nx, int ny, double Lx, double Ly) {
    g->nx = nx;
    g->ny = ny;
    g->N = nx * ny;
    g->Lx = Lx;
    g->Ly = Ly;
    g->dx = Lx / (double)nx;
    g->dy = Ly / (double)ny;
    g->dA = g->dx * g->dy;
    g->kx = (double*)malloc(sizeof(double) * g->N);
    g->ky = (double*)malloc(sizeof(double) * g->N);
    g->k2 = (double*)malloc(sizeof(double) * g->N);
    o2_wavenumbers(nx, ny, Lx, Ly, g->kx, g->ky, g->k2);
}

static void grid_free(o2_grid* g) {
    free(g->kx);
    free(g->ky);
    free(g->k2);
}

/* ---- FFT: iterative radix-2 Cooley-Tukey with the twiddle recurrence
 *      w *= wlen (spectral_pic_part3.cpp:372-404). ---------------------- */
static void fft1d(int n, double* re, double* im, int inverse) {
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double angle = 2.0 * O_PI / (double)len * (inverse ? 1.0 : -1.0);
        const double wr_len = cos(angle), wi_len = sin(angle);
        for (int i = 0; i < n; i += len) {
            double wr = 1.0, wi = 0.0;
            for (int j = 0; j < len / 2; ++j) {
                const double ur = re[i + j], ui = im[i + j];
                const double ar = re[i + j + len / 2], ai = im[i + j + len / 2];
                const double vr = ar * wr - ai * wi;
                const double vi = ar * wi + ai * wr;
                re[i + j] = ur + vr;
                im[i + j] = ui + vi;
                re[i + j + len / 2] = ur - vr;
                im[i + j + len / 2] = ui - vi;
                const double nwr = wr * wr_len - wi * wi_len;
                const double nwi = wr * wi_len + wi * wr_len;
                wr = nwr;
                wi = nwi;
            }
        }
    }
    if (inverse) {
        const double inv_n = 1.0 / (double)n;
        for (int i = 0; i < n; ++i) {
            re[i] *= inv_n;
            im[i] *= inv_n;
        }
    }
}

/* spectral_pic_part3.cpp:406-424: y rows first, then x columns. */
int o2_fft2d(int nx, int ny, double* re, double* im, int inverse) {
    const int nmax = nx > ny ? nx : ny;
    double* tr = (double*)malloc(sizeof(double) * nmax);
    double* ti = (double*)malloc(sizeof(double) * nmax);
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) { tr[j] = re[i * ny + j]; ti[j] = im[i * ny + j]; }
        fft1d(ny, tr, ti, inverse);
        for (int j = 0; j < ny; ++j) { re[i * ny + j] = tr[j]; im[i * ny + j] = ti[j]; }
    }
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) { tr[i] = re[i * ny + j]; ti[i] = im[i * ny + j]; }
        fft1d(nx, tr, ti, inverse);
        for (int i = 0; i < nx; ++i) { re[i * ny + j] = tr[i]; im[i * ny + j] = ti[i]; }
    }
    free(tr);
    free(ti);
    return 0;
}

/* fft_real (spectral_pic_part3.cpp:426-431). */
static void fft_real(const o2_grid* g, const double* f, double* re, double* im) {
    for (int id = 0; id < g->N; ++id) { re[id] = f[id]; im[id] = 0.0; }
    o2_fft2d(g->nx, g->ny, re, im, 0);
}

/* ifft_real (spectral_pic_part3.cpp:433-438): real part of the inverse. */
static void ifft_real(const o2_grid* g, double* re, double* im, double* out) {
    o2_fft2d(g->nx, g->ny, re, im, 1);
    memcpy(out, re, sizeof(double) * g->N);
}

/* ---- Quadratic B-spline (spectral_pic_part3.cpp:537-552) -------------- */
typedef struct {
    int i[3];
    double w[3];
} o2_w1d;

static o2_w1d quadratic_weights(double x, double dx, int n) {
    const double s = x / dx;
    const int ic = (int)floor(s + 0.5);
    const double r = s - (double)ic;
    o2_w1d out;
    out.i[0] = (ic - 1 + n) % n;
    out.i[1] = (ic + n) % n;
    out.i[2] = (ic + 1 + n) % n;
    out.w[0] = 0.5 * (0.5 - r) * (0.5 - r);
    out.w[1] = 0.75 - r * r;
    out.w[2] = 0.5 * (0.5 + r) * (0.5 + r);
    return out;
}

/* Grid::index wrap (spectral_pic_part3.cpp:313-317). */
static int gidx(const o2_grid* g, int i, int j) {
    i = (i % g->nx + g->nx) % g->nx;
    j = (j % g->ny + g->ny) % g->ny;
    return i * g->ny + j;
}

/* spectral_pic_part3.cpp:554-562 */
static void scatter_scalar(double* f, const o2_grid* g, double x, double y, double value) {
    const o2_w1d wx = quadratic_weights(x, g->dx, g->nx);
    const o2_w1d wy = quadratic_weights(y, g->dy, g->ny);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            f[gidx(g, wx.i[a], wy.i[b])] += value * wx.w[a] * wy.w[b] / g->dA;
}

/* spectral_pic_part3.cpp:564-574 */
static double gather_scalar(const double* f, const o2_grid* g, double x, double y) {
    const o2_w1d wx = quadratic_weights(x, g->dx, g->nx);
    const o2_w1d wy = quadratic_weights(y, g->dy, g->ny);
    double value = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            value += f[gidx(g, wx.i[a], wy.i[b])] * wx.w[a] * wy.w[b];
    return value;
}

/* spectral_pic_part3.cpp:747-755 */
static void deposit_current_g(const o2_grid* g, long np, const double* x, const double* y,
                              const double* v, const double* q, double* J) {
    memset(J, 0, sizeof(double) * 3 * (size_t)g->N);
    for (long p = 0; p < np; ++p) {
        scatter_scalar(J, g, x[p], y[p], q[p] * v[3 * p + 0]);
        scatter_scalar(J + g->N, g, x[p], y[p], q[p] * v[3 * p + 1]);
        scatter_scalar(J + 2 * (size_t)g->N, g, x[p], y[p], q[p] * v[3 * p + 2]);
    }
}

/* spectral_pic_part3.cpp:739-745 */
static void deposit_charge_g(const o2_grid* g, double n0, long np, const double* x,
                             const double* y, const double* q, double* rho) {
    for (int id = 0; id < g->N; ++id) rho[id] = n0;
    for (long p = 0; p < np; ++p) scatter_scalar(rho, g, x[p], y[p], q[p]);
}

void o2_deposit_current(int nx, int ny, double Lx, double Ly, long np, const double* x,
                        const double* y, const double* v, const double* q, double* J) {
    o2_grid g;
    grid_init(&g, nx, ny, Lx, Ly);
    deposit_current_g(&g, np, x, y, v, q, J);
    grid_free(&g);
}

void o2_deposit_charge(int nx, int ny, double Lx, double Ly, double n0, long np,
                       const double* x, const double* y, const double* q, double* rho) {
    o2_grid g;
    grid_init(&g, nx, ny, Lx, Ly);
    deposit_charge_g(&g, n0, np, x, y, q, rho);
    grid_free(&g);
}

void o2_gather(int nx, int ny, double Lx, double Ly, const double* f, long np,
               const double* x, const double* y, double* out) {
    o2_grid g;
    grid_init(&g, nx, ny, Lx, Ly);
    for (long p = 0; p < np; ++p) out[p] = gather_scalar(f, &g, x[p], y[p]);
    grid_free(&g);
}

/* ---- Spectral operators (spectral_pic_part3.cpp:440-489) -------------- */
typedef struct {
    double *re, *im, *re2, *im2;
} o2_work;

static void work_init(o2_work* w, int N) {
    w->re = (double*)malloc(sizeof(double) * N);
    w->im = (double*)malloc(sizeof(double) * N);
    w->re2 = (double*)malloc(sizeof(double) * N);
    w->im2 = (double*)malloc(sizeof(double) * N);
}

static void work_free(o2_work* w) {
    free(w->re); free(w->im); free(w->re2); free(w->im2);
}

/* h *= i*k : (a+ib)(0+ik) = (a*0 - b*k) + i(a*k + b*0), as std::complex does. */
static void spectral_derivative_g(const o2_grid* g, o2_work* w, const double* f, int dir,
                                  double* out) {
    fft_real(g, f, w->re, w->im);
    const double* k = dir == 0 ? g->kx : g->ky;
    for (int id = 0; id < g->N; ++id) {
        const double a = w->re[id], b = w->im[id], kk = k[id];
        w->re[id] = a * 0.0 - b * kk;
        w->im[id] = a * kk + b * 0.0;
    }
    ifft_real(g, w->re, w->im, out);
}

/* div = i*(kx*hx + ky*hy) (spectral_pic_part3.cpp:449-455) */
static void spectral_divergence_g(const o2_grid* g, o2_work* w, const double* Vx,
                                  const double* Vy, double* out) {
    fft_real(g, Vx, w->re, w->im);
    fft_real(g, Vy, w->re2, w->im2);
    for (int id = 0; id < g->N; ++id) {
        const double sr = g->kx[id] * w->re[id] + g->ky[id] * w->re2[id];
        const double si = g->kx[id] * w->im[id] + g->ky[id] * w->im2[id];
        /* (0+1i)*(sr+i si) = (0*sr - 1*si) + i(0*si + 1*sr) */
        w->re[id] = 0.0 * sr - 1.0 * si;
        w->im[id] = 0.0 * si + 1.0 * sr;
    }
    ifft_real(g, w->re, w->im, out);
}

void o2_spectral_derivative(int nx, int ny, double Lx, double Ly, const double* f, int dir,
                            double* out) {
    o2_grid g;
    o2_work w;
    grid_init(&g, nx, ny, Lx, Ly);
    work_init(&w, g.N);
    spectral_derivative_g(&g, &w, f, dir, out);
    work_free(&w);
    grid_free(&g);
}

/* spectral_pic_part3.cpp:819-827 */
static void poisson_g(const o2_grid* g, o2_work* w, double eps0, const double* rho, double* phi) {
    fft_real(g, rho, w->re, w->im);
    for (int id = 0; id < g->N; ++id) {
        if (g->k2[id] > 0.0) {
            const double d = eps0 * g->k2[id];
            w->re[id] = w->re[id] / d;
            w->im[id] = w->im[id] / d;
        } else {
            w->re[id] = 0.0;
            w->im[id] = 0.0;
        }
    }
    ifft_real(g, w->re, w->im, phi);
}

void o2_poisson(int nx, int ny, double Lx, double Ly, double eps0, const double* rho,
                double* phi) {
    o2_grid g;
    o2_work w;
    grid_init(&g, nx, ny, Lx, Ly);
    work_init(&w, g.N);
    poisson_g(&g, &w, eps0, rho, phi);
    work_free(&w);
    grid_free(&g);
}

/* ---- BDF machinery (spectral_pic_part3.cpp:764-880) ------------------- */
#define HIST 5
typedef struct {
    double* s[HIST]; /* s[0] = u^n, s[1] = u^{n-1}, ... */
} o2_hist;

static void hist_init(o2_hist* h, const double* f, int N) {
    for (int i = 0; i < HIST; ++i) {
        h->s[i] = (double*)malloc(sizeof(double) * N);
        memcpy(h->s[i], f, sizeof(double) * N);
    }
}

/* push_new: the new field becomes s[0]; the oldest buffer is recycled. */
static void hist_push(o2_hist* h, double* f_new, int N) {
    double* oldest = h->s[HIST - 1];
    for (int i = HIST - 1; i > 0; --i) h->s[i] = h->s[i - 1];
    h->s[0] = oldest;
    memcpy(h->s[0], f_new, sizeof(double) * N);
}

static void hist_free(o2_hist* h) {
    for (int i = 0; i < HIST; ++i) free(h->s[i]);
}

typedef struct {
    int na;
    double a[3];
} o2_bdf;

/* spectral_pic_part3.cpp:769-777 */
static o2_bdf bdf_coeffs(int order) {
    o2_bdf b;
    if (order == 2) { b.na = 3; b.a[0] = 1.5; b.a[1] = -2.0; b.a[2] = 0.5; }
    else { b.na = 2; b.a[0] = 1.0; b.a[1] = -1.0; b.a[2] = 0.0; }
    return b;
}

/* spectral_pic_part3.cpp:829-848 */
static void solve_bdf_wave_g(const o2_grid* g, o2_work* w, const double* src, const o2_hist* h,
                             o2_bdf bdf, double c, double dt, double* out) {
    double b[5] = {0, 0, 0, 0, 0};
    const int nb = 2 * bdf.na - 1;
    for (int i = 0; i < bdf.na; ++i)
        for (int j = 0; j < bdf.na; ++j) b[i + j] += bdf.a[i] * bdf.a[j];
    const double scale = 1.0 / (c * c * dt * dt);
    fft_real(g, src, w->re, w->im);
    for (int l = 1; l < nb; ++l) {
        fft_real(g, h->s[l - 1], w->re2, w->im2);
        const double s = scale * b[l];
        for (int id = 0; id < g->N; ++id) {
            w->re[id] -= s * w->re2[id];
            w->im[id] -= s * w->im2[id];
        }
    }
    for (int id = 0; id < g->N; ++id) {
        const double denom = scale * b[0] + g->k2[id];
        w->re[id] /= denom;
        w->im[id] /= denom;
    }
    ifft_real(g, w->re, w->im, out);
}

/* spectral_pic_part3.cpp:850-863 */
static void bdf_first_derivative_g(const o2_grid* g, const double* u_new, const o2_hist* h,
                                   o2_bdf bdf, double dt, double* out) {
    for (int id = 0; id < g->N; ++id) out[id] = bdf.a[0] * u_new[id];
    for (int l = 1; l < bdf.na; ++l)
        for (int id = 0; id < g->N; ++id) out[id] += bdf.a[l] * h->s[l - 1][id];
    for (int id = 0; id < g->N; ++id) out[id] /= dt;
}

/* spectral_pic_part3.cpp:865-880 */
static void continuity_g(const o2_grid* g, o2_work* w, const o2_hist* rho_h, const double* J,
                         o2_bdf bdf, double dt, double* rho_new, double* scratch) {
    spectral_divergence_g(g, w, J, J + g->N, scratch);
    for (int id = 0; id < g->N; ++id) {
        double hs = 0.0;
        for (int l = 1; l < bdf.na; ++l) hs += bdf.a[l] * rho_h->s[l - 1][id];
        rho_new[id] = -(dt * scratch[id] + hs) / bdf.a[0];
    }
}

/* ---- Particles (spectral_pic_part3.cpp:161-167, 596-612, 1050-1092) ---- */
static double wrap_periodic(double x, double L) {
    x -= floor(x / L) * L;
    if (x >= L) x -= L;
    if (x < 0.0) x += L;
    return x;
}

static double gamma_from_v3(const double* v, double c) {
    const double beta2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / (c * c);
    const double one_m = 1.0 - beta2;
    const double safe = one_m > 1.0e-14 ? one_m : 1.0e-14;
    return 1.0 / sqrt(safe);
}

static void velocity_from_canonical(const double* P, double q, double m, const double* A,
                                    double c, double* v) {
    const double p0 = P[0] - q * A[0], p1 = P[1] - q * A[1], p2 = P[2] - q * A[2];
    const double denom = sqrt(c * c * (p0 * p0 + p1 * p1 + p2 * p2) + (m * c * c) * (m * c * c));
    if (denom == 0.0) { v[0] = v[1] = v[2] = 0.0; return; }
    const double s = c * c / denom;
    v[0] = s * p0;
    v[1] = s * p1;
    v[2] = s * p2;
}

/* Gathered field set used by the IAEM push: A (3), grad phi (x,y), grad A
 * (component c, direction d) at index 5 + 2c + d. */
#define NGF 11

static void push_g(const o2_grid* g, long np, const double* x, const double* y, double* P,
                   double* v, double* vprev, const double* q, const double* m,
                   double* const* F, double c, double dt) {
    for (long p = 0; p < np; ++p) {
        double G[NGF];
        for (int f = 0; f < NGF; ++f) G[f] = gather_scalar(F[f], g, x[p], y[p]);
        double* vp = v + 3 * p;
        double* vq = vprev + 3 * p;
        double* Pp = P + 3 * p;
        const double vs0 = 2.0 * vp[0] - vq[0];
        const double vs1 = 2.0 * vp[1] - vq[1];
        const double vs2 = 2.0 * vp[2] - vq[2];
        /* gather of the (zero) z component of grad phi, as the reference does */
        const double gpz = 0.0;
        const double gdx = G[5] * vs0 + G[7] * vs1 + G[9] * vs2;
        const double gdy = G[6] * vs0 + G[8] * vs1 + G[10] * vs2;
        const double f0 = (-1.0) * G[3] + gdx;
        const double f1 = (-1.0) * G[4] + gdy;
        const double f2 = (-1.0) * gpz + 0.0;
        const double qdt = q[p] * dt;
        double Pn[3] = {Pp[0] + qdt * f0, Pp[1] + qdt * f1, Pp[2] + qdt * f2};
        const double A[3] = {G[0], G[1], G[2]};
        double vn[3];
        velocity_from_canonical(Pn, q[p], m[p], A, c, vn);
        vq[0] = vp[0]; vq[1] = vp[1]; vq[2] = vp[2];
        vp[0] = vn[0]; vp[1] = vn[1]; vp[2] = vn[2];
        Pp[0] = Pn[0]; Pp[1] = Pn[1]; Pp[2] = Pn[2];
    }
}

/* ---- Diagnostics (spectral_pic_part3.cpp:497-523, 902-962) ------------- */
static double rms1(const double* f, int N) {
    long double s = 0.0L;
    for (int i = 0; i < N; ++i) s += (long double)f[i] * (long double)f[i];
    return sqrt((double)(s / (long double)N));
}

static double rms3(const double* a, const double* b, const double* c, int N) {
    long double s = 0.0L;
    for (int i = 0; i < N; ++i)
        s += (long double)a[i] * a[i] + (long double)b[i] * b[i] + (long double)c[i] * c[i];
    return sqrt((double)(s / (long double)N));
}

static double integral_sq3(const double* a, const double* b, const double* c, int N, double dA) {
    long double s = 0.0L;
    for (int i = 0; i < N; ++i)
        s += (long double)a[i] * a[i] + (long double)b[i] * b[i] + (long double)c[i] * c[i];
    return (double)(s * dA);
}

static void diagnostics_g(const o2_grid* g, o2_work* w, long np, const double* v,
                          const double* m, const o2_hist* phi_h, const o2_hist* A_h,
                          const o2_hist* rho_h, const double* phi_new, double* const* A_new,
                          const double* rho_cur, const double* J, o2_bdf bdf, double c,
                          double eps0, double mu0, double dt, double* out) {
    const int N = g->N;
    double* t1 = (double*)malloc(sizeof(double) * N);
    double* t2 = (double*)malloc(sizeof(double) * N);
    double* gauge = (double*)malloc(sizeof(double) * N);
    double* E = (double*)malloc(sizeof(double) * 3 * N);
    double* B = (double*)malloc(sizeof(double) * 3 * N);
    double* gx = (double*)malloc(sizeof(double) * N);
    double* gy = (double*)malloc(sizeof(double) * N);

    /* gauge = phi_t / c^2 + div A */
    bdf_first_derivative_g(g, phi_new, phi_h, bdf, dt, t1);
    spectral_divergence_g(g, w, A_new[0], A_new[1], t2);
    for (int id = 0; id < N; ++id) gauge[id] = t1[id] / (c * c) + t2[id];
    out[0] = rms1(gauge, N);

    /* E = -grad phi - A_t (grad phi z-component is a zero field) */
    spectral_derivative_g(g, w, phi_new, 0, gx);
    spectral_derivative_g(g, w, phi_new, 1, gy);
    for (int comp = 0; comp < 3; ++comp) {
        bdf_first_derivative_g(g, A_new[comp], &A_h[comp], bdf, dt, t1);
        const double* gp = comp == 0 ? gx : (comp == 1 ? gy : NULL);
        for (int id = 0; id < N; ++id)
            E[comp * N + id] = -(gp ? gp[id] : 0.0) - t1[id];
    }
    /* gauss = div E - rho/eps0 */
    spectral_divergence_g(g, w, E, E + N, t2);
    for (int id = 0; id < N; ++id) gauge[id] = t2[id] - rho_cur[id] / eps0;
    out[1] = rms1(gauge, N);

    /* continuity = rho_t + div J */
    spectral_divergence_g(g, w, J, J + N, t2);
    bdf_first_derivative_g(g, rho_cur, rho_h, bdf, dt, t1);
    for (int id = 0; id < N; ++id) gauge[id] = t1[id] + t2[id];
    out[2] = rms1(gauge, N);

    /* B = curl A (spectral_pic_part3.cpp:475-489) */
    spectral_derivative_g(g, w, A_new[2], 0, gx);      /* dAz/dx */
    spectral_derivative_g(g, w, A_new[2], 1, gy);      /* dAz/dy */
    spectral_derivative_g(g, w, A_new[1], 0, t1);      /* dAy/dx */
    spectral_derivative_g(g, w, A_new[0], 1, t2);      /* dAx/dy */
    for (int id = 0; id < N; ++id) {
        B[id] = gy[id];
        B[N + id] = -gx[id];
        B[2 * N + id] = t1[id] - t2[id];
    }
    out[3] = rms1(B + 2 * N, N);
    out[4] = rms3(B, B + N, B + 2 * N, N);
    out[5] = rms3(E, E + N, E + 2 * N, N);
    out[6] = rms1(rho_cur, N);
    out[7] = rms3(J, J + N, J + 2 * N, N);
    out[8] = 0.5 * eps0 * integral_sq3(E, E + N, E + 2 * N, N, g->dA)
           + 0.5 / mu0 * integral_sq3(B, B + N, B + 2 * N, N, g->dA);

    long double kin = 0.0L, gsum = 0.0L;
    double max_speed = 0.0;
    for (long p = 0; p < np; ++p) {
        const double gam = gamma_from_v3(v + 3 * p, c);
        gsum += gam;
        kin += (gam - 1.0) * m[p] * c * c;
        const double* vp = v + 3 * p;
        const double sp = sqrt(vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]);
        if (sp > max_speed) max_speed = sp;
    }
    out[9] = (double)kin;
    out[11] = max_speed;
    out[12] = np == 0 ? 0.0 : (double)(gsum / (long double)np);
    out[10] = out[8] + out[9];

    free(t1); free(t2); free(gauge); free(E); free(B); free(gx); free(gy);
}

/* ---- Step loop (spectral_pic_part3.cpp:1094-1189) --------------------- */
int o2_simulate(const double* params, const int* iparams, long np, double* x, double* y,
                double* P, double* v, double* vprev, const double* q, const double* m,
                double* diag_out, double* fields_out, double* seconds_out) {
    const double Lx = params[0], Ly = params[1], dt = params[2], c = params[3];
    const double eps0 = params[4], mu0 = params[5], n0 = params[6];
    const int nx = iparams[0], ny = iparams[1], order = iparams[2], conserving = iparams[3];
    const int n_steps = iparams[4];
    const int stride = iparams[5] > 1 ? iparams[5] : 1;
    o2_grid g;
    o2_work w;
    grid_init(&g, nx, ny, Lx, Ly);
    work_init(&w, g.N);
    const int N = g.N;

    double* rho0 = (double*)malloc(sizeof(double) * N);
    double* J = (double*)malloc(sizeof(double) * 3 * N);
    double* phi0 = (double*)malloc(sizeof(double) * N);
    double* zero = (double*)calloc((size_t)N, sizeof(double));
    deposit_charge_g(&g, n0, np, x, y, q, rho0);
    deposit_current_g(&g, np, x, y, v, q, J);
    poisson_g(&g, &w, eps0, rho0, phi0);
    o2_hist phi_h, rho_h, A_h[3];
    hist_init(&phi_h, phi0, N);
    hist_init(&rho_h, rho0, N);
    for (int cc = 0; cc < 3; ++cc) hist_init(&A_h[cc], zero, N);

    double* F[NGF];
    for (int f = 0; f < NGF; ++f) F[f] = (double*)malloc(sizeof(double) * N);
    double* phi_new = (double*)malloc(sizeof(double) * N);
    double* rho_new = (double*)malloc(sizeof(double) * N);
    double* src = (double*)malloc(sizeof(double) * N);
    double* scratch = (double*)malloc(sizeof(double) * N);
    double* Anew[3] = {F[0], F[1], F[2]};

    if (diag_out) {
        o2_bdf b0 = bdf_coeffs(1);
        double* Acur[3] = {A_h[0].s[0], A_h[1].s[0], A_h[2].s[0]};
        diagnostics_g(&g, &w, np, v, m, &phi_h, A_h, &rho_h, phi_h.s[0], Acur, rho_h.s[0], J,
                      b0, c, eps0, mu0, dt, diag_out);
    }
    struct timespec ts0, ts1;
    clock_gettime(CLOCK_MONOTONIC, &ts0);
    const o2_bdf bdf = bdf_coeffs(order);
    for (int step = 1; step <= n_steps; ++step) {
        for (long p = 0; p < np; ++p) {
            x[p] = wrap_periodic(x[p] + dt * v[3 * p], Lx);
            y[p] = wrap_periodic(y[p] + dt * v[3 * p + 1], Ly);
        }
        deposit_current_g(&g, np, x, y, v, q, J);
        if (conserving) continuity_g(&g, &w, &rho_h, J, bdf, dt, rho_new, scratch);
        else deposit_charge_g(&g, n0, np, x, y, q, rho_new);
        for (int id = 0; id < N; ++id) src[id] = rho_new[id] / eps0;
        solve_bdf_wave_g(&g, &w, src, &phi_h, bdf, c, dt, phi_new);
        for (int cc = 0; cc < 3; ++cc) {
            for (int id = 0; id < N; ++id) src[id] = mu0 * J[cc * N + id];
            solve_bdf_wave_g(&g, &w, src, &A_h[cc], bdf, c, dt, Anew[cc]);
        }
        spectral_derivative_g(&g, &w, phi_new, 0, F[3]);
        spectral_derivative_g(&g, &w, phi_new, 1, F[4]);
        for (int cc = 0; cc < 3; ++cc) {
            spectral_derivative_g(&g, &w, Anew[cc], 0, F[5 + 2 * cc]);
            spectral_derivative_g(&g, &w, Anew[cc], 1, F[6 + 2 * cc]);
        }
        push_g(&g, np, x, y, P, v, vprev, q, m, F, c, dt);
        if (diag_out && (step % stride == 0 || step == n_steps))
            diagnostics_g(&g, &w, np, v, m, &phi_h, A_h, &rho_h, phi_new, Anew, rho_new, J, bdf,
                          c, eps0, mu0, dt, diag_out + 13 * (size_t)step);
        if (fields_out && step == n_steps) {
            const double* srcs[8] = {phi_new, Anew[0], Anew[1], Anew[2], rho_new, J, J + N, J + 2 * N};
            for (int f = 0; f < 8; ++f) memcpy(fields_out + (size_t)f * N, srcs[f], sizeof(double) * N);
        }
        hist_push(&phi_h, phi_new, N);
        for (int cc = 0; cc < 3; ++cc) hist_push(&A_h[cc], Anew[cc], N);
        hist_push(&rho_h, rho_new, N);
    }
    clock_gettime(CLOCK_MONOTONIC, &ts1);
    if (seconds_out)
        *seconds_out = (double)(ts1.tv_sec - ts0.tv_sec) + 1e-9 * (double)(ts1.tv_nsec - ts0.tv_nsec);

    hist_free(&phi_h);
    hist_free(&rho_h);
    for (int cc = 0; cc < 3; ++cc) hist_free(&A_h[cc]);
    for (int f = 0; f < NGF; ++f) free(F[f]);
    free(rho0); free(J); free(phi0); free(zero); free(phi_new); free(rho_new); free(src);
    free(scratch);
    work_free(&w);
    grid_free(&g);
    return 0;
}

/* ---- Reference Weibel quiet start (spectral_pic_part3.cpp:624-669) ----- */
long o2_init_weibel(int nx, int ny, double Lx, double Ly, int ppc, double c, double n0,
                    double vx, double vy_max, double sine, int mode, unsigned seed,
                    long np_capacity, double* x, double* y, double* P, double* v,
                    double* vprev, double* q, double* m) {
    int nsub = (int)round(sqrt((double)ppc));
    if (nsub < 1) nsub = 1;
    const long total = 2L * nx * ny * nsub * nsub;
    if (total > np_capacity) return -1;
    const double dx = Lx / (double)nx, dy = Ly / (double)ny;
    const double macro = n0 * (Lx * Ly) / (double)total;
    const double qe = -1.0 * macro, me = macro;
    o_mt19937 rng;
    o_mt_seed(&rng, seed);
    long n = 0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int a = 0; a < nsub; ++a)
                for (int b = 0; b < nsub; ++b) {
                    const double px = ((double)i + ((double)a + 0.5) / nsub) * dx;
                    const double py = ((double)j + ((double)b + 0.5) / nsub) * dy;
                    const double sseed = sine * c * sin(2.0 * O_PI * mode * px / Lx);
                    for (int beam = -1; beam <= 1; beam += 2) {
                        const double u = o_mt_canonical(&rng) * (vy_max - (-vy_max)) + (-vy_max);
                        double vv[3] = {(double)beam * vx * c, u + sseed, 0.0};
                        const double gam = gamma_from_v3(vv, c);
                        x[n] = px;
                        y[n] = py;
                        for (int d = 0; d < 3; ++d) {
                            v[3 * n + d] = vv[d];
                            vprev[3 * n + d] = vv[d];
                            P[3 * n + d] = (me * gam) * vv[d] + qe * 0.0;
                        }
                        q[n] = qe;
                        m[n] = me;
                        ++n;
                    }
                }
    return n;
}
