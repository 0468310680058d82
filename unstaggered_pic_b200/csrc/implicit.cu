// Implicit energy-conserving orbit-averaged GM-HC-CN step kernels (sm_100a).
//
// Reference: Project3/ec_pic_nyquist_projected.cpp, the manuscript path
// nonlinear_step_orbit (:6477) -> nonlinear_step_uniform_subcycled (:5878)
// with a level-one layout -> evaluate_selective_current_map_at_layout
// (:5235).  One evaluation of the outer map J -> J_map is: continuity and CN
// potential update in k-space (cn_kspace_kernel), then per particle the
// damped local fixed point on the orbit velocity vbar
// (solve_local_particle_substep :4930, evaluate_local_particle_substep :4843)
// followed by the orbit-averaged current deposit of the accepted orbit
// (path_average_deposit_current :2784) -- all in implicit_map_kernel, one
// thread per particle.  The grid runs in 2D (nz = 1): the z stencil of the
// reference then sums to one, so its z factors and z-knot splits only change
// rounding and are dropped here.
#include <climits>

#include "implicit_kernels.h"
#include "upic_common.cuh"

namespace upic {

namespace {

constexpr int kMapThreads = 128;
// Resident CTAs per SM the map kernel is compiled for (register budget
// 65536 / (128 * kMapMinBlocks) per thread).
#ifndef UPIC_MAP_MIN_BLOCKS
#define UPIC_MAP_MIN_BLOCKS 3
#endif
constexpr int kMapMinBlocks = UPIC_MAP_MIN_BLOCKS;
// A map evaluation runs as one fused launch (kPartFused), or as a local-solve
// launch followed by a deposit launch (kPartSolve, kPartDeposit) that hands
// the orbit velocities over through global memory.  The split keeps the
// solve's code and registers free of the deposit machinery and gives the
// deposit its own occupancy; the sums are the same bit for bit.
#ifndef UPIC_MAP_SPLIT
#define UPIC_MAP_SPLIT 1
#endif
// resident CTAs of the local-solve launch: 3 for the segment-moment
// instances, 4 for the point-by-point ones (orders 3-4 in 2D), each the
// faster of 2, 3 and 4 measured
#ifndef UPIC_SOLVE_MIN_BLOCKS
#define UPIC_SOLVE_MIN_BLOCKS 3
#endif
#ifndef UPIC_SOLVE_POINTS_MIN_BLOCKS
#define UPIC_SOLVE_POINTS_MIN_BLOCKS 4
#endif
// resident CTAs of the deposit launch: 8 for the segment-moment instances
// (one item per segment), 6 for the point-by-point ones (one item per
// quadrature point), whose 8-CTA build measured slower
#ifndef UPIC_DEPOSIT_MIN_BLOCKS
#define UPIC_DEPOSIT_MIN_BLOCKS 6
#endif
#ifndef UPIC_DEPOSIT_MOM_MIN_BLOCKS
#define UPIC_DEPOSIT_MOM_MIN_BLOCKS 8
#endif
constexpr int kPartFused = 0, kPartSolve = 1, kPartDeposit = 2;
constexpr int map_min_blocks(int part, bool mom = false) {
    return part == kPartSolve     ? (mom ? UPIC_SOLVE_MIN_BLOCKS : UPIC_SOLVE_POINTS_MIN_BLOCKS)
           : part == kPartDeposit ? (mom ? UPIC_DEPOSIT_MOM_MIN_BLOCKS : UPIC_DEPOSIT_MIN_BLOCKS)
                                  : kMapMinBlocks;
}
constexpr int kMapWarps = kMapThreads / kWarp;
constexpr int kKeyNone = -1;
constexpr int kKeyEscape = -2;


// wrap1 (:704): x -> [-L/2, L/2), fmod(x + L/2, L) shifted into [0, L).
// For t = x + L/2 in [-L, 2L) -- every orbit point, whose excursion is below
// kappa dt -- fmod(t, L) is t itself or t - L, which is exact (Sterbenz), so
// the branches below return fmod's value without its remainder loop.
UPIC_D double wrap1(double x, double L) {
    double y = x + 0.5 * L;
    if (y >= L) {
        y = y < 2.0 * L ? y - L : fmod(y, L);
    } else if (y < 0.0) {
        if (y < -L) y = fmod(y, L);
        if (y < 0.0) y += L;
    }
    return y - 0.5 * L;
}

// Centered B-spline of degree ORDER on the stencil of grid coordinate u
// (centered_bspline :1856, centered_bspline_derivative :1912, axis_stencil
// :1971).  The stencil's first node is il = floor(u - (ORDER-1)/2); with
// f = u - il each node's offset r_a = f - a lies on a fixed polynomial piece,
// evaluated directly.  dw holds dS/dx = S'(r) / h.
template <int ORDER>
struct Stencil {
    int il;
    double w[ORDER + 1];
    double dw[ORDER + 1];
};

// Weights and dS/dx of the stencil whose first node is il, at f = u - il.
template <int ORDER>
UPIC_D void bspline_f(double f, double inv_h, double* w, double* dw);

template <int ORDER>
UPIC_D void bspline(double u, double inv_h, Stencil<ORDER>& s) {
    const double fl = floor(u - 0.5 * (double)(ORDER - 1));
    s.il = (int)fl;
    bspline_f<ORDER>(u - fl, inv_h, s.w, s.dw);
}

template <int ORDER>
UPIC_D void bspline_f(double f, double inv_h, double* w, double* dw) {
    Stencil<ORDER> s;
    if (ORDER == 1) {
        s.w[0] = 1.0 - f;
        s.w[1] = f;
        s.dw[0] = -inv_h;
        s.dw[1] = inv_h;
    } else if (ORDER == 2) {
        const double z0 = 1.5 - f, r1 = f - 1.0, z2 = f - 0.5;
        s.w[0] = 0.5 * z0 * z0;
        s.w[1] = 0.75 - r1 * r1;
        s.w[2] = 0.5 * z2 * z2;
        s.dw[0] = -z0 * inv_h;
        s.dw[1] = -2.0 * r1 * inv_h;
        s.dw[2] = z2 * inv_h;
    } else if (ORDER == 3) {
        const double z0 = 2.0 - f, a1 = f - 1.0, a2 = 2.0 - f, z3 = f - 1.0;
        s.w[0] = z0 * z0 * z0 / 6.0;
        s.w[1] = (2.0 / 3.0) - a1 * a1 + 0.5 * a1 * a1 * a1;
        s.w[2] = (2.0 / 3.0) - a2 * a2 + 0.5 * a2 * a2 * a2;
        s.w[3] = z3 * z3 * z3 / 6.0;
        s.dw[0] = -0.5 * z0 * z0 * inv_h;
        s.dw[1] = (-2.0 * a1 + 1.5 * a1 * a1) * inv_h;
        s.dw[2] = (2.0 * a2 - 1.5 * a2 * a2) * inv_h;
        s.dw[3] = 0.5 * z3 * z3 * inv_h;
    } else {
        const double z0 = 2.5 - f, a1 = f - 1.0, r2 = f - 2.0, a3 = 3.0 - f, z4 = f - 1.5;
        const double r22 = r2 * r2;
        s.w[0] = z0 * z0 * z0 * z0 / 24.0;
        s.w[1] = 55.0 / 96.0 + (5.0 / 24.0) * a1 - 1.25 * a1 * a1 + (5.0 / 6.0) * a1 * a1 * a1 -
                 (1.0 / 6.0) * a1 * a1 * a1 * a1;
        s.w[2] = 115.0 / 192.0 - (5.0 / 8.0) * r22 + 0.25 * r22 * r22;
        s.w[3] = 55.0 / 96.0 + (5.0 / 24.0) * a3 - 1.25 * a3 * a3 + (5.0 / 6.0) * a3 * a3 * a3 -
                 (1.0 / 6.0) * a3 * a3 * a3 * a3;
        s.w[4] = z4 * z4 * z4 * z4 / 24.0;
        s.dw[0] = -(z0 * z0 * z0 / 6.0) * inv_h;
        s.dw[1] = (5.0 / 24.0 - 2.5 * a1 + 2.5 * a1 * a1 - (2.0 / 3.0) * a1 * a1 * a1) * inv_h;
        s.dw[2] = r2 * (r22 - 1.25) * inv_h;
        s.dw[3] = -(5.0 / 24.0 - 2.5 * a3 + 2.5 * a3 * a3 - (2.0 / 3.0) * a3 * a3 * a3) * inv_h;
        s.dw[4] = (z4 * z4 * z4 / 6.0) * inv_h;
    }
#pragma unroll
    for (int a = 0; a <= ORDER; ++a) {
        w[a] = s.w[a];
        dw[a] = s.dw[a];
    }
}

struct Geo {
    int nx, ny;
    double Lx, Ly, inv_dx, inv_dy;
    // orbit quadrature (map kernel only, in shared memory): the deck's
    // Gauss rule for point-wise orbit sums, and the rule used for segment
    // moments
    const double *qs = nullptr, *qw = nullptr, *ms = nullptr, *mw = nullptr;
    int nq = 0, mnq = 0;
};

// SY: nodes of the y stencil, ORDER + 1, or 1 on a grid one cell high
// (ny = 1), where every y node wraps onto the same row: the weights of the
// ORDER + 1 nodes then add to 1 and their derivatives to 0 (the partition
// of unity), so the y stencil is that one row with weight 1 and
// derivative 0.
template <int ORDER, int SY = ORDER + 1>
UPIC_D void stencil_xy(const Geo& g, double x, double y, Stencil<ORDER>& sx, Stencil<ORDER>& sy) {
    bspline<ORDER>((x + 0.5 * g.Lx) * g.inv_dx, g.inv_dx, sx);
    if constexpr (SY == 1) {
        (void)y;
        sy.il = 0;
        sy.w[0] = 1.0;
        sy.dw[0] = 0.0;
    } else {
        bspline<ORDER>((y + 0.5 * g.Ly) * g.inv_dy, g.inv_dy, sy);
    }
}

// Sum of record component block [off, off+3) at a wrapped position.
template <int ORDER, int STRIDE = kIRec, int SY = ORDER + 1>
UPIC_D void gather_rec3(const Geo& g, const double* __restrict__ rec, int off, double x, double y,
                        double out[3]) {
    Stencil<ORDER> sx, sy;
    stencil_xy<ORDER, SY>(g, x, y, sx, sy);
    out[0] = out[1] = out[2] = 0.0;
#pragma unroll
    for (int a = 0; a <= ORDER; ++a) {
        const int gx = wrap_index(sx.il + a, g.nx);
#pragma unroll
        for (int b = 0; b < SY; ++b) {
            const double* r = rec + (size_t)(gx * g.ny + wrap_index(sy.il + b, g.ny)) * STRIDE + off;
            const double w = sx.w[a] * sy.w[b];
            out[0] = fma(__ldg(r), w, out[0]);
            out[1] = fma(__ldg(r + 1), w, out[1]);
            out[2] = fma(__ldg(r + 2), w, out[2]);
        }
    }
}

// Knot-split breakpoints of the orbit x0 + s dx, s in [0, 1]
// (path_breakpoints_for_particle :2555); returns the count, or -1 when more
// than kMaxBreaks are needed.
template <int ORDER>
UPIC_D int breakpoints(const Geo& g, double x0, double y0, double dxx, double dxy, int split,
                       double* b) {
    int nb = 0;
    b[nb++] = 0.0;
    b[nb++] = 1.0;
    if (split) {
        const double tol = 1.0e-13;
        const double offset = 0.5 * (double)(ORDER - 1);
#pragma unroll
        for (int d = 0; d < 2; ++d) {
            const double L = d == 0 ? g.Lx : g.Ly;
            const double h = L / (double)(d == 0 ? g.nx : g.ny);
            const double u0 = (wrap1(d == 0 ? x0 : y0, L) + 0.5 * L) / h;
            const double du = (d == 0 ? dxx : dxy) / h;
            if (fabs(du) < 1.0e-300) continue;
            const double a0 = u0 - offset;
            const double a1 = a0 + du;
            const double lo = fmin(a0, a1), hi = fmax(a0, a1);
            const long long first = (long long)floor(lo) + 1;
            const long long last = (long long)ceil(hi) - 1;
            for (long long m = first; m <= last; ++m) {
                const double s = ((double)m - a0) / du;
                if (s > tol && s < 1.0 - tol) {
                    if (nb >= kMaxBreaks) return -1;
                    b[nb++] = s;
                }
            }
        }
        // insertion sort, then drop near-duplicates
        for (int i = 1; i < nb; ++i) {
            const double v = b[i];
            int j = i - 1;
            while (j >= 0 && b[j] > v) {
                b[j + 1] = b[j];
                --j;
            }
            b[j + 1] = v;
        }
        int n = 0;
        for (int i = 0; i < nb; ++i)
            if (n == 0 || fabs(b[i] - b[n - 1]) > 1.0e-12) b[n++] = b[i];
        nb = n;
    }
    return nb;
}

UPIC_D double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
UPIC_D double norm3(const double* a) { return sqrt(dot3(a, a)); }

// gamma_from_p (:584)
UPIC_D double gamma_p(const double* p, double mk) { return sqrt(1.0 + dot3(p, p) / (mk * mk)); }

// Higuera-Cary rotation by B_eff (higuera_cary_rotate_with_K :4636,
// beff_from_skew_K :4605).
UPIC_D double hc_rotate(const double* pm, const double* B, double q, double m, double mk, double inv_mk,
                        double dt, double* out) {
    double u[3] = {pm[0] * inv_mk, pm[1] * inv_mk, pm[2] * inv_mk};
    const double gm = sqrt(1.0 + dot3(u, u));
    const double c = q * dt / (2.0 * m);
    const double tau[3] = {c * B[0], c * B[1], c * B[2]};
    const double tau2 = dot3(tau, tau);
    const double udt = dot3(u, tau);
    const double sigma = gm * gm - tau2;
    const double ghc2 = 0.5 * (sigma + sqrt(sigma * sigma + 4.0 * (tau2 + udt * udt)));
    const double inv_ghc = 1.0 / sqrt(fmax(ghc2, 1.0));
    const double t[3] = {tau[0] * inv_ghc, tau[1] * inv_ghc, tau[2] * inv_ghc};
    const double sf = 2.0 / (1.0 + dot3(t, t));
    const double sv[3] = {sf * t[0], sf * t[1], sf * t[2]};
    const double up[3] = {u[0] + (u[1] * t[2] - u[2] * t[1]), u[1] + (u[2] * t[0] - u[0] * t[2]),
                          u[2] + (u[0] * t[1] - u[1] * t[0])};
    const double upl[3] = {u[0] + (up[1] * sv[2] - up[2] * sv[1]), u[1] + (up[2] * sv[0] - up[0] * sv[2]),
                           u[2] + (up[0] * sv[1] - up[1] * sv[0])};
    out[0] = mk * upl[0];
    out[1] = mk * upl[1];
    out[2] = mk * upl[2];
    return gm;  // gamma of pm
}

struct LocalIn {
    double x0, y0;
    double P0[3];
    double A0p[3];
    double pstart[3];
    double q, m;
    // per-particle constants of the local solve: m kappa, 1 / (m kappa) and
    // gamma(pstart) (set by set_local_constants)
    double mk, inv_mk, gstart;
};

struct LocalOut {
    double vbar_map[3];
    double P_end[3];
    double v_end[3];
    double x1, y1;
};

// gamma_from_p (:584) with the particle's 1 / (m kappa)
UPIC_D double gamma_p_inv(const double* p, double inv_mk) {
    return sqrt(1.0 + dot3(p, p) * (inv_mk * inv_mk));
}

UPIC_D void set_local_constants(LocalIn& in, double kappa) {
    in.mk = in.m * kappa;
    in.inv_mk = 1.0 / in.mk;
    in.gstart = gamma_p_inv(in.pstart, in.inv_mk);
}

// The kick-rotate-kick of one local map evaluation over a step h
// (evaluate_local_particle_substep :4843-4929): the orbit averages gp =
// <grad phi_mid> and D = <dA/dx>, A' at the orbit's end (A1p) and at its
// midpoint ((A0p + A1p) / 2) give P_end, v_end and the secant orbit
// velocity vbar_map.  Each gamma is evaluated once (the rotation's gamma of
// p_minus serves its secant, gamma(pstart) is a particle constant, gamma of
// p_end serves both v_end and its secant).
UPIC_D void kick_rotate_kick(const LocalIn& in, const double* guess, double gp0, double gp1, const double (&D)[3][2],
                             const double* A1p, double h, LocalOut& o) {
    const double Aep[3] = {0.5 * (in.A0p[0] + A1p[0]), 0.5 * (in.A0p[1] + A1p[1]),
                           0.5 * (in.A0p[2] + A1p[2])};
    // D vbar and the skew part K = D^T - D as B_eff (:4585-4620); the z
    // columns of D vanish in 2D.
    const double Dv[3] = {D[0][0] * guess[0] + D[0][1] * guess[1], D[1][0] * guess[0] + D[1][1] * guess[1],
                          D[2][0] * guess[0] + D[2][1] * guess[1]};
    const double B[3] = {D[2][1], -D[2][0], D[1][0] - D[0][1]};
    const double q = in.q, m = in.m, hq = 0.5 * q * h;
    const double gpb[3] = {gp0, gp1, 0.0};
    double pm[3], pp[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) pm[c] = ((in.P0[c] - q * Aep[c]) - hq * gpb[c]) + hq * Dv[c];
    const double gm = hc_rotate(pm, B, q, m, in.mk, in.inv_mk, h, pp);
    double pend[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        o.P_end[c] = ((pp[c] + q * Aep[c]) - hq * gpb[c]) + hq * Dv[c];
        pend[c] = o.P_end[c] - q * A1p[c];
    }
    const double gam = gamma_p_inv(pend, in.inv_mk);
    const double inv_mgam = 1.0 / (m * gam);
#pragma unroll
    for (int c = 0; c < 3; ++c) o.v_end[c] = pend[c] * inv_mgam;
    // kinetic_secant_velocity (:682) of (p_minus, pstart) and (p_end, p_plus)
    const double sm = 1.0 / (m * (gm + in.gstart));
    const double sp = 1.0 / (m * (gam + gamma_p_inv(pp, in.inv_mk)));
#pragma unroll
    for (int c = 0; c < 3; ++c) o.vbar_map[c] = 0.5 * (sm * (pm[c] + in.pstart[c]) + sp * (pend[c] + pp[c]));
}

// Orbit averages along x0 + s (dxx, dxy), s in [0, 1] split at the
// breakpoints b[0..nb): gp = <grad phi_mid> and D[c][d] = <d A_c / d x_d>
// with A = (1-s) A^n + s A^{n+1} (path_average_gather_vector_one :2738,
// orbit_discrete_gradient_A_interval :2958), the deck's Gauss rule point by
// point.
template <int ORDER, int SY = ORDER + 1>
UPIC_D void orbit_integrals_points(const Geo& g, const double* __restrict__ rec, double x0, double y0, double dxx,
                                   double dxy, const double* b, int nb, double gp[2], double D[3][2],
                                   double th0 = 0.0, double th1 = 1.0) {
    double gp0 = 0.0, gp1 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) D[c][0] = D[c][1] = 0.0;
    const int nq = g.nq;
    for (int k = 0; k + 1 < nb; ++k) {
        const double sa = b[k], len = b[k + 1] - b[k];
        if (len <= 0.0) continue;
        for (int iq = 0; iq < nq; ++iq) {
            const double s = sa + len * g.qs[iq];
            const double wq = len * g.qw[iq];
            const double xs = wrap1(x0 + s * dxx, g.Lx);
            const double ys = wrap1(y0 + s * dxy, g.Ly);
            Stencil<ORDER> sx, sy;
            stencil_xy<ORDER, SY>(g, xs, ys, sx, sy);
            double g0 = 0.0, g1 = 0.0;
            double d[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
            // A at the orbit's time: (1 - th) A^n + th A^{n+1} with th running
            // over [th0, th1] (orbit_discrete_gradient_A_interval :2958)
            const double th = th0 + s * (th1 - th0);
            const double s1 = 1.0 - th;
#pragma unroll
            for (int a = 0; a <= ORDER; ++a) {
                const int gx = wrap_index(sx.il + a, g.nx);
#pragma unroll
                for (int bb = 0; bb < SY; ++bb) {
                    const double* r = rec + (size_t)(gx * g.ny + wrap_index(sy.il + bb, g.ny)) * kIRec;
                    const double2 r01 = __ldg(reinterpret_cast<const double2*>(r));
                    const double2 r23 = __ldg(reinterpret_cast<const double2*>(r + 2));
                    const double2 r45 = __ldg(reinterpret_cast<const double2*>(r + 4));
                    const double2 r67 = __ldg(reinterpret_cast<const double2*>(r + 6));
                    const double sh = sx.w[a] * sy.w[bb];
                    const double dsx = sx.dw[a] * sy.w[bb];
                    g0 = fma(r01.x, sh, g0);
                    g1 = fma(r01.y, sh, g1);
                    const double av[3] = {s1 * r23.x + th * r45.y, s1 * r23.y + th * r67.x, s1 * r45.x + th * r67.y};
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        d[c][0] = fma(av[c], dsx, d[c][0]);
                        if constexpr (SY > 1) d[c][1] = fma(av[c], sx.w[a] * sy.dw[bb], d[c][1]);
                    }
                }
            }
            gp0 = fma(wq, g0, gp0);
            gp1 = fma(wq, g1, gp1);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                D[c][0] = fma(wq, d[c][0], D[c][0]);
                D[c][1] = fma(wq, d[c][1], D[c][1]);
            }
        }
    }
    gp[0] = gp0;
    gp[1] = gp1;
}

// One evaluation of the particle map at guess vbar (evaluate_local_particle_substep
// :4843 with h = dt, theta0 = 0, theta1 = 1).  b/nb: breakpoints of the orbit.
template <int ORDER, int SY = ORDER + 1>
UPIC_D bool evaluate(const Geo& g, const double* __restrict__ rec, double dt, double kappa, int split,
                     const LocalIn& in, const double* guess, LocalOut& o, double* b, int& nb) {
    const double dxx = dt * guess[0], dxy = dt * guess[1];
    o.x1 = wrap1(in.x0 + dxx, g.Lx);
    o.y1 = wrap1(in.y0 + dxy, g.Ly);
    double A1p[3];
    gather_rec3<ORDER, kIRec, SY>(g, rec, kIRecAe, o.x1, o.y1, A1p);
    nb = breakpoints<ORDER>(g, in.x0, in.y0, dxx, dxy, split, b);
    if (nb < 0) return false;
    double gpv[2], D[3][2];
    orbit_integrals_points<ORDER, SY>(g, rec, in.x0, in.y0, dxx, dxy, b, nb, gpv, D);
    kick_rotate_kick(in, guess, gpv[0], gpv[1], D, A1p, dt, o);
    return true;
}

// One evaluation of the particle map of a substep: h = dt / n over the step
// fraction [th0, th1] (evaluate_local_particle_substep :4843): A at the orbit
// ends and along the orbit is interpolated in time between A^n and A^{n+1};
// grad phi_mid is the step's.
template <int ORDER>
UPIC_D bool evaluate_sub(const Geo& g, const double* __restrict__ rec, double h, double th0, double th1,
                         double kappa, int split, const LocalIn& in, const double* guess, LocalOut& o, double* b,
                         int& nb) {
    const double dxx = h * guess[0], dxy = h * guess[1];
    o.x1 = wrap1(in.x0 + dxx, g.Lx);
    o.y1 = wrap1(in.y0 + dxy, g.Ly);
    double An1[3], Ae1[3], A1p[3];
    gather_rec3<ORDER>(g, rec, kIRecAn, o.x1, o.y1, An1);
    gather_rec3<ORDER>(g, rec, kIRecAe, o.x1, o.y1, Ae1);
#pragma unroll
    for (int c = 0; c < 3; ++c) A1p[c] = (1.0 - th1) * An1[c] + th1 * Ae1[c];
    nb = breakpoints<ORDER>(g, in.x0, in.y0, dxx, dxy, split, b);
    if (nb < 0) return false;
    double gpv[2], D[3][2];
    orbit_integrals_points<ORDER>(g, rec, in.x0, in.y0, dxx, dxy, b, nb, gpv, D, th0, th1);
    kick_rotate_kick(in, guess, gpv[0], gpv[1], D, A1p, h, o);
    return true;
}

// Shape moments of one knot-split orbit segment [sa, sa + len].  Inside a
// segment every point of the orbit has the same stencil (its first node per
// axis is ilx, ily, taken at the segment midpoint), so the Gauss sums
//   sum_q wq S_a S_b,  sum_q wq (1-s_q) S'_a S_b,  sum_q wq s_q S'_a S_b, ...
// are accumulated once per segment and contracted with each node record
// once, instead of gathering the node records at every quadrature point.
// The algebra is that of path_average_gather_vector_one (:2738) and
// orbit_discrete_gradient_A_interval (:2958) with the node and quadrature
// sums exchanged.
template <int ORDER, int SY = ORDER + 1>
struct SegMoments {
    static constexpr int SS = (ORDER + 1) * SY;
    int ilx, ily;
    double m[SS];               // sum wq Sx_a Sy_b
    double x0[SS], x1[SS];      // sum wq (1-s) dSx_a Sy_b, sum wq s dSx_a Sy_b
    double y0[SS], y1[SS];      // sum wq (1-s) Sx_a dSy_b, sum wq s Sx_a dSy_b
};

// Segment stencil origin and the weighted shape sums of one segment.  With
// GRAD false only m is formed (the deposit needs no derivatives).
template <int ORDER, bool GRAD, int SY = ORDER + 1>
UPIC_D void segment_moments(const Geo& g, double x0, double y0, double dxx, double dxy, double sa,
                            double len, SegMoments<ORDER, SY>& M) {
    constexpr int S = ORDER + 1;
    const double off = 0.5 * (double)(ORDER - 1);
    const double ox = x0 + 0.5 * g.Lx, oy = y0 + 0.5 * g.Ly;
    const double sm = sa + 0.5 * len;
    M.ilx = (int)floor((ox + sm * dxx) * g.inv_dx - off);
    M.ily = SY == 1 ? 0 : (int)floor((oy + sm * dxy) * g.inv_dy - off);
    const double fx0 = (double)M.ilx, fy0 = (double)M.ily;
#pragma unroll
    for (int k = 0; k < S * SY; ++k) {
        M.m[k] = 0.0;
        if (GRAD) M.x0[k] = M.x1[k] = M.y0[k] = M.y1[k] = 0.0;
    }
    const int nq = g.mnq;
    for (int iq = 0; iq < nq; ++iq) {
        const double s = sa + len * g.ms[iq];
        const double wq = len * g.mw[iq];
        double wx[S], dwx[S], wy[S], dwy[S];
        bspline_f<ORDER>((ox + s * dxx) * g.inv_dx - fx0, g.inv_dx, wx, dwx);
        if constexpr (SY == 1) {
            wy[0] = 1.0;
            dwy[0] = 0.0;
        } else {
            bspline_f<ORDER>((oy + s * dxy) * g.inv_dy - fy0, g.inv_dy, wy, dwy);
        }
        const double w1 = wq * s, w0 = wq * (1.0 - s);
#pragma unroll
        for (int a = 0; a < S; ++a) {
            const double ta = wq * wx[a];
#pragma unroll
            for (int b = 0; b < SY; ++b) M.m[a * SY + b] = fma(ta, wy[b], M.m[a * SY + b]);
            if (GRAD) {
                const double t0 = w0 * dwx[a], t1 = w1 * dwx[a], u0 = w0 * wx[a], u1 = w1 * wx[a];
#pragma unroll
                for (int b = 0; b < SY; ++b) {
                    M.x0[a * SY + b] = fma(t0, wy[b], M.x0[a * SY + b]);
                    M.x1[a * SY + b] = fma(t1, wy[b], M.x1[a * SY + b]);
                    if constexpr (SY > 1) {  // one row: no y derivative, y0 = y1 = 0
                        M.y0[a * SY + b] = fma(u0, dwy[b], M.y0[a * SY + b]);
                        M.y1[a * SY + b] = fma(u1, dwy[b], M.y1[a * SY + b]);
                    }
                }
            }
        }
    }
}

// orbit_integrals_points through segment moments (ORDER <= 2, knot splitting
// on, so that each segment has one stencil).
template <int ORDER, int SY = ORDER + 1>
UPIC_D void orbit_integrals_moments(const Geo& g, const double* __restrict__ rec, double x0, double y0, double dxx,
                                    double dxy, const double* b, int nb, double gp[2], double D[3][2]) {
    constexpr int S = ORDER + 1;
    double gp0 = 0.0, gp1 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) D[c][0] = D[c][1] = 0.0;
    for (int k = 0; k + 1 < nb; ++k) {
        const double len = b[k + 1] - b[k];
        if (len <= 0.0) continue;
        SegMoments<ORDER, SY> M;
        segment_moments<ORDER, true, SY>(g, x0, y0, dxx, dxy, b[k], len, M);
#pragma unroll
        for (int a = 0; a < S; ++a) {
            const int gx = wrap_index(M.ilx + a, g.nx);
#pragma unroll
            for (int bb = 0; bb < SY; ++bb) {
                const double* r = rec + (size_t)(gx * g.ny + wrap_index(M.ily + bb, g.ny)) * kIRec;
                const double2 r01 = __ldg(reinterpret_cast<const double2*>(r));
                const double2 r23 = __ldg(reinterpret_cast<const double2*>(r + 2));
                const double2 r45 = __ldg(reinterpret_cast<const double2*>(r + 4));
                const double2 r67 = __ldg(reinterpret_cast<const double2*>(r + 6));
                const int j = a * SY + bb;
                gp0 = fma(r01.x, M.m[j], gp0);
                gp1 = fma(r01.y, M.m[j], gp1);
                const double An[3] = {r23.x, r23.y, r45.x}, Ae[3] = {r45.y, r67.x, r67.y};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    D[c][0] = fma(An[c], M.x0[j], fma(Ae[c], M.x1[j], D[c][0]));
                    if constexpr (SY > 1) D[c][1] = fma(An[c], M.y0[j], fma(Ae[c], M.y1[j], D[c][1]));
                }
            }
        }
    }
    gp[0] = gp0;
    gp[1] = gp1;
}

// evaluate() with knot splitting on, through segment moments (ORDER <= 2,
// or any order with a one-row y stencil, SY = 1).
template <int ORDER, int SY = ORDER + 1>
UPIC_D bool evaluate_moments(const Geo& g, const double* __restrict__ rec, double dt, double kappa, int split,
                             const LocalIn& in, const double* guess, LocalOut& o, double* b, int& nb) {
    const double dxx = dt * guess[0], dxy = dt * guess[1];
    o.x1 = wrap1(in.x0 + dxx, g.Lx);
    o.y1 = wrap1(in.y0 + dxy, g.Ly);
    double A1p[3];
    gather_rec3<ORDER, kIRec, SY>(g, rec, kIRecAe, o.x1, o.y1, A1p);
    nb = breakpoints<ORDER>(g, in.x0, in.y0, dxx, dxy, split, b);
    if (nb < 0) return false;
    double gpv[2], D[3][2];
    orbit_integrals_moments<ORDER, SY>(g, rec, in.x0, in.y0, dxx, dxy, b, nb, gpv, D);
    kick_rotate_kick(in, guess, gpv[0], gpv[1], D, A1p, dt, o);
    return true;
}

UPIC_D bool finite3(const double* v) { return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]); }

UPIC_D int window_coord(int s, int origin, int n, int w, int span) {
    const int d = (s - origin) & (n - 1);
    return d <= w - span ? d : -1;
}

// MOM: segment moments (ORDER <= 2 with knot splitting on); otherwise the
// orbit integrals are gathered point by point.  PICARD: the deposit of the
// non-relativistic Picard map (evaluate_picard_map_orbit,
// Project1/ec_pic_serial_demo.cpp:1455-1474): the orbit velocity is
// vbar = (v_guess + v^n) / 2 with no local solve, followed by the same
// orbit-averaged deposit.
// PART: kPartFused (solve and deposit in one launch), kPartSolve (local
// solves only; writes each particle's orbit velocity to vbar_*) or
// kPartDeposit (the deposit of the orbits in vbar_*).
// ONED: a grid one cell high (ny = 1): the y stencil is one row (SY = 1).
template <int ORDER, bool UNIFORM, bool MOM, bool PICARD, int PART = kPartFused, bool ONED = false>
__global__ void __launch_bounds__(kMapThreads, map_min_blocks(PART, MOM))
implicit_map_kernel(ImplicitMapArgs a, TileGeom tg) {
    constexpr bool kSolve = PART != kPartDeposit;
    constexpr bool kDeposit = PART != kPartSolve;
    constexpr int S = ORDER + 1;
    constexpr int SY = ONED ? 1 : S;
    constexpr int SS = S * SY;
    constexpr int NV = 3 * SS;
    constexpr int RW = SS + 3;
    constexpr int NPER = (NV + 31) / 32;
    extern __shared__ unsigned long long smem_u64[];
    const int WN = tg.wx * tg.wy;
    unsigned long long* whi = smem_u64;
    unsigned long long* wlo = whi + 3 * WN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* srow = reinterpret_cast<double*>(wlo + 3 * WN) + warp * 32 * RW;
    int* sgk = reinterpret_cast<int*>(reinterpret_cast<double*>(wlo + 3 * WN) + kMapWarps * 32 * RW) + warp * 32;
    double* squad = reinterpret_cast<double*>(reinterpret_cast<int*>(reinterpret_cast<double*>(wlo + 3 * WN) +
                                                                       kMapWarps * 32 * RW) + kMapWarps * 32);
    for (int i = threadIdx.x; i < 4 * kMaxQuad; i += blockDim.x) squad[i] = a.qtab[i];
    __syncthreads();

    Geo g{tg.nx, tg.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    g.qs = squad;
    g.qw = squad + kMaxQuad;
    g.ms = squad + 2 * kMaxQuad;
    g.mw = squad + 3 * kMaxQuad;
    g.nq = a.nq;
    g.mnq = a.mnq;
    const int nx = tg.nx, ny = tg.ny, N = nx * ny;
    const int nch = *a.nchunks;
    const int c_begin = (int)(((long long)blockIdx.x * nch) / gridDim.x);
    const int c_end = (int)(((long long)(blockIdx.x + 1) * nch) / gridDim.x);

    // values owned by this lane in the grouped reduction
    int t_ab[NPER], t_a[NPER], t_b[NPER], t_c[NPER], t_off[NPER];
#pragma unroll
    for (int r = 0; r < NPER; ++r) {
        const int t = lane + 32 * r;
        const int ab = t < NV ? t / 3 : 0;
        t_ab[r] = ab;
        t_a[r] = ab / SY;
        t_b[r] = ab % SY;
        t_c[r] = t < NV ? t - 3 * ab : 0;
        t_off[r] = t_a[r] * tg.wy + t_b[r];
    }

    unsigned long long it_total = 0;
    int it_max = 0, nfail = 0;
    unsigned long long first_fail = ~0ull;
    double worst = 0.0;

    int cur_tile = -1, ox = 0, oy = 0;
    for (int ci = c_begin; ci < c_end; ++ci) {
        const Chunk ch = a.chunks[ci];
        if (kDeposit && ch.tile != cur_tile) {
            __syncthreads();
            if (cur_tile >= 0) {
                for (int idx = threadIdx.x; idx < 3 * WN; idx += blockDim.x) {
                    const unsigned long long hi = whi[idx], lo = wlo[idx];
                    if ((hi | lo) == 0ull) continue;
                    const int cc = idx / WN, widx = idx - cc * WN;
                    const int lx = widx / tg.wy, ly = widx - lx * tg.wy;
                    const int gx = tg.full_x ? lx : wrap_index(ox + lx, nx);
                    const int gy = tg.full_y ? ly : wrap_index(oy + ly, ny);
                    atomicAdd(&a.acc[(size_t)(2 * cc) * N + gx * ny + gy], hi);
                    atomicAdd(&a.acc[(size_t)(2 * cc + 1) * N + gx * ny + gy], lo);
                }
                __syncthreads();
            }
            for (int idx = threadIdx.x; idx < 6 * WN; idx += blockDim.x) whi[idx] = 0ull;
            cur_tile = ch.tile;
            const int tx = cur_tile / tg.nty, ty = cur_tile - tx * tg.nty;
            ox = tg.full_x ? 0 : tx * tg.tile_x - tg.guard - tg.lo;
            oy = tg.full_y ? 0 : ty * tg.tile_y - tg.guard - tg.lo;
            __syncthreads();
        }
        for (int base = ch.start; base < ch.end; base += kMapThreads) {
            const int p = base + threadIdx.x;
            const bool active = p < ch.end;
            bool ok = false;
            double vb[3] = {0.0, 0.0, 0.0};
            double bk[kMaxBreaks];
            int nb = 0;
            LocalIn in;
            if (PART == kPartDeposit) {
                // the orbit velocity the solve launch accepted (NaN: none)
                if (active) {
                    vb[0] = a.vbar_x[p];
                    vb[1] = a.vbar_y[p];
                    vb[2] = a.vbar_z[p];
                    ok = finite3(vb);
                    if (ok) {
                        in.x0 = a.x[p];
                        in.y0 = a.y[p];
                        in.q = UNIFORM ? a.q0 : a.q[p];
                        nb = breakpoints<ORDER>(g, in.x0, in.y0, a.dt * vb[0], a.dt * vb[1], a.split, bk);
                        ok = nb >= 0;
                    }
                    if (!ok) nb = 0;
                }
            } else if (PICARD && active) {
                in.x0 = a.x[p];
                in.y0 = a.y[p];
                in.q = UNIFORM ? a.q0 : a.q[p];
                vb[0] = 0.5 * (a.gx[p] + a.vx[p]);
                vb[1] = 0.5 * (a.gy[p] + a.vy[p]);
                vb[2] = 0.5 * (a.gz[p] + a.vz[p]);
                int reason = kLocalOk;
                if (!(fabs(vb[0]) <= a.vb_limit && fabs(vb[1]) <= a.vb_limit && fabs(vb[2]) <= a.vb_limit)) {
                    reason = kLocalNonfiniteIterate;
                } else {
                    nb = breakpoints<ORDER>(g, in.x0, in.y0, a.dt * vb[0], a.dt * vb[1], a.split, bk);
                    if (nb < 0) reason = kLocalTooManyCrossings;
                }
                ok = reason == kLocalOk;
                if (!ok) {
                    nb = 0;
                    ++nfail;
                    const unsigned long long key = ((unsigned long long)(unsigned)a.id[p] << 8) | (unsigned)reason;
                    first_fail = key < first_fail ? key : first_fail;
                }
            } else if (active && !(a.nsub && a.nsub[p] > 1)) {
                in.x0 = a.x[p];
                in.y0 = a.y[p];
                in.P0[0] = a.Px[p];
                in.P0[1] = a.Py[p];
                in.P0[2] = a.Pz[p];
                in.q = UNIFORM ? a.q0 : a.q[p];
                in.m = UNIFORM ? a.m0 : a.m[p];
                gather_rec3<ORDER, kIRec, SY>(g, a.rec, kIRecAn, in.x0, in.y0, in.A0p);
#pragma unroll
                for (int c = 0; c < 3; ++c) in.pstart[c] = in.P0[c] - in.q * in.A0p[c];
                set_local_constants(in, a.kappa);
                double guess[3] = {a.vx[p], a.vy[p], a.vz[p]};
                if (a.warm_x) {
                    guess[0] = a.warm_x[p];
                    guess[1] = a.warm_y[p];
                    guess[2] = a.warm_z[p];
                }
                // solve_local_particle_substep (:4930)
                int reason = kLocalMaxIter;
                int iters = 0;
                double scaled = INFINITY;
                LocalOut o;
                for (int it = 0; it < a.loc_maxit; ++it) {
                    bool okev;
                    if constexpr (MOM)
                        okev = evaluate_moments<ORDER, SY>(g, a.rec, a.dt, a.kappa, a.split, in, guess, o, bk, nb);
                    else
                        okev = evaluate<ORDER, SY>(g, a.rec, a.dt, a.kappa, a.split, in, guess, o, bk, nb);
                    if (!okev) {
                        reason = kLocalTooManyCrossings;
                        break;
                    }
                    ++iters;
                    if (!finite3(o.vbar_map)) {
                        reason = kLocalNonfiniteMap;
                        break;
                    }
                    if (norm3(o.vbar_map) >= a.kappa) {
                        reason = kLocalSuperluminalMap;
                        break;
                    }
                    const double res[3] = {o.vbar_map[0] - guess[0], o.vbar_map[1] - guess[1],
                                           o.vbar_map[2] - guess[2]};
                    const double sc = 0.5 * (norm3(o.vbar_map) + norm3(guess));
                    scaled = norm3(res) / (a.loc_atol + a.loc_rtol * sc);
                    if (scaled <= 1.0) {
                        reason = kLocalOk;
                        break;
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) guess[c] += a.loc_damp * res[c];
                    if (!finite3(guess)) {
                        reason = kLocalNonfiniteIterate;
                        break;
                    }
                    if (norm3(guess) >= a.kappa) {
                        reason = kLocalSuperluminalIterate;
                        break;
                    }
                }
                it_total += (unsigned long long)iters;
                it_max = max(it_max, iters);
                worst = fmax(worst, isfinite(scaled) ? scaled : 1.0e300);
                ok = reason == kLocalOk;
                if (!ok) {
                    ++nfail;
                    const unsigned long long key = ((unsigned long long)(unsigned)a.id[p] << 8) | (unsigned)reason;
                    first_fail = key < first_fail ? key : first_fail;
                    if (a.failed) a.failed[atomicAdd(a.nfailed, 1)] = p;
                } else {
                    vb[0] = guess[0];
                    vb[1] = guess[1];
                    vb[2] = guess[2];
                    if (a.keep_x) {
                        a.keep_x[p] = guess[0];
                        a.keep_y[p] = guess[1];
                        a.keep_z[p] = guess[2];
                    }
                    if (a.write_state) {
                        a.ox[p] = o.x1;
                        a.oy[p] = o.y1;
                        a.oPx[p] = o.P_end[0];
                        a.oPy[p] = o.P_end[1];
                        a.oPz[p] = o.P_end[2];
                        a.ovx[p] = o.v_end[0];
                        a.ovy[p] = o.v_end[1];
                        a.ovz[p] = o.v_end[2];
                        a.obx[p] = guess[0];
                        a.oby[p] = guess[1];
                        a.obz[p] = guess[2];
                    }
                }
            }
            if constexpr (PART == kPartSolve) {
                if (active) {
                    const double nan = __longlong_as_double(0x7ff8000000000000ll);
                    a.vbar_x[p] = ok ? vb[0] : nan;
                    a.vbar_y[p] = ok ? vb[1] : nan;
                    a.vbar_z[p] = ok ? vb[2] : nan;
                }
                continue;
            }
            // Orbit-averaged deposit of the accepted orbit (:2784).  Item k of
            // a particle is its k-th segment (MOM: the segment's shape sums,
            // one stencil per segment) or its k-th (segment, quadrature point)
            // pair; the warp works through the items in rounds and reduces
            // equal window keys.
            const double dxx = a.dt * vb[0], dxy = a.dt * vb[1];
            const double qa = ok ? in.q * a.inv_dV : 0.0;
            const double val[3] = {qa * vb[0], qa * vb[1], qa * vb[2]};
            const int nq = MOM ? 1 : g.nq;
            const int nitems = ok ? (nb - 1) * nq : 0;
            const int rounds = __reduce_max_sync(0xffffffffu, nitems);
            for (int rd = 0; rd < rounds; ++rd) {
                int key = kKeyNone, gx0 = 0, gy0 = 0;
                double wgt[SS];
                if (rd < nitems) {
                    const int k = rd / nq, iq = rd - k * nq;
                    const double sa = bk[k], len = bk[k + 1] - bk[k];
                    if (len > 0.0) {
                        int ilx, ily;
                        if constexpr (MOM) {
                            (void)iq;
                            SegMoments<ORDER, SY> M;
                            segment_moments<ORDER, false, SY>(g, in.x0, in.y0, dxx, dxy, sa, len, M);
                            ilx = M.ilx;
                            ily = M.ily;
#pragma unroll
                            for (int j = 0; j < SS; ++j) wgt[j] = M.m[j];
                        } else {
                            const double s = sa + len * g.qs[iq];
                            const double wq = len * g.qw[iq];
                            const double xs = wrap1(in.x0 + s * dxx, g.Lx);
                            const double ys = wrap1(in.y0 + s * dxy, g.Ly);
                            Stencil<ORDER> sx, sy;
                            stencil_xy<ORDER, SY>(g, xs, ys, sx, sy);
                            ilx = sx.il;
                            ily = sy.il;
#pragma unroll
                            for (int ia = 0; ia < S; ++ia)
#pragma unroll
                                for (int ib = 0; ib < SY; ++ib) wgt[ia * SY + ib] = wq * sx.w[ia] * sy.w[ib];
                        }
                        gx0 = wrap_index(ilx, nx);
                        gy0 = wrap_index(ily, ny);
                        const int lx = tg.full_x ? gx0 : window_coord(ilx, ox, nx, tg.wx, S);
                        const int ly = tg.full_y ? gy0 : window_coord(ily, oy, ny, tg.wy, SY);
                        key = (lx < 0 || ly < 0) ? kKeyEscape : lx * tg.wy + ly;
                    }
                }
                const unsigned full = 0xffffffffu;
                const unsigned lt = (1u << lane) - 1u;
                const unsigned valid = __ballot_sync(full, key >= 0);
                const unsigned esc = __ballot_sync(full, key == kKeyEscape);
                const unsigned peers = __match_any_sync(full, key);
                int row = -1, nvalid = 0, ngroups = 0;
                unsigned heads = 0u;
                for (unsigned rem = valid; rem;) {
                    const int l = __ffs(rem) - 1;
                    const unsigned gm = __shfl_sync(full, peers, l);
                    const int gk = __shfl_sync(full, key, l);
                    if ((gm >> lane) & 1u) row = nvalid + __popc(gm & lt);
                    if (lane == 0) sgk[ngroups] = gk;
                    heads |= 1u << nvalid;
                    nvalid += __popc(gm);
                    rem &= ~gm;
                    ++ngroups;
                }
                if (key == kKeyEscape) row = nvalid + __popc(esc & lt);
                if (row >= 0) {
                    double* mine = srow + row * RW;
#pragma unroll
                    for (int j = 0; j < SS; ++j) mine[j] = wgt[j];
                    mine[SS + 0] = val[0];
                    mine[SS + 1] = val[1];
                    mine[SS + 2] = val[2];
                }
                __syncwarp();
                {
                    unsigned e = esc;
                    int erow = nvalid;
                    while (e) {
                        const int j = __ffs(e) - 1;
                        e &= e - 1;
                        const int gxj = __shfl_sync(full, gx0, j);
                        const int gyj = __shfl_sync(full, gy0, j);
#pragma unroll
                        for (int r = 0; r < NPER; ++r) {
                            const int t = lane + 32 * r;
                            if (t < NV) {
                                const double v = srow[erow * RW + SS + t_c[r]] * srow[erow * RW + t_ab[r]];
                                if (v != 0.0) {
                                    const int gi = wrap_index(gxj + t_a[r], nx) * ny + wrap_index(gyj + t_b[r], ny);
                                    const Fixed2 f = to_fixed(v, a.scale[t_c[r]]);
                                    atomicAdd(&a.acc[(size_t)(2 * t_c[r]) * N + gi], f.hi);
                                    atomicAdd(&a.acc[(size_t)(2 * t_c[r] + 1) * N + gi], f.lo);
                                }
                            }
                        }
                        ++erow;
                    }
                }
                {
                    unsigned h = heads;
                    int gi = 0;
                    while (h) {
                        const int rs = __ffs(h) - 1;
                        h &= h - 1;
                        const int re = h ? __ffs(h) - 1 : nvalid;
                        const int kk = sgk[gi++];
#pragma unroll
                        for (int r = 0; r < NPER; ++r) {
                            const int t = lane + 32 * r;
                            if (t < NV) {
                                double s0 = 0.0;
                                const int iw = t_ab[r], iv = SS + t_c[r];
                                for (int j = rs; j < re; ++j) s0 = fma(srow[j * RW + iv], srow[j * RW + iw], s0);
                                if (s0 != 0.0) {
                                    int widx;
                                    if (tg.full_x || tg.full_y) {
                                        const int kx = kk / tg.wy, ky = kk - kx * tg.wy;
                                        int nxl = kx + t_a[r], nyl = ky + t_b[r];
                                        if (tg.full_x) nxl &= tg.wx - 1;
                                        if (tg.full_y) nyl &= tg.wy - 1;
                                        widx = nxl * tg.wy + nyl;
                                    } else {
                                        widx = kk + t_off[r];
                                    }
                                    const Fixed2 f = to_fixed(s0, a.scale[t_c[r]]);
                                    atomicAdd(&whi[t_c[r] * WN + widx], f.hi);
                                    atomicAdd(&wlo[t_c[r] * WN + widx], f.lo);
                                }
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
    }
    if (kDeposit) {
        __syncthreads();
        if (cur_tile >= 0) {
            for (int idx = threadIdx.x; idx < 3 * WN; idx += blockDim.x) {
                const unsigned long long hi = whi[idx], lo = wlo[idx];
                if ((hi | lo) == 0ull) continue;
                const int cc = idx / WN, widx = idx - cc * WN;
                const int lx = widx / tg.wy, ly = widx - lx * tg.wy;
                const int gx = tg.full_x ? lx : wrap_index(ox + lx, nx);
                const int gy = tg.full_y ? ly : wrap_index(oy + ly, ny);
                atomicAdd(&a.acc[(size_t)(2 * cc) * N + gx * ny + gy], hi);
                atomicAdd(&a.acc[(size_t)(2 * cc + 1) * N + gx * ny + gy], lo);
            }
        }
    }
    if (!kSolve) return;
    // statistics (integer atomics and max over bit patterns: order independent)
    MapStats* st = a.stats;
    for (int o = 16; o > 0; o >>= 1) {
        it_total += __shfl_xor_sync(0xffffffffu, it_total, o);
        it_max = max(it_max, __shfl_xor_sync(0xffffffffu, it_max, o));
        nfail += __shfl_xor_sync(0xffffffffu, nfail, o);
        const unsigned long long ff = __shfl_xor_sync(0xffffffffu, first_fail, o);
        first_fail = ff < first_fail ? ff : first_fail;
        worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    }
    if (lane == 0) {
        if (it_total) atomicAdd(&st->iter_total, it_total);
        atomicMax(&st->iter_max, it_max);
        if (nfail) {
            atomicAdd(&st->failures, nfail);
            atomicMin(&st->first_fail_key, first_fail);
        }
        atomicMax(&st->worst_scaled_bits, (unsigned long long)__double_as_longlong(worst));
    }
}

// ---- selective particle sub-cycling ------------------------------------------
// One thread per refined particle (push_particle of
// evaluate_selective_current_map_at_layout, ec_pic_nyquist_projected.cpp:5235):
// n = nsub[p] chained substeps of h = dt / n, each a local fixed point started
// from the particle's current velocity over [k/n, (k+1)/n] of the step; each
// accepted sub-orbit deposits q/n of the particle's current.  A failing
// particle is appended to the failed list and leaves the evaluation (which
// is then discarded and refined again).
template <int ORDER, bool UNIFORM>
__global__ void __launch_bounds__(128) refined_map_kernel(ImplicitMapArgs a, int nx, int ny) {
    constexpr int S = ORDER + 1;
    Geo g{nx, ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    g.qs = a.qtab;
    g.qw = a.qtab + kMaxQuad;
    g.ms = a.qtab + 2 * kMaxQuad;
    g.mw = a.qtab + 3 * kMaxQuad;
    g.nq = a.nq;
    g.mnq = a.mnq;
    const int N = nx * ny;
    unsigned long long it_total = 0;
    int it_max = 0, nfail = 0;
    unsigned long long first_fail = ~0ull;
    double worst = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.nref) {
        const int p = a.refined[i];
        const int n = a.nsub[p];
        const double h = a.dt / (double)n;
        const double q = UNIFORM ? a.q0 : a.q[p];
        const double m = UNIFORM ? a.m0 : a.m[p];
        double x = a.x[p], y = a.y[p];
        double P[3] = {a.Px[p], a.Py[p], a.Pz[p]};
        double v[3] = {a.vx[p], a.vy[p], a.vz[p]};
        double vmacro[3] = {0.0, 0.0, 0.0};
        double bk[kMaxBreaks];
        bool alive = true;
        for (int k = 0; k < n && alive; ++k) {
            const double th0 = (double)k / (double)n, th1 = (double)(k + 1) / (double)n;
            LocalIn in;
            in.x0 = x;
            in.y0 = y;
            in.q = q;
            in.m = m;
            double An0[3], Ae0[3];
            gather_rec3<ORDER>(g, a.rec, kIRecAn, x, y, An0);
            gather_rec3<ORDER>(g, a.rec, kIRecAe, x, y, Ae0);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                in.P0[c] = P[c];
                in.A0p[c] = (1.0 - th0) * An0[c] + th0 * Ae0[c];
                in.pstart[c] = P[c] - q * in.A0p[c];
            }
            set_local_constants(in, a.kappa);
            double guess[3] = {v[0], v[1], v[2]};
            int reason = kLocalMaxIter, iters = 0, nb = 0;
            double scaled = INFINITY;
            LocalOut o;
            for (int it = 0; it < a.loc_maxit; ++it) {
                if (!evaluate_sub<ORDER>(g, a.rec, h, th0, th1, a.kappa, a.split, in, guess, o, bk, nb)) {
                    reason = kLocalTooManyCrossings;
                    break;
                }
                ++iters;
                if (!finite3(o.vbar_map)) {
                    reason = kLocalNonfiniteMap;
                    break;
                }
                if (norm3(o.vbar_map) >= a.kappa) {
                    reason = kLocalSuperluminalMap;
                    break;
                }
                const double res[3] = {o.vbar_map[0] - guess[0], o.vbar_map[1] - guess[1],
                                       o.vbar_map[2] - guess[2]};
                const double sc = 0.5 * (norm3(o.vbar_map) + norm3(guess));
                scaled = norm3(res) / (a.loc_atol + a.loc_rtol * sc);
                if (scaled <= 1.0) {
                    reason = kLocalOk;
                    break;
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) guess[c] += a.loc_damp * res[c];
                if (!finite3(guess)) {
                    reason = kLocalNonfiniteIterate;
                    break;
                }
                if (norm3(guess) >= a.kappa) {
                    reason = kLocalSuperluminalIterate;
                    break;
                }
            }
            it_total += (unsigned long long)iters;
            it_max = max(it_max, iters);
            worst = fmax(worst, isfinite(scaled) ? scaled : 1.0e300);
            if (reason != kLocalOk) {
                ++nfail;
                const unsigned long long key = ((unsigned long long)(unsigned)a.id[p] << 8) | (unsigned)reason;
                first_fail = key < first_fail ? key : first_fail;
                if (a.failed) a.failed[atomicAdd(a.nfailed, 1)] = p;
                alive = false;
                break;
            }
            if (a.write_state && a.sub_rec) {
                double* so = a.sub_rec + (size_t)(a.roff[i] + k) * 5;
                so[0] = x;
                so[1] = y;
                so[2] = guess[0];
                so[3] = guess[1];
                so[4] = guess[2];
            }
            // this sub-orbit's share of the orbit-averaged current (:2784, weight q/n)
            const double dxx = h * guess[0], dxy = h * guess[1];
            const double qa = q / (double)n * a.inv_dV;
            const double val[3] = {qa * guess[0], qa * guess[1], qa * guess[2]};
            for (int kk = 0; kk + 1 < nb; ++kk) {
                const double sa = bk[kk], len = bk[kk + 1] - bk[kk];
                if (len <= 0.0) continue;
                for (int iq = 0; iq < g.nq; ++iq) {
                    const double s = sa + len * g.qs[iq];
                    const double wq = len * g.qw[iq];
                    Stencil<ORDER> sx, sy;
                    stencil_xy<ORDER>(g, wrap1(x + s * dxx, g.Lx), wrap1(y + s * dxy, g.Ly), sx, sy);
#pragma unroll
                    for (int ia = 0; ia < S; ++ia) {
                        const int gx = wrap_index(sx.il + ia, nx);
#pragma unroll
                        for (int ib = 0; ib < S; ++ib) {
                            const int node = gx * ny + wrap_index(sy.il + ib, ny);
                            const double w = wq * sx.w[ia] * sy.w[ib];
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const double dv = val[c] * w;
                                if (dv != 0.0) {
                                    const Fixed2 f = to_fixed(dv, a.scale[c]);
                                    atomicAdd(&a.acc[(size_t)(2 * c) * N + node], f.hi);
                                    atomicAdd(&a.acc[(size_t)(2 * c + 1) * N + node], f.lo);
                                }
                            }
                        }
                    }
                }
            }
            x = o.x1;
            y = o.y1;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                P[c] = o.P_end[c];
                v[c] = o.v_end[c];
                vmacro[c] += (1.0 / (double)n) * guess[c];
            }
        }
        if (alive && a.write_state) {
            a.ox[p] = x;
            a.oy[p] = y;
            a.oPx[p] = P[0];
            a.oPy[p] = P[1];
            a.oPz[p] = P[2];
            a.ovx[p] = v[0];
            a.ovy[p] = v[1];
            a.ovz[p] = v[2];
            a.obx[p] = vmacro[0];
            a.oby[p] = vmacro[1];
            a.obz[p] = vmacro[2];
        }
    }
    MapStats* st = a.stats;
    if (i < a.nref) {
        if (it_total) atomicAdd(&st->iter_total, it_total);
        atomicMax(&st->iter_max, it_max);
        if (nfail) {
            atomicAdd(&st->failures, nfail);
            atomicMin(&st->first_fail_key, first_fail);
        }
        atomicMax(&st->worst_scaled_bits, (unsigned long long)__double_as_longlong(worst));
    }
}

// ---- failed-particle records ---------------------------------------------------
// The report of one local solve (LocalParticleSolveReport :4805, filled as
// solve_local_particle_substep :4930 fills it): iteration count, reason, the
// first and last scaled residuals, the last absolute residual, the last
// iterate and the last map value.
struct SolveTrace {
    int iters = 0, reason = kLocalMaxIter;
    double first_scaled = INFINITY, final_scaled = INFINITY, final_abs = INFINITY;
    double last_guess[3] = {0.0, 0.0, 0.0}, last_map[3] = {0.0, 0.0, 0.0};
};

// The local fixed point of the map kernels with its report; eval(guess, o)
// is one map evaluation (false: too many knot crossings).  The arithmetic of
// every iterate is the map kernels', so a particle fails here exactly as it
// failed there.
template <class Eval>
UPIC_D bool traced_solve(const ImplicitMapArgs& a, const double* start, Eval eval, SolveTrace& t) {
    double guess[3] = {start[0], start[1], start[2]};
    LocalOut o;
    t = SolveTrace{};
#pragma unroll
    for (int c = 0; c < 3; ++c) t.last_guess[c] = guess[c];
    for (int it = 0; it < a.loc_maxit; ++it) {
        if (!eval(guess, o)) {
            t.reason = kLocalTooManyCrossings;
            return false;
        }
        ++t.iters;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            t.last_guess[c] = guess[c];
            t.last_map[c] = o.vbar_map[c];
        }
        if (!finite3(o.vbar_map)) {
            t.reason = kLocalNonfiniteMap;
            return false;
        }
        if (norm3(o.vbar_map) >= a.kappa) {
            t.reason = kLocalSuperluminalMap;
            return false;
        }
        const double res[3] = {o.vbar_map[0] - guess[0], o.vbar_map[1] - guess[1], o.vbar_map[2] - guess[2]};
        const double sc = 0.5 * (norm3(o.vbar_map) + norm3(guess));
        t.final_abs = norm3(res);
        t.final_scaled = t.final_abs / (a.loc_atol + a.loc_rtol * sc);
        if (t.iters == 1) t.first_scaled = t.final_scaled;
        if (t.final_scaled <= 1.0) {
            t.reason = kLocalOk;
            return true;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            guess[c] += a.loc_damp * res[c];
            t.last_guess[c] = guess[c];
        }
        if (!finite3(guess)) {
            t.reason = kLocalNonfiniteIterate;
            return false;
        }
        if (norm3(guess) >= a.kappa) {
            t.reason = kLocalSuperluminalIterate;
            return false;
        }
    }
    t.reason = kLocalMaxIter;
    return false;
}

// One record per failed particle of a map evaluation (failed[0..nf), sorted
// positions; the FailedParticleDiagnostic of :5331-5350): the particle's
// local solves are run again on the evaluation's fields, unit-step particles
// with the map kernel's evaluation (MOM, SY as that launch), sub-cycled ones
// substep by substep as refined_map_kernel advances them, up to the substep
// that fails.  Record (kFailRec doubles): particle id, assigned substeps,
// failed substep, theta0, theta1, h, iterations, reason, first / final
// scaled residual, final absolute residual, q, m, x0 (3), P0 (3), initial
// guess (3), last guess (3), last map (3).
template <int ORDER, bool UNIFORM, bool MOM, int SY>
__global__ void __launch_bounds__(128) failure_report_kernel(ImplicitMapArgs a, int nx, int ny, const int* failed,
                                                             int nf, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    Geo g{nx, ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    g.qs = a.qtab;
    g.qw = a.qtab + kMaxQuad;
    g.ms = a.qtab + 2 * kMaxQuad;
    g.mw = a.qtab + 3 * kMaxQuad;
    g.nq = a.nq;
    g.mnq = a.mnq;
    const int p = failed[i];
    const int n = a.nsub ? a.nsub[p] : 1;
    const double q = UNIFORM ? a.q0 : a.q[p];
    const double m = UNIFORM ? a.m0 : a.m[p];
    double x = a.x[p], y = a.y[p];
    double P[3] = {a.Px[p], a.Py[p], a.Pz[p]};
    double v[3] = {a.vx[p], a.vy[p], a.vz[p]};
    double bk[kMaxBreaks];
    int nb = 0;
    SolveTrace t;
    int k = 0;
    double th0 = 0.0, th1 = 1.0, h = a.dt, x0 = x, y0 = y, P0[3] = {P[0], P[1], P[2]}, start[3];
    if (n <= 1) {
        LocalIn in;
        in.x0 = x;
        in.y0 = y;
        in.q = q;
        in.m = m;
#pragma unroll
        for (int c = 0; c < 3; ++c) in.P0[c] = P[c];
        gather_rec3<ORDER, kIRec, SY>(g, a.rec, kIRecAn, x, y, in.A0p);
#pragma unroll
        for (int c = 0; c < 3; ++c) in.pstart[c] = in.P0[c] - in.q * in.A0p[c];
        set_local_constants(in, a.kappa);
        start[0] = a.warm_x ? a.warm_x[p] : v[0];
        start[1] = a.warm_x ? a.warm_y[p] : v[1];
        start[2] = a.warm_x ? a.warm_z[p] : v[2];
        traced_solve(a, start, [&](const double* gs, LocalOut& o) {
            if constexpr (MOM)
                return evaluate_moments<ORDER, SY>(g, a.rec, a.dt, a.kappa, a.split, in, gs, o, bk, nb);
            else
                return evaluate<ORDER, SY>(g, a.rec, a.dt, a.kappa, a.split, in, gs, o, bk, nb);
        }, t);
    } else {
        h = a.dt / (double)n;
        for (k = 0; k < n; ++k) {
            th0 = (double)k / (double)n;
            th1 = (double)(k + 1) / (double)n;
            LocalIn in;
            in.x0 = x;
            in.y0 = y;
            in.q = q;
            in.m = m;
            double An0[3], Ae0[3];
            gather_rec3<ORDER>(g, a.rec, kIRecAn, x, y, An0);
            gather_rec3<ORDER>(g, a.rec, kIRecAe, x, y, Ae0);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                in.P0[c] = P[c];
                in.A0p[c] = (1.0 - th0) * An0[c] + th0 * Ae0[c];
                in.pstart[c] = P[c] - q * in.A0p[c];
            }
            set_local_constants(in, a.kappa);
            x0 = x;
            y0 = y;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                P0[c] = P[c];
                start[c] = v[c];
            }
            LocalOut last;
            const bool ok = traced_solve(a, start, [&](const double* gs, LocalOut& o) {
                const bool r = evaluate_sub<ORDER>(g, a.rec, h, th0, th1, a.kappa, a.split, in, gs, o, bk, nb);
                last = o;
                return r;
            }, t);
            if (!ok) break;
            // the accepted sub-orbit's end state starts the next substep
            x = last.x1;
            y = last.y1;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                P[c] = last.P_end[c];
                v[c] = last.v_end[c];
            }
        }
    }
    double* r = out + (size_t)i * kFailRec;
    r[0] = (double)a.id[p];
    r[1] = (double)n;
    r[2] = (double)(n <= 1 ? 0 : k);
    r[3] = th0;
    r[4] = th1;
    r[5] = h;
    r[6] = (double)t.iters;
    r[7] = (double)t.reason;
    r[8] = t.first_scaled;
    r[9] = t.final_scaled;
    r[10] = t.final_abs;
    r[11] = q;
    r[12] = m;
    r[13] = x0;
    r[14] = y0;
    r[15] = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r[16 + c] = P0[c];
        r[19 + c] = start[c];
        r[22 + c] = t.last_guess[c];
        r[25 + c] = t.last_map[c];
    }
}

__global__ void fill_int_kernel(int n, int value, int* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = value;
}

// ---- start-up point deposit -------------------------------------------------
template <int ORDER>
__global__ void point_deposit_kernel(PointDepositArgs a) {
    const Geo g{a.nx, a.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    const int N = a.nx * a.ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < a.np; p += (long)gridDim.x * blockDim.x) {
        Stencil<ORDER> sx, sy;
        stencil_xy<ORDER>(g, a.x[p], a.y[p], sx, sy);
        const double q = a.q ? a.q[p] : a.q0;
        const double qa = q * a.inv_dV;
        const double val[4] = {qa * a.vx[p], qa * a.vy[p], qa * a.vz[p], qa};
        for (int ia = 0; ia <= ORDER; ++ia) {
            const int gx = wrap_index(sx.il + ia, a.nx);
            for (int ib = 0; ib <= ORDER; ++ib) {
                const int node = gx * a.ny + wrap_index(sy.il + ib, a.ny);
                const double w = sx.w[ia] * sy.w[ib];
                for (int c = 0; c < 4; ++c) {
                    const double v = val[c] * w;
                    if (v == 0.0) continue;
                    const Fixed2 f = to_fixed(v, a.scale[c]);
                    atomicAdd(&a.acc[(size_t)(2 * c) * N + node], f.hi);
                    atomicAdd(&a.acc[(size_t)(2 * c + 1) * N + node], f.lo);
                }
            }
        }
    }
}

// ---- kernel-level orbit entry points ---------------------------------------
// Orbit x0 + s dx, s in [0, 1], split at knots and summed with the deck's
// Gauss rule point by point, in the reference's order of quadrature points
// (path_average_deposit_current :2784, path_average_gather_and_gradient
// :3016).  One thread per particle; the deposit adds fixed-point integers,
// so its result does not depend on the order of the atomics.
template <int ORDER>
__global__ void orbit_deposit_kernel(OrbitArgs a) {
    constexpr int S = ORDER + 1;
    Geo g{a.nx, a.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    const int N = a.nx * a.ny;
    const double* qs = a.qtab;
    const double* qw = a.qtab + kMaxQuad;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < a.np; p += (long)gridDim.x * blockDim.x) {
        const double x0 = a.x[p], y0 = a.y[p];
        const double dxx = a.dx[3 * p], dxy = a.dx[3 * p + 1];
        double b[kMaxBreaks];
        const int nb = breakpoints<ORDER>(g, x0, y0, dxx, dxy, a.split, b);
        if (nb < 0) {
            atomicOr(a.err, 1);
            continue;
        }
        const double qa = (a.q ? a.q[p] : a.q0) * a.inv_dV;
        const double val[3] = {qa * a.vbar[3 * p], qa * a.vbar[3 * p + 1], qa * a.vbar[3 * p + 2]};
        for (int k = 0; k + 1 < nb; ++k) {
            const double sa = b[k], len = b[k + 1] - b[k];
            if (len <= 0.0) continue;
            for (int iq = 0; iq < a.nq; ++iq) {
                const double s = sa + len * qs[iq];
                const double wq = len * qw[iq];
                Stencil<ORDER> sx, sy;
                stencil_xy<ORDER>(g, wrap1(x0 + s * dxx, g.Lx), wrap1(y0 + s * dxy, g.Ly), sx, sy);
                for (int ia = 0; ia < S; ++ia) {
                    const int gx = wrap_index(sx.il + ia, a.nx);
                    for (int ib = 0; ib < S; ++ib) {
                        const int node = gx * a.ny + wrap_index(sy.il + ib, a.ny);
                        const double w = wq * sx.w[ia] * sy.w[ib];
                        for (int c = 0; c < 3; ++c) {
                            const double v = val[c] * w;
                            if (v == 0.0) continue;
                            const Fixed2 f = to_fixed(v, a.scale[c]);
                            atomicAdd(&a.acc[(size_t)(2 * c) * N + node], f.hi);
                            atomicAdd(&a.acc[(size_t)(2 * c + 1) * N + node], f.lo);
                        }
                    }
                }
            }
        }
    }
}

template <int ORDER>
__global__ void orbit_gather_kernel(OrbitArgs a) {
    constexpr int S = ORDER + 1;
    Geo g{a.nx, a.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    const int N = a.nx * a.ny;
    const double* qs = a.qtab;
    const double* qw = a.qtab + kMaxQuad;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < a.np; p += (long)gridDim.x * blockDim.x) {
        const double x0 = a.x[p], y0 = a.y[p];
        const double dxx = a.dx[3 * p], dxy = a.dx[3 * p + 1];
        double b[kMaxBreaks];
        const int nb = breakpoints<ORDER>(g, x0, y0, dxx, dxy, a.split, b);
        double gat[3] = {0.0, 0.0, 0.0};
        double D[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        if (nb < 0) atomicOr(a.err, 1);
        for (int k = 0; k + 1 < nb; ++k) {
            const double sa = b[k], len = b[k + 1] - b[k];
            if (len <= 0.0) continue;
            for (int iq = 0; iq < a.nq; ++iq) {
                const double s = sa + len * qs[iq];
                const double wq = len * qw[iq];
                Stencil<ORDER> sx, sy;
                stencil_xy<ORDER>(g, wrap1(x0 + s * dxx, g.Lx), wrap1(y0 + s * dxy, g.Ly), sx, sy);
                for (int ia = 0; ia < S; ++ia) {
                    const int gx = wrap_index(sx.il + ia, a.nx);
                    for (int ib = 0; ib < S; ++ib) {
                        const int node = gx * a.ny + wrap_index(sy.il + ib, a.ny);
                        const double shape = sx.w[ia] * sy.w[ib];
                        const double dsx = sx.dw[ia] * sy.w[ib], dsy = sx.w[ia] * sy.dw[ib];
                        for (int c = 0; c < 3; ++c) {
                            gat[c] += wq * a.mesh[(size_t)c * N + node] * shape;
                            const double av = (1.0 - s) * a.An[(size_t)c * N + node] + s * a.Ae[(size_t)c * N + node];
                            D[c][0] += wq * av * dsx;
                            D[c][1] += wq * av * dsy;
                        }
                    }
                }
            }
        }
        for (int c = 0; c < 3; ++c) {
            a.gathered[3 * p + c] = gat[c];
            a.grad[9 * p + 3 * c] = D[c][0];
            a.grad[9 * p + 3 * c + 1] = D[c][1];
            a.grad[9 * p + 3 * c + 2] = 0.0;  // nz = 1: no z derivative
        }
    }
}

template <int ORDER>
__global__ void gather3_kernel(int nx, int ny, double Lx, double Ly, const double* f3, long np,
                               const double* x, const double* y, double* out3) {
    const Geo g{nx, ny, Lx, Ly, nx / Lx, ny / Ly};
    const int N = nx * ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        Stencil<ORDER> sx, sy;
        stencil_xy<ORDER>(g, x[p], y[p], sx, sy);
        double o[3] = {0.0, 0.0, 0.0};
        for (int ia = 0; ia <= ORDER; ++ia) {
            const int gx = wrap_index(sx.il + ia, nx);
            for (int ib = 0; ib <= ORDER; ++ib) {
                const int node = gx * ny + wrap_index(sy.il + ib, ny);
                const double w = sx.w[ia] * sy.w[ib];
                for (int c = 0; c < 3; ++c) o[c] = fma(f3[(size_t)c * N + node], w, o[c]);
            }
        }
        for (int c = 0; c < 3; ++c) out3[3 * p + c] = o[c];
    }
}

// Point probes (evaluate_reconstructed_field_probe :7924): F holds 18
// planar fields phi, psi, rho, A, U, J, E, B; per point the 18 shape
// gathers, grad(S phi) and grad(S A) (row c: dA_c/dx, dA_c/dy, 0), 30
// values in the UPIC_PROBE_* order.
// GM-HC-CN push of a particle list in given fields (upic_push_gmhc): the
// damped local fixed point on the orbit velocity (solve_local_particle_substep
// :4930) with the kick-rotate-kick map (evaluate_local_particle_substep
// :4843, h = dt, theta0 = 0, theta1 = 1), one thread per particle.  rec:
// node records (grad phi_mid, A^n, A^{n+1}; kIRec doubles per node).  in7:
// x, y, Px, Py, Pz, q, m per particle (planar, stride np); guess3: the
// first guesses (planar); out: x1, y1, P_end (3), v_end (3), vbar (3)
// (planar, NaN for a failed particle); rep: iterations and failure reason.
template <int ORDER, bool MOM>
__global__ void gmhc_push_kernel(ImplicitMapArgs a, int nx, int ny, long np, const double* __restrict__ in7,
                                 const double* __restrict__ guess3, double* __restrict__ out, int* __restrict__ rep) {
    Geo g{nx, ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    g.qs = a.qtab;
    g.qw = a.qtab + kMaxQuad;
    g.ms = a.qtab + 2 * kMaxQuad;
    g.mw = a.qtab + 3 * kMaxQuad;
    g.nq = a.nq;
    g.mnq = a.mnq;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        LocalIn in;
        in.x0 = in7[p];
        in.y0 = in7[np + p];
        for (int c = 0; c < 3; ++c) in.P0[c] = in7[(2 + c) * np + p];
        in.q = in7[5 * np + p];
        in.m = in7[6 * np + p];
        gather_rec3<ORDER>(g, a.rec, kIRecAn, in.x0, in.y0, in.A0p);
        for (int c = 0; c < 3; ++c) in.pstart[c] = in.P0[c] - in.q * in.A0p[c];
        set_local_constants(in, a.kappa);
        double guess[3] = {guess3[p], guess3[np + p], guess3[2 * np + p]};
        double bk[kMaxBreaks];
        int nb = 0, iters = 0, reason = kLocalMaxIter;
        LocalOut o;
        for (int it = 0; it < a.loc_maxit; ++it) {
            const bool okev = MOM ? evaluate_moments<ORDER>(g, a.rec, a.dt, a.kappa, a.split, in, guess, o, bk, nb)
                                  : evaluate<ORDER>(g, a.rec, a.dt, a.kappa, a.split, in, guess, o, bk, nb);
            if (!okev) {
                reason = kLocalTooManyCrossings;
                break;
            }
            ++iters;
            if (!finite3(o.vbar_map)) {
                reason = kLocalNonfiniteMap;
                break;
            }
            if (norm3(o.vbar_map) >= a.kappa) {
                reason = kLocalSuperluminalMap;
                break;
            }
            const double res[3] = {o.vbar_map[0] - guess[0], o.vbar_map[1] - guess[1], o.vbar_map[2] - guess[2]};
            const double sc = 0.5 * (norm3(o.vbar_map) + norm3(guess));
            if (norm3(res) / (a.loc_atol + a.loc_rtol * sc) <= 1.0) {
                reason = kLocalOk;
                break;
            }
            for (int c = 0; c < 3; ++c) guess[c] += a.loc_damp * res[c];
            if (!finite3(guess)) {
                reason = kLocalNonfiniteIterate;
                break;
            }
            if (norm3(guess) >= a.kappa) {
                reason = kLocalSuperluminalIterate;
                break;
            }
        }
        const bool ok = reason == kLocalOk;
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        const double vals[11] = {o.x1, o.y1, o.P_end[0], o.P_end[1], o.P_end[2], o.v_end[0], o.v_end[1],
                                 o.v_end[2], guess[0], guess[1], guess[2]};
        for (int k = 0; k < 11; ++k) out[(size_t)k * np + p] = ok ? vals[k] : nan;
        rep[2 * p] = iters;
        rep[2 * p + 1] = reason;
    }
}

template <int ORDER>
__global__ void probe_kernel(int nx, int ny, double Lx, double Ly, const double* __restrict__ F, long np,
                             const double* x, const double* y, double* out) {
    const Geo g{nx, ny, Lx, Ly, nx / Lx, ny / Ly};
    const int N = nx * ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        Stencil<ORDER> sx, sy;
        stencil_xy<ORDER>(g, x[p], y[p], sx, sy);
        double v[18], gp[2] = {0.0, 0.0}, gA[3][2] = {};
        for (int f = 0; f < 18; ++f) v[f] = 0.0;
        for (int ia = 0; ia <= ORDER; ++ia) {
            const int gx = wrap_index(sx.il + ia, nx);
            for (int ib = 0; ib <= ORDER; ++ib) {
                const int node = gx * ny + wrap_index(sy.il + ib, ny);
                const double w = sx.w[ia] * sy.w[ib];
                const double wx = sx.dw[ia] * sy.w[ib], wy = sx.w[ia] * sy.dw[ib];
                for (int f = 0; f < 18; ++f) v[f] = fma(F[(size_t)f * N + node], w, v[f]);
                const double ph = F[node];
                gp[0] = fma(ph, wx, gp[0]);
                gp[1] = fma(ph, wy, gp[1]);
                for (int c = 0; c < 3; ++c) {
                    const double a = F[(size_t)(3 + c) * N + node];
                    gA[c][0] = fma(a, wx, gA[c][0]);
                    gA[c][1] = fma(a, wy, gA[c][1]);
                }
            }
        }
        double* o = out + (size_t)p * 30;
        for (int f = 0; f < 18; ++f) o[f] = v[f];
        o[18] = gp[0];
        o[19] = gp[1];
        o[20] = 0.0;
        for (int c = 0; c < 3; ++c) {
            o[21 + 3 * c] = gA[c][0];
            o[22 + 3 * c] = gA[c][1];
            o[23 + 3 * c] = 0.0;
        }
    }
}

template <int ORDER>
__global__ void add_qA_kernel(int nx, int ny, double Lx, double Ly, const double* A3, long np, const double* x,
                              const double* y, const double* q, double q0, double* Px, double* Py, double* Pz) {
    const Geo g{nx, ny, Lx, Ly, nx / Lx, ny / Ly};
    const int N = nx * ny;
    double* const P[3] = {Px, Py, Pz};
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        Stencil<ORDER> sx, sy;
        stencil_xy<ORDER>(g, x[p], y[p], sx, sy);
        double o[3] = {0.0, 0.0, 0.0};
        for (int ia = 0; ia <= ORDER; ++ia) {
            const int gx = wrap_index(sx.il + ia, nx);
            for (int ib = 0; ib <= ORDER; ++ib) {
                const int node = gx * ny + wrap_index(sy.il + ib, ny);
                const double w = sx.w[ia] * sy.w[ib];
                for (int c = 0; c < 3; ++c) o[c] = fma(A3[(size_t)c * N + node], w, o[c]);
            }
        }
        const double qp = q ? q[p] : q0;
        // m gamma v + q A, the product rounded before the sum as the reference's
        for (int c = 0; c < 3; ++c) P[c][p] = __dadd_rn(P[c][p], __dmul_rn(qp, o[c]));
    }
}

template <int ORDER>
__global__ void history_velocity_kernel(int nx, int ny, double Lx, double Ly, const double* E3,
                                        const double* B3, long np, const double* x, const double* y,
                                        const double* vx, const double* vy, const double* vz,
                                        const double* qa, double q0, const double* ma, double m0,
                                        double kappa, double dt, double* wx, double* wy, double* wz) {
    const Geo g{nx, ny, Lx, Ly, nx / Lx, ny / Ly};
    const int N = nx * ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        Stencil<ORDER> sx, sy;
        stencil_xy<ORDER>(g, x[p], y[p], sx, sy);
        double E[3] = {0.0, 0.0, 0.0}, B[3] = {0.0, 0.0, 0.0};
        for (int ia = 0; ia <= ORDER; ++ia) {
            const int gx = wrap_index(sx.il + ia, nx);
            for (int ib = 0; ib <= ORDER; ++ib) {
                const int node = gx * ny + wrap_index(sy.il + ib, ny);
                const double w = sx.w[ia] * sy.w[ib];
                for (int c = 0; c < 3; ++c) {
                    E[c] = fma(E3[(size_t)c * N + node], w, E[c]);
                    B[c] = fma(B3[(size_t)c * N + node], w, B[c]);
                }
            }
        }
        const double q = qa ? qa[p] : q0, m = ma ? ma[p] : m0;
        const double v[3] = {vx[p], vy[p], vz[p]};
        const double beta2 = dot3(v, v) / (kappa * kappa);
        const double gam = 1.0 / sqrt(fmax(1.0e-300, 1.0 - beta2));
        const double pn[3] = {m * gam * v[0], m * gam * v[1], m * gam * v[2]};
        const double vxb[3] = {v[1] * B[2] - v[2] * B[1], v[2] * B[0] - v[0] * B[2], v[0] * B[1] - v[1] * B[0]};
        const double pp[3] = {pn[0] - dt * (q * (E[0] + vxb[0])), pn[1] - dt * (q * (E[1] + vxb[1])),
                              pn[2] - dt * (q * (E[2] + vxb[2]))};
        const double gp = gamma_p(pp, m * kappa);
        wx[p] = pp[0] * (1.0 / (m * gp));
        wy[p] = pp[1] * (1.0 / (m * gp));
        wz[p] = pp[2] * (1.0 / (m * gp));
    }
}

// ---- k-space map fields -----------------------------------------------------
UPIC_D double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
UPIC_D double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
UPIC_D double2 cik(double k, double2 z) { return make_double2(-k * z.y, k * z.x); }

__global__ void cn_kspace_kernel(CnArgs a) {
    const int N = a.N;
    const double c2 = a.kappa * a.kappa;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const bool ex = a.excl && a.excl[id];
        const double kx = a.kx[id], ky = a.ky[id], k2 = a.k2[id];
        double2 J[3];
        for (int c = 0; c < 3; ++c) J[c] = ex ? make_double2(0.0, 0.0) : a.Jhat[(size_t)c * N + id];
        const double2 phi = a.st[0 * (size_t)N + id], psi = a.st[1 * (size_t)N + id];
        const double2 rho = a.st[2 * (size_t)N + id];
        // continuity_charge_update (:3288): rho - dt div J, zero mean, Nyquist projection
        const double2 divJ = cik(1.0, make_double2(kx * J[0].x + ky * J[1].x, kx * J[0].y + ky * J[1].y));
        double2 rho_end = make_double2(rho.x - a.dt * divJ.x, rho.y - a.dt * divJ.y);
        if (id == 0 || ex) rho_end = make_double2(0.0, 0.0);
        const double2 rho_mid = cscale(0.5, cadd(rho, rho_end));
        // CN step (cn_fft_wave_step_from_spectra :3131)
        const double theta = 0.25 * c2 * a.dt * a.dt * k2;
        const double den = 1.0 + theta;
        auto cn = [&](double2 u, double2 v, double2 S, double sigma, double2& un, double2& vn) {
            if (ex) {
                un = vn = make_double2(0.0, 0.0);
                return;
            }
            const double sc = c2 * sigma;
            un = make_double2(((1.0 - theta) * u.x + a.dt * v.x + 0.5 * sc * a.dt * a.dt * S.x) / den,
                              ((1.0 - theta) * u.y + a.dt * v.y + 0.5 * sc * a.dt * a.dt * S.y) / den);
            vn = make_double2(((1.0 - theta) * v.x - c2 * a.dt * k2 * u.x + sc * a.dt * S.x) / den,
                              ((1.0 - theta) * v.y - c2 * a.dt * k2 * u.y + sc * a.dt * S.y) / den);
        };
        double2 phin, psin;
        cn(phi, psi, rho_mid, a.sigma1, phin, psin);
        if (id == 0) {  // subtract_mean of phi and psi
            phin = make_double2(0.0, 0.0);
            psin = make_double2(0.0, 0.0);
        }
        double2 An[3], Un[3];
        for (int c = 0; c < 3; ++c)
            cn(a.st[(size_t)(3 + c) * N + id], a.st[(size_t)(6 + c) * N + id], J[c], a.sigma2, An[c], Un[c]);
        a.out[0 * (size_t)N + id] = phin;
        a.out[1 * (size_t)N + id] = psin;
        a.out[2 * (size_t)N + id] = rho_end;
        for (int c = 0; c < 3; ++c) {
            a.out[(size_t)(3 + c) * N + id] = An[c];
            a.out[(size_t)(6 + c) * N + id] = Un[c];
        }
        // grad phi_mid = (grad phi^n + grad phi^{n+1}) / 2, and A^{n+1}
        const double2 gx = cscale(0.5, cadd(cik(kx, phi), cik(kx, phin)));
        const double2 gy = cscale(0.5, cadd(cik(ky, phi), cik(ky, phin)));
        a.gspec[0 * (size_t)N + id] = gx;
        a.gspec[1 * (size_t)N + id] = gy;
        for (int c = 0; c < 3; ++c) a.gspec[(size_t)(2 + c) * N + id] = An[c];
    }
}

// Diagnostics spectra of a state (compute_E :3338, spectral_curl :1780,
// compute_diagnostics :3521): E (3), B (3), div E, div A, psi, rho.
__global__ void diag_spectra_kernel(int N, const double* kx, const double* ky, const double2* st,
                                    double2* out) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double kxx = kx[id], kyy = ky[id];
        const double2 phi = st[id], psi = st[N + id], rho = st[2 * (size_t)N + id];
        const double2 A0 = st[3 * (size_t)N + id], A1 = st[4 * (size_t)N + id], A2 = st[5 * (size_t)N + id];
        const double2 U0 = st[6 * (size_t)N + id], U1 = st[7 * (size_t)N + id], U2 = st[8 * (size_t)N + id];
        const double2 gx = cik(kxx, phi), gy = cik(kyy, phi);
        const double2 E0 = make_double2(-gx.x - U0.x, -gx.y - U0.y);
        const double2 E1 = make_double2(-gy.x - U1.x, -gy.y - U1.y);
        const double2 E2 = make_double2(-U2.x, -U2.y);
        out[0 * (size_t)N + id] = E0;
        out[1 * (size_t)N + id] = E1;
        out[2 * (size_t)N + id] = E2;
        out[3 * (size_t)N + id] = cik(kyy, A2);
        out[4 * (size_t)N + id] = cik(-kxx, A2);
        out[5 * (size_t)N + id] = cik(1.0, make_double2(kxx * A1.x - kyy * A0.x, kxx * A1.y - kyy * A0.y));
        out[6 * (size_t)N + id] = cik(1.0, make_double2(kxx * E0.x + kyy * E1.x, kxx * E0.y + kyy * E1.y));
        out[7 * (size_t)N + id] = cik(1.0, make_double2(kxx * A0.x + kyy * A1.x, kxx * A0.y + kyy * A1.y));
        out[8 * (size_t)N + id] = psi;
        out[9 * (size_t)N + id] = rho;
    }
}

// P = m gamma(v) v + q A(x) with A = 0 at start-up (momentum_from_v :645).
__global__ void momentum_from_v_kernel(long np, const double* vx, const double* vy, const double* vz,
                                       const double* m, double m0, double kappa, double* Px, double* Py,
                                       double* Pz) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        const double v[3] = {vx[p], vy[p], vz[p]};
        const double beta2 = dot3(v, v) / (kappa * kappa);
        const double gam = 1.0 / sqrt(fmax(1.0e-300, 1.0 - beta2));
        const double mg = (m ? m[p] : m0) * gam;
        Px[p] = mg * v[0];
        Py[p] = mg * v[1];
        Pz[p] = mg * v[2];
    }
}

// project_nyquist (:2044): per line, subtract the alternating mean.  One
// warp per line: lane l sums entries l, l+32, ... in double-double, then a
// fixed xor tree combines the lanes (the same order on every run).
// Axis 1 (lines along y) reads rows contiguously; axis 0 (lines along x)
// makes 32 lines of consecutive j share each warp's columns via the grid.
__global__ void project_lines_kernel(double* f, int ncomp, int nx, int ny, int axis) {
    const int n = axis == 0 ? nx : ny;
    const int lines = axis == 0 ? ny : nx;
    const int stride = axis == 0 ? ny : 1;
    const long total = (long)ncomp * lines;
    const int lane = threadIdx.x & 31;
    const long warps = (long)gridDim.x * (blockDim.x >> 5);
    for (long L = blockIdx.x * (long)(blockDim.x >> 5) + (threadIdx.x >> 5); L < total; L += warps) {
        const int c = (int)(L / lines), l = (int)(L - (long)c * lines);
        double* base = f + (size_t)c * nx * ny + (axis == 0 ? l : (size_t)l * ny);
        DD s{0.0, 0.0};
        for (int j = lane; j < n; j += 32) {
            const double v = base[(size_t)j * stride];
            s = dd_add(s, (j & 1) ? -v : v);
        }
        s = warp_sum_dd(s);
        const double mean = (s.hi + s.lo) / (double)n;
        for (int j = lane; j < n; j += 32) base[(size_t)j * stride] -= (j & 1) ? -mean : mean;
    }
}

__global__ void kspace_mask_kernel(double2* f, int ncomp, int N, const unsigned char* excl, int zero_mean) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncomp * N; i += gridDim.x * blockDim.x) {
        const int id = i % N;
        if ((zero_mean && id == 0) || (excl && excl[id])) f[i] = make_double2(0.0, 0.0);
    }
}

// ---- outer iteration algebra ------------------------------------------------
constexpr int kRed = 256;

__global__ void __launch_bounds__(kRed)
residual_norms_kernel(int N, const double* map, const double* guess, double floor_rel, double atol,
                      double rtol, double* partials) {
    DD r2{0, 0}, m2{0, 0}, g2{0, 0};
    double mrel = 0.0, msc = 0.0;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        double mv[3], gv[3], rv[3];
        for (int c = 0; c < 3; ++c) {
            mv[c] = map[(size_t)c * N + id];
            gv[c] = guess[(size_t)c * N + id];
            rv[c] = mv[c] - gv[c];
            r2 = dd_add_dd(r2, dd_sq(rv[c]));
            m2 = dd_add_dd(m2, dd_sq(mv[c]));
            g2 = dd_add_dd(g2, dd_sq(gv[c]));
        }
        const double rn = norm3(rv);
        const double vs = 0.5 * (norm3(mv) + norm3(gv));
        mrel = fmax(mrel, rn / fmax(floor_rel, vs));
        msc = fmax(msc, rn / (atol + rtol * vs));
    }
    r2 = warp_sum_dd(r2);
    m2 = warp_sum_dd(m2);
    g2 = warp_sum_dd(g2);
    mrel = warp_max(mrel);
    msc = warp_max(msc);
    __shared__ double red[kRed / kWarp][8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w][0] = r2.hi; red[w][1] = r2.lo; red[w][2] = m2.hi; red[w][3] = m2.lo;
        red[w][4] = g2.hi; red[w][5] = g2.lo; red[w][6] = mrel; red[w][7] = msc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD a{0, 0}, b{0, 0}, c{0, 0};
        double x = 0.0, y = 0.0;
        for (int k = 0; k < kRed / kWarp; ++k) {
            a = dd_add_dd(a, DD{red[k][0], red[k][1]});
            b = dd_add_dd(b, DD{red[k][2], red[k][3]});
            c = dd_add_dd(c, DD{red[k][4], red[k][5]});
            x = fmax(x, red[k][6]);
            y = fmax(y, red[k][7]);
        }
        double* o = partials + (size_t)blockIdx.x * 8;
        o[0] = a.hi; o[1] = a.lo; o[2] = b.hi; o[3] = b.lo; o[4] = c.hi; o[5] = c.lo; o[6] = x; o[7] = y;
    }
}

// One warp: lane l combines the partials l, l+32, ...; a fixed xor tree
// combines the lanes.
__global__ void residual_final_kernel(const double* partials, int grid, NormSums* out) {
    DD a{0, 0}, b{0, 0}, c{0, 0};
    double x = 0.0, y = 0.0;
    for (int k = threadIdx.x; k < grid; k += 32) {
        const double* o = partials + (size_t)k * 8;
        a = dd_add_dd(a, DD{o[0], o[1]});
        b = dd_add_dd(b, DD{o[2], o[3]});
        c = dd_add_dd(c, DD{o[4], o[5]});
        x = fmax(x, o[6]);
        y = fmax(y, o[7]);
    }
    a = warp_sum_dd(a);
    b = warp_sum_dd(b);
    c = warp_sum_dd(c);
    x = warp_max(x);
    y = warp_max(y);
    if (threadIdx.x != 0) return;
    out->r2[0] = a.hi; out->r2[1] = a.lo;
    out->map2[0] = b.hi; out->map2[1] = b.lo;
    out->guess2[0] = c.hi; out->guess2[1] = c.lo;
    out->max_rel = x;
    out->max_scaled = y;
}

struct RPtrs {
    const double* r[8];
};

constexpr int kMaxDots = 14;

__global__ void __launch_bounds__(kRed)
anderson_dots_kernel(int n, RPtrs rp, int m, double* partials) {
    DD s[kMaxDots];
    for (int k = 0; k < kMaxDots; ++k) s[k] = DD{0, 0};
    const int ndots = m * (m + 1) / 2 + m;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double dr[4];
        for (int j = 0; j < m; ++j) dr[j] = rp.r[j + 1][i] - rp.r[j][i];
        const double rl = rp.r[m][i];
        int k = 0;
        for (int a = 0; a < m; ++a)
            for (int b = 0; b <= a; ++b) {
                const double pr = dr[a] * dr[b];
                s[k] = dd_add_dd(s[k], DD{pr, fma(dr[a], dr[b], -pr)});
                ++k;
            }
        for (int a = 0; a < m; ++a) {
            const double pr = dr[a] * rl;
            s[k] = dd_add_dd(s[k], DD{pr, fma(dr[a], rl, -pr)});
            ++k;
        }
    }
    __shared__ double red[kRed / kWarp][2 * kMaxDots];
    const int w = threadIdx.x >> 5;
    for (int k = 0; k < ndots; ++k) {
        s[k] = warp_sum_dd(s[k]);
        if ((threadIdx.x & 31) == 0) {
            red[w][2 * k] = s[k].hi;
            red[w][2 * k + 1] = s[k].lo;
        }
    }
    __syncthreads();
    if (threadIdx.x < ndots) {
        DD t{0, 0};
        for (int q = 0; q < kRed / kWarp; ++q) t = dd_add_dd(t, DD{red[q][2 * threadIdx.x], red[q][2 * threadIdx.x + 1]});
        partials[(size_t)blockIdx.x * 2 * kMaxDots + 2 * threadIdx.x] = t.hi;
        partials[(size_t)blockIdx.x * 2 * kMaxDots + 2 * threadIdx.x + 1] = t.lo;
    }
}

// One warp per dot (blockDim = 32 * ndots), lanes over the partials.
__global__ void dots_final_kernel(const double* partials, int grid, int ndots, double* out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= ndots) return;
    DD t{0, 0};
    for (int b = lane; b < grid; b += 32)
        t = dd_add_dd(t, DD{partials[(size_t)b * 2 * kMaxDots + 2 * k], partials[(size_t)b * 2 * kMaxDots + 2 * k + 1]});
    t = warp_sum_dd(t);
    if (lane == 0) out[k] = t.hi + t.lo;
}

struct GPtrs {
    const double* x[8];
    const double* r[8];
    double gamma[4];
};

__global__ void anderson_candidate_kernel(int n, GPtrs g, int m, double beta, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double c = g.x[m][i] + beta * g.r[m][i];
        for (int j = 0; j < m; ++j) {
            const double dx = g.x[j + 1][i] - g.x[j][i];
            const double dr = g.r[j + 1][i] - g.r[j][i];
            c -= g.gamma[j] * (dx + beta * dr);
        }
        out[i] = c;
    }
}

__global__ void nonfinite_kernel(int n, const double* v, int* flag) {
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        bad |= !isfinite(v[i]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

__global__ void extrapolate_kernel(int n, const double* v, const double* w, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = 2.0 * v[i] - w[i];
}

__global__ void half_sum_kernel(int n, const double* a, const double* b, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = 0.5 * (a[i] + b[i]);
}

__global__ void lerp_kernel(int n, const double* a, const double* b, double s, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = a[i] + s * (b[i] - a[i]);
}

__global__ void axpy_kernel(int n, const double* a, const double* b, double s, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = a[i] + s * b[i];
}

// ---- step diagnostics (compute_subcycled_step_diagnostics :4340 with one
// level per particle, the layout of nonlinear_step_orbit) ---------------------
constexpr int kSdRec = 12;   // An(3), Ae(3), U_mid(3), E_mid(3) per node
constexpr int kSdPart = 16;  // per-CTA partials: 6 double-double sums + max

// Spectra of A^n, A^{n+1}, U_mid = (U^n + U^{n+1})/2 and
// E_mid = -(grad phi^n + grad phi^{n+1})/2 - U_mid.
__global__ void step_diag_spectra_kernel(int N, const double* kx, const double* ky, const double2* s0,
                                         const double2* s1, double2* out) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double kxx = kx[id], kyy = ky[id];
        const double2 phi0 = s0[id], phi1 = s1[id];
        double2 um[3];
        for (int c = 0; c < 3; ++c) {
            out[(size_t)c * N + id] = s0[(size_t)(3 + c) * N + id];
            out[(size_t)(3 + c) * N + id] = s1[(size_t)(3 + c) * N + id];
            const double2 u0 = s0[(size_t)(6 + c) * N + id], u1 = s1[(size_t)(6 + c) * N + id];
            um[c] = make_double2(0.5 * u0.x + 0.5 * u1.x, 0.5 * u0.y + 0.5 * u1.y);
            out[(size_t)(6 + c) * N + id] = um[c];
        }
        const double2 g0 = cik(kxx, phi0), g1 = cik(kxx, phi1), h0 = cik(kyy, phi0), h1 = cik(kyy, phi1);
        out[(size_t)9 * N + id] = make_double2(-0.5 * (g0.x + g1.x) - um[0].x, -0.5 * (g0.y + g1.y) - um[0].y);
        out[(size_t)10 * N + id] = make_double2(-0.5 * (h0.x + h1.x) - um[1].x, -0.5 * (h0.y + h1.y) - um[1].y);
        out[(size_t)11 * N + id] = make_double2(-um[2].x, -um[2].y);
    }
}

struct DDSix {
    DD v[6];
};

// Block reduction of the step-diagnostics sums: six double-double sums and
// the max into out[0..12], path counts into counts by integer atomics.
UPIC_D void sd_block_finish(DDSix sums, double nmax, unsigned long long segs, unsigned long long cross,
                            unsigned long long cpart, int maxseg, unsigned long long* counts, double* out) {
    __shared__ double red[kRed / kWarp][kSdPart];
    const int w = threadIdx.x >> 5;
    for (int k = 0; k < 6; ++k) {
        const DD v = warp_sum_dd(sums.v[k]);
        if ((threadIdx.x & 31) == 0) {
            red[w][2 * k] = v.hi;
            red[w][2 * k + 1] = v.lo;
        }
    }
    nmax = warp_max(nmax);
    if ((threadIdx.x & 31) == 0) red[w][12] = nmax;
    for (int o = 16; o > 0; o >>= 1) {
        segs += __shfl_xor_sync(0xffffffffu, segs, o);
        cross += __shfl_xor_sync(0xffffffffu, cross, o);
        cpart += __shfl_xor_sync(0xffffffffu, cpart, o);
        maxseg = max(maxseg, __shfl_xor_sync(0xffffffffu, maxseg, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counts[0], segs);
        atomicAdd(&counts[1], cross);
        atomicAdd(&counts[2], cpart);
        atomicMax(&counts[3], (unsigned long long)maxseg);
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        const int k = threadIdx.x;
        if (k < 6) {
            DD t{0, 0};
            for (int q = 0; q < kRed / kWarp; ++q) t = dd_add_dd(t, DD{red[q][2 * k], red[q][2 * k + 1]});
            out[2 * k] = t.hi;
            out[2 * k + 1] = t.lo;
        } else {
            double mx = 0.0;
            for (int q = 0; q < kRed / kWarp; ++q) mx = fmax(mx, red[q][12]);
            out[12] = mx;
        }
    }
}

template <int ORDER>
__global__ void __launch_bounds__(kRed) step_diag_kernel(StepDiagArgs a) {
    constexpr int S = ORDER + 1;
    Geo g{a.nx, a.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    const double* qs = a.qtab;
    const double* qw = a.qtab + kMaxQuad;
    DD r2{0, 0}, a2{0, 0}, rhs2{0, 0}, nsum{0, 0}, wdef{0, 0}, pw{0, 0};
    double nmax = 0.0;
    unsigned long long segs = 0, cross = 0, cpart = 0;
    int maxseg = 1;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < a.np; p += (long)gridDim.x * blockDim.x) {
        if (a.nsub && a.nsub[p] > 1) continue;  // sub-cycled: step_diag_refined_kernel
        const double x0 = a.x[p], y0 = a.y[p];
        const double vb[3] = {a.bx[p], a.by[p], a.bz[p]};
        const double q = a.q ? a.q[p] : a.q0;
        const double h = a.dt;
        const double dxx = h * vb[0], dxy = h * vb[1];
        const double x1 = wrap1(x0 + dxx, g.Lx), y1 = wrap1(y0 + dxy, g.Ly);
        double A0p[3], A1p[3];
        gather_rec3<ORDER, kSdRec>(g, a.rec, 0, x0, y0, A0p);
        gather_rec3<ORDER, kSdRec>(g, a.rec, 3, x1, y1, A1p);
        double b[kMaxBreaks];
        const int nb = breakpoints<ORDER>(g, x0, y0, dxx, dxy, a.split, b);
        double Ub[3] = {0.0, 0.0, 0.0}, Eb[3] = {0.0, 0.0, 0.0};
        double D[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        for (int k = 0; k + 1 < nb; ++k) {
            const double sa = b[k], len = b[k + 1] - b[k];
            if (len <= 0.0) continue;
            for (int iq = 0; iq < a.nq; ++iq) {
                const double s = sa + len * qs[iq];
                const double wq = len * qw[iq];
                Stencil<ORDER> sx, sy;
                stencil_xy<ORDER>(g, wrap1(x0 + s * dxx, g.Lx), wrap1(y0 + s * dxy, g.Ly), sx, sy);
                for (int ia = 0; ia < S; ++ia) {
                    const int gx = wrap_index(sx.il + ia, a.nx);
                    for (int ib = 0; ib < S; ++ib) {
                        const double* r = a.rec + (size_t)(gx * a.ny + wrap_index(sy.il + ib, a.ny)) * kSdRec;
                        const double shape = sx.w[ia] * sy.w[ib];
                        const double dsx = sx.dw[ia] * sy.w[ib], dsy = sx.w[ia] * sy.dw[ib];
                        for (int c = 0; c < 3; ++c) {
                            Ub[c] += wq * r[6 + c] * shape;
                            Eb[c] += wq * r[9 + c] * shape;
                            const double av = (1.0 - s) * r[c] + s * r[3 + c];
                            D[c][0] += wq * av * dsx;
                            D[c][1] += wq * av * dsy;
                        }
                    }
                }
            }
        }
        double R[3], Ad[3], rhs[3];
        for (int c = 0; c < 3; ++c) {
            Ad[c] = A1p[c] - A0p[c];
            rhs[c] = h * (Ub[c] + (D[c][0] * vb[0] + D[c][1] * vb[1]));
            R[c] = Ad[c] - rhs[c];
        }
        r2 = dd_add(r2, dot3(R, R));
        a2 = dd_add(a2, dot3(Ad, Ad));
        rhs2 = dd_add(rhs2, dot3(rhs, rhs));
        const double nr = norm3(R);
        nmax = fmax(nmax, nr);
        nsum = dd_add(nsum, nr);
        wdef = dd_add(wdef, -q * dot3(vb, R));
        pw = dd_add(pw, (h * q) * dot3(vb, Eb));
        const int nseg = nb - 1 > 1 ? nb - 1 : 1;
        segs += (unsigned long long)nseg;
        cross += (unsigned long long)(nseg - 1);
        cpart += nseg > 1 ? 1ull : 0ull;
        maxseg = max(maxseg, nseg);
    }
    sd_block_finish(DDSix{r2, a2, rhs2, nsum, wdef, pw}, nmax, segs, cross, cpart, maxseg, a.counts,
                    a.partials + (size_t)blockIdx.x * kSdPart);
}

// Step diagnostics of the refined (sub-cycled) particles
// (compute_subcycled_step_diagnostics :4340): per recorded sub-orbit of
// h = dt/n over [k/n, (k+1)/n], the A-chain defect with time-interpolated A
// (weights 1/n in the rms sums), the work defect and the particle work; path
// segments summed per particle.  Block partials go to a.partials + block.
template <int ORDER>
__global__ void __launch_bounds__(kRed) step_diag_refined_kernel(StepDiagArgs a) {
    constexpr int S = ORDER + 1;
    Geo g{a.nx, a.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    const double* qs = a.qtab;
    const double* qw = a.qtab + kMaxQuad;
    DD r2{0, 0}, a2{0, 0}, rhs2{0, 0}, nsum{0, 0}, wdef{0, 0}, pw{0, 0};
    double nmax = 0.0;
    unsigned long long segs = 0, cross = 0, cpart = 0;
    int maxseg = 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nref; i += gridDim.x * blockDim.x) {
        const int p = a.refined[i];
        const int n = a.nsub[p];
        const double q = a.q ? a.q[p] : a.q0;
        const double h = a.dt / (double)n, wgt = 1.0 / (double)n;
        int psegs = 0;
        bool crossed = false;
        for (int k = 0; k < n; ++k) {
            const double* so = a.sub + (size_t)(a.roff[i] + k) * 5;
            const double x0 = so[0], y0 = so[1];
            const double vb[3] = {so[2], so[3], so[4]};
            const double th0 = (double)k / (double)n, th1 = (double)(k + 1) / (double)n;
            const double dxx = h * vb[0], dxy = h * vb[1];
            const double x1 = wrap1(x0 + dxx, g.Lx), y1 = wrap1(y0 + dxy, g.Ly);
            double An0[3], Ae0[3], An1[3], Ae1[3], A0p[3], A1p[3];
            gather_rec3<ORDER, kSdRec>(g, a.rec, 0, x0, y0, An0);
            gather_rec3<ORDER, kSdRec>(g, a.rec, 3, x0, y0, Ae0);
            gather_rec3<ORDER, kSdRec>(g, a.rec, 0, x1, y1, An1);
            gather_rec3<ORDER, kSdRec>(g, a.rec, 3, x1, y1, Ae1);
            for (int c = 0; c < 3; ++c) {
                A0p[c] = (1.0 - th0) * An0[c] + th0 * Ae0[c];
                A1p[c] = (1.0 - th1) * An1[c] + th1 * Ae1[c];
            }
            double b[kMaxBreaks];
            const int nb = breakpoints<ORDER>(g, x0, y0, dxx, dxy, a.split, b);
            double Ub[3] = {0.0, 0.0, 0.0}, Eb[3] = {0.0, 0.0, 0.0};
            double D[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
            for (int kk = 0; kk + 1 < nb; ++kk) {
                const double sa = b[kk], len = b[kk + 1] - b[kk];
                if (len <= 0.0) continue;
                for (int iq = 0; iq < a.nq; ++iq) {
                    const double s = sa + len * qs[iq];
                    const double wq = len * qw[iq];
                    const double th = th0 + s * (th1 - th0);
                    Stencil<ORDER> sx, sy;
                    stencil_xy<ORDER>(g, wrap1(x0 + s * dxx, g.Lx), wrap1(y0 + s * dxy, g.Ly), sx, sy);
                    for (int ia = 0; ia < S; ++ia) {
                        const int gx = wrap_index(sx.il + ia, a.nx);
                        for (int ib = 0; ib < S; ++ib) {
                            const double* r = a.rec + (size_t)(gx * a.ny + wrap_index(sy.il + ib, a.ny)) * kSdRec;
                            const double shape = sx.w[ia] * sy.w[ib];
                            const double dsx = sx.dw[ia] * sy.w[ib], dsy = sx.w[ia] * sy.dw[ib];
                            for (int c = 0; c < 3; ++c) {
                                Ub[c] += wq * r[6 + c] * shape;
                                Eb[c] += wq * r[9 + c] * shape;
                                const double av = (1.0 - th) * r[c] + th * r[3 + c];
                                D[c][0] += wq * av * dsx;
                                D[c][1] += wq * av * dsy;
                            }
                        }
                    }
                }
            }
            double Rv[3], Ad[3], rhs[3];
            for (int c = 0; c < 3; ++c) {
                Ad[c] = A1p[c] - A0p[c];
                rhs[c] = h * (Ub[c] + (D[c][0] * vb[0] + D[c][1] * vb[1]));
                Rv[c] = Ad[c] - rhs[c];
            }
            r2 = dd_add(r2, wgt * dot3(Rv, Rv));
            a2 = dd_add(a2, wgt * dot3(Ad, Ad));
            rhs2 = dd_add(rhs2, wgt * dot3(rhs, rhs));
            const double nr = norm3(Rv);
            nmax = fmax(nmax, nr);
            nsum = dd_add(nsum, wgt * nr);
            wdef = dd_add(wdef, -q * dot3(vb, Rv));
            pw = dd_add(pw, (h * q) * dot3(vb, Eb));
            const int nseg = nb - 1 > 1 ? nb - 1 : 1;
            psegs += nseg;
            cross += (unsigned long long)(nseg - 1);
            crossed = crossed || nseg > 1;
        }
        segs += (unsigned long long)psegs;
        cpart += crossed ? 1ull : 0ull;
        maxseg = max(maxseg, psegs);
    }
    sd_block_finish(DDSix{r2, a2, rhs2, nsum, wdef, pw}, nmax, segs, cross, cpart, maxseg, a.counts,
                    a.partials + (size_t)blockIdx.x * kSdPart);
}

// One warp per quantity: out[0..11] the six double-double sums, out[12] max.
__global__ void step_diag_final_kernel(const double* partials, int grid, double* out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k < 6) {
        DD t{0, 0};
        for (int b = lane; b < grid; b += 32)
            t = dd_add_dd(t, DD{partials[(size_t)b * kSdPart + 2 * k], partials[(size_t)b * kSdPart + 2 * k + 1]});
        t = warp_sum_dd(t);
        if (lane == 0) {
            out[2 * k] = t.hi;
            out[2 * k + 1] = t.lo;
        }
    } else if (k == 6) {
        double mx = 0.0;
        for (int b = lane; b < grid; b += 32) mx = fmax(mx, partials[(size_t)b * kSdPart + 12]);
        mx = warp_max(mx);
        if (lane == 0) out[12] = mx;
    }
}

// sum_m sum_id J_m(id) E_mid,m(id) in double-double (exact products).
__global__ void __launch_bounds__(kRed) grid_work_kernel(int N, const double* J, const double* rec, double* partials) {
    DD s{0, 0};
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            const double a = J[(size_t)c * N + id], b = rec[(size_t)id * kSdRec + 9 + c];
            const double pr = a * b;
            s = dd_add_dd(s, DD{pr, fma(a, b, -pr)});
        }
    }
    s = warp_sum_dd(s);
    __shared__ double red[kRed / kWarp][2];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w][0] = s.hi;
        red[w][1] = s.lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD t{0, 0};
        for (int q = 0; q < kRed / kWarp; ++q) t = dd_add_dd(t, DD{red[q][0], red[q][1]});
        partials[2 * blockIdx.x] = t.hi;
        partials[2 * blockIdx.x + 1] = t.lo;
    }
}

// ---- non-relativistic Picard push (evaluate_picard_map_orbit,
// Project1/ec_pic_serial_demo.cpp:1455-1506) ---------------------------------
// Per particle: vbar = (v_guess + v^n)/2, x_end = wrap(x + dt vbar), orbit
// averages of grad phi_mid and D_A (A time-interpolated), A^{n+1} at x_end,
// P_end = P + dt (-q <grad phi> + q D_A^T vbar), v_next = (P_end - q A)/m.
// Writes the trial state (sorted order) and per-CTA double-double partials of
// |v_next - v_guess|^2, |v_next|^2, |v_guess|^2 in the residual-norm layout.
template <int ORDER, bool UNIFORM, bool MOM>
__global__ void __launch_bounds__(kRed) picard_push_kernel(PicardPushArgs a) {
    Geo g{a.nx, a.ny, a.Lx, a.Ly, a.inv_dx, a.inv_dy};
    g.qs = a.qtab;
    g.qw = a.qtab + kMaxQuad;
    g.ms = a.qtab + 2 * kMaxQuad;
    g.mw = a.qtab + 3 * kMaxQuad;
    g.nq = a.nq;
    g.mnq = a.mnq;
    DD d2{0, 0}, n2{0, 0}, g2{0, 0};
    int nfail = 0;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < a.np; p += (long)gridDim.x * blockDim.x) {
        const double x0 = a.x[p], y0 = a.y[p];
        const double vg[3] = {a.gx[p], a.gy[p], a.gz[p]};
        const double vb[3] = {0.5 * (vg[0] + a.vx[p]), 0.5 * (vg[1] + a.vy[p]), 0.5 * (vg[2] + a.vz[p])};
        const double q = UNIFORM ? a.q0 : a.q[p];
        const double m = UNIFORM ? a.m0 : a.m[p];
        const double dxx = a.dt * vb[0], dxy = a.dt * vb[1];
        const double x1 = wrap1(x0 + dxx, g.Lx), y1 = wrap1(y0 + dxy, g.Ly);
        double b[kMaxBreaks];
        const int nb = breakpoints<ORDER>(g, x0, y0, dxx, dxy, a.split, b);
        double gp[2] = {0.0, 0.0}, D[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        if (nb < 0) {
            ++nfail;
        } else if constexpr (MOM) {
            orbit_integrals_moments<ORDER>(g, a.rec, x0, y0, dxx, dxy, b, nb, gp, D);
        } else {
            orbit_integrals_points<ORDER>(g, a.rec, x0, y0, dxx, dxy, b, nb, gp, D);
        }
        double A1p[3];
        gather_rec3<ORDER>(g, a.rec, kIRecAe, x1, y1, A1p);
        // D_A^T vbar (the z derivatives vanish in 2D)
        const double DATv[3] = {D[0][0] * vb[0] + D[1][0] * vb[1] + D[2][0] * vb[2],
                                D[0][1] * vb[0] + D[1][1] * vb[1] + D[2][1] * vb[2], 0.0};
        const double gpb[3] = {gp[0], gp[1], 0.0};
        const double P0[3] = {a.Px[p], a.Py[p], a.Pz[p]};
        double Pe[3], vn[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double f = (-q) * gpb[c] + q * DATv[c];
            Pe[c] = P0[c] + a.dt * f;
            vn[c] = (Pe[c] - q * A1p[c]) / m;
            const double dv = vn[c] - vg[c];
            d2 = dd_add_dd(d2, dd_sq(dv));
            n2 = dd_add_dd(n2, dd_sq(vn[c]));
            g2 = dd_add_dd(g2, dd_sq(vg[c]));
        }
        a.ox[p] = x1;
        a.oy[p] = y1;
        a.oPx[p] = Pe[0];
        a.oPy[p] = Pe[1];
        a.oPz[p] = Pe[2];
        a.ovx[p] = vn[0];
        a.ovy[p] = vn[1];
        a.ovz[p] = vn[2];
    }
    if (nfail) atomicAdd(a.err, nfail);
    d2 = warp_sum_dd(d2);
    n2 = warp_sum_dd(n2);
    g2 = warp_sum_dd(g2);
    __shared__ double red[kRed / kWarp][6];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w][0] = d2.hi; red[w][1] = d2.lo; red[w][2] = n2.hi; red[w][3] = n2.lo;
        red[w][4] = g2.hi; red[w][5] = g2.lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD A{0, 0}, B{0, 0}, C{0, 0};
        for (int k = 0; k < kRed / kWarp; ++k) {
            A = dd_add_dd(A, DD{red[k][0], red[k][1]});
            B = dd_add_dd(B, DD{red[k][2], red[k][3]});
            C = dd_add_dd(C, DD{red[k][4], red[k][5]});
        }
        double* o = a.partials + (size_t)blockIdx.x * 8;
        o[0] = A.hi; o[1] = A.lo; o[2] = B.hi; o[3] = B.lo; o[4] = C.hi; o[5] = C.lo; o[6] = 0.0; o[7] = 0.0;
    }
}

// v_prev = v - dt (q/m) E(x) and P = m v: the Taylor start-up of
// Project1's initializers (ec_pic_serial_demo.cpp:1200-1210).
template <int ORDER>
__global__ void picard_startup_kernel(int nx, int ny, double Lx, double Ly, const double* E3, long np,
                                      const double* x, const double* y, const double* vx, const double* vy,
                                      const double* vz, const double* qa, double q0, const double* ma, double m0,
                                      double dt, double* Px, double* Py, double* Pz, double* wx, double* wy,
                                      double* wz) {
    const Geo g{nx, ny, Lx, Ly, nx / Lx, ny / Ly};
    const int N = nx * ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        Stencil<ORDER> sx, sy;
        stencil_xy<ORDER>(g, x[p], y[p], sx, sy);
        double E[3] = {0.0, 0.0, 0.0};
        for (int ia = 0; ia <= ORDER; ++ia) {
            const int gx = wrap_index(sx.il + ia, nx);
            for (int ib = 0; ib <= ORDER; ++ib) {
                const int node = gx * ny + wrap_index(sy.il + ib, ny);
                const double w = sx.w[ia] * sy.w[ib];
                for (int c = 0; c < 3; ++c) E[c] = fma(E3[(size_t)c * N + node], w, E[c]);
            }
        }
        const double q = qa ? qa[p] : q0, m = ma ? ma[p] : m0;
        const double v[3] = {vx[p], vy[p], vz[p]};
        const double qm = q / m;
        Px[p] = m * v[0];
        Py[p] = m * v[1];
        Pz[p] = m * v[2];
        wx[p] = v[0] - dt * (qm * E[0]);
        wy[p] = v[1] - dt * (qm * E[1]);
        wz[p] = v[2] - dt * (qm * E[2]);
    }
}

// Knot-crossing statistics of the orbits x + dt vbar (compute_path_stats,
// ec_pic_serial_demo.cpp:835; PathStats of Project3): vbar from (bx, by)
// or, with vbar null arrays, (v1 + v0) / 2.  counts: total segments,
// crossings, crossing particles, max segments.
template <int ORDER>
__global__ void path_stats_kernel(PathStatsArgs a) {
    const Geo g{a.nx, a.ny, a.Lx, a.Ly, a.nx / a.Lx, a.ny / a.Ly};
    unsigned long long segs = 0, cross = 0, cpart = 0;
    int maxseg = 1;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < a.np; p += (long)gridDim.x * blockDim.x) {
        double vbx, vby;
        if (a.bx) {
            vbx = a.bx[p];
            vby = a.by[p];
        } else {
            vbx = 0.5 * (a.v1x[p] + a.v0x[p]);
            vby = 0.5 * (a.v1y[p] + a.v0y[p]);
        }
        double b[kMaxBreaks];
        const int nb = breakpoints<ORDER>(g, a.x[p], a.y[p], a.dt * vbx, a.dt * vby, a.split, b);
        const int nseg = nb - 1 > 1 ? nb - 1 : 1;
        segs += (unsigned long long)nseg;
        cross += (unsigned long long)(nseg - 1);
        cpart += nseg > 1 ? 1ull : 0ull;
        maxseg = max(maxseg, nseg);
    }
    for (int o = 16; o > 0; o >>= 1) {
        segs += __shfl_xor_sync(0xffffffffu, segs, o);
        cross += __shfl_xor_sync(0xffffffffu, cross, o);
        cpart += __shfl_xor_sync(0xffffffffu, cpart, o);
        maxseg = max(maxseg, __shfl_xor_sync(0xffffffffu, maxseg, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&a.counts[0], segs);
        atomicAdd(&a.counts[1], cross);
        atomicAdd(&a.counts[2], cpart);
        atomicMax(&a.counts[3], (unsigned long long)maxseg);
    }
}

// ---- diagnostics ----------------------------------------------------------------
constexpr int kDiagSums = 9;

__global__ void __launch_bounds__(kRed) implicit_diag_kernel(ImplicitDiagArgs a) {
    const int N = a.N;
    DD s[kDiagSums];
    for (int k = 0; k < kDiagSums; ++k) s[k] = DD{0, 0};
    double gmax = 0.0, gamax = 0.0;
    const double ik2 = 1.0 / (a.kappa * a.kappa);
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double gauss = a.divE[id] - a.sigma1 * a.rho[id];
        const double gauge = a.psi[id] * ik2 + a.divA[id];
        gmax = fmax(gmax, fabs(gauss));
        gamax = fmax(gamax, fabs(gauge));
        s[0] = dd_add_dd(s[0], dd_sq(gauss));
        s[1] = dd_add_dd(s[1], dd_sq(a.divE[id]));
        s[2] = dd_add_dd(s[2], dd_sq(a.rho[id]));
        s[3] = dd_add_dd(s[3], dd_sq(gauge));
        s[4] = dd_add_dd(s[4], dd_sq(a.psi[id]));
        s[5] = dd_add_dd(s[5], dd_sq(a.divA[id]));
        for (int c = 0; c < 3; ++c) {
            s[6] = dd_add_dd(s[6], dd_sq(a.E[(size_t)c * N + id]));
            s[7] = dd_add_dd(s[7], dd_sq(a.B[(size_t)c * N + id]));
        }
        s[8] = dd_add(s[8], a.rho[id]);
    }
    __shared__ double red[kRed / kWarp][2 * kDiagSums + 2];
    const int w = threadIdx.x >> 5;
    for (int k = 0; k < kDiagSums; ++k) {
        s[k] = warp_sum_dd(s[k]);
        if ((threadIdx.x & 31) == 0) {
            red[w][2 * k] = s[k].hi;
            red[w][2 * k + 1] = s[k].lo;
        }
    }
    gmax = warp_max(gmax);
    gamax = warp_max(gamax);
    if ((threadIdx.x & 31) == 0) {
        red[w][2 * kDiagSums] = gmax;
        red[w][2 * kDiagSums + 1] = gamax;
    }
    __syncthreads();
    if (threadIdx.x < kDiagSums + 2) {
        const int k = threadIdx.x;
        double* o = a.partials + (size_t)blockIdx.x * 32;
        if (k < kDiagSums) {
            DD t{0, 0};
            for (int q = 0; q < kRed / kWarp; ++q) t = dd_add_dd(t, DD{red[q][2 * k], red[q][2 * k + 1]});
            o[2 * k] = t.hi;
            o[2 * k + 1] = t.lo;
        } else {
            double mx = 0.0;
            for (int q = 0; q < kRed / kWarp; ++q) mx = fmax(mx, red[q][2 * kDiagSums + (k - kDiagSums)]);
            o[2 * kDiagSums + (k - kDiagSums)] = mx;
        }
    }
}

// One warp per quantity (blockDim = 32 * (kDiagSums + 2)), lanes over the
// partials.
__global__ void implicit_diag_final_kernel(const double* partials, int grid, double* out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k < kDiagSums) {
        DD t{0, 0};
        for (int b = lane; b < grid; b += 32)
            t = dd_add_dd(t, DD{partials[(size_t)b * 32 + 2 * k], partials[(size_t)b * 32 + 2 * k + 1]});
        t = warp_sum_dd(t);
        if (lane == 0) {
            out[2 * k] = t.hi;
            out[2 * k + 1] = t.lo;
        }
    } else if (k < kDiagSums + 2) {
        double mx = 0.0;
        for (int b = lane; b < grid; b += 32) mx = fmax(mx, partials[(size_t)b * 32 + 2 * kDiagSums + (k - kDiagSums)]);
        mx = warp_max(mx);
        if (lane == 0) out[2 * kDiagSums + (k - kDiagSums)] = mx;
    }
}

// Relativistic m kappa^2 (gamma - 1) (compute_kinetic_energy, Project3 :3457)
// or, with nonrel, m v^2 / 2 (Project1 :1031).
__global__ void __launch_bounds__(kRed)
kinetic_kernel(long np, const double* vx, const double* vy, const double* vz, const double* m, double m0,
               double kappa, double* partials, int nonrel) {
    DD s{0, 0};
    const double k2 = kappa * kappa;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        const double v[3] = {vx[p], vy[p], vz[p]};
        const double mm = m ? m[p] : m0;
        if (nonrel) {
            s = dd_add(s, 0.5 * mm * dot3(v, v));
        } else {
            const double beta2 = dot3(v, v) / k2;
            const double gam = 1.0 / sqrt(fmax(1.0e-300, 1.0 - beta2));
            s = dd_add(s, mm * kappa * kappa * (gam - 1.0));
        }
    }
    s = warp_sum_dd(s);
    __shared__ double red[kRed / kWarp][2];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w][0] = s.hi;
        red[w][1] = s.lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD t{0, 0};
        for (int q = 0; q < kRed / kWarp; ++q) t = dd_add_dd(t, DD{red[q][0], red[q][1]});
        partials[2 * blockIdx.x] = t.hi;
        partials[2 * blockIdx.x + 1] = t.lo;
    }
}

__global__ void pair_final_kernel(const double* partials, int grid, double* out) {
    DD t{0, 0};
    for (int b = threadIdx.x; b < grid; b += 32) t = dd_add_dd(t, DD{partials[2 * b], partials[2 * b + 1]});
    t = warp_sum_dd(t);
    if (threadIdx.x != 0) return;
    out[0] = t.hi;
    out[1] = t.lo;
}

int gsize(long n, int threads = 256) {
    long g = (n + threads - 1) / threads;
    if (g > 148 * 8) g = 148 * 8;
    return g < 1 ? 1 : (int)g;
}

using MapKernel = void (*)(ImplicitMapArgs, TileGeom);

// The map kernel instance of (order, uniform q/m, knot splitting, Picard
// deposit, part).
template <bool PICARD, int PART>
MapKernel map_kernel_of(int order, bool uniform, bool split) {
    const bool mom = split && order <= 2;
#define UPIC_K(O, U, M) &implicit_map_kernel<O, U, M, PICARD, PART>
    switch (order) {
        case 1:
            return mom ? (uniform ? UPIC_K(1, true, true) : UPIC_K(1, false, true))
                       : (uniform ? UPIC_K(1, true, false) : UPIC_K(1, false, false));
        case 2:
            return mom ? (uniform ? UPIC_K(2, true, true) : UPIC_K(2, false, true))
                       : (uniform ? UPIC_K(2, true, false) : UPIC_K(2, false, false));
        case 3: return uniform ? UPIC_K(3, true, false) : UPIC_K(3, false, false);
        case 4: return uniform ? UPIC_K(4, true, false) : UPIC_K(4, false, false);
    }
#undef UPIC_K
    return nullptr;
}

// The one-row (ny = 1) instances of the split launches: segment moments for
// every order (knot splitting on; one y node leaves (ORDER + 1) moments per
// segment).
template <int PART>
MapKernel map_kernel_oned(int order, bool uniform) {
#define UPIC_K1(O) (uniform ? &implicit_map_kernel<O, true, true, false, PART, true> \
                            : &implicit_map_kernel<O, false, true, false, PART, true>)
    switch (order) {
        case 1: return UPIC_K1(1);
        case 2: return UPIC_K1(2);
        case 3: return UPIC_K1(3);
        case 4: return UPIC_K1(4);
    }
#undef UPIC_K1
    return nullptr;
}

// oned: the grid is one cell high; its split launches (relativistic map,
// knot splitting on) use the one-row instances.
MapKernel map_kernel(int order, bool uniform, bool split, bool picard, int part = kPartFused, bool oned = false) {
    if (picard) return map_kernel_of<true, kPartFused>(order, uniform, split);
    if (oned && split && part == kPartSolve) return map_kernel_oned<kPartSolve>(order, uniform);
    if (oned && split && part == kPartDeposit) return map_kernel_oned<kPartDeposit>(order, uniform);
    switch (part) {
        case kPartSolve: return map_kernel_of<false, kPartSolve>(order, uniform, split);
        case kPartDeposit: return map_kernel_of<false, kPartDeposit>(order, uniform, split);
        default: return map_kernel_of<false, kPartFused>(order, uniform, split);
    }
}

// Split launches for the relativistic map when the caller supplied the
// hand-over buffers.
bool use_split(const ImplicitMapArgs& a, bool picard) {
    return UPIC_MAP_SPLIT && !picard && a.vbar_x && a.vbar_y && a.vbar_z;
}

}  // namespace

int implicit_map_smem_bytes(const TileGeom& tg, int order) {
    const int S = order + 1;
    const int RW = S * S + 3;
    return 2 * 3 * tg.wx * tg.wy * 8 + kMapWarps * (32 * RW * 8 + 32 * 4) + 4 * kMaxQuad * 8;
}

cudaError_t implicit_configure_smem(const TileGeom& tg, int order, bool split, bool picard) {
    const int b = implicit_map_smem_bytes(tg, order);
    for (int u = 0; u < 2; ++u) {
        for (int part = kPartFused; part <= (picard ? kPartFused : kPartDeposit); ++part) {
            MapKernel k = map_kernel(order, u != 0, split, picard, part, tg.ny == 1);
            if (!k) return cudaErrorInvalidValue;
            const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), b);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

int implicit_map_occupancy(const TileGeom& tg, int order, bool split, bool picard) {
    int n = 0;
    MapKernel k = map_kernel(order, true, split, picard);
    if (!k) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kMapThreads, implicit_map_smem_bytes(tg, order));
    return n;
}

cudaError_t launch_implicit_map(int order, bool uniform, bool split, const TileGeom& tg,
                                const ImplicitMapArgs& a, int grid, cudaStream_t st, bool picard) {
    const int smem = implicit_map_smem_bytes(tg, order);
    if (use_split(a, picard)) {
        MapKernel ks = map_kernel(order, uniform, split, picard, kPartSolve, tg.ny == 1);
        MapKernel kd = map_kernel(order, uniform, split, picard, kPartDeposit, tg.ny == 1);
        if (!ks || !kd) return cudaErrorInvalidValue;
        // grid is sized for the fused kernel's resident CTAs; each part is
        // given as many CTAs as it keeps resident
        const bool mom = (tg.ny == 1 && split) || (split && order <= 2);
        const int gs = grid / kMapMinBlocks * map_min_blocks(kPartSolve, mom);
        const int gd = grid / kMapMinBlocks * map_min_blocks(kPartDeposit, mom);
        ks<<<gs > 0 ? gs : grid, kMapThreads, smem, st>>>(a, tg);
        kd<<<gd > 0 ? gd : grid, kMapThreads, smem, st>>>(a, tg);
        count_launches(2);
        return cudaGetLastError();
    }
    MapKernel k = map_kernel(order, uniform, split, picard);
    if (!k) return cudaErrorInvalidValue;
    k<<<grid, kMapThreads, smem, st>>>(a, tg);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_refined_map(int order, bool uniform, const ImplicitMapArgs& a, cudaStream_t st) {
    if (a.nref <= 0) return cudaSuccess;
    const int g = (a.nref + 127) / 128;
    const int nx = a.grid_nx, ny = a.grid_ny;
#define UPIC_RM(O) \
    if (uniform) refined_map_kernel<O, true><<<g, 128, 0, st>>>(a, nx, ny); \
    else refined_map_kernel<O, false><<<g, 128, 0, st>>>(a, nx, ny);
    switch (order) {
        case 1: UPIC_RM(1) break;
        case 2: UPIC_RM(2) break;
        case 3: UPIC_RM(3) break;
        case 4: UPIC_RM(4) break;
        default: return cudaErrorInvalidValue;
    }
#undef UPIC_RM
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_failure_report(int order, bool uniform, bool split, const TileGeom& tg, const ImplicitMapArgs& a,
                                  const int* failed, int nf, double* out, cudaStream_t st) {
    if (nf <= 0) return cudaSuccess;
    const int g = (nf + 127) / 128;
    // the evaluation form of the map launch (map_kernel): one-row instances for
    // split launches on a grid one cell high, segment moments for split
    // orbits of order <= 2
    const bool oned = tg.ny == 1 && split && use_split(a, false);
    const bool mom = oned || (split && order <= 2);
#define UPIC_FR(O, U, M, SY) failure_report_kernel<O, U, M, SY><<<g, 128, 0, st>>>(a, tg.nx, tg.ny, failed, nf, out)
#define UPIC_FR_ORDER(O)                                                    \
    if (oned) {                                                             \
        if (uniform) UPIC_FR(O, true, true, 1); else UPIC_FR(O, false, true, 1); \
    } else if (mom && O <= 2) {                                             \
        if (uniform) UPIC_FR(O, true, (O <= 2), O + 1); else UPIC_FR(O, false, (O <= 2), O + 1); \
    } else {                                                                \
        if (uniform) UPIC_FR(O, true, false, O + 1); else UPIC_FR(O, false, false, O + 1); \
    }
    switch (order) {
        case 1: UPIC_FR_ORDER(1) break;
        case 2: UPIC_FR_ORDER(2) break;
        case 3: UPIC_FR_ORDER(3) break;
        case 4: UPIC_FR_ORDER(4) break;
        default: return cudaErrorInvalidValue;
    }
#undef UPIC_FR_ORDER
#undef UPIC_FR
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fill_int(int n, int value, int* out, cudaStream_t st) {
    fill_int_kernel<<<gsize(n), 256, 0, st>>>(n, value, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_orbit_deposit(int order, const OrbitArgs& a, cudaStream_t st) {
    const int g = gsize(a.np);
    switch (order) {
        case 1: orbit_deposit_kernel<1><<<g, 128, 0, st>>>(a); break;
        case 2: orbit_deposit_kernel<2><<<g, 128, 0, st>>>(a); break;
        case 3: orbit_deposit_kernel<3><<<g, 128, 0, st>>>(a); break;
        case 4: orbit_deposit_kernel<4><<<g, 128, 0, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_orbit_gather(int order, const OrbitArgs& a, cudaStream_t st) {
    const int g = gsize(a.np);
    switch (order) {
        case 1: orbit_gather_kernel<1><<<g, 128, 0, st>>>(a); break;
        case 2: orbit_gather_kernel<2><<<g, 128, 0, st>>>(a); break;
        case 3: orbit_gather_kernel<3><<<g, 128, 0, st>>>(a); break;
        case 4: orbit_gather_kernel<4><<<g, 128, 0, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_step_diag_spectra(int N, const double* kx, const double* ky, const double2* s0,
                                     const double2* s1, double2* out12, cudaStream_t st) {
    step_diag_spectra_kernel<<<gsize(N), 256, 0, st>>>(N, kx, ky, s0, s1, out12);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_step_diag(int order, const StepDiagArgs& a, int grid, double* out13, cudaStream_t st) {
    switch (order) {
        case 1: step_diag_kernel<1><<<grid, kRed, 0, st>>>(a); break;
        case 2: step_diag_kernel<2><<<grid, kRed, 0, st>>>(a); break;
        case 3: step_diag_kernel<3><<<grid, kRed, 0, st>>>(a); break;
        case 4: step_diag_kernel<4><<<grid, kRed, 0, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    int g2 = 0;
    if (a.nref > 0) {
        // refined particles: their block partials follow the main kernel's
        g2 = std::min((a.nref + kRed - 1) / kRed, a.refined_grid_max);
        StepDiagArgs b = a;
        b.partials = a.partials + (size_t)grid * kSdPart;
        switch (order) {
            case 1: step_diag_refined_kernel<1><<<g2, kRed, 0, st>>>(b); break;
            case 2: step_diag_refined_kernel<2><<<g2, kRed, 0, st>>>(b); break;
            case 3: step_diag_refined_kernel<3><<<g2, kRed, 0, st>>>(b); break;
            case 4: step_diag_refined_kernel<4><<<g2, kRed, 0, st>>>(b); break;
            default: return cudaErrorInvalidValue;
        }
        count_launches(1);
    }
    step_diag_final_kernel<<<1, 32 * 7, 0, st>>>(a.partials, grid + g2, out13);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_grid_work(int N, const double* J, const double* rec12, double* partials, int grid, double* out2,
                             cudaStream_t st) {
    grid_work_kernel<<<grid, kRed, 0, st>>>(N, J, rec12, partials);
    pair_final_kernel<<<1, 32, 0, st>>>(partials, grid, out2);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_picard_push(int order, bool uniform, bool split, const PicardPushArgs& a, int grid,
                              NormSums* out, cudaStream_t st) {
    const bool mom = split && order <= 2;
#define UPIC_PP(O, U, M) picard_push_kernel<O, U, M><<<grid, kRed, 0, st>>>(a)
    switch (order) {
        case 1:
            if (mom) { if (uniform) UPIC_PP(1, true, true); else UPIC_PP(1, false, true); }
            else { if (uniform) UPIC_PP(1, true, false); else UPIC_PP(1, false, false); }
            break;
        case 2:
            if (mom) { if (uniform) UPIC_PP(2, true, true); else UPIC_PP(2, false, true); }
            else { if (uniform) UPIC_PP(2, true, false); else UPIC_PP(2, false, false); }
            break;
        case 3: if (uniform) UPIC_PP(3, true, false); else UPIC_PP(3, false, false); break;
        case 4: if (uniform) UPIC_PP(4, true, false); else UPIC_PP(4, false, false); break;
        default: return cudaErrorInvalidValue;
    }
#undef UPIC_PP
    residual_final_kernel<<<1, 32, 0, st>>>(a.partials, grid, out);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_picard_startup(int order, int nx, int ny, double Lx, double Ly, const double* E3, long np,
                                  const double* x, const double* y, const double* vx, const double* vy,
                                  const double* vz, const double* q, double q0, const double* m, double m0,
                                  double dt, double* Px, double* Py, double* Pz, double* wx, double* wy, double* wz,
                                  cudaStream_t st) {
    const int g = gsize(np);
#define UPIC_PS(O) picard_startup_kernel<O><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, E3, np, x, y, vx, vy, vz, q, q0, m, \
                                                               m0, dt, Px, Py, Pz, wx, wy, wz)
    switch (order) {
        case 1: UPIC_PS(1); break;
        case 2: UPIC_PS(2); break;
        case 3: UPIC_PS(3); break;
        case 4: UPIC_PS(4); break;
        default: return cudaErrorInvalidValue;
    }
#undef UPIC_PS
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_path_stats(int order, const PathStatsArgs& a, cudaStream_t st) {
    const int g = gsize(a.np);
    switch (order) {
        case 1: path_stats_kernel<1><<<g, 256, 0, st>>>(a); break;
        case 2: path_stats_kernel<2><<<g, 256, 0, st>>>(a); break;
        case 3: path_stats_kernel<3><<<g, 256, 0, st>>>(a); break;
        case 4: path_stats_kernel<4><<<g, 256, 0, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_point_deposit(int order, const PointDepositArgs& a, cudaStream_t st) {
    const int g = gsize(a.np);
    switch (order) {
        case 1: point_deposit_kernel<1><<<g, 256, 0, st>>>(a); break;
        case 2: point_deposit_kernel<2><<<g, 256, 0, st>>>(a); break;
        case 3: point_deposit_kernel<3><<<g, 256, 0, st>>>(a); break;
        case 4: point_deposit_kernel<4><<<g, 256, 0, st>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_add_qA(int order, int nx, int ny, double Lx, double Ly, const double* A3, long np,
                          const double* x, const double* y, const double* q, double q0, double* Px, double* Py,
                          double* Pz, cudaStream_t st) {
    const int g = gsize(np);
    switch (order) {
        case 1: add_qA_kernel<1><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, A3, np, x, y, q, q0, Px, Py, Pz); break;
        case 2: add_qA_kernel<2><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, A3, np, x, y, q, q0, Px, Py, Pz); break;
        case 3: add_qA_kernel<3><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, A3, np, x, y, q, q0, Px, Py, Pz); break;
        case 4: add_qA_kernel<4><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, A3, np, x, y, q, q0, Px, Py, Pz); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gather3(int order, int nx, int ny, double Lx, double Ly, const double* f3, long np,
                           const double* x, const double* y, double* out3, cudaStream_t st) {
    const int g = gsize(np);
    switch (order) {
        case 1: gather3_kernel<1><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, f3, np, x, y, out3); break;
        case 2: gather3_kernel<2><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, f3, np, x, y, out3); break;
        case 3: gather3_kernel<3><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, f3, np, x, y, out3); break;
        case 4: gather3_kernel<4><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, f3, np, x, y, out3); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gmhc_push(int order, const ImplicitMapArgs& a, int nx, int ny, long np, const double* in7,
                             const double* guess3, double* out, int* rep, cudaStream_t st) {
    const int gr = gsize(np, 128);
    const bool mom = a.split && order <= 2;
    switch (order) {
        case 1:
            if (mom) gmhc_push_kernel<1, true><<<gr, 128, 0, st>>>(a, nx, ny, np, in7, guess3, out, rep);
            else gmhc_push_kernel<1, false><<<gr, 128, 0, st>>>(a, nx, ny, np, in7, guess3, out, rep);
            break;
        case 2:
            if (mom) gmhc_push_kernel<2, true><<<gr, 128, 0, st>>>(a, nx, ny, np, in7, guess3, out, rep);
            else gmhc_push_kernel<2, false><<<gr, 128, 0, st>>>(a, nx, ny, np, in7, guess3, out, rep);
            break;
        case 3: gmhc_push_kernel<3, false><<<gr, 128, 0, st>>>(a, nx, ny, np, in7, guess3, out, rep); break;
        case 4: gmhc_push_kernel<4, false><<<gr, 128, 0, st>>>(a, nx, ny, np, in7, guess3, out, rep); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_probe(int order, int nx, int ny, double Lx, double Ly, const double* F18, long np,
                         const double* x, const double* y, double* out30, cudaStream_t st) {
    const int g = gsize(np, 128);
    switch (order) {
        case 1: probe_kernel<1><<<g, 128, 0, st>>>(nx, ny, Lx, Ly, F18, np, x, y, out30); break;
        case 2: probe_kernel<2><<<g, 128, 0, st>>>(nx, ny, Lx, Ly, F18, np, x, y, out30); break;
        case 3: probe_kernel<3><<<g, 128, 0, st>>>(nx, ny, Lx, Ly, F18, np, x, y, out30); break;
        case 4: probe_kernel<4><<<g, 128, 0, st>>>(nx, ny, Lx, Ly, F18, np, x, y, out30); break;
        default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_history_velocity(int order, int nx, int ny, double Lx, double Ly, const double* E3,
                                    const double* B3, long np, const double* x, const double* y,
                                    const double* vx, const double* vy, const double* vz,
                                    const double* q, double q0, const double* m, double m0, double kappa,
                                    double dt, double* wx, double* wy, double* wz, cudaStream_t st) {
    const int g = gsize(np);
#define UPIC_HV(O)                                                                                        \
    history_velocity_kernel<O><<<g, 256, 0, st>>>(nx, ny, Lx, Ly, E3, B3, np, x, y, vx, vy, vz, q, q0, m, m0, \
                                                  kappa, dt, wx, wy, wz)
    switch (order) {
        case 1: UPIC_HV(1); break;
        case 2: UPIC_HV(2); break;
        case 3: UPIC_HV(3); break;
        case 4: UPIC_HV(4); break;
        default: return cudaErrorInvalidValue;
    }
#undef UPIC_HV
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_cn_kspace(const CnArgs& a, cudaStream_t st) {
    cn_kspace_kernel<<<gsize(a.N), 256, 0, st>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_diag_spectra(int N, const double* kx, const double* ky, const double2* st_spec, double2* out,
                                cudaStream_t st) {
    diag_spectra_kernel<<<gsize(N), 256, 0, st>>>(N, kx, ky, st_spec, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_momentum_from_v(long np, const double* vx, const double* vy, const double* vz, const double* m,
                                   double m0, double kappa, double* Px, double* Py, double* Pz, cudaStream_t st) {
    momentum_from_v_kernel<<<gsize(np), 256, 0, st>>>(np, vx, vy, vz, m, m0, kappa, Px, Py, Pz);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_project_nyquist(double* f, int ncomp, int nx, int ny, cudaStream_t st) {
    if (nx > 1 && nx % 2 == 0) {
        project_lines_kernel<<<gsize((long)ncomp * ny, 8), 256, 0, st>>>(f, ncomp, nx, ny, 0);
        count_launches(1);
    }
    if (ny > 1 && ny % 2 == 0) {
        project_lines_kernel<<<gsize((long)ncomp * nx, 8), 256, 0, st>>>(f, ncomp, nx, ny, 1);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_kspace_mask(double2* f, int ncomp, int N, const unsigned char* excl, int zero_mean,
                               cudaStream_t st) {
    kspace_mask_kernel<<<gsize((long)ncomp * N), 256, 0, st>>>(f, ncomp, N, excl, zero_mean);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_residual_norms(int N, const double* map, const double* guess, double floor_rel, double atol,
                                  double rtol, double* partials, int grid, NormSums* out, cudaStream_t st) {
    residual_norms_kernel<<<grid, kRed, 0, st>>>(N, map, guess, floor_rel, atol, rtol, partials);
    residual_final_kernel<<<1, 32, 0, st>>>(partials, grid, out);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_anderson_dots(int n, const double* const* r, int m, double* partials, int grid, double* out,
                                 cudaStream_t st) {
    if (m < 1 || m > 4) return cudaErrorInvalidValue;
    RPtrs rp{};
    for (int k = 0; k <= m; ++k) rp.r[k] = r[k];
    anderson_dots_kernel<<<grid, kRed, 0, st>>>(n, rp, m, partials);
    dots_final_kernel<<<1, 32 * (m * (m + 1) / 2 + m), 0, st>>>(partials, grid, m * (m + 1) / 2 + m, out);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_anderson_candidate(int n, const double* const* x, const double* const* r, int m, double beta,
                                      const double* gamma, double* out, cudaStream_t st) {
    if (m < 0 || m > 4) return cudaErrorInvalidValue;
    GPtrs g{};
    for (int k = 0; k <= m; ++k) {
        g.x[k] = x[k];
        g.r[k] = r[k];
    }
    for (int k = 0; k < m; ++k) g.gamma[k] = gamma[k];
    anderson_candidate_kernel<<<gsize(n), 256, 0, st>>>(n, g, m, beta, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_nonfinite_flag(int n, const double* v, int* flag, cudaStream_t st) {
    nonfinite_kernel<<<gsize(n), 256, 0, st>>>(n, v, flag);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_extrapolate(int n, const double* v, const double* w, double* out, cudaStream_t st) {
    extrapolate_kernel<<<gsize(n), 256, 0, st>>>(n, v, w, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_half_sum(int n, const double* a, const double* b, double* out, cudaStream_t st) {
    half_sum_kernel<<<gsize(n), 256, 0, st>>>(n, a, b, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_lerp(int n, const double* a, const double* b, double s, double* out, cudaStream_t st) {
    lerp_kernel<<<gsize(n), 256, 0, st>>>(n, a, b, s, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_axpy(int n, const double* a, const double* b, double s, double* out, cudaStream_t st) {
    axpy_kernel<<<gsize(n), 256, 0, st>>>(n, a, b, s, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_implicit_diag(const ImplicitDiagArgs& a, double* out20, cudaStream_t st) {
    implicit_diag_kernel<<<a.grid, kRed, 0, st>>>(a);
    implicit_diag_final_kernel<<<1, 32 * (kDiagSums + 2), 0, st>>>(a.partials, a.grid, out20);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_kinetic(long np, const double* vx, const double* vy, const double* vz, const double* m,
                           double m0, double kappa, double* partials, int grid, double* out, cudaStream_t st,
                           bool nonrel) {
    kinetic_kernel<<<grid, kRed, 0, st>>>(np, vx, vy, vz, m, m0, kappa, partials, nonrel ? 1 : 0);
    pair_final_kernel<<<1, 32, 0, st>>>(partials, grid, out);
    count_launches(2);
    return cudaGetLastError();
}

}  // namespace upic
