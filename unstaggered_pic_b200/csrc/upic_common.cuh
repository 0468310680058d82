// Shared device helpers for the unstaggered GM-PIC kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define UPIC_HD __host__ __device__ __forceinline__
#define UPIC_D __device__ __forceinline__

namespace upic {

constexpr int kWarp = 32;
constexpr double kPi = 3.141592653589793238462643383279502884;

// Gathered field record of the explicit step: A (3), grad phi (x,y),
// grad A component c direction d at 5 + 2c + d; padded to 12 doubles so a
// node is six 16-byte loads.
constexpr int kGF = 11;
constexpr int kGFStride = 12;

// ---------------------------------------------------------------------------
// Periodic wrap into [0, L): spectral_pic_part3.cpp:161-167.
UPIC_HD double wrap_periodic(double x, double L) {
    x -= floor(x / L) * L;
    if (x >= L) x -= L;
    if (x < 0.0) x += L;
    return x;
}

// Same result with a precomputed 1/L: floor(x*invL) can differ from
// floor(x/L) only when x is within an ulp of a multiple of L, and the two
// correction branches then produce the identical wrapped value.
UPIC_HD double wrap_periodic(double x, double L, double invL) {
    x -= floor(x * invL) * L;
    if (x >= L) x -= L;
    if (x < 0.0) x += L;
    return x;
}

// Quadratic B-spline weights centred on the nearest node:
// spectral_pic_part3.cpp:537-552.  ic is the nearest node (unwrapped).
struct Quad1D {
    int ic;
    double w0, w1, w2;
};

UPIC_HD Quad1D quadratic_weights(double x, double inv_dx) {
    const double s = x * inv_dx;
    const double fl = floor(s + 0.5);
    const double r = s - fl;
    Quad1D q;
    q.ic = (int)fl;
    const double a = 0.5 - r, b = 0.5 + r;
    q.w0 = 0.5 * a * a;
    q.w1 = 0.75 - r * r;
    q.w2 = 0.5 * b * b;
    return q;
}

// Periodic node index; n is a power of two (radix-2 grids), so the wrap is a
// mask (two's complement handles negative i).
UPIC_HD int wrap_index(int i, int n) { return i & (n - 1); }

// ---------------------------------------------------------------------------
// Deterministic fixed-point accumulation.
//
// A double v is represented as the integer N = round(v * 2^F), split into a
// signed high word H = floor(N / 2^32) and an unsigned low word L = N - H*2^32
// in [0, 2^32].  Sums of H and of L are exact integer sums, so the result is
// independent of the order of the additions (atomics included) and therefore
// reproducible bit for bit.  F is chosen per field from a bound B on any node
// value (|sum| <= B): F = 91 - ceil(log2 B), which keeps |sum H| < 2^60 and
// gives an absolute resolution of about B * 2^-91.
struct Fixed2 {
    unsigned long long hi;  // two's-complement signed high word
    unsigned long long lo;  // unsigned low word, < 2^32 + 1
};

UPIC_D Fixed2 to_fixed(double v, double scale) {
    const double s = v * scale;                    // exact power-of-two scaling
    const double hd = floor(s * 2.3283064365386963e-10);  // s / 2^32, exact scaling
    const double rem = fma(-hd, 4294967296.0, s);  // in [0, 2^32), exact
    Fixed2 f;
    f.hi = (unsigned long long)(long long)hd;
    f.lo = (unsigned long long)__double2ll_rn(rem);
    return f;
}

UPIC_HD double from_fixed(unsigned long long hi, unsigned long long lo, double inv_scale) {
    const double h = (double)(long long)hi;
    const double l = (double)lo;
    return fma(h, 4294967296.0 * inv_scale, l * inv_scale);
}

// ---------------------------------------------------------------------------
// Double-double (compensated) accumulation; stands in for the reference's
// long double accumulators (spectral_pic_part3.cpp:497-523, 950-959).
struct DD {
    double hi, lo;
};

UPIC_HD DD dd_add(DD a, double b) {
    const double s = a.hi + b;
    const double bb = s - a.hi;
    const double err = (a.hi - (s - bb)) + (b - bb);
    const double lo = a.lo + err;
    const double hi = s + lo;
    return DD{hi, lo - (hi - s)};
}

UPIC_HD DD dd_add_dd(DD a, DD b) {
    const double s = a.hi + b.hi;
    const double bb = s - a.hi;
    const double err = (a.hi - (s - bb)) + (b.hi - bb);
    const double lo = a.lo + b.lo + err;
    const double hi = s + lo;
    return DD{hi, lo - (hi - s)};
}

// Exact product a*a as a double-double.
UPIC_HD DD dd_sq(double a) {
    const double p = a * a;
    const double e = fma(a, a, -p);
    return DD{p, e};
}

UPIC_D double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

UPIC_D DD warp_sum_dd(DD v) {
    for (int o = 16; o > 0; o >>= 1) {
        DD w{__shfl_xor_sync(0xffffffffu, v.hi, o), __shfl_xor_sync(0xffffffffu, v.lo, o)};
        v = dd_add_dd(v, w);
    }
    return v;
}

UPIC_D double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace upic
