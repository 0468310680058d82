/*
 * TEST INFRASTRUCTURE ONLY (CPU oracle).  Restatement of the random-number
 * sequence the reference's initializers draw from: the C++ standard's
 * mt19937 engine ([rand.eng.mers], w=32 n=624 m=397 r=31 a=0x9908b0df,
 * u=11 d=0xffffffff s=7 b=0x9d2c5680 t=15 c=0xefc60000 l=18, seeding
 * multiplier 1812433253) and libstdc++'s generate_canonical<double,53>, which
 * combines two 32-bit draws as (g1 + g2*2^32) / 2^64 and clamps to below 1.
 * Used by Project2/spectral_pic_part3.cpp:633-634 (std::mt19937 +
 * uniform_real_distribution) for the Weibel quiet start.
 */
#include <math.h>
#include "oracle.h"

void o_mt_seed(o_mt19937* g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i) {
        uint32_t prev = g->mt[i - 1];
        g->mt[i] = 1812433253u * (prev ^ (prev >> 30)) + (uint32_t)i;
    }
    g->idx = 624;
}

static void mt_twist(o_mt19937* g) {
    for (int i = 0; i < 624; ++i) {
        uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
        uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
        if (y & 1u) v ^= 0x9908b0dfu;
        g->mt[i] = v;
    }
    g->idx = 0;
}

uint32_t o_mt_next(o_mt19937* g) {
    if (g->idx >= 624) mt_twist(g);
    uint32_t y = g->mt[g->idx++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

double o_mt_canonical(o_mt19937* g) {
    double sum = 0.0;
    double tmp = 1.0;
    for (int k = 0; k < 2; ++k) {
        sum += (double)o_mt_next(g) * tmp;
        tmp *= 4294967296.0;
    }
    double ret = sum / tmp;
    if (ret >= 1.0) ret = nextafter(1.0, 0.0);
    return ret;
}
