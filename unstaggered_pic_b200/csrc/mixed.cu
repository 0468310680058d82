// Mixed-precision explicit step (UPIC_PRECISION_MIXED, sm_100a).
//
// The same step as push_deposit_kernel (explicit.cu: recompute x^n, gather
// the eleven field records, IAEM push of P and v, deposit of the next step's
// current), with the particle state in FP32: the nearest node of each
// particle as an integer cell and its cell-relative offsets r = x/dx - ix in
// [-1/2, 1/2), so that FP32 keeps the position to 2^-24 of a cell anywhere in
// the box.  Particle arithmetic, gathers and the warp-level deposit sums are
// FP32; the field solve stays FP64 (its node records are rounded to FP32 when
// the gather table is written), and the deposit sums are folded into the grid
// as single-word 64-bit fixed point, so the grid accumulation is exact,
// order-independent and the run reproducible.  Particle diagnostics
// (kinetic energy, gamma sum) accumulate in FP64 double-double.
//
// Streamed state per particle and step: cell, r (2), v (3), v_prev (3), P (3)
// read (48 B) and the same minus P_z written (44 B): 92 B against 176 B in
// FP64.
#include "kernels.h"
#include "upic_common.cuh"

namespace upic {

namespace {

constexpr int kMThreads = 256;
constexpr int kMWarps = kMThreads / kWarp;
constexpr int kKeyNone = -1;
constexpr int kKeyEscape = -2;

template <int NCOMP>
struct MStage {
    static constexpr int kNV = 9 * NCOMP;   // values reduced per particle
    static constexpr int kRow = 9 + NCOMP;  // floats staged per particle
    static constexpr int kFloats = 32 * kRow;
};

UPIC_D int slot_of(int ncomp, int c) { return ncomp == 1 ? 3 : c; }

UPIC_D int mwindow_coord(int s, int origin, int n, int w) {
    const int d = (s - origin) & (n - 1);
    return d <= w - 3 ? d : -1;
}

// Single-word fixed point: round(v * scale) as a two's-complement int64.
// scale is a power of two with headroom over the largest node sum.
UPIC_D unsigned long long fixed1(float v, double scale) {
    return (unsigned long long)__double2ll_rn((double)v * scale);
}

// Move an offset by d cells and carry whole cells into the node index.
UPIC_D void advance(int& i, float& r, float d, int n) {
    r += d;
    const float s = floorf(r + 0.5f);
    r -= s;
    i = (i + (int)s) & (n - 1);
}

// Quadratic B-spline weights of nodes i-1, i, i+1 at offset r
// (quadratic_weights, spectral_pic_part3.cpp:537-552).
UPIC_D void qweights(float r, float* w) {
    const float a = 0.5f - r, b = 0.5f + r;
    w[0] = 0.5f * a * a;
    w[1] = 0.75f - r * r;
    w[2] = 0.5f * b * b;
}

template <int NCOMP>
UPIC_D void fold_window1(const unsigned long long* win, int WN, const TileGeom& tg, int ox, int oy,
                         unsigned long long* acc) {
    const int N = tg.nx * tg.ny;
    for (int idx = threadIdx.x; idx < NCOMP * WN; idx += blockDim.x) {
        const unsigned long long v = win[idx];
        if (v == 0ull) continue;
        const int cc = idx / WN, widx = idx - cc * WN;
        const int lx = widx / tg.wy, ly = widx - lx * tg.wy;
        const int gx = tg.full_x ? lx : wrap_index(ox + lx, tg.nx);
        const int gy = tg.full_y ? ly : wrap_index(oy + ly, tg.ny);
        atomicAdd(&acc[(size_t)(2 * slot_of(NCOMP, cc)) * N + gx * tg.ny + gy], v);
    }
}

template <int MODE, int NCOMP, bool UNIFORM>
__global__ void __launch_bounds__(kMThreads, 4) push_deposit_mixed_kernel(MixedPushArgs a, TileGeom tg) {
    constexpr int NV = MStage<NCOMP>::kNV;
    constexpr int RW = MStage<NCOMP>::kRow;
    constexpr int NPER = (NV + 31) / 32;
    extern __shared__ unsigned long long msmem[];
    const int WN = tg.wx * tg.wy;
    unsigned long long* win = msmem;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* sprod = reinterpret_cast<float*>(win + NCOMP * WN) + warp * MStage<NCOMP>::kFloats;
    int* sgk = reinterpret_cast<int*>(reinterpret_cast<float*>(win + NCOMP * WN) +
                                      kMWarps * MStage<NCOMP>::kFloats) + warp * 32;
    // FP32 field records of the tile's window (kModePush): gathers of
    // stencils inside the window read them from here
    // (16-byte aligned; offset from the shared base, so the pointer keeps the
    // shared state space: LDS, not generic loads)
    unsigned char* const sbytes = reinterpret_cast<unsigned char*>(msmem);
    const unsigned char* const sgk_end = reinterpret_cast<const unsigned char*>(
        reinterpret_cast<int*>(reinterpret_cast<float*>(win + NCOMP * WN) + kMWarps * MStage<NCOMP>::kFloats) +
        kMWarps * 32);
    float4* srec = reinterpret_cast<float4*>(sbytes + (((sgk_end - sbytes) + 15) & ~ptrdiff_t(15)));

    const int nx = tg.nx, ny = tg.ny;
    const int N = nx * ny;
    const int nch = *a.nchunks;
    const int c_begin = (int)(((long long)blockIdx.x * nch) / gridDim.x);
    const int c_end = (int)(((long long)(blockIdx.x + 1) * nch) / gridDim.x);

    DD kin{0.0, 0.0}, gsum{0.0, 0.0};
    double vmax2 = 0.0;  // largest |v|^2 (sqrt taken once: monotonic, correctly rounded)

    int cur_tile = -1, ox = 0, oy = 0;
    for (int ci = c_begin; ci < c_end; ++ci) {
        const Chunk ch = a.chunks[ci];
        if (ch.tile != cur_tile) {
            __syncthreads();
            if (cur_tile >= 0) {
                fold_window1<NCOMP>(win, WN, tg, ox, oy, a.acc);
                __syncthreads();
            }
            for (int idx = threadIdx.x; idx < NCOMP * WN; idx += blockDim.x) win[idx] = 0ull;
            cur_tile = ch.tile;
            const int tx = cur_tile / tg.nty, ty = cur_tile - tx * tg.nty;
            ox = tg.full_x ? 0 : tx * tg.tile_x - tg.guard - 1;
            oy = tg.full_y ? 0 : ty * tg.tile_y - tg.guard - 1;
            if (MODE == kModePush) {
                const float4* g4 = reinterpret_cast<const float4*>(a.gf);
                for (int idx = threadIdx.x; idx < WN * (kGFStride / 4); idx += blockDim.x) {
                    const int node = idx / (kGFStride / 4), f = idx - node * (kGFStride / 4);
                    const int lx = node / tg.wy, ly = node - lx * tg.wy;
                    const int gx = tg.full_x ? lx : ((ox + lx) & (nx - 1));
                    const int gy = tg.full_y ? ly : ((oy + ly) & (ny - 1));
                    srec[idx] = __ldg(g4 + (size_t)(gx * ny + gy) * (kGFStride / 4) + f);
                }
            }
            __syncthreads();
        }
        for (int base = ch.start; base < ch.end; base += kMThreads) {
            const int p = base + threadIdx.x;
            const bool active = p < ch.end;
            int key = kKeyNone, gx0 = 0, gy0 = 0;
            float dwx[3], dwy[3], dval[NCOMP];
            if (active) {
                const float q = UNIFORM ? a.q0f : a.p.q[p];
                const int cell = __ldcs(a.p.cell + p);
                int ix = cell >> a.lny, iy = cell & (ny - 1);
                float rx = __ldcs(a.p.rx + p), ry = __ldcs(a.p.ry + p);
                float v0 = __ldcs(a.p.vx + p), v1 = __ldcs(a.p.vy + p), v2 = __ldcs(a.p.vz + p);
                if (MODE == kModePush) {
                    // x^n = x^{n-1} + dt v^{n-1} (spectral_pic_part3.cpp:1050-1055)
                    advance(ix, rx, v0 * a.dt_dx, nx);
                    advance(iy, ry, v1 * a.dt_dy, ny);
                    // gather A, grad phi, grad A at x^n (:1063-1078)
                    float wxs[3], wys[3];
                    qweights(rx, wxs);
                    qweights(ry, wys);
                    float G[12];
#pragma unroll
                    for (int f = 0; f < 12; ++f) G[f] = 0.0f;
                    const int lx0 = tg.full_x ? 0 : mwindow_coord(ix - 1, ox, nx, tg.wx);
                    const int ly0 = tg.full_y ? 0 : mwindow_coord(iy - 1, oy, ny, tg.wy);
                    if (lx0 >= 0 && ly0 >= 0) {
#pragma unroll
                        for (int ia = 0; ia < 3; ++ia) {
                            const int wxi = tg.full_x ? wrap_index(ix - 1 + ia, nx) : lx0 + ia;
#pragma unroll
                            for (int ib = 0; ib < 3; ++ib) {
                                const int wyi = tg.full_y ? wrap_index(iy - 1 + ib, ny) : ly0 + ib;
                                const float w = wxs[ia] * wys[ib];
                                const float4* rec = srec + (wxi * tg.wy + wyi) * (kGFStride / 4);
#pragma unroll
                                for (int f4 = 0; f4 < kGFStride / 4; ++f4) {
                                    const float4 r = rec[f4];
                                    G[4 * f4] = fmaf(r.x, w, G[4 * f4]);
                                    G[4 * f4 + 1] = fmaf(r.y, w, G[4 * f4 + 1]);
                                    G[4 * f4 + 2] = fmaf(r.z, w, G[4 * f4 + 2]);
                                    G[4 * f4 + 3] = fmaf(r.w, w, G[4 * f4 + 3]);
                                }
                            }
                        }
                    } else
#pragma unroll
                    for (int ia = 0; ia < 3; ++ia) {
                        const int gx = wrap_index(ix - 1 + ia, nx);
#pragma unroll
                        for (int ib = 0; ib < 3; ++ib) {
                            const int gy = wrap_index(iy - 1 + ib, ny);
                            const float w = wxs[ia] * wys[ib];
                            const float4* rec = reinterpret_cast<const float4*>(a.gf + (size_t)(gx * ny + gy) * kGFStride);
#pragma unroll
                            for (int f4 = 0; f4 < kGFStride / 4; ++f4) {
                                const float4 r = __ldg(rec + f4);
                                G[4 * f4] = fmaf(r.x, w, G[4 * f4]);
                                G[4 * f4 + 1] = fmaf(r.y, w, G[4 * f4 + 1]);
                                G[4 * f4 + 2] = fmaf(r.z, w, G[4 * f4 + 2]);
                                G[4 * f4 + 3] = fmaf(r.w, w, G[4 * f4 + 3]);
                            }
                        }
                    }
                    // IAEM momentum update (:1072-1090)
                    const float w0 = __ldcs(a.p.wx + p), w1 = __ldcs(a.p.wy + p), w2 = __ldcs(a.p.wz + p);
                    const float vs0 = 2.0f * v0 - w0, vs1 = 2.0f * v1 - w1, vs2 = 2.0f * v2 - w2;
                    const float gdx = G[5] * vs0 + G[7] * vs1 + G[9] * vs2;
                    const float gdy = G[6] * vs0 + G[8] * vs1 + G[10] * vs2;
                    const float qdt = q * a.dt;
                    const float P0 = __ldcs(a.p.Px + p) + qdt * (gdx - G[3]);
                    const float P1 = __ldcs(a.p.Py + p) + qdt * (gdy - G[4]);
                    const float P2 = __ldcs(a.p.Pz + p);
                    // velocity_from_canonical (:602-607)
                    const float m = UNIFORM ? a.m0f : a.p.m[p];
                    const float p0 = P0 - q * G[0], p1 = P1 - q * G[1], p2 = P2 - q * G[2];
                    const float mc2 = m * a.c2;
                    const float arg = a.c2 * (p0 * p0 + p1 * p1 + p2 * p2) + mc2 * mc2;
                    const float sc = arg == 0.0f ? 0.0f : a.c2 * rsqrtf(arg);
                    const float n0v = sc * p0, n1v = sc * p1, n2v = sc * p2;
                    __stcs(a.p.cell + p, (ix << a.lny) | iy);
                    __stcs(a.p.rx + p, rx);
                    __stcs(a.p.ry + p, ry);
                    __stcs(a.p.Px + p, P0);
                    __stcs(a.p.Py + p, P1);
                    __stcs(a.p.wx + p, v0);
                    __stcs(a.p.wy + p, v1);
                    __stcs(a.p.wz + p, v2);
                    __stcs(a.p.vx + p, n0v);
                    __stcs(a.p.vy + p, n1v);
                    __stcs(a.p.vz + p, n2v);
                    v0 = n0v;
                    v1 = n1v;
                    v2 = n2v;
                }
                // particle diagnostics on the (new) velocity, FP64 (:950-957)
                if (a.diag_part) {
                    const double m = UNIFORM ? a.m0 : (double)a.p.m[p];
                    const double d0 = v0, d1 = v1, d2 = v2;
                    const double sp2 = d0 * d0 + d1 * d1 + d2 * d2;
                    const double one_m = 1.0 - sp2 * a.inv_c2d;
                    const double gam = rsqrt(one_m > 1.0e-14 ? one_m : 1.0e-14);
                    gsum = dd_add(gsum, gam);
                    kin = dd_add(kin, (gam - 1.0) * m * a.cd * a.cd);
                    vmax2 = fmax(vmax2, sp2);
                }
                // deposit position: stored x (kModeDeposit) or one step ahead
                if (MODE != kModeDeposit) {
                    advance(ix, rx, v0 * a.dt_dx, nx);
                    advance(iy, ry, v1 * a.dt_dy, ny);
                }
                qweights(rx, dwx);
                qweights(ry, dwy);
                const float qa = q * a.inv_dA;
                if (NCOMP == 1) {
                    dval[0] = qa;
                } else {
                    dval[0] = qa * v0;
                    dval[1] = qa * v1;
                    dval[2] = qa * v2;
                    if (NCOMP == 4) dval[NCOMP - 1] = qa;
                }
                gx0 = wrap_index(ix - 1, nx);
                gy0 = wrap_index(iy - 1, ny);
                const int lx = tg.full_x ? gx0 : mwindow_coord(ix - 1, ox, nx, tg.wx);
                const int ly = tg.full_y ? gy0 : mwindow_coord(iy - 1, oy, ny, tg.wy);
                key = (lx < 0 || ly < 0) ? kKeyEscape : lx * tg.wy + ly;
            }
            // group the warp's particles by window key (groups in the order of
            // their first particle, rows in index order, escapes last)
            const unsigned full = 0xffffffffu;
            const unsigned lt = (1u << lane) - 1u;
            const unsigned valid = __ballot_sync(full, key >= 0);
            const unsigned esc = __ballot_sync(full, key == kKeyEscape);
            const unsigned peers = __match_any_sync(full, key);
            int row = -1, nvalid = 0, ngroups = 0;
            unsigned heads = 0u;
            for (unsigned rem = valid; rem;) {
                const int l = __ffs(rem) - 1;
                const unsigned g = __shfl_sync(full, peers, l);
                const int gk = __shfl_sync(full, key, l);
                if ((g >> lane) & 1u) row = nvalid + __popc(g & lt);
                if (lane == 0) sgk[ngroups] = gk;
                heads |= 1u << nvalid;
                nvalid += __popc(g);
                rem &= ~g;
                ++ngroups;
            }
            if (key == kKeyEscape) row = nvalid + __popc(esc & lt);
            if (row >= 0) {
                float* mine = sprod + row * RW;
#pragma unroll
                for (int ia = 0; ia < 3; ++ia)
#pragma unroll
                    for (int ib = 0; ib < 3; ++ib) mine[ia * 3 + ib] = dwx[ia] * dwy[ib];
#pragma unroll
                for (int cc = 0; cc < NCOMP; ++cc) mine[9 + cc] = dval[cc];
            }
            __syncwarp();
            // particles whose stencil leaves the window: fixed-point adds to the grid
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
                            const int tab = t / NCOMP, tc = t - tab * NCOMP;
                            const float v = sprod[erow * RW + 9 + tc] * sprod[erow * RW + tab];
                            if (v != 0.0f) {
                                const int g = wrap_index(gxj + tab / 3, nx) * ny + wrap_index(gyj + tab % 3, ny);
                                const int sl = slot_of(NCOMP, tc);
                                atomicAdd(&a.acc[(size_t)(2 * sl) * N + g], fixed1(v, a.scale[sl]));
                            }
                        }
                    }
                    ++erow;
                }
            }
            // warp-level segmented reduction in fixed order, one window add per
            // key group and value
            {
                unsigned h = heads;
                int gi = 0;
                while (h) {
                    const int rs = __ffs(h) - 1;
                    h &= h - 1;
                    const int re = h ? __ffs(h) - 1 : nvalid;
                    const int k = sgk[gi++];
#pragma unroll
                    for (int r = 0; r < NPER; ++r) {
                        const int t = lane + 32 * r;
                        if (t < NV) {
                            const int tab = t / NCOMP, tc = t - tab * NCOMP;
                            float s0 = 0.0f, s1 = 0.0f;
                            int j = rs;
                            for (; j + 1 < re; j += 2) {
                                s0 = fmaf(sprod[j * RW + 9 + tc], sprod[j * RW + tab], s0);
                                s1 = fmaf(sprod[(j + 1) * RW + 9 + tc], sprod[(j + 1) * RW + tab], s1);
                            }
                            if (j < re) s0 = fmaf(sprod[j * RW + 9 + tc], sprod[j * RW + tab], s0);
                            const float sum = s0 + s1;
                            if (sum != 0.0f) {
                                int widx;
                                if (tg.full_x || tg.full_y) {
                                    const int kx = k / tg.wy, ky = k - kx * tg.wy;
                                    int nxl = kx + tab / 3, nyl = ky + tab % 3;
                                    if (tg.full_x) nxl &= tg.wx - 1;
                                    if (tg.full_y) nyl &= tg.wy - 1;
                                    widx = nxl * tg.wy + nyl;
                                } else {
                                    widx = k + (tab / 3) * tg.wy + tab % 3;
                                }
                                atomicAdd(&win[tc * WN + widx], fixed1(sum, a.scale[slot_of(NCOMP, tc)]));
                            }
                        }
                    }
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (cur_tile >= 0) fold_window1<NCOMP>(win, WN, tg, ox, oy, a.acc);
    if (a.diag_part) {
        kin = warp_sum_dd(kin);
        gsum = warp_sum_dd(gsum);
        const double vmax = warp_max(sqrt(vmax2));
        __syncthreads();
        double* red = reinterpret_cast<double*>(msmem);
        if (lane == 0) {
            red[warp * 5 + 0] = kin.hi;
            red[warp * 5 + 1] = kin.lo;
            red[warp * 5 + 2] = gsum.hi;
            red[warp * 5 + 3] = gsum.lo;
            red[warp * 5 + 4] = vmax;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            DD k{0.0, 0.0}, g{0.0, 0.0};
            double vm = 0.0;
            for (int w = 0; w < kMWarps; ++w) {
                k = dd_add_dd(k, DD{red[w * 5 + 0], red[w * 5 + 1]});
                g = dd_add_dd(g, DD{red[w * 5 + 2], red[w * 5 + 3]});
                vm = fmax(vm, red[w * 5 + 4]);
            }
            double* out = a.diag_part + (size_t)blockIdx.x * kDiagPart;
            out[0] = k.hi;
            out[1] = k.lo;
            out[2] = g.hi;
            out[3] = g.lo;
            out[4] = vm;
        }
    }
}

// ---- sorting, layout conversion -------------------------------------------------

__global__ void make_keys_mixed_kernel(TileGeom tg, MixedSoA p, long np, int lny, float sx, float sy,
                                       unsigned* keys) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < np; q += (long)gridDim.x * blockDim.x) {
        const int cell = p.cell[q];
        int ix = cell >> lny, iy = cell & (tg.ny - 1);
        if (sx != 0.0f || sy != 0.0f) {
            float rx = p.rx[q], ry = p.ry[q];
            advance(ix, rx, sx * p.vx[q], tg.nx);
            advance(iy, ry, sy * p.vy[q], tg.ny);
        }
        const int tx = ix / tg.tile_x, lx = ix - tx * tg.tile_x;
        const int ty = iy / tg.tile_y, ly = iy - ty * tg.tile_y;
        const unsigned tile = (unsigned)(tx * tg.nty + ty);
        keys[q] = tile * (unsigned)(tg.tile_x * tg.tile_y) + (unsigned)(lx * tg.tile_y + ly);
    }
}

template <typename T>
__global__ void mgather_kernel(const T* __restrict__ src, T* __restrict__ dst, const int* idx, long n) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        dst[q] = src[idx[q]];
}

__global__ void unpermute_mixed_kernel(MixedSoA s, MixedSoA d, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int o = s.id[k];
        const int cell = s.cell[k];
        const float v[11] = {s.rx[k], s.ry[k], s.Px[k], s.Py[k], s.Pz[k], s.vx[k],
                             s.vy[k], s.vz[k], s.wx[k], s.wy[k], s.wz[k]};
        d.cell[o] = cell;
        d.rx[o] = v[0];
        d.ry[o] = v[1];
        d.Px[o] = v[2];
        d.Py[o] = v[3];
        d.Pz[o] = v[4];
        d.vx[o] = v[5];
        d.vy[o] = v[6];
        d.vz[o] = v[7];
        d.wx[o] = v[8];
        d.wy[o] = v[9];
        d.wz[o] = v[10];
    }
}

// Nearest node and offset of x in [0, L) (quadratic_weights' s = x/dx,
// ic = floor(s + 1/2), r = s - ic), the offset rounded once to FP32.
__global__ void from_positions_kernel(long np, const double* x, const double* y, double inv_dx, double inv_dy,
                                      int nx, int ny, int lny, int* cell, float* rx, float* ry) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < np; q += (long)gridDim.x * blockDim.x) {
        const double sx = x[q] * inv_dx, sy = y[q] * inv_dy;
        const double fx = floor(sx + 0.5), fy = floor(sy + 0.5);
        const int ix = wrap_index((int)fx, nx), iy = wrap_index((int)fy, ny);
        cell[q] = (ix << lny) | iy;
        rx[q] = (float)(sx - fx);
        ry[q] = (float)(sy - fy);
    }
}

// Position in [0, L) of node ix plus offset r.
__global__ void to_positions_kernel(long np, const int* cell, const float* rx, const float* ry, double dx,
                                    double dy, double Lx, double Ly, int lny, int ny, double* x, double* y) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < np; q += (long)gridDim.x * blockDim.x) {
        const int c = cell[q];
        double xv = ((double)(c >> lny) + (double)rx[q]) * dx;
        double yv = ((double)(c & (ny - 1)) + (double)ry[q]) * dy;
        if (xv < 0.0) xv += Lx;
        if (xv >= Lx) xv -= Lx;
        if (yv < 0.0) yv += Ly;
        if (yv >= Ly) yv -= Ly;
        x[q] = xv;
        y[q] = yv;
    }
}

__global__ void split3f_kernel(long n, const double* aos, float* a, float* b, float* c) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
        a[q] = (float)aos[3 * q];
        b[q] = (float)aos[3 * q + 1];
        c[q] = (float)aos[3 * q + 2];
    }
}

__global__ void join3f_kernel(long n, const float* a, const float* b, const float* c, double* aos) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
        aos[3 * q] = a[q];
        aos[3 * q + 1] = b[q];
        aos[3 * q + 2] = c[q];
    }
}

__global__ void to_float_kernel(long n, const double* src, float* dst) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        dst[q] = (float)src[q];
}

__global__ void convert_acc1_kernel(unsigned long long* acc, int N, double s0, double s1, double s2, double s3,
                                    double* J, double* rho, double n0, int mask, const double* bg) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        if (mask & 1) {
            const double sc[3] = {s0, s1, s2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                unsigned long long* h = acc + (size_t)(2 * c) * N;
                J[(size_t)c * N + id] = (double)(long long)h[id] / sc[c];
                h[id] = 0ull;
            }
        }
        if (mask & 2) {
            unsigned long long* h = acc + (size_t)6 * N;
            rho[id] = (bg ? bg[id] : n0) + (double)(long long)h[id] / s3;
            h[id] = 0ull;
        }
    }
}

int mgrid(long n) {
    long g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return g < 1 ? 1 : (int)g;
}

template <int MODE, int NCOMP, bool UNIFORM>
cudaError_t launch_mixed_one(const TileGeom& tg, const MixedPushArgs& a, int grid, cudaStream_t st) {
    push_deposit_mixed_kernel<MODE, NCOMP, UNIFORM>
        <<<grid, kMThreads, push_mixed_smem_bytes(tg, NCOMP), st>>>(a, tg);
    count_launches(1);
    return cudaGetLastError();
}

template <int MODE, int NCOMP, bool UNIFORM>
cudaError_t set_mixed_smem(int bytes) {
    return raise_smem_limit(reinterpret_cast<const void*>(push_deposit_mixed_kernel<MODE, NCOMP, UNIFORM>), bytes);
}

}  // namespace

int push_mixed_smem_bytes(const TileGeom& tg, int ncomp) {
    const int window = ncomp * tg.wx * tg.wy * 8;
    const int stage = kMWarps * (32 * (9 + ncomp) * 4 + 32 * 4);
    const int bytes = window + stage + 16 + tg.wx * tg.wy * kGFStride * 4;
    const int red = kMWarps * 5 * 8;
    return bytes > red ? bytes : red;
}

cudaError_t push_mixed_configure_smem(const TileGeom& tg) {
    cudaError_t e = cudaSuccess;
#define UPIC_SETM(MODE, NC, U)                                      \
    e = set_mixed_smem<MODE, NC, U>(push_mixed_smem_bytes(tg, NC)); \
    if (e != cudaSuccess) return e;
    UPIC_SETM(kModeDeposit, 4, true) UPIC_SETM(kModeDeposit, 4, false)
    UPIC_SETM(kModeAdvanceDeposit, 3, true) UPIC_SETM(kModeAdvanceDeposit, 3, false)
    UPIC_SETM(kModeAdvanceDeposit, 4, true) UPIC_SETM(kModeAdvanceDeposit, 4, false)
    UPIC_SETM(kModePush, 3, true) UPIC_SETM(kModePush, 3, false)
    UPIC_SETM(kModePush, 4, true) UPIC_SETM(kModePush, 4, false)
#undef UPIC_SETM
    return e;
}

int push_mixed_occupancy(const TileGeom& tg, int ncomp) {
    int n = 0;
    if (ncomp == 4)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, push_deposit_mixed_kernel<kModePush, 4, true>, kMThreads,
                                                      push_mixed_smem_bytes(tg, 4));
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, push_deposit_mixed_kernel<kModePush, 3, true>, kMThreads,
                                                      push_mixed_smem_bytes(tg, 3));
    return n;
}

cudaError_t launch_push_mixed(int mode, int ncomp, bool uniform, const TileGeom& tg, const MixedPushArgs& a,
                              int grid, cudaStream_t st) {
#define UPIC_CASEM(MODE, NC)                                                  \
    if (mode == MODE && ncomp == NC)                                          \
        return uniform ? launch_mixed_one<MODE, NC, true>(tg, a, grid, st)    \
                       : launch_mixed_one<MODE, NC, false>(tg, a, grid, st);
    UPIC_CASEM(kModeDeposit, 4)
    UPIC_CASEM(kModeAdvanceDeposit, 3)
    UPIC_CASEM(kModeAdvanceDeposit, 4)
    UPIC_CASEM(kModePush, 3)
    UPIC_CASEM(kModePush, 4)
#undef UPIC_CASEM
    return cudaErrorInvalidValue;
}

cudaError_t launch_convert_acc1(unsigned long long* acc, int N, const double* scale, double* J, double* rho,
                                double n0, int mask, cudaStream_t st, const double* bg) {
    convert_acc1_kernel<<<mgrid(N), 256, 0, st>>>(acc, N, scale[0], scale[1], scale[2], scale[3], J, rho, n0,
                                                  mask, bg);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t sort_mixed_by_tile(const TileGeom& tg, const MixedSoA& p, long np, int lny, float sx, float sy,
                               SortWork& w, cudaStream_t st) {
    if (np > 0) {
        make_keys_mixed_kernel<<<mgrid(np), 256, 0, st>>>(tg, p, np, lny, sx, sy, sort_key_input(tg, w));
        count_launches(1);
    }
    return sort_keys_to_chunks(tg, np, w, st);
}

// Every payload array of the mixed set in one pass over the sorted index.
struct MGatherSet {
    const float* src[13];
    float* dst[13];
    int narr;
    const int *scell, *sid;
    int *dcell, *did;
};

__global__ void mgather_set_kernel(MGatherSet g, const int* __restrict__ idx, long n) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
        const int i = idx[q];
        // all of a particle's values loaded ahead of the stores (13 loads in
        // flight; the arrays may alias as far as the compiler knows): 4.65-4.68
        // against 4.77 ms per mixed step at 512x512 x 256 with one array after
        // the other (the FP64 gather measured the other way round)
        float v[13];
#pragma unroll
        for (int k = 0; k < 13; ++k) v[k] = k < g.narr ? __ldg(g.src[k] + i) : 0.0f;
        const int cell = __ldg(g.scell + i), id = __ldg(g.sid + i);
#pragma unroll
        for (int k = 0; k < 13; ++k)
            if (k < g.narr) g.dst[k][q] = v[k];
        g.dcell[q] = cell;
        g.did[q] = id;
    }
}

cudaError_t permute_mixed(const MixedSoA& s, const MixedSoA& d, long np, const SortWork& w, cudaStream_t st) {
    const int g = mgrid(np);
    float* const src[13] = {s.rx, s.ry, s.Px, s.Py, s.Pz, s.vx, s.vy, s.vz, s.wx, s.wy, s.wz, s.q, s.m};
    float* const dst[13] = {d.rx, d.ry, d.Px, d.Py, d.Pz, d.vx, d.vy, d.vz, d.wx, d.wy, d.wz, d.q, d.m};
    MGatherSet gs{};
    for (int k = 0; k < 13; ++k)
        if (src[k] && dst[k]) {
            gs.src[gs.narr] = src[k];
            gs.dst[gs.narr] = dst[k];
            ++gs.narr;
        }
    gs.scell = s.cell;
    gs.dcell = d.cell;
    gs.sid = s.id;
    gs.did = d.id;
    if (np > 0) {
        mgather_set_kernel<<<g, 256, 0, st>>>(gs, w.vals, np);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t unpermute_mixed(const MixedSoA& s, const MixedSoA& d, long np, cudaStream_t st) {
    unpermute_mixed_kernel<<<mgrid(np), 256, 0, st>>>(s, d, np);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t mixed_from_positions(long np, const double* x, const double* y, double inv_dx, double inv_dy, int nx,
                                 int ny, int lny, int* cell, float* rx, float* ry, cudaStream_t st) {
    from_positions_kernel<<<mgrid(np), 256, 0, st>>>(np, x, y, inv_dx, inv_dy, nx, ny, lny, cell, rx, ry);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t mixed_to_positions(long np, const int* cell, const float* rx, const float* ry, double dx, double dy,
                               double Lx, double Ly, int lny, int ny, double* x, double* y, cudaStream_t st) {
    to_positions_kernel<<<mgrid(np), 256, 0, st>>>(np, cell, rx, ry, dx, dy, Lx, Ly, lny, ny, x, y);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t mixed_split3(long np, const double* aos, float* a, float* b, float* c, cudaStream_t st) {
    split3f_kernel<<<mgrid(np), 256, 0, st>>>(np, aos, a, b, c);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t mixed_join3(long np, const float* a, const float* b, const float* c, double* aos, cudaStream_t st) {
    join3f_kernel<<<mgrid(np), 256, 0, st>>>(np, a, b, c, aos);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t mixed_from_doubles(long np, const double* src, float* dst, cudaStream_t st) {
    to_float_kernel<<<mgrid(np), 256, 0, st>>>(np, src, dst);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace upic
