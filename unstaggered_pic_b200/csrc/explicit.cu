// Explicit spectral BDF / IAEM step kernels (sm_100a).
//
// Reference: Project2/spectral_pic_part3.cpp (run_simulation :1094-1189).
// One step of the reference is
//   x += dt v; J = deposit(x, v); rho (continuity or redeposit); BDF wave
//   solves for phi, A; spectral grad phi, grad A; IAEM push; diagnostics.
// Here the particle work of a step is one fused kernel (push_deposit_kernel,
// kModePush): it recomputes x^n = wrap(x^{n-1} + dt v^{n-1}), gathers the
// eleven field records at x^n, pushes P and v, stores the step-n state, and
// already deposits the NEXT step's current J^{n+1} at wrap(x^n + dt v^n) with
// v^n (what the reference's next iteration deposits).  The field work of a
// step is a handful of grid kernels in k-space (histories kept as spectra).
#include <map>
#include <mutex>
#include <utility>
#include "kernels.h"
#include "upic_common.cuh"

namespace upic {

namespace {

// Threads per CTA and resident CTAs per SM the push kernel is compiled for
// (register budget 65536 / (threads * CTAs) per thread).
#ifndef UPIC_PUSH_THREADS
#define UPIC_PUSH_THREADS 256
#endif
#ifndef UPIC_PUSH_MIN_BLOCKS
#define UPIC_PUSH_MIN_BLOCKS 3
#endif
// 1: the step push stages its tile window's field records in shared memory
// and gathers from there (the same sums in the same order as the global
// gather, which remains for stencils outside the window)
#ifndef UPIC_PUSH_SMEM_GATHER
#define UPIC_PUSH_SMEM_GATHER 1
#endif
constexpr int kPushThreads = UPIC_PUSH_THREADS;
constexpr int kPushWarps = kPushThreads / kWarp;
constexpr int kKeyNone = -1;
constexpr int kKeyEscape = -2;

// Per-warp staging: one row per particle with its 9 tensor-product stencil
// weights S_ab and its NCOMP deposit values (q v_c / dA, or q / dA).
template <int NCOMP>
struct StageLayout {
    static constexpr int kNV = 9 * NCOMP;   // values reduced per particle
    static constexpr int kRow = 9 + NCOMP;  // doubles staged per particle
    static constexpr int kDoubles = 32 * kRow;
};

UPIC_D int acc_slot(int ncomp, int c) { return ncomp == 1 ? 3 : c; }

// Window-local coordinate of a stencil origin node (tiled axis): -1 when the
// three-node stencil does not fit in the window.
UPIC_D int window_coord(int s, int origin, int n, int w) {
    const int d = (s - origin) & (n - 1);
    return d <= w - 3 ? d : -1;
}

// Fold a CTA's window into the global fixed-point accumulators (integer adds:
// order-independent, hence deterministic).
template <int NCOMP>
UPIC_D void fold_window(const unsigned long long* whi, const unsigned long long* wlo, int WN,
                        const TileGeom& tg, int ox, int oy, unsigned long long* acc) {
    const int N = tg.nx * tg.ny;
    for (int idx = threadIdx.x; idx < NCOMP * WN; idx += blockDim.x) {
        const unsigned long long hi = whi[idx], lo = wlo[idx];
        if ((hi | lo) == 0ull) continue;
        const int cc = idx / WN, widx = idx - cc * WN;
        const int lx = widx / tg.wy, ly = widx - lx * tg.wy;
        const int gx = tg.full_x ? lx : wrap_index(ox + lx, tg.nx);
        const int gy = tg.full_y ? ly : wrap_index(oy + ly, tg.ny);
        const int sl = acc_slot(NCOMP, cc);
        atomicAdd(&acc[(size_t)(2 * sl) * N + gx * tg.ny + gy], hi);
        atomicAdd(&acc[(size_t)(2 * sl + 1) * N + gx * tg.ny + gy], lo);
    }
}

// Bulk L2 prefetch (sm_90+ TMA unit) of elements [i0, i1) of a particle
// array.  The range is widened to 16-byte boundaries; particle arrays carry
// two elements of padding (alloc_soa), so the widened range stays inside
// the allocation.  A prefetch is a hint: it moves no data into the SM.
UPIC_D void prefetch_l2(const double* base, int i0, int i1) {
    if (!base || i1 <= i0) return;
    const unsigned long long a0 = reinterpret_cast<unsigned long long>(base + i0) & ~15ull;
    const unsigned long long a1 = (reinterpret_cast<unsigned long long>(base + i1) + 15ull) & ~15ull;
    const unsigned bytes = (unsigned)(a1 - a0);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"(bytes) : "memory");
}

// Prefetch of the particle state the CTA reads in its next batch of
// kPushThreads particles: the rest of this chunk, else the next chunk.
template <int MODE, bool UNIFORM>
UPIC_D void prefetch_next_batch(const PushArgs& a, const Chunk& ch, int base, int ci, int c_end) {
    int n0, n1;
    if (base + kPushThreads < ch.end) {
        n0 = base + kPushThreads;
        n1 = min(n0 + kPushThreads, ch.end);
    } else if (ci + 1 < c_end) {
        const Chunk nx = a.chunks[ci + 1];
        n0 = nx.start;
        n1 = min(nx.start + kPushThreads, nx.end);
    } else {
        return;
    }
    const int t = threadIdx.x;
    const double* arr = nullptr;
    switch (t) {
        case 0: arr = a.p.x; break;
        case 1: arr = a.p.y; break;
        case 2: arr = a.p.vx; break;
        case 3: arr = a.p.vy; break;
        case 4: arr = a.p.vz; break;
        case 5: arr = MODE == kModePush ? a.p.wx : nullptr; break;
        case 6: arr = MODE == kModePush ? a.p.wy : nullptr; break;
        case 7: arr = MODE == kModePush ? a.p.wz : nullptr; break;
        case 8: arr = MODE == kModePush ? a.p.Px : nullptr; break;
        case 9: arr = MODE == kModePush ? a.p.Py : nullptr; break;
        case 10: arr = MODE == kModePush ? a.p.Pz : nullptr; break;
        case 11: arr = UNIFORM ? nullptr : a.p.q; break;
        case 12: arr = UNIFORM ? nullptr : a.p.m; break;
        default: break;
    }
    prefetch_l2(arr, n0, n1);
}

template <int MODE, int NCOMP, bool UNIFORM>
__global__ void __launch_bounds__(kPushThreads, UPIC_PUSH_MIN_BLOCKS)
push_deposit_kernel(PushArgs a, TileGeom tg) {
    constexpr int NV = StageLayout<NCOMP>::kNV;
    constexpr int RW = StageLayout<NCOMP>::kRow;
    constexpr int NPER = (NV + 31) / 32;
    extern __shared__ unsigned long long smem_u64[];
    const int WN = tg.wx * tg.wy;
    unsigned long long* whi = smem_u64;
    unsigned long long* wlo = whi + NCOMP * WN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* sprod = reinterpret_cast<double*>(wlo + NCOMP * WN) + warp * StageLayout<NCOMP>::kDoubles;
    int* sgk = reinterpret_cast<int*>(reinterpret_cast<double*>(wlo + NCOMP * WN) +
                                      kPushWarps * StageLayout<NCOMP>::kDoubles) + warp * 32;
#if UPIC_PUSH_SMEM_GATHER
    // field records of the tile's window (kModePush): the gathers of
    // particles whose stencil lies in the window read them from here
    // (16-byte aligned; the offset is taken from the shared base so that the
    // pointer keeps the shared state space and the gathers are LDS, not
    // generic loads)
    unsigned char* const sbytes = reinterpret_cast<unsigned char*>(smem_u64);
    const unsigned char* const sgk_end = reinterpret_cast<const unsigned char*>(
        reinterpret_cast<int*>(reinterpret_cast<double*>(wlo + NCOMP * WN) +
                               kPushWarps * StageLayout<NCOMP>::kDoubles) + kPushWarps * 32);
    double2* srec = reinterpret_cast<double2*>(sbytes + (((sgk_end - sbytes) + 15) & ~ptrdiff_t(15)));
#endif

    const int nx = tg.nx, ny = tg.ny;
    const int N = nx * ny;
    const int nch = *a.nchunks;
    const int c_begin = (int)(((long long)blockIdx.x * nch) / gridDim.x);
    const int c_end = (int)(((long long)(blockIdx.x + 1) * nch) / gridDim.x);

    // values owned by this lane in the segmented reduction: t = lane + 32 r is
    // stencil node ab = t / NCOMP (a = ab/3 along x, b = ab%3 along y) and
    // deposit component c = t % NCOMP
    int t_off[NPER], t_a[NPER], t_b[NPER], t_c[NPER], t_ab[NPER];
    double t_scale[NPER];
#pragma unroll
    for (int r = 0; r < NPER; ++r) {
        const int t = lane + 32 * r;
        const int ab = t < NV ? t / NCOMP : 0;
        t_ab[r] = ab;
        t_a[r] = ab / 3;
        t_b[r] = ab % 3;
        t_c[r] = t < NV ? t - ab * NCOMP : 0;
        t_off[r] = t_a[r] * tg.wy + t_b[r];
        t_scale[r] = a.scale[acc_slot(NCOMP, t_c[r])];
    }

    DD kin{0.0, 0.0}, gsum{0.0, 0.0};
    double vmax2 = 0.0;  // largest |v|^2 (sqrt taken once: sqrt is monotonic and correctly rounded)
    const double c2 = a.c * a.c;

    int cur_tile = -1, ox = 0, oy = 0;
    for (int ci = c_begin; ci < c_end; ++ci) {
        const Chunk ch = a.chunks[ci];
        if (ch.tile != cur_tile) {
            __syncthreads();
            if (cur_tile >= 0) {
                fold_window<NCOMP>(whi, wlo, WN, tg, ox, oy, a.acc);
                __syncthreads();
            }
            for (int idx = threadIdx.x; idx < 2 * NCOMP * WN; idx += blockDim.x) whi[idx] = 0ull;
            cur_tile = ch.tile;
            const int tx = cur_tile / tg.nty, ty = cur_tile - tx * tg.nty;
            ox = tg.full_x ? 0 : tx * tg.tile_x - tg.guard - 1;
            oy = tg.full_y ? 0 : ty * tg.tile_y - tg.guard - 1;
#if UPIC_PUSH_SMEM_GATHER
            if (MODE == kModePush) {
                const double2* g2 = reinterpret_cast<const double2*>(a.gfields);
                for (int idx = threadIdx.x; idx < WN * (kGFStride / 2); idx += blockDim.x) {
                    const int node = idx / (kGFStride / 2), f = idx - node * (kGFStride / 2);
                    const int lx = node / tg.wy, ly = node - lx * tg.wy;
                    const int gx = tg.full_x ? lx : ((ox + lx) & (nx - 1));
                    const int gy = tg.full_y ? ly : ((oy + ly) & (ny - 1));
                    srec[idx] = __ldg(g2 + (size_t)(gx * ny + gy) * (kGFStride / 2) + f);
                }
            }
#endif
            __syncthreads();
        }
        for (int base = ch.start; base < ch.end; base += kPushThreads) {
            const int p = base + threadIdx.x;
            const bool active = p < ch.end;
            if (threadIdx.x < 13) prefetch_next_batch<MODE, UNIFORM>(a, ch, base, ci, c_end);
            int key = kKeyNone, gx0 = 0, gy0 = 0;
            double dwx[3], dwy[3], dval[NCOMP];
            if (active) {
                const double q = UNIFORM ? a.q0 : a.p.q[p];
                double x = __ldcs(a.p.x + p), y = __ldcs(a.p.y + p);
                double v0 = __ldcs(a.p.vx + p), v1 = __ldcs(a.p.vy + p), v2 = __ldcs(a.p.vz + p);
                if (MODE == kModePush) {
                    // spectral_pic_part3.cpp:1050-1055: x^n = x^{n-1} + dt v^{n-1}
                    x = wrap_periodic(x + a.dt * v0, a.Lx, a.inv_Lx);
                    y = wrap_periodic(y + a.dt * v1, a.Ly, a.inv_Ly);
                    // gather A, grad phi, grad A at x^n (:1063-1078)
                    const Quad1D qx = quadratic_weights(x, a.inv_dx);
                    const Quad1D qy = quadratic_weights(y, a.inv_dy);
                    const double wxs[3] = {qx.w0, qx.w1, qx.w2};
                    const double wys[3] = {qy.w0, qy.w1, qy.w2};
                    double G[12];
#pragma unroll
                    for (int f = 0; f < 12; ++f) G[f] = 0.0;
#if UPIC_PUSH_SMEM_GATHER
                    const int lx0 = tg.full_x ? 0 : window_coord(qx.ic - 1, ox, nx, tg.wx);
                    const int ly0 = tg.full_y ? 0 : window_coord(qy.ic - 1, oy, ny, tg.wy);
                    if (lx0 >= 0 && ly0 >= 0) {
#pragma unroll
                        for (int ia = 0; ia < 3; ++ia) {
                            const int wxi = tg.full_x ? wrap_index(qx.ic - 1 + ia, nx) : lx0 + ia;
#pragma unroll
                            for (int ib = 0; ib < 3; ++ib) {
                                const int wyi = tg.full_y ? wrap_index(qy.ic - 1 + ib, ny) : ly0 + ib;
                                const double w = wxs[ia] * wys[ib];
                                const double2* rec = srec + (wxi * tg.wy + wyi) * (kGFStride / 2);
#pragma unroll
                                for (int f2 = 0; f2 < kGFStride / 2; ++f2) {
                                    const double2 r = rec[f2];
                                    G[2 * f2] = fma(r.x, w, G[2 * f2]);
                                    G[2 * f2 + 1] = fma(r.y, w, G[2 * f2 + 1]);
                                }
                            }
                        }
                    } else
#endif
#pragma unroll
                    for (int ia = 0; ia < 3; ++ia) {
                        const int gx = wrap_index(qx.ic - 1 + ia, nx);
#pragma unroll
                        for (int ib = 0; ib < 3; ++ib) {
                            const int gy = wrap_index(qy.ic - 1 + ib, ny);
                            const double w = wxs[ia] * wys[ib];
                            const double2* rec = reinterpret_cast<const double2*>(
                                a.gfields + (size_t)(gx * ny + gy) * kGFStride);
#pragma unroll
                            for (int f2 = 0; f2 < kGFStride / 2; ++f2) {
                                const double2 r = __ldg(rec + f2);
                                G[2 * f2] = fma(r.x, w, G[2 * f2]);
                                G[2 * f2 + 1] = fma(r.y, w, G[2 * f2 + 1]);
                            }
                        }
                    }
                    // IAEM momentum update (:1072-1090)
                    const double w0 = __ldcs(a.p.wx + p), w1 = __ldcs(a.p.wy + p), w2 = __ldcs(a.p.wz + p);
                    const double vs0 = 2.0 * v0 - w0, vs1 = 2.0 * v1 - w1, vs2 = 2.0 * v2 - w2;
                    const double gdx = G[5] * vs0 + G[7] * vs1 + G[9] * vs2;
                    const double gdy = G[6] * vs0 + G[8] * vs1 + G[10] * vs2;
                    const double qdt = q * a.dt;
                    const double P0 = __ldcs(a.p.Px + p) + qdt * (gdx - G[3]);
                    const double P1 = __ldcs(a.p.Py + p) + qdt * (gdy - G[4]);
                    const double P2 = __ldcs(a.p.Pz + p);
                    // velocity_from_canonical (:602-607)
                    const double m = UNIFORM ? a.m0 : a.p.m[p];
                    const double p0 = P0 - q * G[0], p1 = P1 - q * G[1], p2 = P2 - q * G[2];
                    const double mc2 = m * c2;
                    const double arg = c2 * (p0 * p0 + p1 * p1 + p2 * p2) + mc2 * mc2;
                    const double s = arg == 0.0 ? 0.0 : c2 * rsqrt(arg);
                    const double n0v = s * p0, n1v = s * p1, n2v = s * p2;
                    __stcs(a.p.x + p, x);
                    __stcs(a.p.y + p, y);
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
                // particle diagnostics on the (new) velocity (:950-957)
                if (a.diag_part) {
                    const double m = UNIFORM ? a.m0 : a.p.m[p];
                    const double sp2 = v0 * v0 + v1 * v1 + v2 * v2;
                    const double one_m = 1.0 - sp2 * a.inv_c2;
                    const double gam = rsqrt(one_m > 1.0e-14 ? one_m : 1.0e-14);
                    gsum = dd_add(gsum, gam);
                    kin = dd_add(kin, (gam - 1.0) * m * a.c * a.c);
                    vmax2 = fmax(vmax2, sp2);
                }
                // deposit position: stored x (kModeDeposit) or one step ahead
                if (MODE != kModeDeposit) {
                    x = wrap_periodic(x + a.dt * v0, a.Lx, a.inv_Lx);
                    y = wrap_periodic(y + a.dt * v1, a.Ly, a.inv_Ly);
                }
                const Quad1D dx_ = quadratic_weights(x, a.inv_dx);
                const Quad1D dy_ = quadratic_weights(y, a.inv_dy);
                const double wxs[3] = {dx_.w0, dx_.w1, dx_.w2};
                const double wys[3] = {dy_.w0, dy_.w1, dy_.w2};
                const double qa = q * a.inv_dA;
                if (NCOMP == 1) {
                    dval[0] = qa;
                } else {
                    dval[0] = qa * v0;
                    dval[1] = qa * v1;
                    dval[2] = qa * v2;
                    if (NCOMP == 4) dval[NCOMP - 1] = qa;
                }
                gx0 = wrap_index(dx_.ic - 1, nx);
                gy0 = wrap_index(dy_.ic - 1, ny);
                const int lx = tg.full_x ? gx0 : window_coord(dx_.ic - 1, ox, nx, tg.wx);
                const int ly = tg.full_y ? gy0 : window_coord(dy_.ic - 1, oy, ny, tg.wy);
                key = (lx < 0 || ly < 0) ? kKeyEscape : lx * tg.wy + ly;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    dwx[k] = wxs[k];
                    dwy[k] = wys[k];
                }
            }
            // Group the warp's particles by window key: groups in the order of
            // their first particle, particles in index order inside a group
            // (deterministic), escapes after all groups.
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
                // stage S_ab and q v_c / dA of this particle in its row
                double* mine = sprod + row * RW;
#pragma unroll
                for (int ia = 0; ia < 3; ++ia)
#pragma unroll
                    for (int ib = 0; ib < 3; ++ib) mine[ia * 3 + ib] = dwx[ia] * dwy[ib];
#pragma unroll
                for (int cc = 0; cc < NCOMP; ++cc) mine[9 + cc] = dval[cc];
            }
            __syncwarp();
            // Particles whose stencil leaves the window (rare): exact fixed-point
            // adds straight to the grid.
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
                            const double v = sprod[erow * RW + 9 + t_c[r]] * sprod[erow * RW + t_ab[r]];
                            if (v != 0.0) {
                                const int g = wrap_index(gxj + t_a[r], nx) * ny + wrap_index(gyj + t_b[r], ny);
                                const int sl = acc_slot(NCOMP, t_c[r]);
                                const Fixed2 f = to_fixed(v, t_scale[r]);
                                atomicAdd(&a.acc[(size_t)(2 * sl) * N + g], f.hi);
                                atomicAdd(&a.acc[(size_t)(2 * sl + 1) * N + g], f.lo);
                            }
                        }
                    }
                    ++erow;
                }
            }
            // Warp-level segmented reduction: lane t owns value t and sums it over
            // the rows of each key group (two interleaved partial sums, fixed
            // order); each group adds its sum to the window once per value.
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
                            double s0 = 0.0, s1 = 0.0;
                            // rows rs..re-1, two interleaved partial sums
                            const double* pv = sprod + rs * RW + 9 + t_c[r];
                            const double* pw = sprod + rs * RW + t_ab[r];
                            const double* const pe = sprod + re * RW + 9 + t_c[r];
                            for (; pv + RW < pe; pv += 2 * RW, pw += 2 * RW) {
                                s0 = fma(pv[0], pw[0], s0);
                                s1 = fma(pv[RW], pw[RW], s1);
                            }
                            if (pv < pe) s0 = fma(pv[0], pw[0], s0);
                            const double sum = s0 + s1;
                            if (sum != 0.0) {
                                int widx;
                                if (tg.full_x || tg.full_y) {
                                    const int kx = k / tg.wy, ky = k - kx * tg.wy;
                                    int nxl = kx + t_a[r], nyl = ky + t_b[r];
                                    if (tg.full_x) nxl &= tg.wx - 1;
                                    if (tg.full_y) nyl &= tg.wy - 1;
                                    widx = nxl * tg.wy + nyl;
                                } else {
                                    widx = k + t_off[r];
                                }
                                const Fixed2 f = to_fixed(sum, t_scale[r]);
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
    __syncthreads();
    if (cur_tile >= 0) fold_window<NCOMP>(whi, wlo, WN, tg, ox, oy, a.acc);
    // particle reductions: fixed order (lanes, then warps in index order)
    if (a.diag_part) {
        kin = warp_sum_dd(kin);
        gsum = warp_sum_dd(gsum);
        const double vmax = warp_max(sqrt(vmax2));
        __syncthreads();
        double* red = reinterpret_cast<double*>(smem_u64);
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
            for (int w = 0; w < kPushWarps; ++w) {
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

// acc -> doubles, then clear (kept on device for the next deposit).
__global__ void convert_acc_kernel(unsigned long long* acc, int N, double s0, double s1, double s2,
                                   double s3, double* J, double* rho, double n0, int mask,
                                   const double* bg) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        if (mask & 1) {
            const double sc[3] = {s0, s1, s2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                unsigned long long* h = acc + (size_t)(2 * c) * N;
                unsigned long long* l = acc + (size_t)(2 * c + 1) * N;
                J[(size_t)c * N + id] = from_fixed(h[id], l[id], 1.0 / sc[c]);
                h[id] = 0ull;
                l[id] = 0ull;
            }
        }
        if (mask & 2) {
            unsigned long long* h = acc + (size_t)6 * N;
            unsigned long long* l = acc + (size_t)7 * N;
            rho[id] = (bg ? bg[id] : n0) + from_fixed(h[id], l[id], 1.0 / s3);
            h[id] = 0ull;
            l[id] = 0ull;
        }
    }
}

UPIC_D double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
UPIC_D double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
UPIC_D double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// i*k*z
UPIC_D double2 cik(double k, double2 z) { return make_double2(-k * z.y, k * z.x); }

// k-space BDF step: continuity / naive charge, BDF Helmholtz solves for phi
// and A (spectral_pic_part3.cpp:829-880, 1147-1164), spectra of the eleven
// gathered fields (:1166-1168).
__global__ void bdf_kspace_kernel(KspaceArgs a) {
    const int N = a.N;
    const double scale = 1.0 / (a.c * a.c * a.dt * a.dt);
    const int snew = (a.head + a.R - 1) % a.R;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double kx = a.kx[id], ky = a.ky[id];
        const double denom = scale * a.b[0] + a.k2[id];
        const double2 J0 = a.Jhat[id], J1 = a.Jhat[N + id], J2 = a.Jhat[2 * (size_t)N + id];
        auto H = [&](int field, int past) -> double2 {
            const int slot = (a.head + past) % a.R;
            return a.hist[((size_t)field * a.R + slot) * N + id];
        };
        double2 rho_new;
        if (a.conserving) {
            const double2 div = cik(1.0, make_double2(kx * J0.x + ky * J1.x, kx * J0.y + ky * J1.y));
            double2 hs = make_double2(0.0, 0.0);
            for (int l = 1; l < a.na; ++l) hs = cadd(hs, cscale(a.a[l], H(4, l - 1)));
            const double2 num = cadd(cscale(a.dt, div), hs);
            rho_new = make_double2(-num.x / a.a[0], -num.y / a.a[0]);
        } else {
            rho_new = a.rho_dep[id];
        }
        // phi: (b0 s + k^2) phi = rho/eps0 - s sum b_l phi^{n+1-l}
        double2 rhs = make_double2(rho_new.x / a.eps0, rho_new.y / a.eps0);
        for (int l = 1; l < a.nb; ++l) rhs = csub(rhs, cscale(scale * a.b[l], H(0, l - 1)));
        const double2 phi = make_double2(rhs.x / denom, rhs.y / denom);
        double2 A[3];
        const double2 J[3] = {J0, J1, J2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double2 r = cscale(a.mu0, J[c]);
            for (int l = 1; l < a.nb; ++l) r = csub(r, cscale(scale * a.b[l], H(1 + c, l - 1)));
            A[c] = make_double2(r.x / denom, r.y / denom);
        }
        a.hist[((size_t)0 * a.R + snew) * N + id] = phi;
        for (int c = 0; c < 3; ++c) a.hist[((size_t)(1 + c) * a.R + snew) * N + id] = A[c];
        a.hist[((size_t)4 * a.R + snew) * N + id] = rho_new;
        if (a.gspec) {
            double2* g = a.gspec;
            g[0 * (size_t)N + id] = A[0];
            g[1 * (size_t)N + id] = A[1];
            g[2 * (size_t)N + id] = A[2];
            g[3 * (size_t)N + id] = cik(kx, phi);
            g[4 * (size_t)N + id] = cik(ky, phi);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                g[(5 + 2 * c) * (size_t)N + id] = cik(kx, A[c]);
                g[(6 + 2 * c) * (size_t)N + id] = cik(ky, A[c]);
            }
        }
    }
}

// Diagnostics spectra (spectral_pic_part3.cpp:902-948): gauge, E, gauss,
// continuity, B = curl A, rho, using BDF first derivatives of the histories.
__global__ void diag_kspace_kernel(DiagKArgs a) {
    const int N = a.N;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double kx = a.kx[id], ky = a.ky[id];
        auto H = [&](int field, int slot) -> double2 {
            return a.hist[((size_t)field * a.R + slot) * N + id];
        };
        auto ddt = [&](int field) -> double2 {
            double2 r = cscale(a.a[0], H(field, a.slot_new));
            for (int l = 1; l < a.na; ++l) r = cadd(r, cscale(a.a[l], H(field, (a.slot_prev0 + l - 1) % a.R)));
            return make_double2(r.x / a.dt, r.y / a.dt);
        };
        const double2 phi = H(0, a.slot_new);
        const double2 Ax = H(1, a.slot_new), Ay = H(2, a.slot_new), Az = H(3, a.slot_new);
        const double2 rho = H(4, a.slot_new);
        const double2 phit = ddt(0);
        const double2 divA = cik(1.0, make_double2(kx * Ax.x + ky * Ay.x, kx * Ax.y + ky * Ay.y));
        const double c2 = a.c * a.c;
        const double2 gauge = cadd(make_double2(phit.x / c2, phit.y / c2), divA);
        const double2 Atx = ddt(1), Aty = ddt(2), Atz = ddt(3);
        const double2 gpx = cik(kx, phi), gpy = cik(ky, phi);
        const double2 Ex = make_double2(-gpx.x - Atx.x, -gpx.y - Atx.y);
        const double2 Ey = make_double2(-gpy.x - Aty.x, -gpy.y - Aty.y);
        const double2 Ez = make_double2(-Atz.x, -Atz.y);
        const double2 divE = cik(1.0, make_double2(kx * Ex.x + ky * Ey.x, kx * Ex.y + ky * Ey.y));
        const double2 gauss = csub(divE, make_double2(rho.x / a.eps0, rho.y / a.eps0));
        const double2 J0 = a.Jhat[id], J1 = a.Jhat[N + id];
        const double2 divJ = cik(1.0, make_double2(kx * J0.x + ky * J1.x, kx * J0.y + ky * J1.y));
        const double2 cont = cadd(ddt(4), divJ);
        const double2 Bx = cik(ky, Az);
        const double2 gAzx = cik(kx, Az);
        const double2 By = make_double2(-gAzx.x, -gAzx.y);
        const double2 Bz = csub(cik(kx, Ay), cik(ky, Ax));
        double2* o = a.out;
        o[0 * (size_t)N + id] = gauge;
        o[1 * (size_t)N + id] = Ex;
        o[2 * (size_t)N + id] = Ey;
        o[3 * (size_t)N + id] = Ez;
        o[4 * (size_t)N + id] = gauss;
        o[5 * (size_t)N + id] = cont;
        o[6 * (size_t)N + id] = Bx;
        o[7 * (size_t)N + id] = By;
        o[8 * (size_t)N + id] = Bz;
        o[9 * (size_t)N + id] = rho;
    }
}

constexpr int kRedThreads = 256;
constexpr int kNSums = 8;  // gauge, gauss, cont, Bz, B, E, rho, J

__global__ void __launch_bounds__(kRedThreads) diag_reduce_kernel(DiagReduceArgs a) {
    const int N = a.N;
    const double* f = a.dfields;
    DD s[kNSums];
#pragma unroll
    for (int k = 0; k < kNSums; ++k) s[k] = DD{0.0, 0.0};
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double gauge = f[id], Ex = f[N + id], Ey = f[2 * (size_t)N + id];
        const double Ez = f[3 * (size_t)N + id], gauss = f[4 * (size_t)N + id];
        const double cont = f[5 * (size_t)N + id], Bx = f[6 * (size_t)N + id];
        const double By = f[7 * (size_t)N + id], Bz = f[8 * (size_t)N + id];
        const double rho = f[9 * (size_t)N + id];
        const double Jx = a.J[id], Jy = a.J[N + id], Jz = a.J[2 * (size_t)N + id];
        s[0] = dd_add_dd(s[0], dd_sq(gauge));
        s[1] = dd_add_dd(s[1], dd_sq(gauss));
        s[2] = dd_add_dd(s[2], dd_sq(cont));
        s[3] = dd_add_dd(s[3], dd_sq(Bz));
        s[4] = dd_add_dd(dd_add_dd(dd_add_dd(s[4], dd_sq(Bx)), dd_sq(By)), dd_sq(Bz));
        s[5] = dd_add_dd(dd_add_dd(dd_add_dd(s[5], dd_sq(Ex)), dd_sq(Ey)), dd_sq(Ez));
        s[6] = dd_add_dd(s[6], dd_sq(rho));
        s[7] = dd_add_dd(dd_add_dd(dd_add_dd(s[7], dd_sq(Jx)), dd_sq(Jy)), dd_sq(Jz));
    }
    __shared__ double red[kRedThreads / kWarp][kNSums * 2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kNSums; ++k) {
        s[k] = warp_sum_dd(s[k]);
        if (lane == 0) {
            red[warp][2 * k] = s[k].hi;
            red[warp][2 * k + 1] = s[k].lo;
        }
    }
    __syncthreads();
    if (threadIdx.x < kNSums) {
        DD t{0.0, 0.0};
        for (int w = 0; w < kRedThreads / kWarp; ++w)
            t = dd_add_dd(t, DD{red[w][2 * threadIdx.x], red[w][2 * threadIdx.x + 1]});
        a.partials[(size_t)blockIdx.x * 16 + 2 * threadIdx.x] = t.hi;
        a.partials[(size_t)blockIdx.x * 16 + 2 * threadIdx.x + 1] = t.lo;
    }
}

// Final reduction in a fixed order: lane l sums blocks l, l+32, ... and the
// 32 lane sums are combined by a fixed butterfly; then thread 0 forms the row.
__global__ void diag_final_kernel(DiagReduceArgs a) {
    const int lane = threadIdx.x;
    __shared__ double sums[kNSums + 2][2];
    __shared__ double svmax;
    for (int k = 0; k < kNSums; ++k) {
        DD s{0.0, 0.0};
        for (int b = lane; b < a.grid; b += 32)
            s = dd_add_dd(s, DD{a.partials[b * 16 + 2 * k], a.partials[b * 16 + 2 * k + 1]});
        s = warp_sum_dd(s);
        if (lane == 0) { sums[k][0] = s.hi; sums[k][1] = s.lo; }
    }
    DD kin{0.0, 0.0}, gs{0.0, 0.0};
    double vmax = 0.0;
    for (int b = lane; b < a.pcount; b += 32) {
        const double* p = a.pdiag + (size_t)b * kDiagPart;
        kin = dd_add_dd(kin, DD{p[0], p[1]});
        gs = dd_add_dd(gs, DD{p[2], p[3]});
        vmax = fmax(vmax, p[4]);
    }
    kin = warp_sum_dd(kin);
    gs = warp_sum_dd(gs);
    vmax = warp_max(vmax);
    if (lane == 0) {
        sums[kNSums][0] = kin.hi; sums[kNSums][1] = kin.lo;
        sums[kNSums + 1][0] = gs.hi; sums[kNSums + 1][1] = gs.lo;
        svmax = vmax;
    }
    __syncwarp();
    if (lane != 0) return;
    const double invN = 1.0 / (double)a.N;
    auto tot = [&](int k) { return sums[k][0] + sums[k][1]; };
    double* r = a.row;
    for (int k = 0; k < kNSums; ++k) r[k] = sqrt(tot(k) * invN);
    r[8] = 0.5 * a.eps0 * (tot(5) * a.dA) + 0.5 / a.mu0 * (tot(4) * a.dA);
    r[9] = tot(kNSums);
    r[10] = r[8] + r[9];
    r[11] = svmax;
    r[12] = a.np > 0 ? tot(kNSums + 1) / (double)a.np : 0.0;
}

__global__ void poisson_kspace_kernel(int N, const double* k2, const double2* rh, double eps0,
                                      double2* out) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double kk = k2[id];
        if (kk > 0.0) {
            const double d = eps0 * kk;
            out[id] = make_double2(rh[id].x / d, rh[id].y / d);
        } else {
            out[id] = make_double2(0.0, 0.0);
        }
    }
}

__global__ void derivative_kspace_kernel(int N, const double* k, const double2* in, double2* out) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x)
        out[id] = cik(k[id], in[id]);
}

__global__ void bdf_single_kernel(int N, const double* k2, const double2* src, const double2* hist,
                                  int nb, double b0, double b1, double b2, double b3, double b4,
                                  double scale, double2* out) {
    const double b[5] = {b0, b1, b2, b3, b4};
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        double2 r = src[id];
        for (int l = 1; l < nb; ++l) r = csub(r, cscale(scale * b[l], hist[(size_t)(l - 1) * N + id]));
        const double d = scale * b[0] + k2[id];
        out[id] = make_double2(r.x / d, r.y / d);
    }
}

__global__ void gather_scalar_kernel(int nx, int ny, double inv_dx, double inv_dy, const double* f,
                                     long np, const double* x, const double* y, double* out) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        const Quad1D qx = quadratic_weights(x[p], inv_dx);
        const Quad1D qy = quadratic_weights(y[p], inv_dy);
        const double wxs[3] = {qx.w0, qx.w1, qx.w2};
        const double wys[3] = {qy.w0, qy.w1, qy.w2};
        double v = 0.0;
        for (int ia = 0; ia < 3; ++ia) {
            const int gx = wrap_index(qx.ic - 1 + ia, nx);
            for (int ib = 0; ib < 3; ++ib) {
                const int gy = wrap_index(qy.ic - 1 + ib, ny);
                v = fma(f[gx * ny + gy], wxs[ia] * wys[ib], v);
            }
        }
        out[p] = v;
    }
}

__global__ void fill_hist_kernel(double2* h, int R, int N, const double2* src) {
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x) {
        const double2 v = src[id];
        for (int s = 0; s < R; ++s) h[(size_t)s * N + id] = v;
    }
}

int grid_for(long n, int threads) {
    long g = (n + threads - 1) / threads;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return (int)g;
}

template <int MODE, int NCOMP, bool UNIFORM>
cudaError_t launch_one(const TileGeom& tg, const PushArgs& a, int grid, cudaStream_t st) {
    const int smem = push_deposit_smem_bytes(tg, NCOMP);
    push_deposit_kernel<MODE, NCOMP, UNIFORM><<<grid, kPushThreads, smem, st>>>(a, tg);
    count_launches(1);
    return cudaGetLastError();
}

template <int MODE, int NCOMP, bool UNIFORM>
cudaError_t set_smem_one(int bytes) {
    return raise_smem_limit(reinterpret_cast<const void*>(push_deposit_kernel<MODE, NCOMP, UNIFORM>), bytes);
}

}  // namespace

cudaError_t raise_smem_limit(const void* func, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int& cur = limit[{func, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

static long g_launches = 0;
void count_launches(long n) { __atomic_fetch_add(&g_launches, n, __ATOMIC_RELAXED); }
long launches_total() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int push_deposit_smem_bytes(const TileGeom& tg, int ncomp) {
    const int WN = tg.wx * tg.wy;
    const int window = 2 * ncomp * WN * 8;
    const int stage = kPushWarps * (32 * (9 + ncomp) * 8 + 32 * 4);
    int bytes = window + stage;
#if UPIC_PUSH_SMEM_GATHER
    bytes += 16 + WN * kGFStride * 8;
#endif
    const int red = kPushWarps * 5 * 8;
    return bytes > red ? bytes : red;
}

cudaError_t push_configure_smem(const TileGeom& tg) {
    cudaError_t e = cudaSuccess;
#define UPIC_SET(MODE, NC, U)                                                   \
    e = set_smem_one<MODE, NC, U>(push_deposit_smem_bytes(tg, NC));              \
    if (e != cudaSuccess) return e;
    UPIC_SET(kModeDeposit, 1, true) UPIC_SET(kModeDeposit, 1, false)
    UPIC_SET(kModeDeposit, 3, true) UPIC_SET(kModeDeposit, 3, false)
    UPIC_SET(kModeDeposit, 4, true) UPIC_SET(kModeDeposit, 4, false)
    UPIC_SET(kModeAdvanceDeposit, 3, true) UPIC_SET(kModeAdvanceDeposit, 3, false)
    UPIC_SET(kModeAdvanceDeposit, 4, true) UPIC_SET(kModeAdvanceDeposit, 4, false)
    UPIC_SET(kModePush, 3, true) UPIC_SET(kModePush, 3, false)
    UPIC_SET(kModePush, 4, true) UPIC_SET(kModePush, 4, false)
#undef UPIC_SET
    return e;
}

int push_occupancy(const TileGeom& tg, int ncomp) {
    int n = 0;
    if (ncomp == 4)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, push_deposit_kernel<kModePush, 4, true>, kPushThreads,
                                                      push_deposit_smem_bytes(tg, 4));
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, push_deposit_kernel<kModePush, 3, true>, kPushThreads,
                                                      push_deposit_smem_bytes(tg, 3));
    return n;
}

// IAEM momentum push of a particle list in given fields
// (push_particles_momentum_and_velocity, spectral_pic_part3.cpp:1057-1090):
// quadratic gathers of A, grad phi and grad A at (x, y), P += q dt
// (-grad phi + (grad A) . v*), v* = 2 v - v_prev, then v from the canonical
// momentum (velocity_from_canonical :602).  F: 11 planar fields A (3),
// grad phi (2), dAx/dx, dAx/dy, dAy/dx, dAy/dy, dAz/dx, dAz/dy.  P, v,
// v_prev: xyz triples, updated in place.
__global__ void iaem_push_kernel(long np, const double* __restrict__ x, const double* __restrict__ y,
                                 double* __restrict__ P, double* __restrict__ v, double* __restrict__ vp,
                                 const double* __restrict__ q, const double* __restrict__ m,
                                 const double* __restrict__ F, int nx, int ny, double inv_dx, double inv_dy,
                                 double dt, double c) {
    const int N = nx * ny;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        const Quad1D qx = quadratic_weights(x[p], inv_dx);
        const Quad1D qy = quadratic_weights(y[p], inv_dy);
        const double wx[3] = {qx.w0, qx.w1, qx.w2}, wy[3] = {qy.w0, qy.w1, qy.w2};
        double G[11];
        for (int f = 0; f < 11; ++f) G[f] = 0.0;
        for (int a = 0; a < 3; ++a) {
            const int gx = wrap_index(qx.ic - 1 + a, nx);
            for (int b = 0; b < 3; ++b) {
                const int node = gx * ny + wrap_index(qy.ic - 1 + b, ny);
                for (int f = 0; f < 11; ++f) G[f] += F[(size_t)f * N + node] * wx[a] * wy[b];
            }
        }
        const double vs[3] = {2.0 * v[3 * p] - vp[3 * p], 2.0 * v[3 * p + 1] - vp[3 * p + 1],
                              2.0 * v[3 * p + 2] - vp[3 * p + 2]};
        const double gv[2] = {G[5] * vs[0] + G[7] * vs[1] + G[9] * vs[2], G[6] * vs[0] + G[8] * vs[1] + G[10] * vs[2]};
        const double force[3] = {-G[3] + gv[0], -G[4] + gv[1], 0.0};
        const double qdt = q[p] * dt;
        double Pn[3], pm[3];
        for (int k = 0; k < 3; ++k) {
            Pn[k] = P[3 * p + k] + qdt * force[k];
            pm[k] = Pn[k] - q[p] * G[k];
        }
        const double mc2 = m[p] * c * c;
        const double den = sqrt(c * c * (pm[0] * pm[0] + pm[1] * pm[1] + pm[2] * pm[2]) + mc2 * mc2);
        const double s = den == 0.0 ? 0.0 : c * c / den;
        for (int k = 0; k < 3; ++k) {
            vp[3 * p + k] = v[3 * p + k];
            v[3 * p + k] = s * pm[k];
            P[3 * p + k] = Pn[k];
        }
    }
}

cudaError_t launch_iaem_push(long np, const double* x, const double* y, double* P, double* v, double* vp,
                             const double* q, const double* m, const double* F, int nx, int ny, double inv_dx,
                             double inv_dy, double dt, double c, cudaStream_t st) {
    long g = (np + 127) / 128;
    if (g > 148 * 16) g = 148 * 16;
    iaem_push_kernel<<<(int)(g < 1 ? 1 : g), 128, 0, st>>>(np, x, y, P, v, vp, q, m, F, nx, ny, inv_dx, inv_dy, dt,
                                                           c);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_push_deposit(int mode, int ncomp, bool uniform, const TileGeom& tg,
                                const PushArgs& a, int grid, cudaStream_t st) {
#define UPIC_CASE(MODE, NC)                                                     \
    if (mode == MODE && ncomp == NC)                                            \
        return uniform ? launch_one<MODE, NC, true>(tg, a, grid, st)            \
                       : launch_one<MODE, NC, false>(tg, a, grid, st);
    UPIC_CASE(kModeDeposit, 1)
    UPIC_CASE(kModeDeposit, 3)
    UPIC_CASE(kModeDeposit, 4)
    UPIC_CASE(kModeAdvanceDeposit, 3)
    UPIC_CASE(kModeAdvanceDeposit, 4)
    UPIC_CASE(kModePush, 3)
    UPIC_CASE(kModePush, 4)
#undef UPIC_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_convert_acc(unsigned long long* acc, int N, const double* scale, double* J,
                               double* rho, double n0, int mask, cudaStream_t st, const double* bg) {
    convert_acc_kernel<<<grid_for(N, 256), 256, 0, st>>>(acc, N, scale[0], scale[1], scale[2],
                                                         scale[3], J, rho, n0, mask, bg);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bdf_kspace(const KspaceArgs& a, cudaStream_t st) {
    bdf_kspace_kernel<<<grid_for(a.N, 256), 256, 0, st>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_diag_kspace(const DiagKArgs& a, cudaStream_t st) {
    diag_kspace_kernel<<<grid_for(a.N, 256), 256, 0, st>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_diag_reduce(const DiagReduceArgs& a, cudaStream_t st) {
    diag_reduce_kernel<<<a.grid, kRedThreads, 0, st>>>(a);
    diag_final_kernel<<<1, 32, 0, st>>>(a);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_poisson_kspace(int N, const double* k2, const double2* rho_hat, double eps0,
                                  double2* out, cudaStream_t st) {
    poisson_kspace_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, k2, rho_hat, eps0, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_derivative_kspace(int N, const double* k, const double2* in, double2* out,
                                     cudaStream_t st) {
    derivative_kspace_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, k, in, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bdf_single(int N, const double* k2, const double2* src, const double2* hist,
                              int nb, const double* b, double scale, double2* out,
                              cudaStream_t st) {
    bdf_single_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, k2, src, hist, nb, b[0], b[1], b[2], b[3],
                                                        b[4], scale, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gather_scalar(int nx, int ny, double inv_dx, double inv_dy, const double* f,
                                 long np, const double* x, const double* y, double* out,
                                 cudaStream_t st) {
    gather_scalar_kernel<<<grid_for(np, 256), 256, 0, st>>>(nx, ny, inv_dx, inv_dy, f, np, x, y, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_fill_hist(double2* h, int R, int N, const double2* src, cudaStream_t st) {
    fill_hist_kernel<<<grid_for(N, 256), 256, 0, st>>>(h, R, N, src);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace upic
