// C-ABI implementation (include/upic.h): device context, memory layout and
// the explicit BDF/IAEM step driver.
//
// HBM layout of a context (N = nx*ny nodes, np particles):
//   particles   2 x SoA {x, y, Px, Py, Pz, vx, vy, vz, wx, wy, wz (v_prev), id
//               [, q, m when not uniform]}: the active set and a sort target
//   acc         8 x N uint64: fixed-point (hi, lo) accumulators for J (3) and rho
//   J, rho      3 x N, N doubles: current deposit of this time level
//   gf          12 x N doubles: interleaved gather records (A, grad phi, grad A)
//   spec        16 x N complex: J^ (3), deposited rho^ (1), gather spectra (11)
//   hist        5 fields x 5 slots x N complex: phi^, A^ (3), rho^ ring buffers
//   dspec/dreal 10 x N complex / real: diagnostics fields
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "upic_common.cuh"

#include "context.h"

using namespace upic;
using namespace upic_host;

namespace {
thread_local std::string g_create_error;
}  // namespace

namespace upic_host {

int fail(upic_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

int dalloc_bytes(upic_ctx* c, void** p, size_t bytes) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, bytes);
    if (e != cudaSuccess)
        return fail(c, UPIC_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    c->allocs.push_back(v);
    *p = v;
    return 0;
}

void dfree(upic_ctx* c, void* p) {
    if (!p) return;
    for (auto& a : c->allocs)
        if (a == p) {
            cudaFree(p);
            a = nullptr;
        }
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Integer Fourier mode of FFT index i on an n-point axis.
enum ModeConvention {
    kModesP2,        // spectral_pic_part3.cpp:320-330: Nyquist zeroed (n = 1 gives -1)
    kModesP3,        // ec_pic_nyquist_projected.cpp:1485-1504: Nyquist zeroed, n = 1 gives 0
    kModesKeepNyq    // ec_pic_serial_demo.cpp:385-391: Nyquist kept as +n/2, n = 1 gives 0
};
int mode_number(int i, int n, ModeConvention conv = kModesP2) {
    if (conv != kModesP2 && n == 1) return 0;
    if (conv == kModesKeepNyq) return (i <= n / 2) ? i : i - n;
    if (n > 1 && i == n / 2) return 0;
    return (i < n / 2) ? i : i - n;
}

std::vector<double2> twiddles(int n) {
    std::vector<double2> t(n > 1 ? n / 2 : 1);
    for (int m = 0; m < (int)t.size(); ++m) {
        const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
        t[m] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return t;
}

// A tiled axis' window covers the nodes that the stencils of particles in
// the tile, or up to `guard` cells outside it, can touch: `lo` nodes below
// and `hi` nodes above a particle's key cell.  An axis whose window would
// cover the whole axis becomes one periodic window.
TileGeom make_tiles(int nx, int ny, int tile, int guard, int lo, int hi) {
    TileGeom g{};
    g.nx = nx;
    g.ny = ny;
    g.guard = guard;
    g.lo = lo;
    g.span = lo + hi + 1;
    auto axis = [&](int n, int& t, int& nt, int& w, int& full) {
        t = tile < n ? tile : n;
        const int wt = t + 2 * guard + lo + hi;
        if (n <= wt) {
            full = 1;
            t = n;
            w = n;
        } else {
            full = 0;
            w = wt;
        }
        nt = n / t;
    };
    axis(nx, g.tile_x, g.ntx, g.wx, g.full_x);
    axis(ny, g.tile_y, g.nty, g.wy, g.full_y);
    g.chunk = 2048;
    g.key_origin_x = 0.0;
    g.key_origin_y = 0.0;
    g.key_shift = 0.5;
    return g;
}

int iota(upic_ctx* c, int* id, long n);

int choose_chunk(long np, int grid, int max_chunk) {
    long t = (np + grid - 1) / (grid > 0 ? grid : 1);
    t = (t + kMinChunk - 1) / kMinChunk * kMinChunk;
    if (t < kMinChunk) t = kMinChunk;
    if (t > max_chunk) t = max_chunk;
    return (int)t;
}

int alloc_soa(upic_ctx* c, ParticleSoA& s, long cap, bool with_state, bool with_qm) {
    int rc = 0;
    // two elements of padding: bulk prefetches widen their ranges to 16-byte
    // boundaries (explicit.cu prefetch_l2)
    cap += 2;
    double** arrs[] = {&s.x, &s.y, &s.vx, &s.vy, &s.vz};
    for (double** a : arrs)
        if ((rc = dalloc(c, a, cap))) return rc;
    if (with_state) {
        double** st[] = {&s.Px, &s.Py, &s.Pz, &s.wx, &s.wy, &s.wz};
        for (double** a : st)
            if ((rc = dalloc(c, a, cap))) return rc;
    }
    if (with_qm) {
        if ((rc = dalloc(c, &s.q, cap))) return rc;
        if ((rc = dalloc(c, &s.m, cap))) return rc;
    }
    return dalloc(c, &s.id, cap);
}

void free_soa(upic_ctx* c, ParticleSoA& s) {
    void* ps[] = {s.x, s.y, s.Px, s.Py, s.Pz, s.vx, s.vy, s.vz, s.wx, s.wy, s.wz, s.q, s.m, s.id};
    for (void* p : ps) dfree(c, p);
    s = ParticleSoA{};
}

int alloc_mixed(upic_ctx* c, MixedSoA& s, long cap, bool with_qm) {
    int rc;
    float** arrs[] = {&s.rx, &s.ry, &s.Px, &s.Py, &s.Pz, &s.vx, &s.vy, &s.vz, &s.wx, &s.wy, &s.wz};
    for (float** a : arrs)
        if ((rc = dalloc(c, a, cap))) return rc;
    if (with_qm && ((rc = dalloc(c, &s.q, cap)) || (rc = dalloc(c, &s.m, cap)))) return rc;
    if ((rc = dalloc(c, &s.cell, cap))) return rc;
    return dalloc(c, &s.id, cap);
}

void free_mixed(upic_ctx* c, MixedSoA& s) {
    void* ps[] = {s.cell, s.rx, s.ry, s.Px, s.Py, s.Pz, s.vx, s.vy, s.vz, s.wx, s.wy, s.wz, s.q, s.m, s.id};
    for (void* p : ps) dfree(c, p);
    s = MixedSoA{};
}

// Single-word fixed-point scale: 2^F with |sum| * 2^F < 2^59 for any sum
// bounded by `bound` (four bits of headroom in the int64).
double fixed_scale1(double bound) {
    if (!(bound > 0.0) || !std::isfinite(bound)) return 1.0;
    int e = 0;
    std::frexp(bound, &e);
    int F = 59 - e;
    if (F > 1000) F = 1000;
    if (F < -1000) F = -1000;
    return std::ldexp(1.0, F);
}

int alloc_sortwork(upic_ctx* c, SortWork& w, long cap, const TileGeom& tg) {
    int rc;
    if ((rc = dalloc(c, &w.keys, cap))) return rc;
    if ((rc = dalloc(c, &w.keys_alt, cap))) return rc;
    if ((rc = dalloc(c, &w.vals, cap))) return rc;
    if ((rc = dalloc(c, &w.vals_alt, cap))) return rc;
    const long nblocks = (cap + 4095) / 4096;
    const long hist = 256 * nblocks;
    if ((rc = dalloc(c, &w.hist, hist))) return rc;
    const long scan_blocks = (hist + 1023) / 1024 + 16;
    if ((rc = dalloc(c, &w.scan_tmp, scan_blocks))) return rc;
    const int ntiles = tg.ntx * tg.nty;
    if ((rc = dalloc(c, &w.tile_count, ntiles))) return rc;
    if ((rc = dalloc(c, &w.tile_start, ntiles + 1))) return rc;
    if ((rc = dalloc(c, &w.tile_chunks, ntiles))) return rc;
    // chunk table for the smallest chunk size choose_chunk picks
    const long chunks = cap / kMinChunk + ntiles + 1;
    if ((rc = dalloc(c, &w.chunks, chunks))) return rc;
    if ((rc = dalloc(c, &w.nchunks, 1))) return rc;
    w.cap = cap;
    return 0;
}

void free_sortwork(upic_ctx* c, SortWork& w) {
    void* ps[] = {w.keys, w.keys_alt, w.vals, w.vals_alt, w.hist, w.scan_tmp, w.tile_count,
                  w.tile_start, w.tile_chunks, w.chunks, w.nchunks};
    for (void* p : ps) dfree(c, p);
    w = SortWork{};
}

// Fixed-point scale 2^F with F = 91 - ceil(log2 B) for a node-value bound B.
double fixed_scale(double bound) {
    if (!(bound > 0.0) || !std::isfinite(bound)) return 1.0;
    int e = 0;
    std::frexp(bound, &e);  // bound < 2^e
    int F = 91 - e;  // two bits of headroom over the bound
    if (F > 1000) F = 1000;
    if (F < -1000) F = -1000;
    return std::ldexp(1.0, F);
}

int sync(upic_ctx* c) {
    UPIC_CUDA(c, cudaStreamSynchronize(c->st));
    return 0;
}

// Split host xyz triples into three device arrays.
__global__ void split3_kernel(const double* t, long n, double* a, double* b, double* c) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        a[i] = t[3 * i];
        b[i] = t[3 * i + 1];
        c[i] = t[3 * i + 2];
    }
}

__global__ void join3_kernel(double* t, long n, const double* a, const double* b, const double* c) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        t[3 * i] = a[i];
        t[3 * i + 1] = b[i];
        t[3 * i + 2] = c[i];
    }
}

__global__ void iota_kernel(int* id, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        id[i] = (int)i;
}

int iota(upic_ctx* c, int* id, long n) {
    if (n <= 0) return 0;
    iota_kernel<<<gridn(n), 256, 0, c->st>>>(id, n);
    count_launches(1);
    UPIC_CUDA(c, cudaGetLastError());
    return 0;
}

__global__ void interleave_kernel(const double* re, const double* im, double2* out, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = make_double2(re[i], im ? im[i] : 0.0);
}

__global__ void deinterleave_kernel(const double2* in, double* re, double* im, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        re[i] = in[i].x;
        if (im) im[i] = in[i].y;
    }
}

int gridn(long n) {
    long g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return g < 1 ? 1 : (int)g;
}

int upload3(upic_ctx* c, const double* host, long n, double* a, double* b, double* d) {
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_tmp3, host, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    split3_kernel<<<gridn(n), 256, 0, c->st>>>(c->d_tmp3, n, a, b, d);
    count_launches(1);
    UPIC_CUDA(c, cudaGetLastError());
    return 0;
}

int download3(upic_ctx* c, double* host, long n, const double* a, const double* b, const double* d) {
    join3_kernel<<<gridn(n), 256, 0, c->st>>>(c->d_tmp3, n, a, b, d);
    count_launches(1);
    UPIC_CUDA(c, cudaGetLastError());
    UPIC_CUDA(c, cudaMemcpyAsync(host, c->d_tmp3, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
    return 0;
}

#ifndef UPIC_DEVICE_SCAN
#define UPIC_DEVICE_SCAN 1
#endif

// Finiteness and speed bounds of an uploaded particle state (the x, y, v
// part of scan_particles, on the device copy): out[0] counts non-finite
// particles, out[1] and out[2] hold the bit patterns of the largest speed
// and velocity component (non-negative doubles order as their bits).  The
// speed is summed without fused multiply-adds, as the host scan sums it.
__global__ void scan_state_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                  const double* __restrict__ vx, const double* __restrict__ vy,
                                  const double* __restrict__ vz, long n, unsigned long long* out) {
    unsigned long long bad = 0;
    double smax = 0.0, cmax = 0.0;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
        const double a = vx[p], b = vy[p], c = vz[p];
        const double sp = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)));
        if (!isfinite(sp) || !isfinite(x[p]) || !isfinite(y[p])) {
            ++bad;
        } else {
            smax = fmax(smax, sp);
            cmax = fmax(cmax, fmax(fabs(a), fmax(fabs(b), fabs(c))));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
        smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(&out[0], bad);
        atomicMax(&out[1], (unsigned long long)__double_as_longlong(smax));
        atomicMax(&out[2], (unsigned long long)__double_as_longlong(cmax));
    }
}

// x == nullptr: q and m only (finite, speed_max and comp_max left as they are).
HostScan scan_particles(long np, const double* x, const double* y, const double* v, const double* q,
                        const double* m) {
    constexpr int kChunks = 64;
    HostScan part[kChunks];
    if (np <= 0) return HostScan{};
    const double q0 = q[0], m0 = m[0];
    auto run = [&](int k) {
        HostScan& h = part[k];
        const long b = np * k / kChunks, e = np * (k + 1) / kChunks;
        for (long p = b; p < e; ++p) {
            if (q[p] != q0 || m[p] != m0) h.uniform = false;
            if (!(m[p] > 0.0)) h.positive_m = false;
            h.qabs += std::fabs(q[p]);
            if (!x) continue;
            const double* vp = v + 3 * p;
            const double s = std::sqrt(vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]);
            if (!std::isfinite(s) || !std::isfinite(x[p]) || !std::isfinite(y[p])) h.finite = false;
            h.speed_max = std::max(h.speed_max, s);
            h.comp_max = std::max(h.comp_max, std::max(std::fabs(vp[0]), std::max(std::fabs(vp[1]), std::fabs(vp[2]))));
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = np < (1L << 20) ? 1 : (int)std::min<unsigned>(16u, hw ? hw : 1u);
    if (nt <= 1) {
        for (int k = 0; k < kChunks; ++k) run(k);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (int k = t; k < kChunks; k += nt) run(k);
            });
        for (auto& t : th) t.join();
    }
    HostScan r;
    for (int k = 0; k < kChunks; ++k) {
        r.finite = r.finite && part[k].finite;
        r.uniform = r.uniform && part[k].uniform;
        r.positive_m = r.positive_m && part[k].positive_m;
        r.qabs += part[k].qabs;
        r.speed_max = std::max(r.speed_max, part[k].speed_max);
        r.comp_max = std::max(r.comp_max, part[k].comp_max);
    }
    return r;
}

int ensure_tmp3(upic_ctx* c, long n) {
    static_assert(sizeof(long) == 8, "64-bit long expected");
    if (c->d_tmp3 && n <= c->cap && n <= c->kcap) return 0;
    long want = n;
    if (c->cap > want) want = c->cap;
    if (c->kcap > want) want = c->kcap;
    dfree(c, c->d_tmp3);
    c->d_tmp3 = nullptr;
    return dalloc(c, &c->d_tmp3, 3 * want);
}

bool is_bdf(int m) { return m == UPIC_METHOD_BDF1 || m == UPIC_METHOD_BDF2; }

void bdf_coeffs(int method, int& na, double* a, int& nb, double* b) {
    if (method == UPIC_METHOD_BDF2) {
        na = 3;
        a[0] = 1.5; a[1] = -2.0; a[2] = 0.5;
    } else {
        na = 2;
        a[0] = 1.0; a[1] = -1.0; a[2] = 0.0;
    }
    nb = 2 * na - 1;
    for (int i = 0; i < 5; ++i) b[i] = 0.0;
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < na; ++j) b[i + j] += a[i] * a[j];
}

PushArgs push_args(upic_ctx* c, const ParticleSoA& p, long np, bool uniform) {
    PushArgs a{};
    a.p = p;
    a.np = np;
    a.q0 = c->q0;
    a.m0 = c->m0;
    a.Lx = c->cfg.Lx;
    a.Ly = c->cfg.Ly;
    a.inv_dx = 1.0 / c->dx;
    a.inv_dy = 1.0 / c->dy;
    a.inv_dA = 1.0 / c->dA;
    a.inv_Lx = 1.0 / c->cfg.Lx;
    a.inv_Ly = 1.0 / c->cfg.Ly;
    a.dt = c->cfg.dt;
    a.c = c->cfg.c;
    a.inv_c2 = 1.0 / (c->cfg.c * c->cfg.c);
    a.gfields = c->d_gf;
    a.acc = c->d_acc;
    for (int k = 0; k < 4; ++k) a.scale[k] = c->scale[k];
    (void)uniform;
    return a;
}

// Diagnostics row of the current spectra (hist slot_new with derivatives
// against slot_prev0) into c->h_row.
int run_diag(upic_ctx* c, int slot_new, int slot_prev0, int na, const double* acoef) {
    DiagKArgs d{};
    d.N = c->N;
    d.kx = c->d_kx;
    d.ky = c->d_ky;
    d.k2 = c->d_k2;
    d.Jhat = c->d_spec;
    d.hist = c->d_hist;
    d.R = kHistSlots;
    d.slot_new = slot_new;
    d.slot_prev0 = slot_prev0;
    d.na = na;
    for (int k = 0; k < 3; ++k) d.a[k] = acoef[k];
    d.dt = c->cfg.dt;
    d.c = c->cfg.c;
    d.eps0 = c->cfg.eps0;
    d.out = c->d_dspec;
    UPIC_CUDA(c, launch_diag_kspace(d, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec, kDiagFields, 1, c->st, nullptr, 1, c->d_dreal));
    DiagReduceArgs r{};
    r.N = c->N;
    r.dfields = c->d_dreal;
    r.J = c->d_J;
    r.partials = c->d_partials;
    r.grid = kRedGrid;
    r.pdiag = c->d_pdiag;
    r.pcount = c->push_grid;
    r.np = c->np;
    r.dA = c->dA;
    r.eps0 = c->cfg.eps0;
    r.mu0 = c->cfg.mu0;
    r.row = c->d_row;
    UPIC_CUDA(c, launch_diag_reduce(r, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(c->h_row, c->d_row, sizeof(double) * UPIC_DIAG_COUNT,
                                 cudaMemcpyDeviceToHost, c->st));
    return 0;
}

// Sort the active particle set by the cell of wrap(x + shift v) and make the
// sorted copy active.
int sort_active(upic_ctx* c, double shift) {
    if (c->mixed) {
        const float sx = (float)(shift / c->dx), sy = (float)(shift / c->dy);
        UPIC_CUDA(c, sort_mixed_by_tile(c->tg, c->M[c->cur], c->np, c->lny, sx, sy, c->sw, c->st));
        UPIC_CUDA(c, permute_mixed(c->M[c->cur], c->M[1 - c->cur], c->np, c->sw, c->st));
        c->cur = 1 - c->cur;
        c->steps_since_sort = 0;
        return 0;
    }
    ParticleSoA& src = c->P[c->cur];
    ParticleSoA& dst = c->P[1 - c->cur];
    UPIC_CUDA(c, sort_particles_by_tile(c->tg, src, c->np, c->cfg.Lx, c->cfg.Ly, shift, c->sw, c->st));
    UPIC_CUDA(c, permute_particles(src, dst, c->np, c->sw, c->st));
    c->cur = 1 - c->cur;
    c->steps_since_sort = 0;
    return 0;
}

int launch_push_mixed_ctx(upic_ctx* c, int mode, int ncomp, long np, bool uniform, const SortWork& w,
                          double* pdiag) {
    MixedPushArgs a{};
    a.p = c->M[c->cur];
    a.np = np;
    a.q0f = (float)c->q0;
    a.m0f = (float)c->m0;
    a.m0 = c->m0;
    a.dt = (float)c->cfg.dt;
    a.dt_dx = (float)(c->cfg.dt / c->dx);
    a.dt_dy = (float)(c->cfg.dt / c->dy);
    a.c = (float)c->cfg.c;
    a.c2 = (float)(c->cfg.c * c->cfg.c);
    a.inv_dA = (float)(1.0 / c->dA);
    a.cd = c->cfg.c;
    a.inv_c2d = 1.0 / (c->cfg.c * c->cfg.c);
    a.lny = c->lny;
    a.gf = c->d_gf32;
    a.chunks = w.chunks;
    a.nchunks = w.nchunks;
    a.acc = c->d_acc;
    for (int k = 0; k < 4; ++k) a.scale[k] = c->scale[k];
    a.diag_part = pdiag;
    const bool prof = c->profiling && mode == kModePush;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof) {
        UPIC_CUDA(c, cudaEventCreate(&e0));
        UPIC_CUDA(c, cudaEventCreate(&e1));
        UPIC_CUDA(c, cudaEventRecord(e0, c->st));
    }
    UPIC_CUDA(c, launch_push_mixed(mode, ncomp, uniform, c->tg, a, c->push_grid, c->st));
    if (prof) {
        UPIC_CUDA(c, cudaEventRecord(e1, c->st));
        c->prof_events.emplace_back(e0, e1);
    }
    return 0;
}

int launch_push(upic_ctx* c, int mode, int ncomp, const ParticleSoA& p, long np, bool uniform,
                const SortWork& w, double* pdiag) {
    if (c->mixed) return launch_push_mixed_ctx(c, mode, ncomp, np, uniform, w, pdiag);
    PushArgs a = push_args(c, p, np, uniform);
    a.chunks = w.chunks;
    a.nchunks = w.nchunks;
    a.diag_part = pdiag;
    const bool prof = c->profiling && mode == kModePush;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof) {
        UPIC_CUDA(c, cudaEventCreate(&e0));
        UPIC_CUDA(c, cudaEventCreate(&e1));
        UPIC_CUDA(c, cudaEventRecord(e0, c->st));
    }
    UPIC_CUDA(c, launch_push_deposit(mode, ncomp, uniform, c->tg, a, c->push_grid, c->st));
    if (prof) {
        UPIC_CUDA(c, cudaEventRecord(e1, c->st));
        c->prof_events.emplace_back(e0, e1);
    }
    return 0;
}

void clear_profile(upic_ctx* c) {
    for (auto& e : c->prof_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    c->prof_events.clear();
}

int grid_ncomp(const upic_ctx* c) { return c->cfg.charge_update == UPIC_CHARGE_NAIVE ? 4 : 3; }

}  // namespace upic_host

// ===========================================================================
extern "C" {

int upic_abi_version(void) { return UPIC_ABI_VERSION; }

int upic_config_default(upic_config* cfg) {
    if (!cfg) return UPIC_ERR_ARGUMENT;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->nx = 32;
    cfg->ny = 32;
    cfg->Lx = 2.0 * kPi;
    cfg->Ly = 2.0 * kPi;
    cfg->dt = 0.05;
    cfg->method = UPIC_METHOD_BDF1;
    cfg->charge_update = UPIC_CHARGE_CONSERVING;
    cfg->c = 1.0;
    cfg->eps0 = 1.0;
    cfg->mu0 = 1.0;
    cfg->n0 = 1.0;
    cfg->precision = UPIC_PRECISION_FP64;
    cfg->sort_interval = 0;
    cfg->tile = 0;
    cfg->guard = -1;
    // implicit method: the Config defaults of ec_pic_nyquist_projected.cpp:837-1005
    cfg->Lz = 2.0 * kPi;
    cfg->kappa = 1.0;
    cfg->sigma1 = 1.0;
    cfg->sigma2 = 1.0;
    cfg->spline_order = 2;
    cfg->orbit_quad_order = 16;
    cfg->split_orbit_at_knots = 1;
    cfg->nyquist_projection = 0;
    cfg->nonlinear_solver = UPIC_SOLVER_ANDERSON;
    cfg->nonlinear_max_iter = 32;
    cfg->anderson_memory = 4;
    cfg->anderson_start = 2;
    cfg->local_max_iter = 24;
    cfg->nonlinear_rtol = 1.0e-12;
    cfg->nonlinear_atol = 1.0e-13;
    cfg->anderson_damping = 0.7;
    cfg->anderson_regularization = 1.0e-12;
    cfg->anderson_growth_limit = 1.2;
    cfg->local_rtol = 1.0e-11;
    cfg->local_atol = 1.0e-13;
    cfg->local_damping = 1.0;
    cfg->perturbation_mode = 1;
    // non-relativistic implicit method: ec_pic_serial_demo.cpp:232-301
    cfg->picard_tol = 1.0e-11;
    cfg->picard_max_iter = 16;
    cfg->final_consistency_sweep = 1;
    cfg->current_predictor = UPIC_PREDICTOR_PREVIOUS;
    cfg->local_warm_start = 0;
    cfg->selective_particle_fallback = 0;
    cfg->selective_particle_max_substeps = 64;
    cfg->learned_train_steps = 200;
    cfg->learned_train_iters = 4;
    cfg->learned_rate = 1.0e-3;
    cfg->learned_seed = 20261203ull;
    return UPIC_OK;
}

const char* upic_last_error(const upic_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int upic_create(const upic_config* cfg, upic_ctx** out) {
    if (!cfg || !out) return fail(nullptr, UPIC_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    // read_config validation (spectral_pic_part3.cpp:281-293)
    if (!pow2(cfg->nx) || !pow2(cfg->ny) || cfg->nx > 8192 || cfg->ny > 8192)
        return fail(nullptr, UPIC_ERR_CONFIG,
                    "the radix-2 FFT requires nx and ny to be powers of two (<= 8192)");
    const bool nonrel = cfg->method == UPIC_METHOD_CN_ORBIT_NONREL;
    const bool implicit = cfg->method == UPIC_METHOD_CN_ORBIT || nonrel;
    if (!is_bdf(cfg->method) && !implicit)
        return fail(nullptr, UPIC_ERR_CONFIG, "method must be bdf1, bdf2, cn_orbit or cn_orbit_nonrel");
    if (cfg->current_predictor == UPIC_PREDICTOR_LEARNED && cfg->method != UPIC_METHOD_CN_ORBIT)
        return fail(nullptr, UPIC_ERR_CONFIG, "the learned predictor needs method cn_orbit");
    if (nonrel) {
        // Config of ec_pic_serial_demo.cpp:232-301 and the checks of make_grid
        // / bspline (:396, :565)
        if (!(cfg->Lx > 0) || !(cfg->Ly > 0) || !(cfg->Lz > 0) || !(cfg->dt > 0) || !(cfg->c > 0) ||
            !(cfg->eps0 > 0) || !(cfg->mu0 > 0))
            return fail(nullptr, UPIC_ERR_CONFIG, "Lx, Ly, Lz, dt, c, eps0, mu0 must be positive");
        if (cfg->spline_order < 1 || cfg->spline_order > 4)
            return fail(nullptr, UPIC_ERR_CONFIG, "spline_order must be 1, 2, 3 or 4");
        if (cfg->orbit_quad_order < 1 || cfg->orbit_quad_order > 32)
            return fail(nullptr, UPIC_ERR_CONFIG, "orbit_quad_order must be in 1..32");
        if (cfg->picard_max_iter < 1) return fail(nullptr, UPIC_ERR_CONFIG, "picard_max_iter must be positive");
        if (!(cfg->picard_tol >= 0)) return fail(nullptr, UPIC_ERR_CONFIG, "picard_tol must be non-negative");
    } else if (implicit) {
        // validation of ec_pic_nyquist_projected.cpp read_config / make_grid
        if (!(cfg->Lx > 0) || !(cfg->Ly > 0) || !(cfg->Lz > 0) || !(cfg->dt > 0) || !(cfg->kappa > 0) ||
            !(cfg->sigma1 > 0) || !(cfg->sigma2 > 0))
            return fail(nullptr, UPIC_ERR_CONFIG, "Lx, Ly, Lz, dt, kappa, sigma1, sigma2 must be positive");
        if (cfg->spline_order < 1 || cfg->spline_order > 4)
            return fail(nullptr, UPIC_ERR_CONFIG, "spline_order must be 1, 2, 3 or 4");
        if (cfg->orbit_quad_order < 1 || cfg->orbit_quad_order > 32)
            return fail(nullptr, UPIC_ERR_CONFIG, "orbit_quad_order must be in 1..32");
        if (cfg->nonlinear_solver != UPIC_SOLVER_ANDERSON && cfg->nonlinear_solver != UPIC_SOLVER_PICARD)
            return fail(nullptr, UPIC_ERR_CONFIG, "nonlinear_solver must be anderson or picard");
        if (cfg->anderson_memory < 1 || cfg->anderson_memory > 4)
            return fail(nullptr, UPIC_ERR_CONFIG, "anderson_memory must be in 1..4");
        if (cfg->nonlinear_max_iter < 1 || cfg->local_max_iter < 1 || cfg->anderson_start < 0)
            return fail(nullptr, UPIC_ERR_CONFIG, "iteration limits must be positive");
        if (!(cfg->nonlinear_rtol >= 0) || !(cfg->nonlinear_atol >= 0) || !(cfg->local_rtol >= 0) ||
            !(cfg->local_atol >= 0) || !(cfg->nonlinear_rtol + cfg->nonlinear_atol > 0) ||
            !(cfg->local_rtol + cfg->local_atol > 0))
            return fail(nullptr, UPIC_ERR_CONFIG, "tolerances must be non-negative and not both zero");
        if (!(cfg->anderson_damping > 0) || !(cfg->local_damping > 0) || !(cfg->anderson_growth_limit > 0) ||
            !(cfg->anderson_regularization >= 0))
            return fail(nullptr, UPIC_ERR_CONFIG, "damping and growth limits must be positive");
        if (cfg->current_predictor != UPIC_PREDICTOR_PREVIOUS && cfg->current_predictor != UPIC_PREDICTOR_EXTRAPOLATED &&
            cfg->current_predictor != UPIC_PREDICTOR_LEARNED)
            return fail(nullptr, UPIC_ERR_CONFIG, "current_predictor must be previous, extrapolated or learned");
        if (cfg->current_predictor == UPIC_PREDICTOR_LEARNED) {
            if (cfg->learned_train_steps < 0 || cfg->learned_train_iters < 1 || !(cfg->learned_rate > 0))
                return fail(nullptr, UPIC_ERR_CONFIG,
                            "learned_train_steps >= 0, learned_train_iters >= 1 and learned_rate > 0 required");
        }
        {
            const int ms = cfg->selective_particle_max_substeps;
            if (ms < 1 || ms > 64 || (ms & (ms - 1)) != 0)
                return fail(nullptr, UPIC_ERR_CONFIG,
                            "selective particle fallback requires a power-of-two max_substeps in [1,64]");
        }
    } else {
        if (cfg->charge_update != UPIC_CHARGE_CONSERVING && cfg->charge_update != UPIC_CHARGE_NAIVE)
            return fail(nullptr, UPIC_ERR_CONFIG, "charge_update must be conserving or naive");
        if (!(cfg->Lx > 0) || !(cfg->Ly > 0) || !(cfg->dt > 0) || !(cfg->c > 0) || !(cfg->eps0 > 0) ||
            !(cfg->mu0 > 0))
            return fail(nullptr, UPIC_ERR_CONFIG, "Lx, Ly, dt, c, eps0, mu0 must be positive");
    }
    if (cfg->precision != UPIC_PRECISION_FP64 && !(cfg->precision == UPIC_PRECISION_MIXED && !implicit))
        return fail(nullptr, UPIC_ERR_CONFIG,
                    "precision must be fp64, or mixed with the explicit methods (bdf1, bdf2)");

    upic_ctx* c = new upic_ctx();
    c->cfg = *cfg;
    c->nx = cfg->nx;
    c->ny = cfg->ny;
    c->N = cfg->nx * cfg->ny;
    c->dx = cfg->Lx / cfg->nx;
    c->dy = cfg->Ly / cfg->ny;
    c->dA = c->dx * c->dy;
    // Defaults from a sweep on the 512x512, 256 e-/cell workload: re-sort
    // every 4 steps, 8x8-cell tiles, 2 guard cells.
    c->sort_interval = cfg->sort_interval > 0 ? cfg->sort_interval : 4;
    const int tile = cfg->tile > 0 ? cfg->tile : 8;
    const int guard = cfg->guard >= 0 ? cfg->guard : 2;
    c->tg = make_tiles(c->nx, c->ny, tile, guard, 1, 1);

    auto bail = [&](int rc) {
        g_create_error = c->err;
        upic_destroy(c);
        return rc;
    };
    int rc;
    if (cudaGetDevice(&c->device) != cudaSuccess)
        return bail(fail(c, UPIC_ERR_CUDA, "no CUDA device"));
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(c, UPIC_ERR_CUDA, "cudaStreamCreate failed"));
    c->st = c->own;
    c->mixed = cfg->precision == UPIC_PRECISION_MIXED;
    while ((1 << c->lny) < c->ny) ++c->lny;
    if (fft_configure_smem() != cudaSuccess || push_configure_smem(c->tg) != cudaSuccess ||
        (c->mixed && push_mixed_configure_smem(c->tg) != cudaSuccess))
        return bail(fail(c, UPIC_ERR_CUDA, "cudaFuncSetAttribute failed"));
    // persistent grid: as many push CTAs as fit on the GPU at once
    const int ncomp_step = cfg->charge_update == UPIC_CHARGE_NAIVE ? 4 : 3;
    const int occ = c->mixed ? push_mixed_occupancy(c->tg, ncomp_step) : push_occupancy(c->tg, ncomp_step);
    c->push_grid = c->nsm * (occ > 0 ? occ : 1);

    const int N = c->N;
    auto tw_x = twiddles(c->nx), tw_y = twiddles(c->ny);
    if ((rc = dalloc(c, &c->d_twx, tw_x.size())) || (rc = dalloc(c, &c->d_twy, tw_y.size())) ||
        (rc = dalloc(c, &c->d_kx, N)) || (rc = dalloc(c, &c->d_ky, N)) || (rc = dalloc(c, &c->d_k2, N)) ||
        (rc = dalloc(c, &c->d_acc, 8 * (size_t)N)) || (rc = dalloc(c, &c->d_J, 3 * (size_t)N)) ||
        (rc = dalloc(c, &c->d_rho, N)) || (rc = dalloc(c, &c->d_gf, (size_t)kGFStride * N)) ||
        (rc = dalloc(c, &c->d_spec, 16 * (size_t)N)) ||
        (rc = dalloc(c, &c->d_hist, 5 * (size_t)kHistSlots * N)) ||
        (rc = dalloc(c, &c->d_dspec, (size_t)kDiagFields * N)) ||
        (rc = dalloc(c, &c->d_dreal, (size_t)kDiagFields * N)) ||
        (rc = dalloc(c, &c->d_partials, (size_t)kRedGrid * 16)) ||
        (rc = dalloc(c, &c->d_pdiag, (size_t)c->push_grid * kDiagPart)) ||
        (rc = dalloc(c, &c->d_row, UPIC_DIAG_COUNT)) || (rc = dalloc(c, &c->d_scan, 3)) ||
        (c->mixed && (rc = dalloc(c, &c->d_gf32, (size_t)kGFStride * N))))
        return bail(rc);
    if (cudaMallocHost(&c->h_row, sizeof(double) * UPIC_DIAG_COUNT) != cudaSuccess ||
        cudaMallocHost(&c->h_scan, 3 * sizeof(unsigned long long)) != cudaSuccess)
        return bail(fail(c, UPIC_ERR_NOMEM, "cudaMallocHost failed"));
    std::vector<double> kx(N), ky(N), k2(N);
    const ModeConvention dconv = implicit ? kModesP3 : kModesP2;
    const ModeConvention lconv = nonrel ? kModesKeepNyq : dconv;
    for (int i = 0; i < c->nx; ++i) {
        const double kxi = 2.0 * kPi * (double)mode_number(i, c->nx, dconv) / cfg->Lx;
        const double kxf = 2.0 * kPi * (double)mode_number(i, c->nx, lconv) / cfg->Lx;
        for (int j = 0; j < c->ny; ++j) {
            const double kyj = 2.0 * kPi * (double)mode_number(j, c->ny, dconv) / cfg->Ly;
            const double kyf = 2.0 * kPi * (double)mode_number(j, c->ny, lconv) / cfg->Ly;
            const int id = i * c->ny + j;
            // First derivatives take the zeroed Nyquist wave number in every
            // method: Project1 keeps +n/2 but returns the real part of each
            // inverse transform, which removes the i k_Nyquist component.
            // Its k^2 (Poisson, wave step) keeps the Nyquist value.
            kx[id] = kxi;
            ky[id] = kyj;
            k2[id] = kxf * kxf + kyf * kyf;
        }
    }
    if (cudaMemcpy(c->d_twx, tw_x.data(), sizeof(double2) * tw_x.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->d_twy, tw_y.data(), sizeof(double2) * tw_y.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->d_kx, kx.data(), sizeof(double) * N, cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->d_ky, ky.data(), sizeof(double) * N, cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->d_k2, k2.data(), sizeof(double) * N, cudaMemcpyHostToDevice) ||
        cudaMemset(c->d_acc, 0, sizeof(unsigned long long) * 8 * (size_t)N))
        return bail(fail(c, UPIC_ERR_CUDA, "initial device copies failed"));
    c->plan.nx = c->nx;
    c->plan.ny = c->ny;
    c->plan.tw_x = c->d_twx;
    c->plan.tw_y = c->d_twy;
    if (implicit && (rc = implicit_create(c))) return bail(rc);
    *out = c;
    return UPIC_OK;
}

}  // extern "C"

// ---- state files -------------------------------------------------------------

namespace upic_host {

int state_bytes(upic_ctx* c, StateIO& io, void* host, size_t n) {
    if (n == 0) return 0;
    const size_t done = io.writing ? std::fwrite(host, 1, n, io.f) : std::fread(host, 1, n, io.f);
    if (done != n) return fail(c, UPIC_ERR_ARGUMENT, io.writing ? "state file write failed" : "state file truncated");
    return 0;
}

int state_device(upic_ctx* c, StateIO& io, void* dev, size_t n) {
    constexpr size_t kPiece = size_t(64) << 20;
    if (io.buf.size() < std::min(n, kPiece)) io.buf.resize(std::min(n, kPiece));
    char* d = static_cast<char*>(dev);
    for (size_t off = 0; off < n; off += kPiece) {
        const size_t k = std::min(kPiece, n - off);
        int rc;
        if (io.writing) {
            UPIC_CUDA(c, cudaMemcpyAsync(io.buf.data(), d + off, k, cudaMemcpyDeviceToHost, c->st));
            if ((rc = sync(c)) || (rc = state_bytes(c, io, io.buf.data(), k))) return rc;
        } else {
            if ((rc = state_bytes(c, io, io.buf.data(), k))) return rc;
            UPIC_CUDA(c, cudaMemcpyAsync(d + off, io.buf.data(), k, cudaMemcpyHostToDevice, c->st));
            if ((rc = sync(c))) return rc;
        }
    }
    return 0;
}

}  // namespace upic_host

namespace {

constexpr char kStateMagic[8] = {'U', 'P', 'I', 'C', 'S', 'T', 'A', 'T'};
constexpr unsigned kStateVersion = 1;

// Every configuration field that shapes the state or its evolution, as
// doubles (struct padding never enters the comparison).
std::vector<double> config_signature(const upic_config& f) {
    return {(double)f.nx, (double)f.ny, f.Lx, f.Ly, f.dt, (double)f.method, (double)f.charge_update, f.c, f.eps0,
            f.mu0, f.n0, (double)f.precision, (double)f.sort_interval, (double)f.tile, (double)f.guard, f.Lz,
            f.kappa, f.sigma1, f.sigma2, (double)f.spline_order, (double)f.orbit_quad_order,
            (double)f.split_orbit_at_knots, (double)f.nyquist_projection, (double)f.nonlinear_solver,
            (double)f.nonlinear_max_iter, (double)f.anderson_memory, (double)f.anderson_start,
            (double)f.local_max_iter, f.nonlinear_rtol, f.nonlinear_atol, f.anderson_damping,
            f.anderson_regularization, f.anderson_growth_limit, f.local_rtol, f.local_atol, f.local_damping,
            (double)f.perturbation_mode, f.picard_tol, (double)f.picard_max_iter,
            (double)f.final_consistency_sweep, (double)f.current_predictor, (double)f.local_warm_start,
            (double)f.selective_particle_fallback, (double)f.selective_particle_max_substeps,
            (double)f.learned_train_steps, (double)f.learned_train_iters, f.learned_rate,
            (double)(f.learned_seed >> 32), (double)(f.learned_seed & 0xFFFFFFFFull)};
}

// Everything the next explicit step reads: the particle set in its current
// (sorted) order with the chunk list of the last sort, the field spectra and
// BDF histories, the gathered field records, the deposit accumulators of the
// next step's current, the charge and current, and the step counters.
int explicit_state_io(upic_ctx* c, StateIO& io) {
    int rc;
    long np = c->np;
    int uniform = c->uniform_qm ? 1 : 0, ready = c->fields_ready ? 1 : 0, has_bg = c->d_bg ? 1 : 0;
    if ((rc = state_value(c, io, np)) || (rc = state_value(c, io, uniform)) || (rc = state_value(c, io, ready)) ||
        (rc = state_value(c, io, has_bg)) || (rc = state_value(c, io, c->q0)) || (rc = state_value(c, io, c->m0)) ||
        (rc = state_bytes(c, io, c->scale, sizeof(c->scale))) || (rc = state_value(c, io, c->head)) ||
        (rc = state_value(c, io, c->steps)) || (rc = state_value(c, io, c->steps_since_sort)))
        return rc;
    if (!io.writing) {
        if (np < 0 || np > 0x7fffffffL) return fail(c, UPIC_ERR_ARGUMENT, "state file: bad particle count");
        if (c->mixed && (np > c->cap || (!uniform && !c->M[0].q))) {
            free_mixed(c, c->M[0]);
            free_mixed(c, c->M[1]);
            free_sortwork(c, c->sw);
            const long cap = std::max(np, c->cap);
            if ((rc = alloc_mixed(c, c->M[0], cap + 2, !uniform)) || (rc = alloc_mixed(c, c->M[1], cap + 2, !uniform)) ||
                (rc = alloc_sortwork(c, c->sw, cap, c->tg)))
                return rc;
            c->cap = cap;
        } else if (!c->mixed && (np > c->cap || (!uniform && !c->P[0].q))) {
            free_soa(c, c->P[0]);
            free_soa(c, c->P[1]);
            free_sortwork(c, c->sw);
            const long cap = std::max(np, c->cap);
            if ((rc = alloc_soa(c, c->P[0], cap, true, !uniform)) ||
                (rc = alloc_soa(c, c->P[1], cap, true, !uniform)) || (rc = alloc_sortwork(c, c->sw, cap, c->tg)))
                return rc;
            c->cap = cap;
        }
        if ((rc = ensure_tmp3(c, np))) return rc;
        if (has_bg && !c->d_bg && (rc = dalloc(c, &c->d_bg, c->N))) return rc;
        c->cur = 0;
        c->np = np;
        c->uniform_qm = uniform != 0;
        c->fields_ready = ready != 0;
    }
    if (c->mixed) {
        MixedSoA& p = c->M[c->cur];
        const size_t fb = sizeof(float) * np;
        float* arrs[] = {p.rx, p.ry, p.Px, p.Py, p.Pz, p.vx, p.vy, p.vz, p.wx, p.wy, p.wz};
        for (float* a : arrs)
            if ((rc = state_device(c, io, a, fb))) return rc;
        if ((rc = state_device(c, io, p.cell, sizeof(int) * np)) || (rc = state_device(c, io, p.id, sizeof(int) * np)))
            return rc;
        if (!uniform && ((rc = state_device(c, io, p.q, fb)) || (rc = state_device(c, io, p.m, fb)))) return rc;
    } else {
        ParticleSoA& p = c->P[c->cur];
        const size_t pb = sizeof(double) * np;
        double* arrs[] = {p.x, p.y, p.Px, p.Py, p.Pz, p.vx, p.vy, p.vz, p.wx, p.wy, p.wz};
        for (double* a : arrs)
            if ((rc = state_device(c, io, a, pb))) return rc;
        if ((rc = state_device(c, io, p.id, sizeof(int) * np))) return rc;
        if (!uniform && ((rc = state_device(c, io, p.q, pb)) || (rc = state_device(c, io, p.m, pb)))) return rc;
    }
    int nch = 0;
    if (io.writing && np > 0) {
        UPIC_CUDA(c, cudaMemcpy(&nch, c->sw.nchunks, sizeof(int), cudaMemcpyDeviceToHost));
    }
    if ((rc = state_value(c, io, nch))) return rc;
    if (nch > 0) {
        const long chunk_cap = c->cap / kMinChunk + c->tg.ntx * c->tg.nty + 1;
        if (nch > chunk_cap) return fail(c, UPIC_ERR_ARGUMENT, "state file: chunk list larger than the context's");
        if ((rc = state_device(c, io, c->sw.chunks, sizeof(Chunk) * nch))) return rc;
        if (!io.writing) UPIC_CUDA(c, cudaMemcpy(c->sw.nchunks, &nch, sizeof(int), cudaMemcpyHostToDevice));
    }
    const size_t N = (size_t)c->N;
    if ((rc = state_device(c, io, c->d_spec, sizeof(double2) * 16 * N)) ||
        (rc = state_device(c, io, c->d_hist, sizeof(double2) * 5 * kHistSlots * N)) ||
        (c->mixed ? (rc = state_device(c, io, c->d_gf32, sizeof(float) * kGFStride * N))
                  : (rc = state_device(c, io, c->d_gf, sizeof(double) * kGFStride * N))) ||
        (rc = state_device(c, io, c->d_acc, sizeof(unsigned long long) * 8 * N)) ||
        (rc = state_device(c, io, c->d_J, sizeof(double) * 3 * N)) ||
        (rc = state_device(c, io, c->d_rho, sizeof(double) * N)))
        return rc;
    if (has_bg && (rc = state_device(c, io, c->d_bg, sizeof(double) * N))) return rc;
    return 0;
}

int state_file(upic_ctx* c, const char* path, bool writing) {
    if (!c || !path) return UPIC_ERR_ARGUMENT;
    StateIO io;
    io.writing = writing;
    io.f = std::fopen(path, writing ? "wb" : "rb");
    if (!io.f) return fail(c, UPIC_ERR_ARGUMENT, std::string("cannot open state file ") + path);
    int rc = 0;
    char magic[8];
    unsigned version = kStateVersion;
    std::vector<double> sig = config_signature(c->cfg);
    long nsig = (long)sig.size();
    if (writing) std::memcpy(magic, kStateMagic, 8);
    if ((rc = state_bytes(c, io, magic, 8)) || (rc = state_value(c, io, version)) || (rc = state_value(c, io, nsig))) {
        std::fclose(io.f);
        return rc;
    }
    if (!writing && (std::memcmp(magic, kStateMagic, 8) != 0 || version != kStateVersion ||
                     nsig != (long)sig.size())) {
        std::fclose(io.f);
        return fail(c, UPIC_ERR_ARGUMENT, "not a state file of this library version");
    }
    std::vector<double> file_sig(sig);
    if ((rc = state_bytes(c, io, file_sig.data(), sizeof(double) * sig.size()))) {
        std::fclose(io.f);
        return rc;
    }
    if (!writing && std::memcmp(file_sig.data(), sig.data(), sizeof(double) * sig.size()) != 0) {
        std::fclose(io.f);
        return fail(c, UPIC_ERR_CONFIG, "state file was written by a context with a different configuration");
    }
    rc = c->imp ? implicit_state_io(c, io) : explicit_state_io(c, io);
    if (std::fclose(io.f) != 0 && rc == 0) rc = fail(c, UPIC_ERR_ARGUMENT, "state file close failed");
    if (rc && !writing) {
        // a partly read state is unusable: the context waits for particles again
        c->np = 0;
        c->fields_ready = false;
        if (c->imp) implicit_mark_unloaded(c);
    }
    return rc;
}

}  // namespace

extern "C" {

int upic_save_state(upic_ctx* ctx, const char* path) {
    if (ctx && ctx->st) {
        const cudaError_t e = cudaStreamSynchronize(ctx->st);
        if (e != cudaSuccess) return fail(ctx, UPIC_ERR_CUDA, cudaGetErrorString(e));
    }
    return state_file(ctx, path, true);
}

int upic_load_state(upic_ctx* ctx, const char* path) {
    if (ctx) ++ctx->generation;
    if (ctx && ctx->st) {
        const cudaError_t e = cudaStreamSynchronize(ctx->st);
        if (e != cudaSuccess) return fail(ctx, UPIC_ERR_CUDA, cudaGetErrorString(e));
    }
    return state_file(ctx, path, false);
}

int upic_destroy(upic_ctx* c) {
    if (!c) return UPIC_OK;
    if (c->st) cudaStreamSynchronize(c->st);
    clear_profile(c);
    implicit_destroy(c);
    for (void* p : c->allocs)
        if (p) cudaFree(p);
    if (c->h_row) cudaFreeHost(c->h_row);
    if (c->h_scan) cudaFreeHost(c->h_scan);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return UPIC_OK;
}

int upic_set_stream(upic_ctx* c, void* stream) {
    if (!c) return UPIC_ERR_ARGUMENT;
    ++c->generation;
    UPIC_CUDA(c, cudaStreamSynchronize(c->st));
    c->st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own;
    return UPIC_OK;
}

// Mixed precision: the host set in the reference's layout becomes nearest
// nodes, FP32 offsets and FP32 momenta and velocities (the conversions run
// on the device from the FP64 staging buffer).
static int set_particles_mixed(upic_ctx* c, long np, const double* x, const double* y, const double* P,
                               const double* v, const double* v_prev, const double* q, const double* m) {
    int rc;
    c->fields_ready = false;
    if (np > c->cap) {
        const bool had_qm = c->M[0].q != nullptr;
        free_mixed(c, c->M[0]);
        free_mixed(c, c->M[1]);
        free_sortwork(c, c->sw);
        if ((rc = alloc_mixed(c, c->M[0], np + 2, had_qm)) || (rc = alloc_mixed(c, c->M[1], np + 2, had_qm)) ||
            (rc = alloc_sortwork(c, c->sw, np, c->tg)))
            return rc;
        c->cap = np;
    }
    if ((rc = ensure_tmp3(c, np))) return rc;
    MixedSoA& s = c->M[0];
    double* t = c->d_tmp3;
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(t, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(t + np, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, mixed_from_positions(np, t, t + np, 1.0 / c->dx, 1.0 / c->dy, c->nx, c->ny, c->lny, s.cell,
                                          s.rx, s.ry, c->st));
        const double* trip[3] = {P, v, v_prev};
        float* dst[3][3] = {{s.Px, s.Py, s.Pz}, {s.vx, s.vy, s.vz}, {s.wx, s.wy, s.wz}};
        for (int k = 0; k < 3; ++k) {
            UPIC_CUDA(c, cudaMemcpyAsync(t, trip[k], sizeof(double) * 3 * np, cudaMemcpyHostToDevice, c->st));
            UPIC_CUDA(c, mixed_split3(np, t, dst[k][0], dst[k][1], dst[k][2], c->st));
        }
    }
    const HostScan hs = scan_particles(np, x, y, v, q, m);
    if (!hs.finite) {
        c->np = 0;
        sync(c);
        return fail(c, UPIC_ERR_NONFINITE, "non-finite particle position or velocity");
    }
    const bool uniform = hs.uniform;
    if (!uniform && !s.q) {
        for (int k = 0; k < 2; ++k)
            if ((rc = dalloc(c, &c->M[k].q, c->cap + 2)) || (rc = dalloc(c, &c->M[k].m, c->cap + 2))) return rc;
    }
    c->np = np;
    c->cur = 0;
    c->uniform_qm = uniform;
    c->q0 = np ? q[0] : 0.0;
    c->m0 = np ? m[0] : 0.0;
    if (np > 0) {
        if (!uniform) {
            UPIC_CUDA(c, cudaMemcpyAsync(t, q, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
            UPIC_CUDA(c, mixed_from_doubles(np, t, c->M[0].q, c->st));
            UPIC_CUDA(c, cudaMemcpyAsync(t + np, m, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
            UPIC_CUDA(c, mixed_from_doubles(np, t + np, c->M[0].m, c->st));
        }
        if ((rc = iota(c, c->M[0].id, np))) return rc;
    }
    const double vb = hs.speed_max > c->cfg.c ? hs.speed_max : c->cfg.c;
    c->scale[0] = c->scale[1] = c->scale[2] = fixed_scale1(hs.qabs * vb / c->dA);
    c->scale[3] = fixed_scale1(hs.qabs / c->dA);
    c->steps = 0;
    return sync(c);
}

static int get_particles_mixed(upic_ctx* c, long np, double* x, double* y, double* P, double* v, double* v_prev) {
    if (np == 0) return UPIC_OK;
    MixedSoA& s = c->M[c->cur];
    MixedSoA& d = c->M[1 - c->cur];
    UPIC_CUDA(c, unpermute_mixed(s, d, np, c->st));
    double* t = c->d_tmp3;
    UPIC_CUDA(c, mixed_to_positions(np, d.cell, d.rx, d.ry, c->dx, c->dy, c->cfg.Lx, c->cfg.Ly, c->lny, c->ny, t,
                                    t + np, c->st));
    if (x) UPIC_CUDA(c, cudaMemcpyAsync(x, t, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    if (y) UPIC_CUDA(c, cudaMemcpyAsync(y, t + np, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    double* out[3] = {P, v, v_prev};
    const float* src[3][3] = {{d.Px, d.Py, d.Pz}, {d.vx, d.vy, d.vz}, {d.wx, d.wy, d.wz}};
    for (int k = 0; k < 3; ++k) {
        if (!out[k]) continue;
        // the staging buffer is reused in stream order
        UPIC_CUDA(c, mixed_join3(np, src[k][0], src[k][1], src[k][2], t, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(out[k], t, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, c->st));
    }
    return sync(c);
}

int upic_set_particles(upic_ctx* c, long np, const double* x, const double* y, const double* P,
                       const double* v, const double* v_prev, const double* q, const double* m) {
    if (!c) return UPIC_ERR_ARGUMENT;
    ++c->generation;
    if (np < 0 || np > 0x7fffffffL) return fail(c, UPIC_ERR_ARGUMENT, "particle count out of range");
    if (np > 0 && (!x || !y || !P || !v || !v_prev || !q || !m))
        return fail(c, UPIC_ERR_ARGUMENT, "null particle array");
    if (c->imp) {
        const int rc = implicit_set_particles(c, np, x, y, P, v, v_prev, q, m);
        if (rc == 0) {
            c->np = np;
            c->fields_ready = false;
            c->steps = 0;
        }
        return rc;
    }
    if (c->mixed) return set_particles_mixed(c, np, x, y, P, v, v_prev, q, m);
    int rc;
    c->fields_ready = false;
    if (np > c->cap) {
        const bool had_qm = c->P[0].q != nullptr;
        free_soa(c, c->P[0]);
        free_soa(c, c->P[1]);
        free_sortwork(c, c->sw);
        if ((rc = alloc_soa(c, c->P[0], np, true, had_qm)) || (rc = alloc_soa(c, c->P[1], np, true, had_qm)) ||
            (rc = alloc_sortwork(c, c->sw, np, c->tg)))
            return rc;
        c->cap = np;
    }
    if ((rc = ensure_tmp3(c, np))) return rc;
    ParticleSoA& s = c->P[0];
    // the state copies run while the host validates the set
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(s.x, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.y, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        if ((rc = upload3(c, P, np, s.Px, s.Py, s.Pz))) return rc;
        if ((rc = upload3(c, v, np, s.vx, s.vy, s.vz))) return rc;
        if ((rc = upload3(c, v_prev, np, s.wx, s.wy, s.wz))) return rc;
    }
    // uniform charge/mass (the reference stores them per particle); the
    // device checks the uploaded positions and velocities meanwhile
#if UPIC_DEVICE_SCAN
    HostScan hs;
    if (np > 0) {
        UPIC_CUDA(c, cudaMemsetAsync(c->d_scan, 0, 3 * sizeof(unsigned long long), c->st));
        scan_state_kernel<<<148 * 8, 256, 0, c->st>>>(s.x, s.y, s.vx, s.vy, s.vz, np, c->d_scan);
        count_launches(1);
        UPIC_CUDA(c, cudaMemcpyAsync(c->h_scan, c->d_scan, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                     c->st));
        hs = scan_particles(np, nullptr, nullptr, nullptr, q, m);
        if ((rc = sync(c))) return rc;
        hs.finite = c->h_scan[0] == 0;
        std::memcpy(&hs.speed_max, &c->h_scan[1], sizeof(double));
        std::memcpy(&hs.comp_max, &c->h_scan[2], sizeof(double));
    }
#else
    const HostScan hs = scan_particles(np, x, y, v, q, m);
#endif
    if (!hs.finite) {
        c->np = 0;  // the context holds no particle set until a valid one is loaded
        sync(c);
        return fail(c, UPIC_ERR_NONFINITE, "non-finite particle position or velocity");
    }
    const bool uniform = hs.uniform;
    const double qabs = hs.qabs, vmax = hs.speed_max;
    if (!uniform && !s.q) {
        for (int k = 0; k < 2; ++k)
            if ((rc = dalloc(c, &c->P[k].q, c->cap + 2)) || (rc = dalloc(c, &c->P[k].m, c->cap + 2))) return rc;
    }
    c->np = np;
    c->cur = 0;
    c->uniform_qm = uniform;
    c->q0 = np ? q[0] : 0.0;
    c->m0 = np ? m[0] : 0.0;
    if (np > 0) {
        if (!uniform) {
            UPIC_CUDA(c, cudaMemcpyAsync(s.q, q, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
            UPIC_CUDA(c, cudaMemcpyAsync(s.m, m, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        }
        if ((rc = iota(c, s.id, np))) return rc;
    }
    const double vb = vmax > c->cfg.c ? vmax : c->cfg.c;
    const double bJ = qabs * vb / c->dA;
    c->scale[0] = c->scale[1] = c->scale[2] = fixed_scale(bJ);
    c->scale[3] = fixed_scale(qabs / c->dA);
    c->fields_ready = false;
    c->steps = 0;
    return sync(c);
}

int upic_get_particles(upic_ctx* c, long np, double* x, double* y, double* P, double* v,
                       double* v_prev) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (np != c->np) return fail(c, UPIC_ERR_ARGUMENT, "particle count does not match the context");
    if (c->imp) return implicit_get_particles(c, np, x, y, P, v, v_prev);
    if (c->mixed) return get_particles_mixed(c, np, x, y, P, v, v_prev);
    if (np == 0) return UPIC_OK;
    ParticleSoA& s = c->P[c->cur];
    ParticleSoA& d = c->P[1 - c->cur];
    UPIC_CUDA(c, unpermute_particles(s, d, np, c->st));
    int rc;
    if (x) UPIC_CUDA(c, cudaMemcpyAsync(x, d.x, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    if (y) UPIC_CUDA(c, cudaMemcpyAsync(y, d.y, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    // the staging buffer is reused in stream order: each join waits for the
    // previous copy out of it
    if (P && (rc = download3(c, P, np, d.Px, d.Py, d.Pz))) return rc;
    if (v && (rc = download3(c, v, np, d.vx, d.vy, d.vz))) return rc;
    if (v_prev && (rc = download3(c, v_prev, np, d.wx, d.wy, d.wz))) return rc;
    return sync(c);
}

int upic_init_fields(upic_ctx* c, double* diag_row) {
    if (c) ++c->generation;
    if (!c) return UPIC_ERR_ARGUMENT;
    if (c->imp) return implicit_init_fields(c, diag_row);
    if (c->cap == 0 && c->np == 0) return fail(c, UPIC_ERR_STATE, "upic_set_particles first");
    const int N = c->N;
    int rc;
    // rho0 = n0 + electrons, J0 (spectral_pic_part3.cpp:1102-1103)
    if (c->np > 0) {
        if ((rc = sort_active(c, 0.0))) return rc;
        UPIC_CUDA(c, cudaMemsetAsync(c->d_acc, 0, sizeof(unsigned long long) * 8 * (size_t)N, c->st));
        if ((rc = launch_push(c, kModeDeposit, 4, c->P[c->cur], c->np, c->uniform_qm, c->sw, c->d_pdiag)))
            return rc;
    } else {
        UPIC_CUDA(c, cudaMemsetAsync(c->d_pdiag, 0, sizeof(double) * c->push_grid * kDiagPart, c->st));
    }
    if (c->mixed)
        UPIC_CUDA(c, launch_convert_acc1(c->d_acc, N, c->scale, c->d_J, c->d_rho, c->cfg.n0, 3, c->st, c->d_bg));
    else
        UPIC_CUDA(c, launch_convert_acc(c->d_acc, N, c->scale, c->d_J, c->d_rho, c->cfg.n0, 3, c->st, c->d_bg));
    // phi0 from Poisson (:1104, :819-827), histories (:1107-1111)
    double2* sp = c->d_spec;
    UPIC_CUDA(c, fft2d_batched(c->plan, sp + 3 * (size_t)N, 1, 0, c->st, c->d_rho));
    UPIC_CUDA(c, launch_poisson_kspace(N, c->d_k2, sp + 3 * (size_t)N, c->cfg.eps0, sp + 4 * (size_t)N, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, sp + 4 * (size_t)N, 1, 1, c->st, nullptr, 1, c->d_dreal));
    UPIC_CUDA(c, fft2d_batched(c->plan, sp + 4 * (size_t)N, 1, 0, c->st, c->d_dreal));
    double2* H = c->d_hist;
    const size_t fs = (size_t)kHistSlots * N;
    UPIC_CUDA(c, launch_fill_hist(H + 0 * fs, kHistSlots, N, sp + 4 * (size_t)N, c->st));
    UPIC_CUDA(c, cudaMemsetAsync(H + 1 * fs, 0, sizeof(double2) * 3 * fs, c->st));
    UPIC_CUDA(c, launch_fill_hist(H + 4 * fs, kHistSlots, N, sp + 3 * (size_t)N, c->st));
    c->head = 0;
    // J0 spectra for the step-0 diagnostics
    UPIC_CUDA(c, fft2d_batched(c->plan, sp, 3, 0, c->st, c->d_J));
    if (diag_row) {
        const double a1[3] = {1.0, -1.0, 0.0};
        if ((rc = run_diag(c, c->head, c->head, 2, a1))) return rc;
    }
    // first step's current, deposited one step ahead (:1137-1141)
    if (c->np > 0) {
        if ((rc = sort_active(c, c->cfg.dt))) return rc;
        if ((rc = launch_push(c, kModeAdvanceDeposit, grid_ncomp(c), c->P[c->cur], c->np, c->uniform_qm,
                              c->sw, nullptr)))
            return rc;
    }
    c->steps = 0;
    c->fields_ready = true;
    if ((rc = sync(c))) return rc;
    if (diag_row) std::memcpy(diag_row, c->h_row, sizeof(double) * UPIC_DIAG_COUNT);
    return UPIC_OK;
}

int upic_step(upic_ctx* c, int nsteps, int diag_stride, double* diag) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (c->imp) return fail(c, UPIC_ERR_STATE, "the implicit method advances with upic_step_implicit");
    if (!c->fields_ready) return fail(c, UPIC_ERR_STATE, "upic_init_fields first");
    if (nsteps < 0) return fail(c, UPIC_ERR_ARGUMENT, "nsteps < 0");
    return upic_host::explicit_advance(c, nsteps, diag_stride, diag, true);
}

}  // extern "C"

namespace upic_host {

// The explicit step loop of upic_step.  Without diagnostics rows and with
// final_sync false it only queues work on the context's stream (no host
// synchronisation, no allocation), so it can be captured into a CUDA graph.
int explicit_advance(upic_ctx* c, int nsteps, int diag_stride, double* diag, bool final_sync) {
    const int N = c->N;
    int na, nb;
    double a[3], b[5];
    bdf_coeffs(c->cfg.method, na, a, nb, b);
    const bool naive = c->cfg.charge_update == UPIC_CHARGE_NAIVE;
    double2* sp = c->d_spec;
    int rc;
    for (int s = 0; s < nsteps; ++s) {
        const long step = c->steps + 1;
        const bool want_diag = diag && diag_stride > 0 && (step % diag_stride == 0 || s == nsteps - 1);
        if (c->np > 0 && c->steps_since_sort >= c->sort_interval) {
            if ((rc = sort_active(c, c->cfg.dt))) return rc;
        }
        // J^n (and rho^n) were deposited by the previous particle kernel
        if (c->mixed)
            UPIC_CUDA(c, launch_convert_acc1(c->d_acc, N, c->scale, c->d_J, c->d_rho, c->cfg.n0, naive ? 3 : 1,
                                             c->st, c->d_bg));
        else
            UPIC_CUDA(c, launch_convert_acc(c->d_acc, N, c->scale, c->d_J, c->d_rho, c->cfg.n0, naive ? 3 : 1,
                                            c->st, c->d_bg));
        UPIC_CUDA(c, fft2d_batched(c->plan, sp, 3, 0, c->st, c->d_J));
        if (naive) UPIC_CUDA(c, fft2d_batched(c->plan, sp + 3 * (size_t)N, 1, 0, c->st, c->d_rho));
        KspaceArgs k{};
        k.N = N;
        k.kx = c->d_kx;
        k.ky = c->d_ky;
        k.k2 = c->d_k2;
        k.Jhat = sp;
        k.rho_dep = naive ? sp + 3 * (size_t)N : nullptr;
        k.hist = c->d_hist;
        k.R = kHistSlots;
        k.head = c->head;
        k.na = na;
        k.nb = nb;
        for (int i = 0; i < 3; ++i) k.a[i] = a[i];
        for (int i = 0; i < 5; ++i) k.b[i] = b[i];
        k.dt = c->cfg.dt;
        k.c = c->cfg.c;
        k.eps0 = c->cfg.eps0;
        k.mu0 = c->cfg.mu0;
        k.conserving = naive ? 0 : 1;
        k.gspec = sp + 4 * (size_t)N;
        UPIC_CUDA(c, launch_bdf_kspace(k, c->st));
        if (c->mixed)
            UPIC_CUDA(c, fft2d_batched(c->plan, sp + 4 * (size_t)N, kGF, 1, c->st, nullptr, 3,
                                       reinterpret_cast<double*>(c->d_gf32), kGFStride, 0));
        else
            UPIC_CUDA(c, fft2d_batched(c->plan, sp + 4 * (size_t)N, kGF, 1, c->st, nullptr, 2, c->d_gf,
                                       kGFStride, 0));
        if (c->np > 0) {
            if ((rc = launch_push(c, kModePush, grid_ncomp(c), c->P[c->cur], c->np, c->uniform_qm, c->sw,
                                  c->d_pdiag)))
                return rc;
        } else {
            UPIC_CUDA(c, cudaMemsetAsync(c->d_pdiag, 0, sizeof(double) * c->push_grid * kDiagPart, c->st));
        }
        const int snew = (c->head + kHistSlots - 1) % kHistSlots;
        if (want_diag) {
            if ((rc = run_diag(c, snew, c->head, na, a))) return rc;
            if ((rc = sync(c))) return rc;
            std::memcpy(diag + (size_t)s * UPIC_DIAG_COUNT, c->h_row, sizeof(double) * UPIC_DIAG_COUNT);
        } else if (diag) {
            for (int i = 0; i < UPIC_DIAG_COUNT; ++i) diag[(size_t)s * UPIC_DIAG_COUNT + i] = NAN;
        }
        c->head = snew;
        c->steps = step;
        c->steps_since_sort++;
    }
    return final_sync ? sync(c) : 0;
}

}  // namespace upic_host

extern "C" {

int upic_profile_enable(upic_ctx* c, int on) {
    if (!c) return UPIC_ERR_ARGUMENT;
    UPIC_CUDA(c, cudaStreamSynchronize(c->st));
    clear_profile(c);
    c->profiling = on != 0;
    return UPIC_OK;
}

int upic_profile_read(upic_ctx* c, double* push_ms, long* push_launches, long* kernel_launches) {
    if (!c) return UPIC_ERR_ARGUMENT;
    UPIC_CUDA(c, cudaStreamSynchronize(c->st));
    double total = 0.0;
    for (auto& e : c->prof_events) {
        float ms = 0.0f;
        UPIC_CUDA(c, cudaEventElapsedTime(&ms, e.first, e.second));
        total += ms;
    }
    if (push_ms) *push_ms = total;
    if (push_launches) *push_launches = (long)c->prof_events.size();
    if (kernel_launches) *kernel_launches = launches_total();
    return UPIC_OK;
}

int upic_set_background(upic_ctx* c, const double* rho_bg) {
    if (c) ++c->generation;
    if (!c) return UPIC_ERR_ARGUMENT;
    if (c->imp) return fail(c, UPIC_ERR_STATE, "the implicit method has a uniform background (n0)");
    if (!rho_bg) {
        dfree(c, c->d_bg);
        c->d_bg = nullptr;
    } else {
        for (int id = 0; id < c->N; ++id)
            if (!std::isfinite(rho_bg[id])) return fail(c, UPIC_ERR_NONFINITE, "non-finite background charge");
        int rc;
        if (!c->d_bg && (rc = dalloc(c, &c->d_bg, c->N))) return rc;
        UPIC_CUDA(c, cudaMemcpyAsync(c->d_bg, rho_bg, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
        if ((rc = sync(c))) return rc;
    }
    c->fields_ready = false;
    return UPIC_OK;
}

int upic_step_count(const upic_ctx* c, long* steps) {
    if (!c || !steps) return UPIC_ERR_ARGUMENT;
    *steps = c->steps;
    return UPIC_OK;
}

int upic_particle_count(const upic_ctx* c, long* np) {
    if (!c || !np) return UPIC_ERR_ARGUMENT;
    *np = c->np;
    return UPIC_OK;
}

int upic_get_field(upic_ctx* c, int which, double* host) {
    if (!c || !host) return UPIC_ERR_ARGUMENT;
    if (!c->fields_ready) return fail(c, UPIC_ERR_STATE, "upic_init_fields first");
    if (c->imp) return implicit_get_field(c, which, host);
    const int N = c->N;
    if (which >= UPIC_FIELD_JX && which <= UPIC_FIELD_JZ) {
        UPIC_CUDA(c, cudaMemcpyAsync(host, c->d_J + (size_t)(which - UPIC_FIELD_JX) * N, sizeof(double) * N,
                                     cudaMemcpyDeviceToHost, c->st));
        return sync(c);
    }
    if (which >= UPIC_FIELD_EX && which <= UPIC_FIELD_BZ) {
        // E = -grad phi - dA/dt (the BDF derivative of the last step, or zero
        // at start-up as in the step-0 diagnostics row) and B = curl A, from
        // the history spectra (compute_diagnostics :918-944)
        int na, nb;
        double a[3], b[5];
        int prev = c->head;
        if (c->steps == 0) {
            na = 2;
            a[0] = 1.0, a[1] = -1.0, a[2] = 0.0;
        } else {
            bdf_coeffs(c->cfg.method, na, a, nb, b);
            prev = (c->head + 1) % kHistSlots;
        }
        DiagKArgs d{};
        d.N = N;
        d.kx = c->d_kx;
        d.ky = c->d_ky;
        d.k2 = c->d_k2;
        d.Jhat = c->d_spec;
        d.hist = c->d_hist;
        d.R = kHistSlots;
        d.slot_new = c->head;
        d.slot_prev0 = prev;
        d.na = na;
        for (int k = 0; k < 3; ++k) d.a[k] = a[k];
        d.dt = c->cfg.dt;
        d.c = c->cfg.c;
        d.eps0 = c->cfg.eps0;
        d.out = c->d_dspec;
        UPIC_CUDA(c, launch_diag_kspace(d, c->st));
        // diag_kspace output slots: E 1..3, B 6..8
        const int slot = which <= UPIC_FIELD_EZ ? 1 + which - UPIC_FIELD_EX : 6 + which - UPIC_FIELD_BX;
        UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec + (size_t)slot * N, 1, 1, c->st, nullptr, 1, c->d_dreal));
        UPIC_CUDA(c, cudaMemcpyAsync(host, c->d_dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
        return sync(c);
    }
    if (which < 0 || which > UPIC_FIELD_RHO) return fail(c, UPIC_ERR_ARGUMENT, "unknown field");
    const int f = which;  // phi 0, A 1..3, rho 4 share the history field index
    const double2* src = c->d_hist + ((size_t)f * kHistSlots + c->head) * N;
    double2* tmp = c->d_dspec;
    UPIC_CUDA(c, cudaMemcpyAsync(tmp, src, sizeof(double2) * N, cudaMemcpyDeviceToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, tmp, 1, 1, c->st, nullptr, 1, c->d_dreal));
    UPIC_CUDA(c, cudaMemcpyAsync(host, c->d_dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

// ---- kernel-level entry points --------------------------------------------
namespace {

int ensure_kparticles(upic_ctx* c, long np) {
    if (np <= c->kcap) return 0;
    free_soa(c, c->K[0]);
    free_soa(c, c->K[1]);
    free_sortwork(c, c->ksw);
    int rc;
    if ((rc = alloc_soa(c, c->K[0], np, false, true)) || (rc = alloc_soa(c, c->K[1], np, false, true)) ||
        (rc = alloc_sortwork(c, c->ksw, np, c->tg)))
        return rc;
    c->kcap = np;
    return ensure_tmp3(c, np);
}

// Upload (x, y, v, q), sort, deposit with ncomp (1 charge, 3 current).
int kernel_deposit(upic_ctx* c, long np, const double* x, const double* y, const double* v,
                   const double* q, int ncomp) {
    int rc;
    if ((rc = ensure_kparticles(c, np))) return rc;
    const int N = c->N;
    ParticleSoA& s = c->K[0];
    double qabs = 0.0, vmax = 0.0;
    for (long p = 0; p < np; ++p) {
        qabs += std::fabs(q[p]);
        if (v) {
            const double sp = std::sqrt(v[3 * p] * v[3 * p] + v[3 * p + 1] * v[3 * p + 1] +
                                        v[3 * p + 2] * v[3 * p + 2]);
            if (sp > vmax) vmax = sp;
        }
    }
    double scale[4];
    scale[0] = scale[1] = scale[2] = fixed_scale(qabs * vmax / c->dA);
    scale[3] = fixed_scale(qabs / c->dA);
    UPIC_CUDA(c, cudaMemsetAsync(c->d_acc, 0, sizeof(unsigned long long) * 8 * (size_t)N, c->st));
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(s.x, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.y, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.q, q, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        if (v) {
            if ((rc = upload3(c, v, np, s.vx, s.vy, s.vz))) return rc;
        } else {
            UPIC_CUDA(c, cudaMemsetAsync(s.vx, 0, sizeof(double) * np, c->st));
            UPIC_CUDA(c, cudaMemsetAsync(s.vy, 0, sizeof(double) * np, c->st));
            UPIC_CUDA(c, cudaMemsetAsync(s.vz, 0, sizeof(double) * np, c->st));
        }
        iota_kernel<<<gridn(np), 256, 0, c->st>>>(s.id, np);
        count_launches(1);
        UPIC_CUDA(c, sort_particles_by_tile(c->tg, s, np, c->cfg.Lx, c->cfg.Ly, 0.0, c->ksw, c->st));
        UPIC_CUDA(c, permute_particles(s, c->K[1], np, c->ksw, c->st));
        PushArgs a = push_args(c, c->K[1], np, false);
        for (int k = 0; k < 4; ++k) a.scale[k] = scale[k];
        a.m0 = 1.0;
        a.c = c->cfg.c;
        a.chunks = c->ksw.chunks;
        a.nchunks = c->ksw.nchunks;
        a.diag_part = nullptr;
        UPIC_CUDA(c, launch_push_deposit(kModeDeposit, ncomp, false, c->tg, a, c->push_grid, c->st));
    }
    UPIC_CUDA(c, launch_convert_acc(c->d_acc, N, scale, c->d_J, c->d_rho, c->cfg.n0,
                                    ncomp == 1 ? 2 : 1, c->st));
    return 0;
}

}  // namespace

int upic_deposit_current(upic_ctx* c, long np, const double* x, const double* y, const double* v,
                         const double* q, double* J) {
    if (!c || !J || np < 0 || (np > 0 && (!x || !y || !v || !q))) return UPIC_ERR_ARGUMENT;
    int rc = kernel_deposit(c, np, x, y, v, q, 3);
    if (rc) return rc;
    UPIC_CUDA(c, cudaMemcpyAsync(J, c->d_J, sizeof(double) * 3 * (size_t)c->N, cudaMemcpyDeviceToHost, c->st));
    c->fields_ready = false;
    return sync(c);
}

int upic_deposit_charge(upic_ctx* c, long np, const double* x, const double* y, const double* q,
                        double* rho) {
    if (!c || !rho || np < 0 || (np > 0 && (!x || !y || !q))) return UPIC_ERR_ARGUMENT;
    int rc = kernel_deposit(c, np, x, y, nullptr, q, 1);
    if (rc) return rc;
    UPIC_CUDA(c, cudaMemcpyAsync(rho, c->d_rho, sizeof(double) * (size_t)c->N, cudaMemcpyDeviceToHost, c->st));
    c->fields_ready = false;
    return sync(c);
}

int upic_gather(upic_ctx* c, const double* f, long np, const double* x, const double* y, double* out) {
    if (!c || !f || !out || np < 0 || (np > 0 && (!x || !y))) return UPIC_ERR_ARGUMENT;
    int rc;
    if ((rc = ensure_kparticles(c, np))) return rc;
    double* df = c->d_dreal;
    UPIC_CUDA(c, cudaMemcpyAsync(df, f, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(c->K[0].x, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(c->K[0].y, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, launch_gather_scalar(c->nx, c->ny, 1.0 / c->dx, 1.0 / c->dy, df, np, c->K[0].x,
                                          c->K[0].y, c->K[0].vx, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(out, c->K[0].vx, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    }
    return sync(c);
}

int upic_fft2d(upic_ctx* c, double* re, double* im, int inverse) {
    if (!c || !re || !im) return UPIC_ERR_ARGUMENT;
    const long N = c->N;
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_dreal, re, sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_dreal + N, im, sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
    interleave_kernel<<<gridn(N), 256, 0, c->st>>>(c->d_dreal, c->d_dreal + N, c->d_dspec, N);
    count_launches(1);
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec, 1, inverse ? 1 : 0, c->st));
    deinterleave_kernel<<<gridn(N), 256, 0, c->st>>>(c->d_dspec, c->d_dreal, c->d_dreal + N, N);
    count_launches(1);
    UPIC_CUDA(c, cudaMemcpyAsync(re, c->d_dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(im, c->d_dreal + N, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

int upic_spectral_derivative(upic_ctx* c, const double* f, int dir, double* out) {
    if (!c || !f || !out || (dir != 0 && dir != 1)) return UPIC_ERR_ARGUMENT;
    const long N = c->N;
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_dreal, f, sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec, 1, 0, c->st, c->d_dreal));
    UPIC_CUDA(c, launch_derivative_kspace(N, dir == 0 ? c->d_kx : c->d_ky, c->d_dspec, c->d_dspec + N, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec + N, 1, 1, c->st, nullptr, 1, c->d_dreal));
    UPIC_CUDA(c, cudaMemcpyAsync(out, c->d_dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

int upic_push_iaem(upic_ctx* c, long np, const double* x, const double* y, double* P, double* v, double* v_prev,
                   const double* q, const double* m, const double* phi, const double* A) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (c->imp) return fail(c, UPIC_ERR_STATE, "upic_push_iaem needs an explicit method (bdf1, bdf2)");
    if (np < 0 || !phi || !A || (np > 0 && (!x || !y || !P || !v || !v_prev || !q || !m)))
        return fail(c, UPIC_ERR_ARGUMENT, "upic_push_iaem: null array or negative particle count");
    if (np == 0) return UPIC_OK;
    for (long p = 0; p < np; ++p)
        if (!std::isfinite(x[p]) || !std::isfinite(y[p]) || !std::isfinite(q[p]) || !(m[p] > 0.0))
            return fail(c, UPIC_ERR_NONFINITE, "upic_push_iaem: non-finite position or charge, or mass <= 0");
    const size_t N = (size_t)c->N, n = (size_t)np;
    // device scratch of this call, freed on every return path
    struct Buf {
        std::vector<void*> p;
        ~Buf() {
            for (void* q : p) cudaFree(q);
        }
        double* get(size_t k) {
            void* v = nullptr;
            if (cudaMalloc(&v, k * sizeof(double) + 16) != cudaSuccess) return nullptr;
            p.push_back(v);
            return static_cast<double*>(v);
        }
    } b;
    double* F = b.get(11 * N);
    double* fin = b.get(N);
    double2* spec = reinterpret_cast<double2*>(b.get(4 * N));
    double *dx_ = b.get(n), *dy_ = b.get(n), *dP = b.get(3 * n), *dv = b.get(3 * n), *dvp = b.get(3 * n);
    double *dq = b.get(n), *dm = b.get(n);
    if (!F || !fin || !spec || !dx_ || !dy_ || !dP || !dv || !dvp || !dq || !dm)
        return fail(c, UPIC_ERR_NOMEM, "upic_push_iaem: device allocation failed");
    // F: A (3), grad phi (2), dA_c/dx, dA_c/dy (spectral_gradient_scalar,
    // spectral_gradient_vector: spectral_derivative :440 with the Nyquist
    // wave number zeroed)
    UPIC_CUDA(c, cudaMemcpyAsync(F, A, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c->st));
    const double* src[4] = {phi, A, A + N, A + 2 * N};
    const size_t dst[4] = {3, 5, 7, 9};
    for (int f = 0; f < 4; ++f) {
        UPIC_CUDA(c, cudaMemcpyAsync(fin, src[f], sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, fft2d_batched(c->plan, spec, 1, 0, c->st, fin));
        for (int d = 0; d < 2; ++d) {
            UPIC_CUDA(c, launch_derivative_kspace((int)N, d == 0 ? c->d_kx : c->d_ky, spec, spec + N, c->st));
            UPIC_CUDA(c, fft2d_batched(c->plan, spec + N, 1, 1, c->st, nullptr, 1, F + (dst[f] + d) * N));
        }
    }
    UPIC_CUDA(c, cudaMemcpyAsync(dx_, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dy_, y, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dP, P, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dv, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dvp, v_prev, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dq, q, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dm, m, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, launch_iaem_push(np, dx_, dy_, dP, dv, dvp, dq, dm, F, c->nx, c->ny, 1.0 / c->dx, 1.0 / c->dy,
                                  c->cfg.dt, c->cfg.c, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(P, dP, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(v, dv, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(v_prev, dvp, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

int upic_poisson(upic_ctx* c, const double* rho, double* phi) {
    if (!c || !rho || !phi) return UPIC_ERR_ARGUMENT;
    const long N = c->N;
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_dreal, rho, sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec, 1, 0, c->st, c->d_dreal));
    UPIC_CUDA(c, launch_poisson_kspace(N, c->d_k2, c->d_dspec, c->cfg.eps0, c->d_dspec + N, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec + N, 1, 1, c->st, nullptr, 1, c->d_dreal));
    UPIC_CUDA(c, cudaMemcpyAsync(phi, c->d_dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

int upic_solve_bdf(upic_ctx* c, const double* source, const double* hist, double* out) {
    if (!c || !source || !hist || !out) return UPIC_ERR_ARGUMENT;
    const long N = c->N;
    int na, nb;
    double a[3], b[5];
    bdf_coeffs(c->cfg.method, na, a, nb, b);
    const int nh = nb - 1;
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_dreal, source, sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(c->d_dreal + N, hist, sizeof(double) * N * nh, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec, 1 + nh, 0, c->st, c->d_dreal));
    const double scale = 1.0 / (c->cfg.c * c->cfg.c * c->cfg.dt * c->cfg.dt);
    UPIC_CUDA(c, launch_bdf_single(N, c->d_k2, c->d_dspec, c->d_dspec + N, nb, b, scale,
                                   c->d_dspec + (size_t)(1 + nh) * N, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, c->d_dspec + (size_t)(1 + nh) * N, 1, 1, c->st, nullptr, 1, c->d_dreal));
    UPIC_CUDA(c, cudaMemcpyAsync(out, c->d_dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

}  // extern "C"
