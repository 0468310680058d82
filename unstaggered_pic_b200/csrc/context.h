// Device context shared by the C-ABI implementation files (api.cu for the
// explicit BDF/IAEM method, api_implicit.cu for the implicit orbit-averaged
// GM-HC-CN method).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "../../include/upic.h"
#include "kernels.h"

namespace upic_host {

constexpr int kHistSlots = 5;
constexpr int kDiagFields = 10;
constexpr int kRedGrid = 148 * 2;

struct ImplicitState;  // api_implicit.cu

}  // namespace upic_host

using upic::FftPlan;
using upic::MixedSoA;
using upic::ParticleSoA;
using upic::SortWork;
using upic::TileGeom;

struct upic_ctx {
    upic_config cfg{};
    std::string err;
    int nx = 0, ny = 0, N = 0;
    double dx = 0, dy = 0, dA = 0;
    cudaStream_t own = nullptr, st = nullptr;
    int device = 0, nsm = 148;

    FftPlan plan{};
    double2* d_twx = nullptr;
    double2* d_twy = nullptr;
    double *d_kx = nullptr, *d_ky = nullptr, *d_k2 = nullptr;

    // particle state
    long np = 0, cap = 0;
    ParticleSoA P[2];
    int cur = 0;
    bool uniform_qm = true;
    double q0 = 0, m0 = 0;
    double scale[4] = {1, 1, 1, 1};
    double* d_tmp3 = nullptr;  // 3*cap staging for xyz triples

    // mixed precision (UPIC_PRECISION_MIXED): the particle state lives in
    // M[cur] instead of P[cur]; scale[] then holds single-word fixed-point
    // scales; d_gf32 holds the FP32 node records
    bool mixed = false;
    MixedSoA M[2];
    float* d_gf32 = nullptr;
    int lny = 0;  // log2(ny)

    // kernel-level entry points use their own particle buffers
    long kcap = 0;
    ParticleSoA K[2];

    // grid state
    unsigned long long* d_acc = nullptr;
    double* d_J = nullptr;
    double* d_rho = nullptr;
    double* d_gf = nullptr;
    double2* d_spec = nullptr;
    double2* d_hist = nullptr;
    double2* d_dspec = nullptr;
    double* d_dreal = nullptr;
    double* d_partials = nullptr;
    double* d_pdiag = nullptr;
    double* d_row = nullptr;
    double* d_bg = nullptr;   // fixed background charge (upic_set_background) or null: uniform n0
    double* h_row = nullptr;  // pinned
    // particle-state scan of upic_set_particles (non-finite count, largest
    // speed and velocity component bits): device words and their pinned copy
    unsigned long long* d_scan = nullptr;
    unsigned long long* h_scan = nullptr;

    int head = 0;
    long steps = 0;
    // bumped by every call that may reallocate or reset the state (particle
    // upload, start-up, state load, stream or background change): a CUDA
    // graph recorded before such a call is stale
    long generation = 0;
    bool fields_ready = false;
    int steps_since_sort = 0;
    int sort_interval = 4;

    // profiling: CUDA events around every particle push kernel
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;

    TileGeom tg{};
    SortWork sw{};
    SortWork ksw{};
    int push_grid = 148;

    std::vector<void*> allocs;

    // implicit orbit-averaged method (api_implicit.cu); null for BDF methods
    upic_host::ImplicitState* imp = nullptr;
};

namespace upic_host {

using upic::MixedSoA;
using upic::ParticleSoA;
using upic::SortWork;
using upic::TileGeom;

int fail(upic_ctx* c, int code, const std::string& msg);

#define UPIC_CUDA(ctx, call)                                                                     \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return ::upic_host::fail(ctx, UPIC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int dalloc_bytes(upic_ctx* c, void** p, size_t bytes);
template <typename T>
int dalloc(upic_ctx* c, T** p, size_t count) {
    void* v = nullptr;
    const int rc = dalloc_bytes(c, &v, sizeof(T) * (count ? count : 1));
    if (rc == 0) *p = reinterpret_cast<T*>(v);
    return rc;
}
void dfree(upic_ctx* c, void* p);
int sync(upic_ctx* c);
int gridn(long n);
int upload3(upic_ctx* c, const double* host, long n, double* a, double* b, double* d);
int download3(upic_ctx* c, double* host, long n, const double* a, const double* b, const double* d);
int ensure_tmp3(upic_ctx* c, long n);
// Validation scan of a host particle set (positions x, y; velocities v as
// xyz triples; q, m): finiteness, uniform q/m, sum |q|, largest speed and
// largest velocity component, positive masses.  Runs in 64 fixed chunks on
// up to 16 host threads; partial sums combine in chunk order, so the result
// does not depend on the thread count.
struct HostScan {
    bool finite = true, uniform = true, positive_m = true;
    double qabs = 0.0, speed_max = 0.0, comp_max = 0.0;
};
// State files (upic_save_state / upic_load_state).  One routine per state
// serialises in both directions: with writing set it writes host/device
// bytes to the file, otherwise it reads them back into the same places.
struct StateIO {
    FILE* f = nullptr;
    bool writing = false;
    std::vector<char> buf;  // host staging of device ranges
};
int state_bytes(upic_ctx* c, StateIO& io, void* host, size_t n);
int state_device(upic_ctx* c, StateIO& io, void* dev, size_t n);
template <typename T>
int state_value(upic_ctx* c, StateIO& io, T& v) {
    return state_bytes(c, io, &v, sizeof(T));
}
int implicit_state_io(upic_ctx* c, StateIO& io);
int explicit_advance(upic_ctx* c, int nsteps, int diag_stride, double* diag, bool final_sync);
void implicit_mark_unloaded(upic_ctx* c);

HostScan scan_particles(long np, const double* x, const double* y, const double* v, const double* q,
                        const double* m);
double fixed_scale(double bound);
TileGeom make_tiles(int nx, int ny, int tile, int guard, int lo, int hi);
// Particles per deposit chunk of the implicit map kernel: enough chunks for
// every resident CTA of a `grid`-CTA launch (a small particle set would
// otherwise keep most SMs idle behind a few long per-particle solves), a
// multiple of kMinChunk in [kMinChunk, max_chunk].  The explicit push keeps
// 2048-particle chunks: its per-particle work is short, and many small
// explicit runs are better served by an ensemble.  Chunk tables are
// allocated for kMinChunk.
constexpr int kMinChunk = 128;
int choose_chunk(long np, int grid, int max_chunk);
int alloc_soa(upic_ctx* c, ParticleSoA& s, long cap, bool with_state, bool with_qm);
void free_soa(upic_ctx* c, ParticleSoA& s);
int alloc_sortwork(upic_ctx* c, SortWork& w, long cap, const TileGeom& tg);
void free_sortwork(upic_ctx* c, SortWork& w);
int iota(upic_ctx* c, int* id, long n);

// implicit method (api_implicit.cu)
int implicit_create(upic_ctx* c);
void implicit_destroy(upic_ctx* c);
int implicit_set_particles(upic_ctx* c, long np, const double* x, const double* y, const double* P,
                           const double* v, const double* v_prev, const double* q, const double* m);
int implicit_get_particles(upic_ctx* c, long np, double* x, double* y, double* P, double* v,
                           double* v_prev);
int implicit_init_fields(upic_ctx* c, double* diag_row);
int implicit_get_field(upic_ctx* c, int which, double* host);

}  // namespace upic_host
