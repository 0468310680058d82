// Internal launch interface between the C-ABI layer (api.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace upic {

// Number of kernels this library has launched (all contexts); read through
// upic_profile_read.  Each launcher adds the kernels it starts.
void count_launches(long n);
long launches_total();
// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device.  The limit belongs to the function, not to a context, so
// it only ever grows: contexts with different tile windows in one process
// each keep room for their own launches.
cudaError_t raise_smem_limit(const void* func, int bytes);

// ---------------------------------------------------------------------------
// FFT (fft.cu)
struct FftPlan {
    int nx, ny;
    const double2* tw_x;  // exp(-2 pi i m / nx), m < nx/2
    const double2* tw_y;  // exp(-2 pi i m / ny), m < ny/2
};

// 2D transform of ncomp stacked complex grids (component stride nx*ny).
// real_in != NULL: the input is the real planar array real_in (imag 0), the
// transform result lands in data.  out_mode 0: complex result in data;
// 1: real part to real_out planar (component stride nx*ny); 2: real part to
// interleaved records real_out[node*rec_stride + comp_offset + c]; 3: the
// same records as floats (real_out then points to float storage).
cudaError_t fft2d_batched(const FftPlan& p, double2* data, int ncomp, int inverse, cudaStream_t st,
                          const double* real_in = nullptr, int out_mode = 0,
                          double* real_out = nullptr, int rec_stride = 0, int comp_offset = 0);
cudaError_t fft_configure_smem();

// ---------------------------------------------------------------------------
// Particles (explicit.cu, sort.cu)
struct ParticleSoA {
    double *x = nullptr, *y = nullptr;
    double *Px = nullptr, *Py = nullptr, *Pz = nullptr;
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;
    double *wx = nullptr, *wy = nullptr, *wz = nullptr;  // previous velocity
    double *q = nullptr, *m = nullptr;                    // per particle, or null (uniform)
    int* id = nullptr;                                    // original index
};

// Deposit tiling.  Tiles are tile_x x tile_y cells in tile-major order; a
// window of wx x wy nodes (the tile plus guard cells and the stencil halo)
// accumulates a chunk's deposit in shared memory.  An axis whose window would
// cover the whole axis is handled as one periodic "full" window.
struct TileGeom {
    int nx, ny;
    int tile_x, tile_y;   // cells per tile
    int ntx, nty;         // tiles per axis
    int guard;            // guard cells around a tile (tiled axes)
    int lo;               // stencil nodes below a particle's key cell
    int span;             // stencil nodes per axis
    int wx, wy;           // window extents in nodes
    int full_x, full_y;   // 1 if the axis window is the whole periodic axis
    int chunk;            // particles per chunk
    // particle key cell = floor((x + key_origin) / dx + key_shift): the
    // nearest node for the explicit method (origin 0, shift 1/2), the cell
    // floor((x + L/2) / dx) for the implicit method (origin L/2, shift 0)
    double key_origin_x, key_origin_y, key_shift;
};

struct Chunk {
    int start, end, tile;
};

struct SortWork {
    unsigned* keys = nullptr;
    unsigned* keys_alt = nullptr;
    int* vals = nullptr;
    int* vals_alt = nullptr;
    int* hist = nullptr;        // digit-major block histograms
    int* scan_tmp = nullptr;    // block sums for the scan
    int* tile_count = nullptr;  // per tile
    int* tile_start = nullptr;  // per tile (exclusive scan)
    int* tile_chunks = nullptr; // chunks per tile, then their exclusive scan
    Chunk* chunks = nullptr;
    int* nchunks = nullptr;     // device scalar
    long cap = 0;
    int hist_cap = 0;
    int ntiles_cap = 0;
    int chunk_cap = 0;
};

// Compute tile-major cell keys of wrap(x + shift*v) and sort the particle
// order; then build the chunk table.  perm receives the sorted source index.
// shift = 0 sorts by the stored positions.
cudaError_t sort_particles_by_tile(const TileGeom& tg, const ParticleSoA& p, long np, double Lx,
                                   double Ly, double shift, SortWork& w, cudaStream_t st);
// Gather every non-null array of src by w.vals (the sorted order) into dst.
cudaError_t permute_particles(const ParticleSoA& src, const ParticleSoA& dst, long np,
                              const SortWork& w, cudaStream_t st);
// dst[id[k]] = src[k] for the arrays x..wz (restores the caller's order).
cudaError_t unpermute_particles(const ParticleSoA& src, const ParticleSoA& dst, long np,
                                cudaStream_t st);
// The buffer a key kernel writes the unsorted cell keys into (the radix
// passes alternate between two buffers and end in w.keys).
unsigned* sort_key_input(const TileGeom& tg, SortWork& w);
// The radix sort of the keys in sort_key_input(tg, w) into w.keys, with the
// sorted source indices in w.vals, and the chunk table (shared by both
// particle formats).
cudaError_t sort_keys_to_chunks(const TileGeom& tg, long np, SortWork& w, cudaStream_t st);

// ---------------------------------------------------------------------------
// Mixed-precision particle state of the explicit step (UPIC_PRECISION_MIXED,
// mixed.cu): per particle the nearest node cell = ix * ny + iy and the
// cell-relative offsets r = x / dx - ix in [-1/2, 1/2), FP32 momenta and
// velocities.
struct MixedSoA {
    int* cell = nullptr;
    float *rx = nullptr, *ry = nullptr;
    float *Px = nullptr, *Py = nullptr, *Pz = nullptr;
    float *vx = nullptr, *vy = nullptr, *vz = nullptr;
    float *wx = nullptr, *wy = nullptr, *wz = nullptr;  // previous velocity
    float *q = nullptr, *m = nullptr;                    // per particle, or null (uniform)
    int* id = nullptr;
};

// Keys of the nearest-node cell after advancing the offsets by (sx vx, sy vy)
// (sx = shift / dx), then sort_keys_to_chunks.
cudaError_t sort_mixed_by_tile(const TileGeom& tg, const MixedSoA& p, long np, int lny, float sx, float sy,
                               SortWork& w, cudaStream_t st);
cudaError_t permute_mixed(const MixedSoA& src, const MixedSoA& dst, long np, const SortWork& w,
                          cudaStream_t st);
// Host layout -> mixed: x, y in [0, L) (doubles), P, v, v_prev as xyz triples
// (doubles, in tmp3 staging on the device) -> the mixed arrays.
cudaError_t mixed_from_positions(long np, const double* x, const double* y, double inv_dx, double inv_dy, int nx,
                                 int ny, int lny, int* cell, float* rx, float* ry, cudaStream_t st);
cudaError_t mixed_split3(long np, const double* aos, float* a, float* b, float* c, cudaStream_t st);
cudaError_t mixed_from_doubles(long np, const double* src, float* dst, cudaStream_t st);
// Mixed (sorted order) -> caller order in dst, then positions / triples as doubles.
cudaError_t unpermute_mixed(const MixedSoA& src, const MixedSoA& dst, long np, cudaStream_t st);
cudaError_t mixed_to_positions(long np, const int* cell, const float* rx, const float* ry, double dx, double dy,
                               double Lx, double Ly, int lny, int ny, double* x, double* y, cudaStream_t st);
cudaError_t mixed_join3(long np, const float* a, const float* b, const float* c, double* aos, cudaStream_t st);

// ---------------------------------------------------------------------------
// Explicit BDF/IAEM step (explicit.cu)
enum DepositMode { kModeDeposit = 0, kModeAdvanceDeposit = 1, kModePush = 2 };

struct PushArgs {
    ParticleSoA p;
    long np;
    double q0, m0;          // uniform charge and mass when p.q / p.m are null
    double Lx, Ly, inv_dx, inv_dy, inv_dA;
    double inv_Lx, inv_Ly;
    double dt, c, inv_c2;
    const double* gfields;  // interleaved node records, kGFStride doubles
    const Chunk* chunks;
    const int* nchunks;
    unsigned long long* acc; // [comp][2][N] fixed-point accumulators (hi, lo)
    double scale[4];         // fixed-point scale per component slot (J x,y,z, rho)
    double* diag_part;       // per-CTA particle reductions (kDiagPart doubles)
};
constexpr int kDiagPart = 5;  // kinetic hi/lo, gamma-sum hi/lo, max speed

// ncomp: 1 (charge only), 3 (current), 4 (current + charge).
cudaError_t launch_push_deposit(int mode, int ncomp, bool uniform_qm, const TileGeom& tg,
                                const PushArgs& a, int grid, cudaStream_t st);
// IAEM momentum push of a particle list in given fields (kernel-level entry
// upic_push_iaem): F = A (3), grad phi (2), grad A (6, dA_c/dx, dA_c/dy per
// component), planar; P, v, v_prev xyz triples updated in place.
cudaError_t launch_iaem_push(long np, const double* x, const double* y, double* P, double* v, double* vp,
                             const double* q, const double* m, const double* F, int nx, int ny, double inv_dx,
                             double inv_dy, double dt, double c, cudaStream_t st);
int push_deposit_smem_bytes(const TileGeom& tg, int ncomp);
cudaError_t push_configure_smem(const TileGeom& tg);
// Resident CTAs per SM of the step's push kernel (ncomp 3 or 4).
int push_occupancy(const TileGeom& tg, int ncomp);

// Mixed-precision step kernel (mixed.cu): the FP32 counterpart of
// push_deposit_kernel with single-word fixed-point deposits.
struct MixedPushArgs {
    MixedSoA p;
    long np;
    float q0f, m0f;          // uniform charge and mass (FP32 arithmetic)
    double m0;               // uniform mass for the FP64 diagnostics
    float dt, dt_dx, dt_dy;  // dt and dt / dx, dt / dy (offsets advance in cells)
    float c, c2, inv_dA;
    double cd, inv_c2d;      // c and 1 / c^2 of the FP64 diagnostics
    int lny;                 // log2(ny)
    const float* gf;         // FP32 node records, kGFStride floats
    const Chunk* chunks;
    const int* nchunks;
    unsigned long long* acc; // [slot][2][N]: the single-word sums go to the first word of a slot
    double scale[4];         // single-word fixed-point scale per slot
    double* diag_part;       // per-CTA particle reductions (kDiagPart doubles)
};
cudaError_t launch_push_mixed(int mode, int ncomp, bool uniform_qm, const TileGeom& tg, const MixedPushArgs& a,
                              int grid, cudaStream_t st);
int push_mixed_smem_bytes(const TileGeom& tg, int ncomp);
cudaError_t push_mixed_configure_smem(const TileGeom& tg);
int push_mixed_occupancy(const TileGeom& tg, int ncomp);
// Single-word accumulators -> J (slots 0..2, mask & 1) and rho = background +
// slot 3 (mask & 2); clears the converted slots.
cudaError_t launch_convert_acc1(unsigned long long* acc, int N, const double* scale, double* J, double* rho,
                                double n0, int ncomp_mask, cudaStream_t st, const double* bg);

// acc -> real fields: J (3 x N) from slots 0..2 when ncomp_mask & 1;
// rho = background + slot 3 when ncomp_mask & 2, the background being bg[id]
// (a fixed charge field) or, with bg null, the uniform n0.  Zeroes the
// converted slots.
cudaError_t launch_convert_acc(unsigned long long* acc, int N, const double* scale,
                               double* J, double* rho, double n0, int ncomp_mask,
                               cudaStream_t st, const double* bg = nullptr);

struct KspaceArgs {
    int N;
    const double *kx, *ky, *k2;
    const double2* Jhat;       // 3 x N
    const double2* rho_dep;    // N (naive charge spectrum) or null
    double2* hist;             // ring: [field(5: phi, Ax, Ay, Az, rho)][slot R][N]
    int R, head;               // slots; head = slot of u^n
    int na;                    // BDF coefficients a[0..na)
    double a[3];
    int nb;
    double b[5];
    double dt, c, eps0, mu0;
    int conserving;
    double2* gspec;            // 11 x N gather-field spectra (output) or null
};
cudaError_t launch_bdf_kspace(const KspaceArgs& a, cudaStream_t st);

// Diagnostics spectra (10 x N): gauge, E (3), gauss, continuity, B (3), rho.
struct DiagKArgs {
    int N;
    const double *kx, *ky, *k2;
    const double2* Jhat;
    const double2* hist;
    int R, slot_new, slot_prev0;  // u^{n+1} slot; past(0) slot
    int na;
    double a[3];
    double dt, c, eps0;
    double2* out;
};
cudaError_t launch_diag_kspace(const DiagKArgs& a, cudaStream_t st);

// Sum-of-squares reductions over the diagnostics fields; writes the row.
struct DiagReduceArgs {
    int N;
    const double* dfields;  // 10 x N real (gauge, Ex, Ey, Ez, gauss, cont, Bx, By, Bz, rho)
    const double* J;        // 3 x N
    double* partials;       // grid x 16
    int grid;
    const double* pdiag;    // particle partials (count x kDiagPart)
    int pcount;
    long np;
    double dA, eps0, mu0;
    double* row;            // 13 doubles (device)
};
cudaError_t launch_diag_reduce(const DiagReduceArgs& a, cudaStream_t st);

// phi_hat = rho_hat/(eps0 k2), 0 at k2 == 0 (into out).
cudaError_t launch_poisson_kspace(int N, const double* k2, const double2* rho_hat, double eps0,
                                  double2* out, cudaStream_t st);
// out = i k_dir * in.
cudaError_t launch_derivative_kspace(int N, const double* k, const double2* in, double2* out,
                                     cudaStream_t st);
// Single BDF solve on explicit spectra (upic_solve_bdf).
cudaError_t launch_bdf_single(int N, const double* k2, const double2* src, const double2* hist,
                              int nb, const double* b, double scale, double2* out, cudaStream_t st);

// out[p] = sum f S(x_p) (quadratic).
cudaError_t launch_gather_scalar(int nx, int ny, double inv_dx, double inv_dy, const double* f,
                                 long np, const double* x, const double* y, double* out,
                                 cudaStream_t st);

// Fill each ring slot of a field with the same spectrum.
cudaError_t launch_fill_hist(double2* hist_field, int R, int N, const double2* src,
                             cudaStream_t st);

}  // namespace upic
