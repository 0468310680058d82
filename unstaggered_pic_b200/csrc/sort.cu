// Particle ordering for the tiled deposit (sm_100a).
//
// The reference keeps particles in a fixed array order and scatters them one
// by one (Project2/spectral_pic_part3.cpp:747-755); it has no sorting.  Here
// particles are periodically reordered by the nearest-node cell of their next
// gather position, in tile-major cell order, so that a warp's 32 particles
// share a handful of cells (broadcast gathers, long runs in the segmented
// deposit reduction) and a CTA's chunk fits one shared-memory window.
//
// The sort is a stable LSD radix sort of (cell key, index) pairs written for
// this purpose: block histograms, a device-wide exclusive scan, and a scatter
// whose in-block ranks come from warp match/popc and per-warp counts in fixed
// order.  It is therefore deterministic: equal inputs give equal orders, and
// with it the deposit's fixed summation order.
#include "kernels.h"
#include "upic_common.cuh"

namespace upic {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // elements per block
constexpr int kSortWarps = kSortThreads / kWarp;
constexpr int kMaxDigits = 256;                       // 8-bit digits at most
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void make_keys_kernel(TileGeom tg, ParticleSoA p, long np, double Lx, double Ly,
                                 double inv_dx, double inv_dy, double shift, unsigned* keys) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < np; q += (long)gridDim.x * blockDim.x) {
        double x = p.x[q], y = p.y[q];
        if (shift != 0.0) {
            x = wrap_periodic(x + shift * p.vx[q], Lx, 1.0 / Lx);
            y = wrap_periodic(y + shift * p.vy[q], Ly, 1.0 / Ly);
        }
        const int icx = wrap_index((int)floor((x + tg.key_origin_x) * inv_dx + tg.key_shift), tg.nx);
        const int icy = wrap_index((int)floor((y + tg.key_origin_y) * inv_dy + tg.key_shift), tg.ny);
        const int tx = icx / tg.tile_x, lx = icx - tx * tg.tile_x;
        const int ty = icy / tg.tile_y, ly = icy - ty * tg.tile_y;
        const unsigned tile = (unsigned)(tx * tg.nty + ty);
        keys[q] = tile * (unsigned)(tg.tile_x * tg.tile_y) + (unsigned)(lx * tg.tile_y + ly);
    }
}

// Digit histogram of one block's kSortTile keys.  Each warp reads its
// kSortItems * 32 keys ahead of counting and adds one shared atomic per
// distinct digit of each 32 (match/popc): the keys of a re-sort are nearly
// sorted already, so most rounds cost one atomic instead of 32 on one word.
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const unsigned* __restrict__ keys, long n, int shift, int digits, int nblocks,
                  int* hist) {
    __shared__ int cnt[kMaxDigits];
    for (int d = threadIdx.x; d < digits; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const unsigned mask = (unsigned)digits - 1u;
    const long wbase = (long)blockIdx.x * kSortTile + (long)warp * (kSortItems * kWarp) + lane;
    unsigned key[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const long e = wbase + r * kWarp;
        key[r] = e < n ? keys[e] : 0u;
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const bool valid = wbase + r * kWarp < n;
        const int d = valid ? (int)((key[r] >> shift) & mask) : digits;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && (peers & lt) == 0) atomicAdd(&cnt[d], __popc(peers));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < digits; d += blockDim.x) hist[(long)d * nblocks + blockIdx.x] = cnt[d];
}

// Stable scatter of one digit pass, 256 keys per round: a key's in-block
// rank is the digit's count in the block's earlier rounds, plus its count in
// the round's earlier warps, plus its rank among its own warp's equal digits
// (match/popc); offs holds the scanned histograms (digit-major).  IDENT: the
// values are the source indices (the first pass of a sort, so the key kernel
// writes no values).
template <bool IDENT>
__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const unsigned* __restrict__ keys, const int* __restrict__ vals, long n, int shift,
                     int digits, int nblocks, const int* __restrict__ offs, unsigned* __restrict__ okeys,
                     int* __restrict__ ovals) {
    __shared__ int base_cnt[kMaxDigits];
    __shared__ int gofs[kMaxDigits];
    __shared__ int wcnt[kSortWarps][kMaxDigits];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = threadIdx.x; d < digits; d += blockDim.x) {
        base_cnt[d] = 0;
        gofs[d] = offs[(long)d * nblocks + blockIdx.x];
    }
    const unsigned mask = (unsigned)digits - 1u;
    const unsigned lt = (1u << lane) - 1u;
    const long base = (long)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortItems; ++r) {
        for (int k = threadIdx.x; k < kSortWarps * kMaxDigits; k += blockDim.x) (&wcnt[0][0])[k] = 0;
        __syncthreads();
        const long e = base + r * kSortThreads + threadIdx.x;
        const bool valid = e < n;
        unsigned key = 0;
        int d = digits;  // sentinel for inactive lanes
        if (valid) {
            key = keys[e];
            d = (int)((key >> shift) & mask);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int lrank = __popc(peers & lt);
        if (valid && lrank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int rank = base_cnt[d] + lrank;
            for (int w = 0; w < warp; ++w) rank += wcnt[w][d];
            const int dst = gofs[d] + rank;
            okeys[dst] = key;
            ovals[dst] = IDENT ? (int)e : vals[e];
        }
        __syncthreads();
        for (int dd = threadIdx.x; dd < digits; dd += blockDim.x) {
            int s = 0;
            for (int w = 0; w < kSortWarps; ++w) s += wcnt[w][dd];
            base_cnt[dd] += s;
        }
        __syncthreads();
    }
}

// ---- exclusive scan of int arrays ------------------------------------------
__device__ int block_exclusive_scan(int v, int* total) {
    __shared__ int ws[kScanThreads / kWarp];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = lane < kScanThreads / kWarp ? ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanThreads / kWarp) ws[lane] = s;
    }
    __syncthreads();
    const int warp_excl = warp > 0 ? ws[warp - 1] : 0;
    *total = ws[kScanThreads / kWarp - 1];
    __syncthreads();
    return warp_excl + x - v;
}

__global__ void __launch_bounds__(kScanThreads)
scan_blocks_kernel(const int* in, int* out, long n, int* block_sums) {
    const long base = (long)blockIdx.x * kScanTile + (long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int ex = block_exclusive_scan(s, &total);
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(int* sums, int nb, int* grand) {
    int carry = 0;
    for (int base = 0; base < nb; base += kScanThreads) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        int total;
        const int ex = block_exclusive_scan(v, &total);
        if (i < nb) sums[i] = ex + carry;
        carry += total;
    }
    if (threadIdx.x == 0 && grand) *grand = carry;
}

__global__ void scan_add_kernel(int* out, long n, const int* sums) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kScanTile];
}

cudaError_t exclusive_scan(const int* in, int* out, long n, int* tmp, int* grand, cudaStream_t st) {
    const int nb = (int)((n + kScanTile - 1) / kScanTile);
    scan_blocks_kernel<<<nb, kScanThreads, 0, st>>>(in, out, n, tmp);
    scan_sums_kernel<<<1, kScanThreads, 0, st>>>(tmp, nb, grand);
    scan_add_kernel<<<(int)((n + 255) / 256), 256, 0, st>>>(out, n, tmp);
    count_launches(3);
    return cudaGetLastError();
}

// ---- chunk table ----------------------------------------------------------
// Tile extents of the sorted keys without atomics: position q opens every
// tile in (tile(key[q-1]), tile(key[q])]; tile_start[ntiles] = n.
__global__ void tile_bounds_kernel(const unsigned* keys, long n, unsigned cells_per_tile, int ntiles,
                                   int* tstart) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q <= n; q += (long)gridDim.x * blockDim.x) {
        const int t = q < n ? (int)(keys[q] / cells_per_tile) : ntiles;
        const int tp = q > 0 ? (int)(keys[q - 1] / cells_per_tile) : -1;
        for (int k = tp + 1; k <= t; ++k) tstart[k] = (int)q;
    }
}

__global__ void tile_counts_kernel(const int* tstart, int ntiles, int* cnt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntiles) cnt[t] = tstart[t + 1] - tstart[t];
}

__global__ void tile_chunks_kernel(const int* cnt, int ntiles, int chunk, int* nch) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntiles) nch[t] = (cnt[t] + chunk - 1) / chunk;
}

__global__ void fill_chunks_kernel(const int* cnt, const int* tstart, const int* cstart, int ntiles,
                                   int chunk, Chunk* chunks) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int c = cnt[t];
    const int s = tstart[t];
    int o = cstart[t];
    for (int k = 0; k < c; k += chunk) {
        Chunk ch;
        ch.start = s + k;
        ch.end = s + (k + chunk < c ? k + chunk : c);
        ch.tile = t;
        chunks[o++] = ch;
    }
}

template <typename T>
__global__ void gather_array_kernel(const T* __restrict__ src, T* __restrict__ dst, const int* idx,
                                    long n) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        dst[q] = src[idx[q]];
}

// All payload arrays of the particle set gathered by one pass over the
// sorted index: dst_k[q] = src_k[idx[q]] for the double arrays present (and
// the original index); the index is read once instead of once per array.
struct GatherSet {
    const double* src[13];
    double* dst[13];
    int narr;
    const int* sid;
    int* did;
};

// One array after the other: each store waits for its load, so a thread
// has one load in flight.  Loading all of a particle's values ahead of the
// stores (13 loads in flight) measured slower on the nearly sorted re-sort
// gathers (7.15-7.21 against 6.85 ms per explicit step at 512x512 x 256).
__global__ void gather_set_kernel(GatherSet g, const int* __restrict__ idx, long n) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
        const int i = idx[q];
#pragma unroll
        for (int k = 0; k < 13; ++k)
            if (k < g.narr) g.dst[k][q] = g.src[k][i];
        if (g.did) g.did[q] = g.sid[i];
    }
}

// All of a particle's values are loaded before the scattered stores (the
// arrays may alias as far as the compiler knows, so a load placed after a
// store stays after it).
__global__ void unpermute_kernel(ParticleSoA s, ParticleSoA d, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int o = s.id[k];
        const double v[11] = {s.x[k],  s.y[k],  s.Px[k], s.Py[k], s.Pz[k], s.vx[k],
                              s.vy[k], s.vz[k], s.wx[k], s.wy[k], s.wz[k]};
        d.x[o] = v[0];
        d.y[o] = v[1];
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

int grid_for(long n) {
    long g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return g < 1 ? 1 : (int)g;
}

// Digit passes of the radix sort for the grid's cell keys: ceil(bits / 8)
// passes of equal width (at most 8 bits).
int radix_passes(const TileGeom& tg, int* dbits) {
    const long ncells = (long)tg.nx * tg.ny;
    int bits = 0;
    while ((1L << bits) < ncells) ++bits;
    if (bits == 0) bits = 1;
    const int passes = (bits + 7) / 8;
    *dbits = (bits + passes - 1) / passes;
    return passes;
}

}  // namespace

unsigned* sort_key_input(const TileGeom& tg, SortWork& w) {
    int dbits;
    return (radix_passes(tg, &dbits) & 1) ? w.keys_alt : w.keys;
}

cudaError_t sort_particles_by_tile(const TileGeom& tg, const ParticleSoA& p, long np, double Lx,
                                   double Ly, double shift, SortWork& w, cudaStream_t st) {
    if (np <= 0) {
        cudaMemsetAsync(w.nchunks, 0, sizeof(int), st);
        return cudaGetLastError();
    }
    const double inv_dx = (double)tg.nx / Lx, inv_dy = (double)tg.ny / Ly;
    make_keys_kernel<<<grid_for(np), 256, 0, st>>>(tg, p, np, Lx, Ly, inv_dx, inv_dy, shift,
                                                   sort_key_input(tg, w));
    count_launches(1);
    return sort_keys_to_chunks(tg, np, w, st);
}

cudaError_t sort_keys_to_chunks(const TileGeom& tg, long np, SortWork& w, cudaStream_t st) {
    if (np <= 0) {
        cudaMemsetAsync(w.nchunks, 0, sizeof(int), st);
        return cudaGetLastError();
    }
    int dbits;
    const int passes = radix_passes(tg, &dbits);
    const int digits = 1 << dbits;
    const int nblocks = (int)((np + kSortTile - 1) / kSortTile);
    // The passes alternate between the two buffers and end in w.keys / w.vals;
    // the key kernel wrote the first pass's input (sort_key_input).
    const bool odd = passes & 1;
    unsigned* kin = odd ? w.keys_alt : w.keys;
    unsigned* kout = odd ? w.keys : w.keys_alt;
    int* vin = nullptr;
    int* vout = odd ? w.vals : w.vals_alt;
    for (int ps = 0; ps < passes; ++ps) {
        const int shift_bits = ps * dbits;
        radix_hist_kernel<<<nblocks, kSortThreads, 0, st>>>(kin, np, shift_bits, digits, nblocks, w.hist);
        exclusive_scan(w.hist, w.hist, (long)digits * nblocks, w.scan_tmp, nullptr, st);
        if (ps == 0)
            radix_scatter_kernel<true><<<nblocks, kSortThreads, 0, st>>>(kin, nullptr, np, shift_bits, digits,
                                                                         nblocks, w.hist, kout, vout);
        else
            radix_scatter_kernel<false><<<nblocks, kSortThreads, 0, st>>>(kin, vin, np, shift_bits, digits,
                                                                          nblocks, w.hist, kout, vout);
        count_launches(2);
        unsigned* tk = kin; kin = kout; kout = tk;
        vin = vout;
        vout = vout == w.vals ? w.vals_alt : w.vals;
    }
    // chunk table
    const int ntiles = tg.ntx * tg.nty;
    tile_bounds_kernel<<<grid_for(np + 1), 256, 0, st>>>(w.keys, np, (unsigned)(tg.tile_x * tg.tile_y),
                                                         ntiles, w.tile_start);
    tile_counts_kernel<<<(ntiles + 255) / 256, 256, 0, st>>>(w.tile_start, ntiles, w.tile_count);
    count_launches(2);
    tile_chunks_kernel<<<(ntiles + 255) / 256, 256, 0, st>>>(w.tile_count, ntiles, tg.chunk, w.tile_chunks);
    exclusive_scan(w.tile_chunks, w.tile_chunks, ntiles, w.scan_tmp, w.nchunks, st);
    fill_chunks_kernel<<<(ntiles + 255) / 256, 256, 0, st>>>(w.tile_count, w.tile_start, w.tile_chunks,
                                                             ntiles, tg.chunk, w.chunks);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t permute_particles(const ParticleSoA& s, const ParticleSoA& d, long np, const SortWork& w,
                              cudaStream_t st) {
    const int g = grid_for(np);
    double* const src[13] = {s.x, s.y, s.Px, s.Py, s.Pz, s.vx, s.vy, s.vz, s.wx, s.wy, s.wz, s.q, s.m};
    double* const dst[13] = {d.x, d.y, d.Px, d.Py, d.Pz, d.vx, d.vy, d.vz, d.wx, d.wy, d.wz, d.q, d.m};
    GatherSet gs{};
    for (int k = 0; k < 13; ++k)
        if (src[k] && dst[k]) {
            gs.src[gs.narr] = src[k];
            gs.dst[gs.narr] = dst[k];
            ++gs.narr;
        }
    if (s.id && d.id) {
        gs.sid = s.id;
        gs.did = d.id;
    }
    if (np > 0) {
        gather_set_kernel<<<g, 256, 0, st>>>(gs, w.vals, np);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t unpermute_particles(const ParticleSoA& s, const ParticleSoA& d, long np, cudaStream_t st) {
    unpermute_kernel<<<grid_for(np), 256, 0, st>>>(s, d, np);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace upic
