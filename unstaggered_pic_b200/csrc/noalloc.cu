// Current deposit that allocates no device memory (sm_100a).
//
// Some host programs cannot call cudaMalloc at the point where they want a
// deposit: applications that reserve all device memory up front through
// their own allocator and forbid raw allocations, or latency-critical loops
// that must not risk the implicit device synchronization a cudaMalloc or
// cudaFree can cause.  For them this entry point keeps its scratch -- the
// fixed-point accumulators of the grid and three status words -- in one
// file-scope __device__ array of fixed size, which every GPU that loads
// this library holds until the process exits.  The caller passes device
// pointers for the particles and for the output current.
//
// The kernel is the plain-order variant of the deposit: each particle adds
// its 27 fixed-point contributions (q v_c S_ab / dA, quadratic B-spline of
// Project2/spectral_pic_part3.cpp:537-562, 747-755) straight into the
// global accumulators with integer atomics, so the result is independent of
// the order of the additions and reproducible.  It needs no sort and no
// tile windows, at the price of more atomics than upic_deposit_current.
#include <mutex>

#include "../../include/upic.h"
#include "kernels.h"
#include "upic_common.cuh"

namespace {

using namespace upic;

constexpr long kNoAllocMaxNodes = UPIC_NOALLOC_MAX_NODES;
constexpr long kScratchWords = 6 * kNoAllocMaxNodes + 3;

// Accumulators (hi, lo) x (J_x, J_y, J_z) x nodes, then the bit patterns of
// max|q| and max|v| (non-negative doubles order like their bits), then a
// flag word that is non-zero when a particle value is not finite.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned long long* g_scratch_ptr[kMaxDevices] = {};

// Bounds max|q|, max|v| and the non-finite flag.  fmax drops a NaN operand,
// so non-finite values are caught by an explicit test, not by the bound.
__global__ void noalloc_bound_kernel(long np, const double* __restrict__ x, const double* __restrict__ y,
                                     const double* __restrict__ v, const double* __restrict__ q,
                                     unsigned long long* words) {
    double mq = 0.0, mv = 0.0;
    bool bad = false;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        const double a = v[3 * p], b = v[3 * p + 1], c = v[3 * p + 2];
        const double qp = q[p], sp = sqrt(a * a + b * b + c * c);
        bad |= !(isfinite(qp) && isfinite(sp) && isfinite(x[p]) && isfinite(y[p]));
        mq = fmax(mq, fabs(qp));
        mv = fmax(mv, sp);
    }
    mq = warp_max(mq);
    mv = warp_max(mv);
    const unsigned any_bad = __ballot_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&words[0], (unsigned long long)__double_as_longlong(mq));
        atomicMax(&words[1], (unsigned long long)__double_as_longlong(mv));
        if (any_bad) atomicOr(&words[2], 1ull);
    }
}

__global__ void noalloc_deposit_kernel(int nx, int ny, double inv_dx, double inv_dy, double inv_dA,
                                       long np, const double* __restrict__ x, const double* __restrict__ y,
                                       const double* __restrict__ v, const double* __restrict__ q,
                                       unsigned long long* acc, const unsigned long long* words) {
    const int N = nx * ny;
    if (words[2]) return;  // non-finite input: nothing is deposited, J becomes NaN
    // fixed-point scale from the bound np * max|q| * max|v| / dA on any node
    // value (2^(91 - ceil(log2 bound)), as the context-based deposit uses)
    const double bound = (double)np * __longlong_as_double((long long)words[0]) *
                         __longlong_as_double((long long)words[1]) * inv_dA;
    double scale = 1.0;
    if (bound > 0.0 && isfinite(bound)) {
        int e;
        frexp(bound, &e);
        scale = ldexp(1.0, max(-1000, min(1000, 91 - e)));
    }
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < np; p += (long)gridDim.x * blockDim.x) {
        const Quad1D wx = quadratic_weights(x[p], inv_dx);
        const Quad1D wy = quadratic_weights(y[p], inv_dy);
        const double wxs[3] = {wx.w0, wx.w1, wx.w2};
        const double wys[3] = {wy.w0, wy.w1, wy.w2};
        const double qa = q[p] * inv_dA;
        const double val[3] = {qa * v[3 * p], qa * v[3 * p + 1], qa * v[3 * p + 2]};
        for (int a = 0; a < 3; ++a) {
            const int gx = wrap_index(wx.ic - 1 + a, nx);
            for (int b = 0; b < 3; ++b) {
                const int node = gx * ny + wrap_index(wy.ic - 1 + b, ny);
                const double w = wxs[a] * wys[b];
                for (int c = 0; c < 3; ++c) {
                    const double contrib = val[c] * w;
                    if (contrib == 0.0) continue;
                    const Fixed2 f = to_fixed(contrib, scale);
                    atomicAdd(&acc[(size_t)(2 * c) * N + node], f.hi);
                    atomicAdd(&acc[(size_t)(2 * c + 1) * N + node], f.lo);
                }
            }
        }
    }
}

__global__ void noalloc_convert_kernel(int N, long np, double inv_dA, const unsigned long long* acc,
                                       const unsigned long long* words, double* J) {
    const double bound = (double)np * __longlong_as_double((long long)words[0]) *
                         __longlong_as_double((long long)words[1]) * inv_dA;
    double inv_scale = 1.0;
    if (bound > 0.0 && isfinite(bound)) {
        int e;
        frexp(bound, &e);
        inv_scale = ldexp(1.0, -max(-1000, min(1000, 91 - e)));
    }
    const bool bad = words[2] != 0ull;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < N; id += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c)
            J[(size_t)c * N + id] = bad ? __longlong_as_double(0x7ff8000000000000ll)
                                        : from_fixed(acc[(size_t)(2 * c) * N + id],
                                                     acc[(size_t)(2 * c + 1) * N + id], inv_scale);
}

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

int grid_blocks(long n) {
    long g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return g < 1 ? 1 : (int)g;
}

}  // namespace

extern "C" int upic_deposit_current_noalloc(int nx, int ny, double Lx, double Ly, long np,
                                            const double* x, const double* y, const double* v,
                                            const double* q, double* J, void* stream) {
    if (!is_pow2(nx) || !is_pow2(ny) || !(Lx > 0.0) || !(Ly > 0.0) || np < 0 || !J ||
        (np > 0 && (!x || !y || !v || !q)))
        return UPIC_ERR_ARGUMENT;
    if ((long)nx * ny > kNoAllocMaxNodes) return UPIC_ERR_TOO_LARGE;  // grid larger than the scratch
    // an error left pending by the caller's own earlier launches is not this
    // call's to consume: report it and leave it in place
    if (cudaPeekAtLastError() != cudaSuccess) return UPIC_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return UPIC_ERR_CUDA;
    unsigned long long* scratch = nullptr;
    {
        // once per device, with that device current: the device address of the
        // scratch array (its host-side name is only a stand-in)
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return UPIC_ERR_CUDA;
            g_scratch_ptr[dev] = static_cast<unsigned long long*>(ptr);
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int N = nx * ny;
    unsigned long long* acc = scratch;
    unsigned long long* words = scratch + 6 * (size_t)N;
    // the array keeps the previous call's contents: clear what this call sums into
    if (cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * (6 * (size_t)N + 3), st) != cudaSuccess)
        return UPIC_ERR_CUDA;
    const double dx = Lx / nx, dy = Ly / ny;
    const double inv_dA = 1.0 / (dx * dy);
    if (np > 0) {
        noalloc_bound_kernel<<<grid_blocks(np), 256, 0, st>>>(np, x, y, v, q, words);
        noalloc_deposit_kernel<<<grid_blocks(np), 256, 0, st>>>(nx, ny, 1.0 / dx, 1.0 / dy, inv_dA, np, x, y,
                                                                v, q, acc, words);
        count_launches(2);
    }
    noalloc_convert_kernel<<<grid_blocks(N), 256, 0, st>>>(N, np, inv_dA, acc, words, J);
    count_launches(1);
    if (cudaGetLastError() != cudaSuccess) return UPIC_ERR_CUDA;
    // the non-finite flag decides the return code, so the call waits for its
    // own kernels on `stream` (one 8-byte read into host stack memory)
    unsigned long long flag = 0;
    if (cudaMemcpyAsync(&flag, words + 2, sizeof(flag), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return UPIC_ERR_CUDA;
    return flag ? UPIC_ERR_NONFINITE : UPIC_OK;
}
