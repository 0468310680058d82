// Learned first guess of the implicit outer current iteration: a 4-layer
// 3x3 periodic conv net (32 channels, BF16 weights and activations, FP32
// accumulation) whose convolutions run as implicit GEMMs on the tcgen05
// tensor cores, trained online by Adam.  See guess_net.h.
//
// Conv tile (one CTA of 128 threads per 128-pixel tile, persistent over
// tiles): the im2col rows of the tile (128 x 288 bf16) and the weights
// (32 x 288 bf16) are staged in shared memory in the no-swizzle K-major
// core-matrix layout (8 rows x 16 B per core matrix, 8-row groups 4608 B
// apart, K chunks 128 B apart); one thread issues 18 tcgen05.mma (M = 128,
// N = 32, K = 16) into a 32-column TMEM accumulator and commits them to an
// mbarrier; each warp reads its 32 accumulator lanes back with tcgen05.ld
// for the epilogue (bias, ReLU or the backward ReLU mask).  Every wait is
// bounded: on time-out the kernel sets an error flag, stops issuing work and
// still frees its TMEM.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "guess_net.h"
#include "kernels.h"

namespace upic {
namespace gnet {
namespace {

constexpr int kConvThreads = 128;
constexpr int kTileM = 128;
constexpr int kChunks = kK / 8;                          // 36 16-byte chunks per GEMM row
constexpr int kGroupBytes = kChunks * 128;               // one 8-row group of core matrices
constexpr int kATileBytes = kTileM / 8 * kGroupBytes;    // 73,728
constexpr int kBTileBytes = kC / 8 * kGroupBytes;        // 18,432
constexpr int kSmemConv = kATileBytes + kBTileBytes + 64;
constexpr int kMmaSteps = kK / 16;                       // 18
constexpr uint32_t kTmemCols = 32;
constexpr long kWaitLimit = 1L << 20;
// tcgen05 instruction descriptor, kind::f16: D fp32 (bits 4-5 = 1), A and B
// bf16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at
// bit 24.
constexpr uint32_t kIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kC >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, leading (K-direction)
// and stride (8-row group) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    for (long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ float bf2f(uint16_t b) {
    return __uint_as_float((uint32_t)b << 16);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ int wrapi(int i, int n) {
    return i < 0 ? i + n : (i >= n ? i - n : i);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kConvThreads) conv_tc_kernel(ConvArgs a, int f_ld) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;
    unsigned char* sB = smem + kATileBytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kATileBytes + kBTileBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kATileBytes + kBTileBytes + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: row n, chunk c -> 8-row group n/8, core matrix c, row n%8
    for (int i = tid; i < kC * kChunks; i += kConvThreads) {
        const int n = i / kChunks, c = i - (i / kChunks) * kChunks;
        const uint4 v = *reinterpret_cast<const uint4*>(a.w + (size_t)n * kK + c * 8);
        *reinterpret_cast<uint4*>(sB + (n >> 3) * kGroupBytes + c * 128 + (n & 7) * 16) = v;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB), mAddr = smem_u32(mbar);
    const int ntiles = (a.P + kTileM - 1) / kTileM;
    uint32_t parity = 0;
    bool ok = true;
    // im2col mapping: thread tid fills channel quarter q = tid % 4 of rows
    // r_j = tid / 4 + 32 j (j < 4) for all 9 taps; the loads of three taps
    // (12 x 16 B) are issued before any of their shared-memory stores
    const int q = tid & 3;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int ixs[4], iys[4];
        bool valid[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int p = tile * kTileM + (tid >> 2) + 32 * j;
            valid[j] = p < a.P;
            ixs[j] = valid[j] ? p / a.ny : 0;
            iys[j] = valid[j] ? p - ixs[j] * a.ny : 0;
        }
#pragma unroll
        for (int t0 = 0; t0 < kTaps; t0 += 3) {
            uint4 v[3][4];
#pragma unroll
            for (int dt = 0; dt < 3; ++dt) {
                const int t = t0 + dt;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    v[dt][j] = make_uint4(0u, 0u, 0u, 0u);
                    if (valid[j]) {
                        const int jx = wrapi(ixs[j] + a.sign * (t / 3 - 1), a.nx);
                        const int jy = wrapi(iys[j] + a.sign * (t % 3 - 1), a.ny);
                        v[dt][j] = __ldg(reinterpret_cast<const uint4*>(a.in + ((size_t)jx * a.ny + jy) * kC + q * 8));
                    }
                }
            }
#pragma unroll
            for (int dt = 0; dt < 3; ++dt)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int r = (tid >> 2) + 32 * j;
                    *reinterpret_cast<uint4*>(sA + (r >> 3) * kGroupBytes + ((t0 + dt) * 4 + q) * 128 + (r & 7) * 16) =
                        v[dt][j];
                }
        }
        // make the generic-proxy stores visible to the tensor core
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            for (int s = 0; s < kMmaSteps; ++s) {
                const uint64_t da = umma_desc(aBase + s * 256, 128, kGroupBytes);
                const uint64_t db = umma_desc(bBase + s * 256, 128, kGroupBytes);
                const uint32_t accum = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kIdesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mAddr)
                         : "memory");
        }
        const bool done = mbar_wait(mAddr, parity);
        parity ^= 1u;
        if (!__syncthreads_and(done ? 1 : 0)) {
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t acc[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16), acc);
        const int p = tile * kTileM + warp * 32 + lane;
        if (p < a.P) {
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(acc[j]) + (a.bias ? a.bias[j] : 0.0f);
            if (a.mode == kConvLinear) {
                for (int j = 0; j < f_ld; ++j) a.out_f[(size_t)p * f_ld + j] = v[j];
            } else {
                if (a.mode == kConvRelu) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.0f);
                } else {
                    const uint4* m4 = reinterpret_cast<const uint4*>(a.mask + (size_t)p * kC);
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        const uint4 mv = m4[g];
                        const uint32_t w4[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
                        for (int h = 0; h < 4; ++h) {
                            if (!(bf2f((uint16_t)(w4[h] & 0xFFFFu)) > 0.0f)) v[g * 8 + 2 * h] = 0.0f;
                            if (!(bf2f((uint16_t)(w4[h] >> 16)) > 0.0f)) v[g * 8 + 2 * h + 1] = 0.0f;
                        }
                    }
                }
                uint4* o4 = reinterpret_cast<uint4*>(a.out_bf + (size_t)p * kC);
#pragma unroll
                for (int g = 0; g < 4; ++g)
                    o4[g] = make_uint4(pack2(v[g * 8], v[g * 8 + 1]), pack2(v[g * 8 + 2], v[g * 8 + 3]),
                                       pack2(v[g * 8 + 4], v[g * 8 + 5]), pack2(v[g * 8 + 6], v[g * 8 + 7]));
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (!ok) {
        if (tid == 0) atomicExch(a.err, 1);
        // the committed MMAs of the abandoned tile: wait for them once more
        mbar_wait(mAddr, parity ^ 1u);
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

constexpr int kWgThreads = 256;
constexpr int kWgBatch = 32;

// Weight gradient partials of one block's pixel range (CUDA cores, FP32):
// thread tid owns the 4 x 9 block of outputs co = 4 (tid % 8) + c, k =
// 9 (tid / 8) + kk, so each pixel costs it 13 shared-memory loads for 36
// fused multiply-adds.
__global__ void __launch_bounds__(kWgThreads)
    wgrad_kernel(const uint16_t* dz, const uint16_t* x, int nx, int ny, int P, float* partials) {
    __shared__ __align__(16) float sdz[kWgBatch][kC];
    __shared__ float sx[kWgBatch][kK];
    const int tid = threadIdx.x, cb = (tid & 7) * 4, kb = (tid >> 3) * 9;
    float acc[4][9];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[c][k] = 0.0f;
    float bacc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const int per = (P + gridDim.x - 1) / gridDim.x;
    const int p0 = blockIdx.x * per, p1 = min(P, p0 + per);
    for (int pb = p0; pb < p1; pb += kWgBatch) {
        for (int i = tid; i < kWgBatch * kC; i += kWgThreads) {
            const int q = i / kC, ch = i % kC, p = pb + q;
            sdz[q][ch] = p < p1 ? bf2f(dz[(size_t)p * kC + ch]) : 0.0f;
        }
        for (int i = tid; i < kWgBatch * kTaps * 4; i += kWgThreads) {
            const int q = i / (kTaps * 4), rem = i % (kTaps * 4), t = rem / 4, qq = rem % 4;
            const int p = pb + q;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (p < p1) {
                const int ix = p / ny, iy = p - (p / ny) * ny;
                const int jx = wrapi(ix + t / 3 - 1, nx), jy = wrapi(iy + t % 3 - 1, ny);
                v = __ldg(reinterpret_cast<const uint4*>(x + ((size_t)jx * ny + jy) * kC + qq * 8));
            }
            const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
            float* d = &sx[q][t * kC + qq * 8];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                d[2 * h] = bf2f((uint16_t)(w4[h] & 0xFFFFu));
                d[2 * h + 1] = bf2f((uint16_t)(w4[h] >> 16));
            }
        }
        __syncthreads();
#pragma unroll 4
        for (int q = 0; q < kWgBatch; ++q) {
            const float4 g = *reinterpret_cast<const float4*>(&sdz[q][cb]);
            const float gv[4] = {g.x, g.y, g.z, g.w};
            float xv[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) xv[k] = sx[q][kb + k];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                bacc[c] += gv[c];
#pragma unroll
                for (int k = 0; k < 9; ++k) acc[c][k] = fmaf(gv[c], xv[k], acc[c][k]);
            }
        }
        __syncthreads();
    }
    float* o = partials + (size_t)blockIdx.x * kParams;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 9; ++k) o[(cb + c) * kK + kb + k] = acc[c][k];
    if (kb == 0)
#pragma unroll
        for (int c = 0; c < 4; ++c) o[kW + cb + c] = bacc[c];
}

// grad[j] = sum_b partials[b][j] in block order
__global__ void wgrad_reduce_kernel(const float* partials, int grid, float* grad) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kParams) return;
    float s = 0.0f;
    for (int b = 0; b < grid; ++b) s += partials[(size_t)b * kParams + j];
    grad[j] = s;
}

// Adam on all layers' parameters; refreshes the bf16 weights, their
// per-tap transposes (backward convs) and the fp32 biases.
__global__ void adam_kernel(float* master, float* m1, float* m2, const float* grad, float lr, float b1, float b2,
                            float eps, float c1, float c2, uint16_t* w_bf, uint16_t* wt_bf, float* bias) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kLayers * kParams) return;
    const float g = grad[j];
    const float m = b1 * m1[j] + (1.0f - b1) * g;
    const float v = b2 * m2[j] + (1.0f - b2) * g * g;
    m1[j] = m;
    m2[j] = v;
    const float w = master[j] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    master[j] = w;
    const int L = j / kParams, r = j - L * kParams;
    if (r < kW) {
        const int co = r / kK, k = r - co * kK, t = k / kC, ci = k - t * kC;
        const uint16_t hb = __bfloat16_as_ushort(__float2bfloat16_rn(w));
        w_bf[(size_t)L * kW + r] = hb;
        wt_bf[(size_t)L * kW + ci * kK + t * kC + co] = hb;
    } else {
        bias[L * kC + (r - kW)] = w;
    }
}

constexpr int kRedThreads = 256;
constexpr int kRedGrid = 148;

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    __syncthreads();
    return t;
}

// Sums of squares of the newest frame's J (3 comps), A (3 comps), phi and of
// the second difference J^n - 2 J^(n-1) + J^(n-2); block partials.
__global__ void __launch_bounds__(kRedThreads)
    frame_sums_kernel(const double* fn, const double* f1, const double* f2, int N, double* partials) {
    __shared__ double sh[kRedThreads / 32];
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            const double j = fn[(size_t)c * N + p];
            s[0] += j * j;
            const double a = fn[(size_t)(3 + c) * N + p];
            s[1] += a * a;
            const double d2 = j - 2.0 * f1[(size_t)c * N + p] + f2[(size_t)c * N + p];
            s[3] += d2 * d2;
        }
        const double ph = fn[(size_t)6 * N + p];
        s[2] += ph * ph;
    }
    for (int k = 0; k < 4; ++k) {
        const double t = block_sum(s[k], sh);
        if (threadIdx.x == 0) partials[k * gridDim.x + blockIdx.x] = t;
    }
}

// scales = {1/rms J, 1/rms A, 1/rms phi, rms of the second difference}
__global__ void frame_scales_kernel(const double* partials, int grid, int N, double* scales) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[4];
    for (int k = 0; k < 4; ++k) {
        double t = 0.0;
        for (int b = 0; b < grid; ++b) t += partials[k * grid + b];
        s[k] = t;
    }
    const double rj = sqrt(s[0] / (3.0 * N)), ra = sqrt(s[1] / (3.0 * N)), rp = sqrt(s[2] / (double)N);
    const double rd = sqrt(s[3] / (3.0 * N));
    scales[0] = rj > 0.0 ? 1.0 / rj : 1.0;
    scales[1] = ra > 0.0 ? 1.0 / ra : 1.0;
    scales[2] = rp > 0.0 ? 1.0 / rp : 1.0;
    scales[3] = rd > 0.0 ? rd : (rj > 0.0 ? 1.0e-12 * rj : 1.0e-300);
}

// Network input: J (3 frames), A (3 frames), phi (3 frames), scaled; 21
// channels of 32, the rest zero.
__global__ void features_kernel(const double* fn, const double* f1, const double* f2, int N,
                                const double* scales, uint16_t* x0) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const double* fr[3] = {fn, f1, f2};
    float v[kC];
#pragma unroll
    for (int j = 0; j < kC; ++j) v[j] = 0.0f;
    for (int f = 0; f < 3; ++f)
        for (int c = 0; c < 3; ++c) {
            v[f * 3 + c] = (float)(fr[f][(size_t)c * N + p] * scales[0]);
            v[9 + f * 3 + c] = (float)(fr[f][(size_t)(3 + c) * N + p] * scales[1]);
        }
    for (int f = 0; f < 3; ++f) v[18 + f] = (float)(fr[f][(size_t)6 * N + p] * scales[2]);
    uint4* o4 = reinterpret_cast<uint4*>(x0 + (size_t)p * kC);
#pragma unroll
    for (int g = 0; g < 4; ++g)
        o4[g] = make_uint4(pack2(v[g * 8], v[g * 8 + 1]), pack2(v[g * 8 + 2], v[g * 8 + 3]),
                           pack2(v[g * 8 + 4], v[g * 8 + 5]), pack2(v[g * 8 + 6], v[g * 8 + 7]));
}

// target[p][c] = (J_next - (2 J^n - J^(n-1))) / s
__global__ void target_kernel(const double* jnext, const double* fn, const double* f1, int N, const double* scales,
                              float* target) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const double inv = 1.0 / scales[3];
    for (int c = 0; c < 3; ++c) {
        const double ex = 2.0 * fn[(size_t)c * N + p] - f1[(size_t)c * N + p];
        target[(size_t)p * 4 + c] = (float)((jnext[(size_t)c * N + p] - ex) * inv);
    }
    target[(size_t)p * 4 + 3] = 0.0f;
}

// guess = 2 J^n - J^(n-1) (+ s * out)
__global__ void guess_kernel(const double* fn, const double* f1, int N, const double* scales, const float* out,
                             double* guess) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * N) return;
    const int c = i / N, p = i - c * N;
    double g = 2.0 * fn[i] - f1[i];
    if (out) g += scales[3] * (double)out[(size_t)p * 4 + c];
    guess[i] = g;
}

// dz = out - target on channels 0..2 (bf16, other channels zero); block
// partial sums of the squared error.
__global__ void __launch_bounds__(kRedThreads)
    loss_kernel(const float* out, const float* target, int P, uint16_t* dz, double* partials) {
    __shared__ double sh[kRedThreads / 32];
    double s = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        float d[3];
        for (int c = 0; c < 3; ++c) {
            d[c] = out[(size_t)p * 4 + c] - target[(size_t)p * 4 + c];
            s += (double)d[c] * (double)d[c];
        }
        uint4* o4 = reinterpret_cast<uint4*>(dz + (size_t)p * kC);
        o4[0] = make_uint4(pack2(d[0], d[1]), pack2(d[2], 0.0f), 0u, 0u);
        o4[1] = make_uint4(0u, 0u, 0u, 0u);
        o4[2] = make_uint4(0u, 0u, 0u, 0u);
        o4[3] = make_uint4(0u, 0u, 0u, 0u);
    }
    const double t = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void loss_final_kernel(const double* partials, int grid, int P, double* loss) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (int b = 0; b < grid; ++b) t += partials[b];
    *loss = t / (3.0 * (double)P);
}

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// standard normal by Box-Muller on two 53-bit uniforms
double normal(uint64_t& s) {
    const double u1 = ((splitmix64(s) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

uint16_t host_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even (finite values)
    return (uint16_t)(r >> 16);
}

}  // namespace

cudaError_t launch_conv_tc(const ConvArgs& a, int nsm, cudaStream_t st) {
    const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(conv_tc_kernel), kSmemConv);
    if (e != cudaSuccess) return e;
    const int ntiles = (a.P + kTileM - 1) / kTileM;
    const int grid = std::min(ntiles, 2 * nsm);
    if (grid <= 0) return cudaSuccess;
    conv_tc_kernel<<<grid, kConvThreads, kSmemConv, st>>>(a, 4);
    count_launches(1);
    return cudaGetLastError();
}

// Test form: linear outputs of all 32 channels (out_f: P x 32).
cudaError_t launch_conv_tc_full(const ConvArgs& a, int nsm, cudaStream_t st) {
    const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(conv_tc_kernel), kSmemConv);
    if (e != cudaSuccess) return e;
    const int ntiles = (a.P + kTileM - 1) / kTileM;
    const int grid = std::min(ntiles, 2 * nsm);
    if (grid <= 0) return cudaSuccess;
    conv_tc_kernel<<<grid, kConvThreads, kSmemConv, st>>>(a, kC);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_conv_wgrad(const uint16_t* dz, const uint16_t* x, int nx, int ny, float* partials, int grid,
                              float* grad, cudaStream_t st) {
    wgrad_kernel<<<grid, kWgThreads, 0, st>>>(dz, x, nx, ny, nx * ny, partials);
    wgrad_reduce_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(partials, grid, grad);
    count_launches(2);
    return cudaGetLastError();
}

struct Net {
    int nx = 0, ny = 0, N = 0, nsm = 148;
    int wg_grid = 0;
    double* frames = nullptr;  // 3 slots x 7 x N
    int newest = -1, count = 0;
    uint16_t *x0 = nullptr, *y[3] = {nullptr, nullptr, nullptr}, *dza = nullptr, *dzb = nullptr;
    float *out = nullptr, *target = nullptr;
    float *master = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *bias = nullptr;
    uint16_t *w_bf = nullptr, *wt_bf = nullptr;
    float* wg_part = nullptr;
    double* red = nullptr;     // reduction partials (4 x kRedGrid)
    double* scales = nullptr;  // 4
    int* err = nullptr;
    long adam_t = 0;
    std::vector<void*> allocs;
};

namespace {
template <typename T>
cudaError_t nalloc(Net* n, T** p, size_t count) {
    void* v = nullptr;
    const cudaError_t e = cudaMalloc(&v, sizeof(T) * (count ? count : 1));
    if (e != cudaSuccess) return e;
    n->allocs.push_back(v);
    *p = reinterpret_cast<T*>(v);
    return cudaMemset(v, 0, sizeof(T) * (count ? count : 1));
}

const double* slot(const Net* n, int back) {
    const int s = ((n->newest - back) % kFrames + kFrames) % kFrames;
    return n->frames + (size_t)s * kFrameFields * n->N;
}

cudaError_t conv(Net* n, int layer, const uint16_t* in, int sign, int mode, const uint16_t* mask, uint16_t* out_bf,
                 float* out_f, cudaStream_t st) {
    ConvArgs a{};
    a.in = in;
    a.w = (sign > 0 ? n->w_bf : n->wt_bf) + (size_t)layer * kW;
    a.bias = sign > 0 ? n->bias + layer * kC : nullptr;
    a.mask = mask;
    a.out_bf = out_bf;
    a.out_f = out_f;
    a.nx = n->nx;
    a.ny = n->ny;
    a.P = n->N;
    a.sign = sign;
    a.mode = mode;
    a.err = n->err;
    return launch_conv_tc(a, n->nsm, st);
}

cudaError_t scales_and_features(Net* n, cudaStream_t st) {
    const double *fn = slot(n, 0), *f1 = slot(n, 1), *f2 = slot(n, 2);
    frame_sums_kernel<<<kRedGrid, kRedThreads, 0, st>>>(fn, f1, f2, n->N, n->red);
    frame_scales_kernel<<<1, 32, 0, st>>>(n->red, kRedGrid, n->N, n->scales);
    features_kernel<<<(n->N + 255) / 256, 256, 0, st>>>(fn, f1, f2, n->N, n->scales, n->x0);
    count_launches(3);
    return cudaGetLastError();
}

cudaError_t forward(Net* n, cudaStream_t st) {
    cudaError_t e;
    if ((e = conv(n, 0, n->x0, 1, kConvRelu, nullptr, n->y[0], nullptr, st))) return e;
    if ((e = conv(n, 1, n->y[0], 1, kConvRelu, nullptr, n->y[1], nullptr, st))) return e;
    if ((e = conv(n, 2, n->y[1], 1, kConvRelu, nullptr, n->y[2], nullptr, st))) return e;
    return conv(n, 3, n->y[2], 1, kConvLinear, nullptr, nullptr, n->out, st);
}
}  // namespace

cudaError_t net_create(Net** out, int nx, int ny, uint64_t seed, int nsm) {
    Net* n = new Net();
    n->nx = nx;
    n->ny = ny;
    n->N = nx * ny;
    n->nsm = nsm > 0 ? nsm : 148;
    n->wg_grid = std::max(1, std::min(2 * n->nsm, (n->N + 255) / 256));
    const size_t N = (size_t)n->N;
    cudaError_t e;
    if ((e = nalloc(n, &n->frames, (size_t)kFrames * kFrameFields * N)) || (e = nalloc(n, &n->x0, N * kC)) ||
        (e = nalloc(n, &n->y[0], N * kC)) || (e = nalloc(n, &n->y[1], N * kC)) || (e = nalloc(n, &n->y[2], N * kC)) ||
        (e = nalloc(n, &n->dza, N * kC)) || (e = nalloc(n, &n->dzb, N * kC)) || (e = nalloc(n, &n->out, N * 4)) ||
        (e = nalloc(n, &n->target, N * 4)) || (e = nalloc(n, &n->master, (size_t)kLayers * kParams)) ||
        (e = nalloc(n, &n->m1, (size_t)kLayers * kParams)) || (e = nalloc(n, &n->m2, (size_t)kLayers * kParams)) ||
        (e = nalloc(n, &n->grad, (size_t)kLayers * kParams)) || (e = nalloc(n, &n->bias, (size_t)kLayers * kC)) ||
        (e = nalloc(n, &n->w_bf, (size_t)kLayers * kW)) || (e = nalloc(n, &n->wt_bf, (size_t)kLayers * kW)) ||
        (e = nalloc(n, &n->wg_part, (size_t)n->wg_grid * kParams)) || (e = nalloc(n, &n->red, 4 * kRedGrid)) ||
        (e = nalloc(n, &n->scales, 4)) || (e = nalloc(n, &n->err, 1))) {
        net_destroy(n);
        return e;
    }
    // He-normal hidden layers over the real inputs; a small output layer on
    // the three real outputs; padded rows and columns zero; biases zero.
    std::vector<float> w((size_t)kLayers * kParams, 0.0f);
    std::vector<uint16_t> wb((size_t)kLayers * kW, 0), wt((size_t)kLayers * kW, 0);
    uint64_t s = seed;
    for (int L = 0; L < kLayers; ++L) {
        const int cin = L == 0 ? kInputs : kC;
        const int cout = L == kLayers - 1 ? kOutputs : kC;
        const double sd = (L == kLayers - 1 ? 0.1 : 1.0) * std::sqrt((L == kLayers - 1 ? 1.0 : 2.0) / (kTaps * cin));
        for (int co = 0; co < cout; ++co)
            for (int t = 0; t < kTaps; ++t)
                for (int ci = 0; ci < cin; ++ci) {
                    const float v = (float)(sd * normal(s));
                    const int r = co * kK + t * kC + ci;
                    w[(size_t)L * kParams + r] = v;
                    wb[(size_t)L * kW + r] = host_bf16(v);
                    wt[(size_t)L * kW + ci * kK + t * kC + co] = host_bf16(v);
                }
    }
    if ((e = cudaMemcpy(n->master, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(n->w_bf, wb.data(), sizeof(uint16_t) * wb.size(), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(n->wt_bf, wt.data(), sizeof(uint16_t) * wt.size(), cudaMemcpyHostToDevice))) {
        net_destroy(n);
        return e;
    }
    *out = n;
    return cudaSuccess;
}

void net_destroy(Net* n) {
    if (!n) return;
    for (void* p : n->allocs) cudaFree(p);
    delete n;
}

cudaError_t net_push_frame(Net* n, const double* J, const double* A, const double* phi, cudaStream_t st) {
    n->newest = (n->newest + 1) % kFrames;
    n->count = std::min(n->count + 1, kFrames);
    double* f = n->frames + (size_t)n->newest * kFrameFields * n->N;
    const size_t b = sizeof(double) * n->N;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(f, J, 3 * b, cudaMemcpyDeviceToDevice, st)) ||
        (e = cudaMemcpyAsync(f + 3 * (size_t)n->N, A, 3 * b, cudaMemcpyDeviceToDevice, st)) ||
        (e = cudaMemcpyAsync(f + 6 * (size_t)n->N, phi, b, cudaMemcpyDeviceToDevice, st)))
        return e;
    return cudaSuccess;
}

int net_frames(const Net* n) {
    return n->count;
}

cudaError_t net_extrapolate(Net* n, double* guess, cudaStream_t st) {
    if (n->count < 2) return cudaErrorInvalidValue;
    guess_kernel<<<(3 * n->N + 255) / 256, 256, 0, st>>>(slot(n, 0), slot(n, 1), n->N, n->scales, nullptr, guess);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t net_predict(Net* n, double* guess, cudaStream_t st) {
    if (n->count < kFrames) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = scales_and_features(n, st)) || (e = forward(n, st))) return e;
    guess_kernel<<<(3 * n->N + 255) / 256, 256, 0, st>>>(slot(n, 0), slot(n, 1), n->N, n->scales, n->out, guess);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t net_train(Net* n, const double* Jnext, int iters, float lr, double* loss_out, cudaStream_t st) {
    if (n->count < kFrames) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = scales_and_features(n, st))) return e;
    target_kernel<<<(n->N + 255) / 256, 256, 0, st>>>(Jnext, slot(n, 0), slot(n, 1), n->N, n->scales, n->target);
    count_launches(1);
    const float b1 = 0.9f, b2 = 0.999f;
    for (int it = 0; it < iters; ++it) {
        if ((e = forward(n, st))) return e;
        loss_kernel<<<kRedGrid, kRedThreads, 0, st>>>(n->out, n->target, n->N, n->dza, n->red);
        loss_final_kernel<<<1, 32, 0, st>>>(n->red, kRedGrid, n->N, loss_out);
        count_launches(2);
        // layer 3 (output), then back through the ReLU layers
        float* g = n->grad;
        if ((e = launch_conv_wgrad(n->dza, n->y[2], n->nx, n->ny, n->wg_part, n->wg_grid, g + 3 * kParams, st)))
            return e;
        if ((e = conv(n, 3, n->dza, -1, kConvMask, n->y[2], n->dzb, nullptr, st))) return e;
        if ((e = launch_conv_wgrad(n->dzb, n->y[1], n->nx, n->ny, n->wg_part, n->wg_grid, g + 2 * kParams, st)))
            return e;
        if ((e = conv(n, 2, n->dzb, -1, kConvMask, n->y[1], n->dza, nullptr, st))) return e;
        if ((e = launch_conv_wgrad(n->dza, n->y[0], n->nx, n->ny, n->wg_part, n->wg_grid, g + kParams, st))) return e;
        if ((e = conv(n, 1, n->dza, -1, kConvMask, n->y[0], n->dzb, nullptr, st))) return e;
        if ((e = launch_conv_wgrad(n->dzb, n->x0, n->nx, n->ny, n->wg_part, n->wg_grid, g, st))) return e;
        ++n->adam_t;
        const float c1 = 1.0f - (float)std::pow((double)b1, (double)n->adam_t);
        const float c2 = 1.0f - (float)std::pow((double)b2, (double)n->adam_t);
        adam_kernel<<<(kLayers * kParams + 255) / 256, 256, 0, st>>>(n->master, n->m1, n->m2, n->grad, lr, b1, b2,
                                                                      1e-8f, c1, c2, n->w_bf, n->wt_bf, n->bias);
        count_launches(1);
        if ((e = cudaGetLastError())) return e;
    }
    return cudaSuccess;
}

const int* net_error_flag(const Net* n) {
    return n->err;
}

size_t net_state_ranges(Net* n, void** ptrs, size_t* sizes, size_t max_ranges) {
    const size_t N = (size_t)n->N;
    void* p[] = {n->frames, n->master, n->m1, n->m2, n->bias, n->w_bf, n->wt_bf};
    const size_t s[] = {sizeof(double) * kFrames * kFrameFields * N, sizeof(float) * kLayers * kParams,
                        sizeof(float) * kLayers * kParams,           sizeof(float) * kLayers * kParams,
                        sizeof(float) * kLayers * kC,                sizeof(uint16_t) * kLayers * kW,
                        sizeof(uint16_t) * kLayers * kW};
    const size_t k = sizeof(p) / sizeof(p[0]);
    for (size_t i = 0; i < k && i < max_ranges; ++i) {
        ptrs[i] = p[i];
        sizes[i] = s[i];
    }
    return k;
}

// Host-side scalar state (frame ring position, Adam step) for checkpoints.
void net_host_state(Net* n, int* newest, int* count, long* adam_t, bool write) {
    if (write) {
        n->newest = *newest;
        n->count = *count;
        n->adam_t = *adam_t;
    } else {
        *newest = n->newest;
        *count = n->count;
        *adam_t = n->adam_t;
    }
}

}  // namespace gnet
}  // namespace upic
