// Batched radix-2 complex FFT for the collocated periodic grid (sm_100a).
//
// Replaces the reference's fft1d/fft2d (Project2/spectral_pic_part3.cpp:372-424;
// Project3/ec_pic_nyquist_projected.cpp:1566-1670): forward
// f_hat[k] = sum_j f[j] exp(-2 pi i jk/n); the inverse is scaled by 1/n in
// each 1D pass, and a 2D transform is the y-line pass followed by the x-line
// pass, as in the reference.
//
// Each CTA stages whole lines in shared memory (bit-reversed on load, then
// log2(n) in-place radix-2 butterfly passes, twiddles from an accurate table
// rather than the reference's w *= wlen recurrence).  y lines are contiguous;
// an x-pass CTA loads a block of adjacent columns so every global access is a
// coalesced run along y.
#include "kernels.h"
#include "upic_common.cuh"

namespace upic {

namespace {

constexpr int kFftThreads = 256;
// Complex elements staged per CTA (64 KB of shared memory); a single line
// longer than this stages alone (up to 8192 elements, 128 KB).
constexpr int kFftSmemElems = 4096;
constexpr int kFftMaxN = 8192;

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) {
    return bits == 0 ? 0u : (__brev(v) >> (32 - bits));
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place radix-2 DIT passes over `lines` bit-reversed lines of length n
// stored contiguously in s.  tw[m] = exp(-2 pi i m / n), m < n/2.
__device__ void butterflies(double2* s, int lines, int n, int log2n, const double2* __restrict__ tw,
                            bool inverse) {
    const int half_total = lines * (n >> 1);
    for (int st = 1; st <= log2n; ++st) {
        const int half = 1 << (st - 1);
        const int tstride = n >> st;  // twiddle index step
        for (int b = threadIdx.x; b < half_total; b += blockDim.x) {
            const int line = b >> (log2n - 1);
            const int k = b & ((n >> 1) - 1);
            const int j = k & (half - 1);
            const int grp = k >> (st - 1);
            const int i0 = line * n + grp * 2 * half + j;
            const int i1 = i0 + half;
            double2 w = __ldg(&tw[j * tstride]);
            if (inverse) w.y = -w.y;
            const double2 u = s[i0];
            const double2 v = cmul(s[i1], w);
            s[i0] = make_double2(u.x + v.x, u.y + v.y);
            s[i1] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

// y-lines: line index L in [0, ncomp*nx), elements contiguous (stride 1).
// in_mode 0: complex in place; 1: real planar input (imag = 0) from `rin`
// (component stride N).  out_mode 0: complex to `data`.
__global__ void __launch_bounds__(kFftThreads)
fft_y_kernel(double2* __restrict__ data, const double* __restrict__ rin, int in_mode, int nlines,
             int n, int log2n, int lines_per_cta, const double2* __restrict__ tw, int inverse) {
    extern __shared__ double2 smem[];
    const int line0 = blockIdx.x * lines_per_cta;
    const int lines = min(lines_per_cta, nlines - line0);
    if (lines <= 0) return;
    const int total = lines * n;
    const size_t base = (size_t)line0 * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int l = e / n, j = e - l * n;
        double2 v;
        if (in_mode == 1) v = make_double2(rin[base + e], 0.0);
        else v = data[base + e];
        smem[l * n + bitrev(j, log2n)] = v;
    }
    __syncthreads();
    butterflies(smem, lines, n, log2n, tw, inverse != 0);
    const double sc = inverse ? 1.0 / (double)n : 1.0;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        double2 v = smem[e];
        if (inverse) { v.x *= sc; v.y *= sc; }
        data[base + e] = v;
    }
}

// x-lines: for component c and column block [j0, j0+cols), element i of
// column j lives at c*N + i*ny + j.  out_mode 0: complex in place;
// 1: real part to rout[(c*N + node) ...] planar (rout_comp_stride = N,
// rout_node_stride = 1); 2: real part to interleaved records
// rout[node*rec_stride + comp_offset + c]; 3: the same records in FP32 (rout
// then points to floats).
__global__ void __launch_bounds__(kFftThreads)
fft_x_kernel(double2* __restrict__ data, int ncomp, int nx, int ny, int log2nx, int cols_per_cta,
             const double2* __restrict__ tw, int inverse, int out_mode, double* __restrict__ rout,
             int rec_stride, int comp_offset) {
    extern __shared__ double2 smem[];
    const int blocks_per_comp = ny / cols_per_cta;
    const int c = blockIdx.x / blocks_per_comp;
    const int j0 = (blockIdx.x - c * blocks_per_comp) * cols_per_cta;
    if (c >= ncomp) return;
    const size_t N = (size_t)nx * ny;
    double2* d = data + c * N;
    const int total = nx * cols_per_cta;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int i = e / cols_per_cta, cc = e - i * cols_per_cta;
        smem[cc * nx + bitrev(i, log2nx)] = d[(size_t)i * ny + j0 + cc];
    }
    __syncthreads();
    butterflies(smem, cols_per_cta, nx, log2nx, tw, inverse != 0);
    const double sc = inverse ? 1.0 / (double)nx : 1.0;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int i = e / cols_per_cta, cc = e - i * cols_per_cta;
        double2 v = smem[cc * nx + i];
        if (inverse) { v.x *= sc; v.y *= sc; }
        const size_t node = (size_t)i * ny + j0 + cc;
        if (out_mode == 0) d[node] = v;
        else if (out_mode == 1) rout[c * N + node] = v.x;
        else if (out_mode == 2) rout[node * rec_stride + comp_offset + c] = v.x;
        else reinterpret_cast<float*>(rout)[node * rec_stride + comp_offset + c] = (float)v.x;
    }
}

int ilog2(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

}  // namespace

// Lines-per-CTA choices keep every CTA at <= kFftSmemElems staged elements.
static int y_lines_per_cta(int ny) { return ny >= kFftSmemElems ? 1 : kFftSmemElems / ny; }
static int x_cols_per_cta(int nx, int ny) {
    int c = nx >= kFftSmemElems ? 1 : kFftSmemElems / nx;
    if (c > ny) c = ny;
    return c;
}

cudaError_t fft2d_batched(const FftPlan& p, double2* data, int ncomp, int inverse, cudaStream_t st,
                          const double* real_in, int out_mode, double* real_out, int rec_stride,
                          int comp_offset) {
    const int nx = p.nx, ny = p.ny;
    const int nl = ncomp * nx;
    const int lpc = y_lines_per_cta(ny);
    const int gy = (nl + lpc - 1) / lpc;
    const size_t smy = sizeof(double2) * (size_t)lpc * ny;
    fft_y_kernel<<<gy, kFftThreads, smy, st>>>(data, real_in, real_in ? 1 : 0, nl, ny, ilog2(ny),
                                               lpc, p.tw_y, inverse);
    const int cpc = x_cols_per_cta(nx, ny);
    const int gx = ncomp * (ny / cpc);
    const size_t smx = sizeof(double2) * (size_t)cpc * nx;
    fft_x_kernel<<<gx, kFftThreads, smx, st>>>(data, ncomp, nx, ny, ilog2(nx), cpc, p.tw_x, inverse,
                                               out_mode, real_out, rec_stride, comp_offset);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t fft_configure_smem() {
    const int bytes = (int)(sizeof(double2) * kFftMaxN);
    cudaError_t e = cudaFuncSetAttribute(fft_y_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fft_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace upic
