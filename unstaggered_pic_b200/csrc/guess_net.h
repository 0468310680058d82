// Learned first guess of the implicit step's outer current iteration
// (UPIC_PREDICTOR_LEARNED): a 4-layer 3x3 periodic conv net, 32 channels,
// BF16 weights and activations with FP32 accumulation on the tcgen05 tensor
// cores (TMEM accumulators), trained online by Adam on the currents and
// potentials the solver itself produces.  It predicts the correction to the
// polynomial extrapolation 2 J^n - J^(n-1) of the next converged current;
// the outer iteration still runs to the solver tolerance, so the guess
// changes the iteration count, never the accepted solution.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace upic {
namespace gnet {

constexpr int kC = 32;              // channels of every activation (inputs zero-padded)
constexpr int kTaps = 9;            // 3x3 stencil, tap t = (dx+1)*3 + (dy+1)
constexpr int kK = kTaps * kC;      // 288: GEMM depth of one conv
constexpr int kLayers = 4;
constexpr int kW = kC * kK;         // weights of one layer (rows: output channel, k = tap*32 + cin)
constexpr int kParams = kW + kC;    // weights + bias of one layer
constexpr int kInputs = 21;         // J^n, J^(n-1), J^(n-2), A^n, A^(n-1), A^(n-2) (3 each), phi (3)
constexpr int kOutputs = 3;         // correction of J (x, y, z)
constexpr int kFrames = 3;          // field frames kept
constexpr int kFrameFields = 7;     // J (3), A (3), phi

// Conv epilogue modes
enum { kConvRelu = 0, kConvLinear = 1, kConvMask = 2 };

struct ConvArgs {
    const uint16_t* in;    // P x 32 bf16, pixel p = ix*ny + iy
    const uint16_t* w;     // 32 x 288 bf16, row n (output channel), k = tap*32 + cin
    const float* bias;     // 32 or null
    const uint16_t* mask;  // P x 32 bf16 or null (kConvMask: output x (mask > 0))
    uint16_t* out_bf;      // P x 32 bf16 (kConvRelu, kConvMask)
    float* out_f;          // P x 4 fp32, channels 0..2 (kConvLinear)
    int nx, ny, P;
    int sign;              // +1: tap t reads pixel p + d_t; -1: p - d_t (transposed conv)
    int mode;
    int* err;              // set when a bounded wait gives up
};

// One periodic 3x3 conv as an implicit GEMM on the tensor cores: 128-pixel
// tiles (M = 128), N = 32 output channels, K = 288 in 18 tcgen05.mma steps.
cudaError_t launch_conv_tc(const ConvArgs& a, int nsm, cudaStream_t st);
// Test form of kConvLinear: all 32 output channels (out_f: P x 32 fp32).
cudaError_t launch_conv_tc_full(const ConvArgs& a, int nsm, cudaStream_t st);
// Weight and bias gradients of one conv: dW[co][t*32+ci] = sum_p dz[p][co]
// x[p + d_t][ci], db[co] = sum_p dz[p][co], block partials reduced in a
// fixed order (deterministic).  partials: grid x kParams floats.
cudaError_t launch_conv_wgrad(const uint16_t* dz, const uint16_t* x, int nx, int ny, float* partials, int grid,
                              float* grad, cudaStream_t st);

struct Net;

// Create / destroy the network of an nx x ny grid (weights from seed).
cudaError_t net_create(Net** net, int nx, int ny, uint64_t seed, int nsm);
void net_destroy(Net* net);
// Append a field frame (J: 3 x N, A: 3 x N, phi: N; fp64, grid order).
cudaError_t net_push_frame(Net* net, const double* J, const double* A, const double* phi, cudaStream_t st);
// Frames held (0..3).
int net_frames(const Net* net);
// First guess from the last three frames: 2 J^n - J^(n-1) + s * net(frames),
// s the rms of the second difference of J.  guess: 3 x N fp64.
cudaError_t net_predict(Net* net, double* guess, cudaStream_t st);
// Polynomial extrapolation 2 J^n - J^(n-1) of the last two frames.
cudaError_t net_extrapolate(Net* net, double* guess, cudaStream_t st);
// iters Adam steps on the sample (last three frames -> Jnext); loss_out
// (device, 1 double) receives the last step's mean squared error in units
// of the target scale.
cudaError_t net_train(Net* net, const double* Jnext, int iters, float lr, double* loss_out, cudaStream_t st);
// Device error flag (nonzero after a bounded wait gave up).
const int* net_error_flag(const Net* net);
// Serialised weights and optimiser state (checkpoints): bytes and device ranges.
size_t net_state_ranges(Net* net, void** ptrs, size_t* sizes, size_t max_ranges);
// Host-side scalars of the same state (frame ring, Adam step): read
// (write = false) or restore (write = true).
void net_host_state(Net* net, int* newest, int* count, long* adam_t, bool write);

}  // namespace gnet
}  // namespace upic
