// net.cuh -- the learned coarse proposal: a small convolutional network that predicts the displacement field at 1/8
// resolution from an image pair (net.cu). It stands in for the POC coarse stage (python/optflow_ref/poc.py:216-239,
// rust/crates/optflow-core/src/poc.rs:694 coarse_flow), never for the refinement that follows it.
//
// Architecture (activations NHWC bfloat16, every convolution a tensor-core GEMM with float32 accumulation):
//   encoder, shared by both images (run as one batch of 2B images):
//     E1 3x3 stride 2, 1 -> 16, ReLU;  E2 3x3 stride 2, 16 -> 32, ReLU;  E3 3x3 stride 2, 32 -> 32, ReLU;
//     E4 3x3, 32 -> 32                                        -> features f at 1/8 resolution
//   correlation C(p, d) = <f1(p), f2(p + d)> / 32 for d in [-5, 5]^2 cells (121 channels; zero outside the image)
//   decoder on [C, f1, 7 zero channels] (160 channels):
//     D1 3x3, 160 -> 64, ReLU;  D2 3x3 dilation 2, 64 -> 64, ReLU;  D3 3x3 dilation 4, 64 -> 32, ReLU;
//     D4 3x3, 32 -> 16 (the first two channels used)
//   flow (px, at the cell centres 8 i + 3.5) = 8 * soft-argmax_d C(p, d) + D4[0:2]
// Parameters: per layer a weight matrix [cout][kpad] (kpad = 9 cin rounded up to 16; column (ky 3 + kx) cin + c)
// followed by cout biases, all float32 in one vector (param_count()).
#pragma once
#include <cstdint>
#include <functional>
#include <string>

#include <cuda_runtime.h>

namespace ofc {
namespace net {

struct ConvSpec {
  int cin, cout, stride, dil, relu;
};
constexpr int NCONV = 8;
constexpr ConvSpec SPECS[NCONV] = {{1, 16, 2, 1, 1},   {16, 32, 2, 1, 1}, {32, 32, 2, 1, 1}, {32, 32, 1, 1, 0},
                                   {160, 64, 1, 1, 1}, {64, 64, 1, 2, 1}, {64, 32, 1, 4, 1}, {32, 16, 1, 1, 0}};
constexpr int CORR_R = 5, CORR_D = 2 * CORR_R + 1, CORR_N = CORR_D * CORR_D, FEAT = 32, DEC_IN = 160;
constexpr int SCALE = 8;  // the network's output grid: one cell per 8 x 8 pixels

inline int kpad(int cin) { return (9 * cin + 15) / 16 * 16; }
size_t param_offset(int layer);  // float index of layer's weights; its biases follow
size_t param_count();

// device memory for the network's work buffers, by name (reused across calls of the same size)
using Alloc = std::function<void*(const std::string&, size_t)>;

struct Workspace {
  Alloc alloc;
  cudaStream_t st;
};

// forward pass on nb image pairs of h x w float32 pixels (i1, i2: nb images each, contiguous), h and w multiples of 8;
// weights16: the bfloat16 copy of the weights (param layout), params: float32 parameters (biases are read from it).
// flow: nb x (h / 8) x (w / 8) x 2 floats (ux, uy in px at the cell centres).
void forward(const Workspace& ws, const float* params, const uint16_t* weights16, const float* i1, const float* i2,
             int nb, int h, int w, float* flow);

// forward + backward of the loss (1 / cells) sum over the masked cells of sqrt(|flow - target|^2 + 0.01) (target and
// mask at the cells); grads (param layout, float32) are overwritten; loss (device double) receives the loss.
void forward_backward(const Workspace& ws, const float* params, const uint16_t* weights16, const float* i1,
                      const float* i2, int nb, int h, int w, const float* target, const uint8_t* mask, float* flow,
                      float* grads, double* loss);

// Adam step (float32 master weights, moments m and v) and the bfloat16 copy of the updated weights
void adam(const Workspace& ws, float* params, const float* grads, float* m, float* v, uint16_t* weights16, float lr,
          float beta1, float beta2, float eps, int step);

// the bfloat16 copy of the weights from the float32 parameters
void to_bf16(const Workspace& ws, const float* params, uint16_t* weights16);

}  // namespace net
}  // namespace ofc
