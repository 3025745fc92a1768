// U-Net of the learned preconditioner: 4 levels (16/32/64/64 channels),
// 3x3 convolutions on the tcgen05 kernels of conv_tc.cuh, BF16 weights and
// activations, FP32 accumulation, additive skips (unet.cu).
//
//   L1 (H x W):      A1 = relu(c0(X0))   S1 = relu(c1(A1)), P1 = pool(S1)
//   L2 (H/2 x W/2):  A2 = relu(c2(P1))   S2 = relu(c3(A2)), P2 = pool(S2)
//   L3 (H/4 x W/4):  A3 = relu(c4(P2))   S3 = relu(c5(A3)), P3 = pool(S3)
//   L4 (H/8 x W/8):  A4 = relu(c6(P3))   B4 = relu(c7(A4))
//   decoder:         U3 = relu(up(c8(B4)) + S3)
//                    U2 = relu(up(c9(U3)) + S2)
//                    U1 = relu(up(c10(U2)) + S1)
//   output:          z  = channel 0 of c11(U1)      (f32, H x W)
//
// X0 has 16 channels (4 used: scaled residual, mask, 1/H, cos(lat)).  H and
// W are multiples of 8.  Parameters are f32 master copies (weights in
// PyTorch order, then biases) packed to bf16 for the kernels after every
// update.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyomgpu {

constexpr int kUNetLayers = 12;

struct UNetLayer {
  int cin, cout;
  int level;  // resolution level of the convolution's input (0 = L1)
  int epi;    // ConvEpilogue
};
extern const UNetLayer kUNet[kUNetLayers];

size_t unet_weight_offset(int layer);  // f32 index of layer's weights in the parameter vector
size_t unet_bias_offset(int layer);
size_t unet_num_params();

struct UNet {
  int H = 0, W = 0, nsm = 1;
  float* params = nullptr;  // unet_num_params() f32
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  int adam_t = 0;
  uint16_t* wpack[kUNetLayers] = {};
  uint16_t* wflip[kUNetLayers] = {};
  // activations (planar bf16)
  uint16_t *X0 = nullptr, *A1 = nullptr, *S1 = nullptr, *U1 = nullptr;
  uint16_t *P1 = nullptr, *A2 = nullptr, *S2 = nullptr, *U2 = nullptr;
  uint16_t *P2 = nullptr, *A3 = nullptr, *S3 = nullptr, *U3 = nullptr;
  uint16_t *P3 = nullptr, *A4 = nullptr, *B4 = nullptr;
  float* z = nullptr;  // [H][W]
  // gradients (planar bf16)
  uint16_t *gO = nullptr, *gU1 = nullptr, *gv10 = nullptr, *gU2 = nullptr, *gv9 = nullptr, *gU3 = nullptr,
           *gv8 = nullptr;
  uint16_t *gB4 = nullptr, *gA4 = nullptr, *gP3 = nullptr, *gS3 = nullptr, *gA3 = nullptr, *gP2 = nullptr;
  uint16_t *gS2 = nullptr, *gA2 = nullptr, *gP1 = nullptr, *gS1 = nullptr, *gA1 = nullptr;
  int* err = nullptr;
  unsigned long long timeout_ns = 2000000000ull;
  bool training = false;
};

// Allocates the buffers for an H x W input (multiples of 8); training adds
// the gradient and optimiser buffers.  Returns 0 or a negative code.
int unet_alloc(UNet& n, int H, int W, bool training);
void unet_free(UNet& n);
// Repacks the bf16 weights (forward, and flipped when training) from params.
void unet_pack(UNet& n, cudaStream_t st);
// X0 -> z.  Returns 0 or a conv launch error.
int unet_forward(UNet& n, cudaStream_t st);
// grads = d loss / d params for gz = d loss / d z (f32 [H][W]); after a forward.
int unet_backward(UNet& n, const float* gz, cudaStream_t st);
// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on params, then repack.
void unet_adam(UNet& n, float lr, cudaStream_t st);

}  // namespace pyomgpu
