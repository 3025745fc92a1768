// 3x3 convolution (stride 1, zero padding 1) as an implicit GEMM on the
// tcgen05 tensor cores, for the learned preconditioner (conv_tc.cu).
//
// Activation layout ("channel-group planar"): a C-channel H x W image is
// stored as [C/8][H][W][8] bf16, i.e. one plane per group of 8 channels with
// the 8 channels of a pixel in one 16-byte chunk.  In that layout 8
// consecutive pixels of one channel group form exactly one tcgen05 core
// matrix (8 rows x 16 bytes), so a TMA-loaded input box is a valid K-major
// MMA operand for every one of the 9 taps by an address offset alone.
//
// Weights are packed once per update as [tap][Cin/8][Cout][8] bf16 (the
// shared-memory image of the B operand); PyTorch's [Cout][Cin][3][3] order
// is the interchange format.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyomgpu {

constexpr int kConvTileX = 128;   // output pixels per row tile (MMA M)
constexpr int kConvThreads = 256;  // 2 warpgroups: TMEM lane quarter = warp % 4, channel half = warp / 4

// Epilogue of one convolution: v = acc + bias, then
//   kEpiPlain: y = act(v (+ addend)) at the input resolution, optional gate
//              (y = 0 where gate <= 0: ReLU backward) and optional 2x2
//              average pool of y into pool_out;
//   kEpiUp:    y (2H x 2W) = act(v broadcast to its 2x2 block + addend), the
//              decoder's upsample + skip (addend required, fine resolution);
//   kEpiF32:   y = v of channel 0 as f32 [H][W].
enum ConvEpilogue : int { kEpiPlain = 0, kEpiUp = 1, kEpiF32 = 2 };

struct ConvArgs {
  CUtensorMap map_x;      // input, box (8, 130, rows+2, Cin/8), rows = the instantiation's tile height
  const uint16_t* wpack;  // [9][Cin/8][Cout][8] bf16
  const float* bias;      // [Cout] or null
  void* y;
  const uint16_t* gate;
  const uint16_t* addend;
  uint16_t* pool_out;
  int H, W, tiles_x, ntiles;
  int relu, epi;
  int* err;               // set to PYOMGPU_TIMEOUT if a wait runs out
  unsigned long long timeout_ns;
};

struct ConvSpec {
  int cin, cout, H, W;    // input channels / size; output channels
  const uint16_t* x;      // device planar input
  const uint16_t* wpack;  // device packed weights
  const float* bias;
  void* y;
  const uint16_t* gate;
  const uint16_t* addend;
  uint16_t* pool_out;
  int relu, epi;
  int* err;
  unsigned long long timeout_ns;
};

// Launches the matching instantiation; returns 0, -1 for an unsupported
// channel pair or shape, -2 for a tensor-map failure, or a cudaError_t.
int conv3x3_launch(const ConvSpec& s, int nsm, cudaStream_t st);
bool conv3x3_supported(int cin, int cout);

// Packs f32 weights [Cout][Cin][3][3] into [tap][Cin/8][Cout][8] bf16 (round
// to nearest even).  flip packs the backward-data kernel instead: channels
// transposed and taps rotated by 180 degrees (its input channels are the
// forward Cout).
void launch_pack_weights(const float* w, int cout, int cin, bool flip, uint16_t* wpack, cudaStream_t st);

}  // namespace pyomgpu
