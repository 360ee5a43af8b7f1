// conv_tc.cuh — 3x3 convolutions (stride 1, zero padding 1) over NHWC BF16
// activations as implicit GEMMs on the tcgen05 tensor cores, FP32
// accumulation in tensor memory. Used by the learned denoiser.
//
//   forward / backward-data:  Y[p, co] = sum_{tap, ci} X[p + off(tap), ci] * W[tap][co][ci]
//   backward-weights:         dW[tap][co][ci] += sum_p dY[p, co] * X[p + off(tap), ci]
//
// Backward-data is the forward kernel with the weights rearranged as
// W'[tap][ci][co] = W[8 - tap][co][ci] (a 3x3 "full" convolution with the
// kernel rotated by 180 degrees).
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace nr {

struct ConvFwdArgs {
  const __nv_bfloat16* x;  // [P, x_stride], channels [x_off, x_off + cin)
  int32_t x_stride, x_off;
  const __nv_bfloat16* w;  // [9][cout][cin]
  const float* bias;       // [cout] or null
  __nv_bfloat16* y;        // [P, y_stride], channels [y_off, y_off + cout)
  int32_t y_stride, y_off;
  int32_t cin, cout;       // multiples of 16; cin <= 256, cout <= 256
  int32_t B, H, W;         // images of H x W pixels; P = B * H * W, a multiple of 128
  int32_t relu;
  uint32_t* err;           // bit 1: a tensor-core wait timed out
  int32_t taps;            // 9: 3x3 convolution; 1: centre tap only, i.e. the
                           // GEMM y[p] = W x[p] (w is then [1][cout][cin])
};

struct ConvWgradArgs {
  const __nv_bfloat16* dy;  // [P, dy_stride], channels [dy_off, dy_off + cout)
  int32_t dy_stride, dy_off;
  const __nv_bfloat16* x;   // [P, x_stride], channels [x_off, x_off + cin)
  int32_t x_stride, x_off;
  float* dw;                // [9][cout][cin], accumulated with atomics
  int32_t cin, cout;        // multiples of 16; cout <= 128, cin <= 256
  int32_t B, H, W;
  int32_t chunks_per_cta;   // 128-pixel chunks reduced by one CTA
  uint32_t* err;
  int32_t taps;             // 9, or 1: dw[0] += dy^T x (a GEMM over pixels)
};

size_t conv_fwd_smem_bytes(int cin, int cout);
size_t conv_wgrad_smem_bytes(int cin);
cudaError_t launch_conv_fwd(const ConvFwdArgs& a, cudaStream_t st);
cudaError_t launch_conv_wgrad(const ConvWgradArgs& a, cudaStream_t st);

}  // namespace nr
