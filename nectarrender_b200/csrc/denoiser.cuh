// denoiser.cuh — learned denoiser: a five-level U-Net over the beauty,
// diffuse and world-normal layers, trained and run on the GPU with the
// tcgen05 convolutions of conv_tc.cu. It takes the place of the reference's
// OIDN stage (nectar_render/csrc/data/include/data/denoise.h:21-104), which
// reads the same three layers.
//
// Network (channels per level, 3x3 convolutions + ReLU, 2x2 average pooling,
// nearest 2x upsampling, skip connections by channel concatenation):
//   input 16 = log(1 + beauty) 3, diffuse 3, normal 3, log(1 + depth) 1,
//            zeros 6
//   encoder  32, 48, 64, 96, 128 (two convolutions per level)
//   decoder  96, 64, 48, 32 (two convolutions per level, after concat)
//   output   16 (first 3 = correction to log(1 + beauty), no activation:
//            the prediction is log(1 + noisy beauty) + output)
// Loss: absolute error in log space (or squared error); Adam.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>
#include <string>
#include <vector>

namespace nr {

struct DenoiserNet;  // defined in denoiser.cu

struct Denoiser {
  DenoiserNet* net = nullptr;
  ~Denoiser();
};

// All image arguments are device float planar CHW, B images of H x W
// (H and W multiples of 16), stacked: [B][3][H][W].
std::string denoiser_create(Denoiser& d, uint32_t max_pixels, uint32_t seed);
// depth: [B][1][H][W] first-hit distances, or null (zeros)
std::string denoiser_forward_backward(Denoiser& d, const float* beauty, const float* diffuse,
                                      const float* normal, const float* depth, const float* target,
                                      int B, int H, int W, double* loss, cudaStream_t st);
std::string denoiser_adam(Denoiser& d, float lr, cudaStream_t st);
std::string denoiser_infer(Denoiser& d, const float* beauty, const float* diffuse,
                           const float* normal, const float* depth, float* out, int B, int H, int W,
                           cudaStream_t st);
std::string denoiser_set_loss(Denoiser& d, int kind);  // 1 absolute, 0 squared
size_t denoiser_param_count(const Denoiser& d);
std::string denoiser_get(const Denoiser& d, int what, float* host);  // 0 weights, 1 gradients
std::string denoiser_set_weights(Denoiser& d, const float* host);
int denoiser_layer_count(const Denoiser& d);
void denoiser_layer_shape(const Denoiser& d, int i, int* cin, int* cout);

}  // namespace nr
