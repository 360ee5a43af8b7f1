// image_ops.cuh — accumulate and display-transform launchers.
#pragma once
#include "vecmath.cuh"

namespace nr {

// StreamConfig display fields (nectar_render/csrc/data/include/data/stream.h:13-30)
// with the white-balance gains resolved on the device.
struct DisplayParams {
  int32_t linear_to_gamma;
  int32_t apply_white_balance;
  float wb_tint;
  int32_t apply_tonemapping;
  int32_t tm_method;
  float tm_white_point;
  float tm_alpha;
  int32_t aligned;
  V3 wb_ratio;
};

cudaError_t display_params_resolve(DisplayParams& p, float temperature, V3* scratch,
                                   cudaStream_t st);
// src: planar float CHW with 3 channels of hw pixels; dst8 (uint8 CHW) and/or
// dstf (float CHW, the pre-quantisation values) may be null.
cudaError_t launch_display(const float* src, uint8_t* dst8, float* dstf, size_t hw,
                           const DisplayParams& p, cudaStream_t st);
cudaError_t launch_accumulate(float* avg, const float* smp, size_t n, uint32_t sample_idx,
                              cudaStream_t st);

}  // namespace nr
