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

// white_balance (stream.cu:88-109), tonemaps (stream.cu:7-59), gamma (:115-121)
__device__ __forceinline__ V3 display_pixel(V3 c, const DisplayParams& p) {
  if (p.apply_white_balance) {
    c = c * p.wb_ratio;
    float tint = p.wb_tint * 0.0025f;
    c = V3{c.x * (1.0f + tint * 0.5f), c.y * (1.0f - tint), c.z * (1.0f + tint * 0.5f)};
  }
  if (p.apply_tonemapping) {
    V3 col = c;
    if (p.tm_method == 1) {  // REINHARD_EXTENDED
      float inv_white2 = 1.0f / (p.tm_white_point * p.tm_white_point);
      V3 num = col * (v3(1.0f) + col * inv_white2);
      col = num / (v3(1.0f) + col);
    } else if (p.tm_method == 2) {  // ACES fit
      const float a = 2.51f, b = 0.03f, cc = 2.43f, d = 0.59f, e = 0.14f;
      V3 x = col;
      V3 num = x * (x * a + b);
      V3 den = x * (x * cc + d) + e;
      col = V3{fminf(1.0f, fmaxf(0.0f, num.x / den.x)), fminf(1.0f, fmaxf(0.0f, num.y / den.y)),
               fminf(1.0f, fmaxf(0.0f, num.z / den.z))};
    }
    // REINHARD leaves col unchanged: the reference discards its result.
    float alpha = p.tm_alpha;
    c = ((1.0f - alpha) * c + alpha * col);
    c = V3{fminf(1.0f, fmaxf(0.0f, c.x)), fminf(1.0f, fmaxf(0.0f, c.y)),
           fminf(1.0f, fmaxf(0.0f, c.z))};
  }
  if (p.linear_to_gamma) {
    c = V3{c.x > 0.0f ? sqrtf(c.x) : 0.0f, c.y > 0.0f ? sqrtf(c.y) : 0.0f,
           c.z > 0.0f ? sqrtf(c.z) : 0.0f};
  }
  return c;
}

// to_image (stream.cu:123-140): NaN -> 0, clamp, *255, truncate.
__device__ __forceinline__ float quant_pre(float v) {
  if (isnan(v)) v = 0.0f;
  v = fmaxf(0.0f, fminf(1.0f, v));
  return v * 255.0f;
}

cudaError_t display_params_resolve(DisplayParams& p, float temperature, V3* scratch,
                                   cudaStream_t st);
// src: planar float CHW with 3 channels of hw pixels; dst8 (uint8 CHW) and/or
// dstf (float CHW, the pre-quantisation values) may be null.
cudaError_t launch_display(const float* src, uint8_t* dst8, float* dstf, size_t hw,
                           const DisplayParams& p, cudaStream_t st);
cudaError_t launch_accumulate(float* avg, const float* smp, size_t n, uint32_t sample_idx,
                              cudaStream_t st);

}  // namespace nr
