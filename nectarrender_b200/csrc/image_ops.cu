// image_ops.cu — accumulation and display transform of planar CHW layers.
//
// Both kernels are HBM-bound streaming passes: each thread handles four
// consecutive pixels of every channel plane (16-byte float loads, 4-byte
// uint8 stores), the grid is a multiple of the SM count, and the tail is
// bounds-checked (the reference's 2D kernels have no guard,
// nectar_render/csrc/data/include/data/utils.h:12-21, so widths or heights
// not divisible by 16 write out of range there).
#include "image_ops.cuh"

namespace nr {

// kelvin_to_rgb (nectar_render/csrc/data/src/stream.cu:65-86)
__device__ __forceinline__ V3 kelvin_to_rgb(float kelvin) {
  float temp = kelvin / 100.0f;
  float r, g, b;
  if (temp <= 66.0f) {
    r = 255.0f;
    g = 99.4708025861f * logf(temp) - 161.1195681661f;
  } else {
    r = 329.698727446f * powf(temp - 60.0f, -0.1332047592f);
    g = 288.1221695283f * powf(temp - 60.0f, -0.0755148492f);
  }
  if (temp >= 66.0f) b = 255.0f;
  else if (temp <= 19.0f) b = 0.0f;
  else b = 138.5177312231f * logf(temp - 10.0f) - 305.0447927307f;
  return V3{fminf(1.0f, fmaxf(0.0f, r / 255.0f)), fminf(1.0f, fmaxf(0.0f, g / 255.0f)),
            fminf(1.0f, fmaxf(0.0f, b / 255.0f))};
}

__global__ void k_display(const float* __restrict__ src, uint8_t* __restrict__ dst8,
                          float* __restrict__ dstf, size_t hw, DisplayParams p) {
  size_t n4 = hw / 4;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (hw + 3) / 4;
       q += (size_t)gridDim.x * blockDim.x) {
    size_t i0 = q * 4;
    float r[4], g[4], b[4];
    if (q < n4 && p.aligned) {
      float4 R = __ldg(reinterpret_cast<const float4*>(src) + q);
      float4 G = __ldg(reinterpret_cast<const float4*>(src + hw) + q);
      float4 B = __ldg(reinterpret_cast<const float4*>(src + 2 * hw) + q);
      r[0] = R.x; r[1] = R.y; r[2] = R.z; r[3] = R.w;
      g[0] = G.x; g[1] = G.y; g[2] = G.z; g[3] = G.w;
      b[0] = B.x; b[1] = B.y; b[2] = B.z; b[3] = B.w;
    } else {
      for (int k = 0; k < 4; ++k) {
        size_t i = i0 + k;
        r[k] = i < hw ? src[i] : 0.f;
        g[k] = i < hw ? src[hw + i] : 0.f;
        b[k] = i < hw ? src[2 * hw + i] : 0.f;
      }
    }
    uint8_t o8[3][4];
    for (int k = 0; k < 4; ++k) {
      V3 c = display_pixel(V3{r[k], g[k], b[k]}, p);
      if (dstf) {
        size_t i = i0 + k;
        if (i < hw) {
          dstf[i] = c.x;
          dstf[hw + i] = c.y;
          dstf[2 * hw + i] = c.z;
        }
      }
      o8[0][k] = (uint8_t)quant_pre(c.x);
      o8[1][k] = (uint8_t)quant_pre(c.y);
      o8[2][k] = (uint8_t)quant_pre(c.z);
    }
    if (dst8) {
      if (q < n4 && p.aligned) {
        for (int ch = 0; ch < 3; ++ch) {
          uint32_t w = (uint32_t)o8[ch][0] | ((uint32_t)o8[ch][1] << 8) |
                       ((uint32_t)o8[ch][2] << 16) | ((uint32_t)o8[ch][3] << 24);
          reinterpret_cast<uint32_t*>(dst8 + ch * hw)[q] = w;
        }
      } else {
        for (int k = 0; k < 4; ++k) {
          size_t i = i0 + k;
          if (i < hw)
            for (int ch = 0; ch < 3; ++ch) dst8[ch * hw + i] = o8[ch][k];
        }
      }
    }
  }
}

// accumulate_samples_kernel (nectar_render/csrc/data/src/data.cu:28-50)
__global__ void k_accumulate(float* __restrict__ avg, const float* __restrict__ smp, size_t n,
                             uint32_t sample_idx) {
  float fn = (float)sample_idx;
  float k_old = (fn - 1.0f) / fn, k_new = 1.0f / fn;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    avg[i] = avg[i] * k_old + smp[i] * k_new;
  }
}

static int grid_for(size_t work) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
  }
  size_t blocks = (work + 255) / 256;
  size_t cap = (size_t)sms * 8;
  return (int)(blocks < cap ? (blocks ? blocks : 1) : cap);
}

// White-balance gains are per-frame constants; the reference evaluates them per
// pixel with device math, so they are evaluated here by one device thread.
__global__ void k_wb_ratio(float temperature, V3* out) {
  V3 reference = kelvin_to_rgb(6500.0f);
  V3 target = kelvin_to_rgb(fmaxf(1000.0f, fminf(temperature, 40000.0f)));
  *out = V3{target.x / fmaxf(reference.x, 1e-4f), target.y / fmaxf(reference.y, 1e-4f),
            target.z / fmaxf(reference.z, 1e-4f)};
}

cudaError_t display_params_resolve(DisplayParams& p, float temperature, V3* scratch,
                                   cudaStream_t st) {
  if (!p.apply_white_balance) return cudaSuccess;
  k_wb_ratio<<<1, 1, 0, st>>>(temperature, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(&p.wb_ratio, scratch, sizeof(V3), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

cudaError_t launch_display(const float* src, uint8_t* dst8, float* dstf, size_t hw,
                           const DisplayParams& p, cudaStream_t st) {
  DisplayParams q = p;
  q.aligned = ((reinterpret_cast<uintptr_t>(src) & 15u) == 0 && (hw % 4) == 0 &&
               (reinterpret_cast<uintptr_t>(dst8) & 3u) == 0)
                  ? 1
                  : 0;
  k_display<<<grid_for((hw + 3) / 4), 256, 0, st>>>(src, dst8, dstf, hw, q);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(float* avg, const float* smp, size_t n, uint32_t sample_idx,
                              cudaStream_t st) {
  k_accumulate<<<grid_for(n), 256, 0, st>>>(avg, smp, n, sample_idx);
  return cudaGetLastError();
}

}  // namespace nr
