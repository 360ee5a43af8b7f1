// integrator.cuh — launch interface of the path-tracing kernels.
#pragma once
#include "pathcore.cuh"

namespace nr {

constexpr int kMegaThreads = 128;

struct KernelParams {
  DevScene scene;
  DevCamera cam;
  uint32_t W, H;
  uint32_t first_sample, n_samples;
  uint32_t seed, depth;
  int32_t rr_enabled;
  uint32_t rr_start;
  float rr_survival;
  int32_t mode;       // NR_MODE_*
  int32_t rtl;        // multi-draw constructor arguments consume draws right to left
  int32_t write_raw;  // write the raw sample instead of folding it into the mean
  float* beauty;      // planar CHW, 3 channels
  float* diffuse;
  float* normal;
  float* depth_layer; // planar 1-channel first-hit distance (wavefront only), or null
  double* beauty64;   // FP64 running sum of beauty, or null
  uint32_t* primary;  // raw mode: primary hit id per pixel, or null
  uint32_t* work_counter;
  uint32_t* err;
  unsigned long long* counters;  // rays, nodes, tris, objects, paths
};

cudaError_t launch_init_constants(float hdri_rotation_deg, CubeFace* d_faces, M3* host_hdri_rot,
                                  cudaStream_t st);
cudaError_t launch_megakernel(const KernelParams& P, bool counters, cudaStream_t st);
int mega_grid_blocks();

}  // namespace nr
