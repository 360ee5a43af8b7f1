// viewport.cuh — launch interface of the viewport, picking and selection
// kernels (viewport.cu).
#pragma once
#include "pathstep.cuh"

namespace nr {

// Result of a picking ray: the fields of the reference's HitRecord a caller
// reads (hittable/include/hittable/hit_record.h:9-22).
struct PickOut {
  int32_t hit;
  uint32_t object_id;
  uint32_t material_id;
  float t;
  float p[3];
  float n[3];
  float uv[2];
  int32_t front_face;
};

cudaError_t launch_viewport(const KernelParams& P, int32_t show_axis_grid, cudaStream_t st);
cudaError_t launch_pick(const KernelParams& P, float su, float sv, PickOut* d_out, cudaStream_t st);
cudaError_t launch_selection_mask(const KernelParams& P, uint32_t object_id, int radius,
                                  uint8_t* d_base, uint8_t* d_out, cudaStream_t st);

}  // namespace nr
