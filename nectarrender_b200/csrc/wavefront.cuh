// wavefront.cuh — launch interface of the wavefront integrator.
#pragma once
#include "integrator.cuh"
#include "../../include/nectar_b200.h"

namespace nr {

struct WfParams {
  KernelParams kp;
  uint32_t base;   // first sample index of the wave (host side; the kernels
                   // read it from ctr, set by wf_set_base and advanced by
                   // each wave's last launch)
  uint32_t count;  // sample indices in the wave
  uint32_t capacity;
  int32_t extend_variant;  // traversal kernel (see extend_fn)
  uint32_t tail_max_paths; // tail hand-off bound (0: none)
  int32_t shade_variant;   // 5 or 6: register budget for that many CTAs per SM; else none
  float4* ray_o;
  float4* ray_d;
  float4* atten;
  float4* acc_b;
  float4* acc_d;
  float4* acc_n;
  uint4* hit;
  float* hit_t;
  uint32_t* queue0;
  uint32_t* queue1;
  uint32_t* ctr;
  // NR_MODE_PERF only (null otherwise): BSDF pdf of each path's current
  // direction, and one shadow ray per path per bounce (origin + max t,
  // direction, contribution) with its queue
  float* mis_pdf;
  float4* sh_o;
  float4* sh_d;
  float4* sh_c;
  uint32_t* sh_queue;
};

size_t wf_state_bytes(uint32_t n_paths, bool perf = false);
cudaError_t wf_alloc(WfParams& W, uint32_t n_paths, bool perf = false);
void wf_free(WfParams& W);
// static_wave.cu: address of the library-owned wave buffer on the current
// device, and its division into the wave's arrays (capacity
// NR_STATIC_WAVE_PATHS paths).
cudaError_t static_wave_address(void** out);
void static_wave_carve(void* base, WfParams& W);
// Optional timing of a wave: an event is recorded after every launch and
// tagged with the launch's kernel class (NR_KERNEL_*); the host attributes
// the time between consecutive events to the later launch.
struct WaveTimer {
  cudaEvent_t* ev = nullptr;
  uint8_t* kind = nullptr;
  int cap = 0;
  int n = 0;
  void mark(int k, cudaStream_t st) {
    if (n < cap) {
      cudaEventRecord(ev[n], st);
      kind[n++] = (uint8_t)k;
    }
  }
};

// Launches one wave: generate, depth x (extend, shade, rotate), accumulate,
// advance. The wave's first sample index must have been set on the stream by
// wf_set_base (for the first wave of a run; each wave advances it).
cudaError_t wf_launch_wave(const WfParams& W, bool counters, cudaStream_t st,
                           WaveTimer* timer = nullptr);
cudaError_t wf_set_base(const WfParams& W, uint32_t first_sample, cudaStream_t st);

}  // namespace nr
