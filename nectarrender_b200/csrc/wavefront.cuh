// wavefront.cuh — launch interface of the wavefront integrator.
#pragma once
#include "image_ops.cuh"
#include "integrator.cuh"
#include "../../include/nectar_b200.h"

namespace nr {

// Fields of the per-path record WfParams::path.
constexpr int kRecWords = 4;
constexpr int kRecO = 0, kRecD = 1, kRecAtten = 2, kRecBeauty = 3;
// the kernels move (origin, direction) and (throughput, beauty) as 32-byte
// sectors of a 64-byte aligned record
static_assert(kRecWords == 4 && kRecD == kRecO + 1 && kRecAtten == 2 && kRecBeauty == 3,
              "path record layout");
__host__ __device__ __forceinline__ size_t path_at(uint32_t p, int field) {
  return (size_t)kRecWords * p + (size_t)field;
}

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
  // one 64-byte record per path, kRecWords float4 (path_at(p, field)): ray
  // origin + time, ray direction + bounce, throughput + draw counter, beauty
  // + primary id. A path's state is two whole 32-byte sectors, so the
  // sorted (scattered) shading reads and writes no half-used sectors.
  float4* path;
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
  // radiance cache (perf mode with a cache attached; nrc_bounce = 0: off).
  // Paths other than training paths stop at hit index nrc_bounce and leave
  // a query (features, and throughput + path index); training paths (one in
  // nrc_train_one_in) run to full depth and leave a record at every hit from
  // index 1 on: features, throughput + path index, beauty before the hit.
  uint32_t nrc_bounce, nrc_train_one_in;
  uint32_t nrc_q_cap, nrc_t_cap;
  float4* nrc_q;       // [cap][4] (NrcQuery layout)
  float4* nrc_q_beta;  // xyz throughput, w path index
  float4* nrc_t;       // [cap][4]
  float4* nrc_t_beta;  // xyz throughput, w path index
  float4* nrc_t_before;
  // material-key sort of each bounce's queue before shading (null: off):
  // skey[p] is path p's key (miss, then material type) written by the
  // extend kernel, queue_s receives the queue grouped by key, sort_ctr holds
  // 8 key counts followed by 8 fill cursors
  uint32_t* queue_s;
  uint8_t* skey;
  uint32_t* sort_ctr;
  // fused display (null: off): the accumulate kernel also writes the beauty
  // layer's display transform as uint8 CHW
  uint8_t* disp8;
  DisplayParams disp_p;
  // per-bounce trace log of the wave's first sample index (null: off;
  // NR_MODE_REFERENCE shading only): kTraceLogFloats floats per pixel and
  // bounce, for bounces below log_bounces (see nr_render_trace_log)
  float* trace_log;
  uint32_t log_bounces;
};
constexpr int kTraceLogFloats = 16;

size_t wf_state_bytes(uint32_t n_paths, bool perf = false, bool sort = false);
cudaError_t wf_alloc(WfParams& W, uint32_t n_paths, bool perf = false, bool sort = false);
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
// Called after the last bounce of a wave, before its samples are folded into
// the layers (the radiance cache queries and trains there).
struct WaveHook {
  cudaError_t (*fn)(void* ctx, const WfParams& W, cudaStream_t st) = nullptr;
  void* ctx = nullptr;
};

cudaError_t wf_launch_wave(const WfParams& W, bool counters, cudaStream_t st,
                           WaveTimer* timer = nullptr, const WaveHook* hook = nullptr);
// Radiance-cache helpers for the hook: counts of queries and training
// records of the wave just traced, adding the cache's answers to the paths'
// beauty, and the training targets (beauty after the hit minus beauty
// before it, over the throughput at the hit).
cudaError_t wf_nrc_counts(const WfParams& W, uint32_t* n_q, uint32_t* n_t, cudaStream_t st);
cudaError_t wf_nrc_apply(const WfParams& W, const float* radiance, uint32_t n_q, cudaStream_t st);
// Training targets of the wave's n_t records, regrouped into `groups`
// interleaved batches: record i goes to slot (i % groups) * per + i / groups
// of target (float3) and of records (4 float4), per = ceil(n_t / groups).
cudaError_t wf_nrc_targets(const WfParams& W, float* target, float4* records, uint32_t n_t,
                           uint32_t groups, cudaStream_t st);
cudaError_t wf_set_base(const WfParams& W, uint32_t first_sample, cudaStream_t st);

}  // namespace nr
