// static_wave.cu — a library-owned device buffer for one wave of path state.
//
// Used by nr_render_samples_static, which renders without allocating: the
// wave's rays, throughputs, per-sample layers, hit records and both path
// queues are carved out of this file-scope array instead of cudaMalloc'd
// memory. The array lives in its own translation unit so that its module,
// and with it the array's device memory, is only loaded by processes that
// call that entry point (CUDA's lazy module loading).
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/nectar_b200.h"
#include "wavefront.cuh"

namespace nr {

static __device__ __align__(256) unsigned char g_static_wave[NR_STATIC_WAVE_BYTES];

namespace {
constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kPaths = NR_STATIC_WAVE_PATHS;
constexpr size_t kLayoutBytes = 7 * round_up(kPaths * 16)  // 6 float4 arrays + uint4 hits
                                + 3 * round_up(kPaths * 4)  // hit_t, queue0, queue1
                                + round_up(16 * sizeof(uint32_t));
static_assert(kPaths % 64 == 0, "path capacity is a multiple of 64");
static_assert(kLayoutBytes <= NR_STATIC_WAVE_BYTES, "wave layout exceeds the static buffer");
}  // namespace

cudaError_t static_wave_address(void** out) {
  return cudaGetSymbolAddress(out, g_static_wave);
}

void static_wave_carve(void* base, WfParams& W) {
  unsigned char* p = static_cast<unsigned char*>(base);
  auto take = [&](size_t bytes) {
    unsigned char* q = p;
    p += round_up(bytes);
    return q;
  };
  W.path = reinterpret_cast<float4*>(take(kRecWords * kPaths * sizeof(float4)));
  W.acc_d = reinterpret_cast<float4*>(take(kPaths * sizeof(float4)));
  W.acc_n = reinterpret_cast<float4*>(take(kPaths * sizeof(float4)));
  W.hit = reinterpret_cast<uint4*>(take(kPaths * sizeof(uint4)));
  W.hit_t = reinterpret_cast<float*>(take(kPaths * sizeof(float)));
  W.queue0 = reinterpret_cast<uint32_t*>(take(kPaths * sizeof(uint32_t)));
  W.queue1 = reinterpret_cast<uint32_t*>(take(kPaths * sizeof(uint32_t)));
  W.ctr = reinterpret_cast<uint32_t*>(take(16 * sizeof(uint32_t)));
  W.capacity = (uint32_t)kPaths;
}

}  // namespace nr
