// integrator.cu — persistent path-tracing megakernel.
//
// Replaces the reference's per-pixel trace_full_kernel (one launch per
// sample, 16x16 blocks, nectar_render/csrc/engine/src/trace.cu:47-94) plus its
// three accumulate launches and three memsets per sample
// (nectar_render/csrc/engine/src/engine.cpp:52-64,
// nectar_render/csrc/data/src/data.cu:28-50).
//
// Schedule: a grid of a few CTAs per SM runs until the work counter is
// exhausted. A lane owns one pixel for all sample indices of the launch; when
// its path ends it folds the sample into the pixel's running mean, kept in
// registers, and regenerates the next sample's camera ray in the same loop
// iteration (path regeneration), so lanes stay busy while their warp-mates
// still trace long paths. Pixels are fetched 32 at a time in 8x4 tiles with
// one warp-aggregated atomic. The running mean is the reference's
// avg*(n-1)/n + s/n applied in sample order, so the accumulated layers equal
// the reference's sample by sample.
#include "integrator.cuh"
#include "pathstep.cuh"

namespace nr {

// ---------------------------------------------------------------------------
// Device-side constants built with device math, as the reference builds them.

// Transform(position, rotation_deg, scale) rotation for the cube faces: the
// reference constructs Cube::face_xforms inside the device constructor
// (shapes.h:192-223 via device_build), so cosf/sinf here are the device
// versions, like the reference's.
__device__ M3 rot_x(float a) {
  float c = cosf(a), s = sinf(a);
  return M3{{{1, 0, 0}, {0, c, -s}, {0, s, c}}};
}
__device__ M3 rot_y(float a) {
  float c = cosf(a), s = sinf(a);
  return M3{{{c, 0, s}, {0, 1, 0}, {-s, 0, c}}};
}
__device__ M3 rot_z(float a) {
  float c = cosf(a), s = sinf(a);
  return M3{{{c, -s, 0}, {s, c, 0}, {0, 0, 1}}};
}
__device__ M3 mat_mul(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      r.m[i][j] = 0;
      for (int k = 0; k < 3; k++) r.m[i][j] += a.m[i][k] * b.m[k][j];
    }
  return r;
}
__device__ M3 transpose(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r.m[i][j] = a.m[j][i];
  return r;
}
// deg2rad multiplies by a double constant (core/utils.h:12-14)
__device__ float d2r(float deg) { return (float)((double)deg * 0.01745329); }
__device__ M3 euler(float rx, float ry, float rz) {
  return mat_mul(mat_mul(rot_z(d2r(rz)), rot_y(d2r(ry))), rot_x(d2r(rx)));
}

__global__ void init_device_constants(CubeFace* faces, float hdri_rotation_deg, M3* hdri_rot) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const float P[6][3] = {{0, 0, 0.5f}, {0, 0, -0.5f}, {0.5f, 0, 0},
                         {-0.5f, 0, 0}, {0, 0.5f, 0}, {0, -0.5f, 0}};
  const float E[6][3] = {{90, 0, 0}, {-90, 0, 0}, {0, 0, -90},
                         {0, 0, 90}, {0, 0, 0},   {180, 0, 0}};
  for (int i = 0; i < 6; ++i) {
    M3 R = euler(E[i][0], E[i][1], E[i][2]);
    faces[i].R = R;
    faces[i].invR = transpose(euler(E[i][0], E[i][1], E[i][2]));
    faces[i].pos = V3{P[i][0], P[i][1], P[i][2]};
  }
  // Sky::HDRI::sample builds rotation_y(deg2rad(rotation)) per call (skylight.h:76)
  *hdri_rot = rot_y(d2r(hdri_rotation_deg));
}

template <bool kCounters, int kMode>
__global__ void __launch_bounds__(kMegaThreads) megakernel(KernelParams P) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tiles_x = (P.W + 7u) / 8u;
  const uint32_t tiles_y = (P.H + 3u) / 4u;
  const uint32_t n_work = tiles_x * tiles_y * 32u;
  const uint32_t last_sample = P.first_sample + P.n_samples;
  const size_t hw = (size_t)P.W * P.H;

  TraceStats st{0u, 0u, 0u};
  uint32_t paths = 0u, rays = 0u;

  PathState s;
  Rng g;
  uint32_t x = 0, y = 0, sample = 0;
  bool alive = false;  // lane holds a pixel with samples left
  bool exhausted = false;
  V3 avg_b{0, 0, 0}, avg_d{0, 0, 0}, avg_n{0, 0, 0};
  double acc64[3] = {0, 0, 0};

  while (true) {
    // --- fetch a pixel for lanes without one (warp-aggregated atomic)
    bool need = !alive && !exhausted;
    uint32_t need_mask = __ballot_sync(0xffffffffu, need);
    if (need_mask) {
      uint32_t base = 0;
      uint32_t leader = __ffs(need_mask) - 1u;
      if (lane == leader) base = atomicAdd(P.work_counter, __popc(need_mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        uint32_t w = base + __popc(need_mask & ((1u << lane) - 1u));
        bool inside = false;
        if (w >= n_work) {
          exhausted = true;
        } else {
          pixel_of(w, P.W, tiles_x, x, y);
          // indices of edge tiles that fall outside the image are consumed
          // and skipped; the lane fetches again on the next iteration
          inside = x < P.W && y < P.H;
        }
        if (inside) {
          alive = true;
          sample = P.first_sample;
          size_t pi = (size_t)y * P.W + x;
          if (P.write_raw == 0) {
            if (P.beauty) avg_b = load3(P.beauty, hw, pi);
            if (P.diffuse) avg_d = load3(P.diffuse, hw, pi);
            if (P.normal) avg_n = load3(P.normal, hw, pi);
            if (P.beauty64) {
              acc64[0] = P.beauty64[pi];
              acc64[1] = P.beauty64[hw + pi];
              acc64[2] = P.beauty64[2 * hw + pi];
            }
          }
          start_path(P, s, g, x, y, sample);
        }
      }
    }
    if (__all_sync(0xffffffffu, !alive && exhausted)) break;
    if (!alive) continue;

    // --- one bounce
    bool cont = bounce_ref(P, s, g, st);
    rays++;
    if (cont) continue;

    // --- path finished: fold the sample, then regenerate
    paths++;
    size_t pi = (size_t)y * P.W + x;
    if (P.write_raw) {
      if (P.beauty) store3(P.beauty, hw, pi, s.beauty);
      if (P.diffuse) store3(P.diffuse, hw, pi, s.diffuse);
      if (P.normal) store3(P.normal, hw, pi, s.normal);
      if (P.primary) P.primary[pi] = s.primary;
    } else {
      avg_b = running_mean(avg_b, s.beauty, sample);
      avg_d = running_mean(avg_d, s.diffuse, sample);
      avg_n = running_mean(avg_n, s.normal, sample);
      acc64[0] += (double)s.beauty.x;
      acc64[1] += (double)s.beauty.y;
      acc64[2] += (double)s.beauty.z;
    }
    sample += 1u;
    if (sample < last_sample && !P.write_raw) {
      start_path(P, s, g, x, y, sample);
    } else {
      if (!P.write_raw) {
        if (P.beauty) store3(P.beauty, hw, pi, avg_b);
        if (P.diffuse) store3(P.diffuse, hw, pi, avg_d);
        if (P.normal) store3(P.normal, hw, pi, avg_n);
        if (P.beauty64) {
          P.beauty64[pi] = acc64[0];
          P.beauty64[hw + pi] = acc64[1];
          P.beauty64[2 * hw + pi] = acc64[2];
        }
      }
      alive = false;
    }
  }

  if (kCounters) {
    unsigned long long v[5] = {rays, st.nodes, st.tris, st.objs, paths};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      unsigned long long a = v[k];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) atomicAdd(P.counters + k, a);
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers

cudaError_t launch_init_constants(float hdri_rotation_deg, CubeFace* d_faces, M3* host_hdri_rot,
                                  cudaStream_t st) {
  M3* d_rot = nullptr;
  cudaError_t e = cudaMalloc(&d_rot, sizeof(M3));
  if (e != cudaSuccess) return e;
  init_device_constants<<<1, 32, 0, st>>>(d_faces, hdri_rotation_deg, d_rot);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_hdri_rot, d_rot, sizeof(M3), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_rot);
  return e;
}

int mega_grid_blocks() {
  static int blocks = 0;
  if (blocks == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, megakernel<false, 0>, kMegaThreads, 0);
    if (per_sm < 1) per_sm = 1;
    blocks = sms * per_sm;
  }
  return blocks;
}

cudaError_t launch_megakernel(const KernelParams& P, bool counters, cudaStream_t st) {
  int blocks = mega_grid_blocks();
  if (counters)
    megakernel<true, 0><<<blocks, kMegaThreads, 0, st>>>(P);
  else
    megakernel<false, 0><<<blocks, kMegaThreads, 0, st>>>(P);
  return cudaGetLastError();
}

}  // namespace nr
