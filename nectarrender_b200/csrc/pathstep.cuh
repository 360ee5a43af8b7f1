// pathstep.cuh — one bounce of the reference integrator and the running
// mean, shared by the megakernel and the wavefront kernels.
#pragma once
#include "integrator.cuh"

namespace nr {

// ---------------------------------------------------------------------------
// path state

struct PathState {
  Ray ray;
  V3 atten;
  V3 beauty, diffuse, normal;
  uint32_t bounce;
  uint32_t primary;
};

__device__ __forceinline__ void pixel_of(uint32_t w, uint32_t W, uint32_t tiles_x, uint32_t& x,
                                         uint32_t& y) {
  uint32_t tile = w >> 5, j = w & 31u;
  x = (tile % tiles_x) * 8u + (j & 7u);
  y = (tile / tiles_x) * 4u + (j >> 3);
}

__device__ __forceinline__ void start_path(const KernelParams& P, PathState& s, Rng& g,
                                           uint32_t x, uint32_t y, uint32_t sample) {
  uint32_t pixel_idx = y * P.W + x;
  g.init(P.seed, pixel_idx + sample * (P.W * P.H));
  s.atten = V3{1.f, 1.f, 1.f};
  s.beauty = V3{0.f, 0.f, 0.f};
  s.diffuse = V3{0.f, 0.f, 0.f};
  s.normal = V3{0.f, 0.f, 0.f};
  s.bounce = 0u;
  s.primary = 0xffffffffu;
  s.ray = camera_ray(P.cam, x, y, pixel_idx, sample, P.seed, g, P.rtl != 0);
}

// sample_cosine_brdf (nectar_render/csrc/engine/src/brdf.cu:4-35)
__device__ __forceinline__ bool sample_brdf(const KernelParams& P, const DevMaterial& m,
                                            const Hit& rec, const Scatter& sr, const Ray& r_in,
                                            PathState& s, Rng& g, TraceStats& st) {
  V3 dir;
  float pdf_val;
  const DevScene& sc = P.scene;
  bool rtl = P.rtl != 0;
  if (sc.light >= 0) {
    if (g.random_float() < 0.5f)
      dir = pdf_generate(sr.pdf, g, rtl);
    else
      dir = light_random(sc, rec.p, g, rtl);
    pdf_val = 0.5f * pdf_value(sr.pdf, dir) + 0.5f * light_pdf_value(sc, rec.p, dir, st, P.err);
  } else {
    dir = pdf_generate(sr.pdf, g, rtl);
    pdf_val = pdf_value(sr.pdf, dir);
  }
  if (pdf_val <= 0.0f) return false;
  s.ray = make_ray(rec.p, dir, r_in.tm);
  V3 brdf = mat_evaluate(m, rec, normalize(-r_in.d), dir);
  s.atten *= brdf / pdf_val;
  return true;
}

// One bounce of trace_full_kernel's loop body (trace.cu:11-41, 63-78).
// Returns false when the path ends.
__device__ __forceinline__ bool bounce_ref(const KernelParams& P, PathState& s, Rng& g,
                                           TraceStats& st) {
  const DevScene& sc = P.scene;
  Hit rec;
  bool hit = scene_hit(sc, s.ray, rec, true, st, P.err);
  if (s.bounce == 0u && hit) {
    uint32_t oid = sc.objects[rec.obj].object_id;
    s.primary = (oid << 22) | (rec.prim == 0xffffffffu ? 0u : ((rec.prim + 1u) & 0x3fffffu));
  }
  if (!hit) {
    s.beauty += s.atten * sky_sample(sc.sky, s.ray);
    return false;
  }
  const DevMaterial& m = sc.materials[sc.objects[rec.obj].material];
  Ray r_in = s.ray;
  s.beauty += s.atten * mat_emitted(m, rec);
  Scatter sr;
  if (!mat_scatter(m, rec, s.ray, sr, g)) return false;
  if (sr.skip_pdf) {
    s.atten *= sr.atten;
    s.ray = make_ray(rec.p, sr.skip_dir, s.ray.tm);
  } else if (!sample_brdf(P, m, rec, sr, r_in, s, g, st)) {
    return false;
  }
  if (s.bounce == 0u) {
    s.diffuse += s.atten;
    s.normal += rec.n;
  }
  if (P.rr_enabled && s.bounce >= P.rr_start) {
    float survival = fmaxf(s.atten.x, fmaxf(s.atten.y, s.atten.z));
    survival = fminf(survival, P.rr_survival);
    if (g.uniform() > survival) return false;
    s.atten *= v3(1.0f / survival);
  }
  s.bounce += 1u;
  return s.bounce < P.depth;
}

// Running mean of accumulate_samples_kernel (data.cu:28-50).
__device__ __forceinline__ V3 running_mean(const V3& avg, const V3& smp, uint32_t n) {
  float fn = (float)n;
  return avg * ((fn - 1.0f) / fn) + smp * (1.0f / fn);
}

__device__ __forceinline__ V3 load3(const float* p, size_t hw, size_t i) {
  return V3{p[i], p[hw + i], p[2 * hw + i]};
}
__device__ __forceinline__ void store3(float* p, size_t hw, size_t i, const V3& v) {
  p[i] = v.x;
  p[hw + i] = v.y;
  p[2 * hw + i] = v.z;
}


}  // namespace nr
