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

// ---------------------------------------------------------------------------
// NR_MODE_PERF: next-event estimation toward lights[0] and the HDRI with
// power-heuristic multiple importance sampling (Veach 1997, ch. 9). The BSDF
// strategy keeps every material's own sampler; the integrand is the one the
// reference's BSDF-only estimator converges to (the isotropic phase function
// is used normalised, 1/(4*pi): its f/p ratio is the reference's).

__device__ __forceinline__ V3 mul_transpose(const M3& a, const V3& v) {
  return V3{a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z,
            a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z,
            a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z};
}

__device__ __forceinline__ bool sky_nee_ready(const DevSky& s) {
  return s.type == 2 && s.data != nullptr && s.texel_pdf != nullptr;
}

// Solid-angle density with which sky_sample_dir produces direction d: texel
// chosen with probability texel_pdf, uniform in (u, v) inside the texel.
__device__ __forceinline__ float sky_dir_pdf(const DevSky& s, const V3& d) {
  const V3 dr = mul(s.rot, normalize(d));
  const float sin_t = sqrtf(fmaxf(0.0f, dr.x * dr.x + dr.z * dr.z));
  if (sin_t <= 1e-7f) return 0.0f;
  const float u = atan2f(dr.z, dr.x) / PI2 + 0.5f;
  const float v = acosf(fminf(fmaxf(dr.y, -1.0f), 1.0f)) / PI;
  const int x = min(s.W - 1, max(0, (int)(u * (float)s.W)));
  const int y = min(s.H - 1, max(0, (int)(v * (float)s.H)));
  const float n = (float)s.W * (float)s.H;
  return __ldg(s.texel_pdf + (size_t)y * s.W + x) * n / (2.0f * PI * PI * sin_t);
}

// Alias-table sample of a texel (Walker 1977): a row from the row table,
// then a column from that row's table; then a uniform point inside the
// texel, as a world direction.
__device__ __forceinline__ V3 sky_sample_dir(const DevSky& s, Rng& g, float& pdf) {
  const uint32_t n = (uint32_t)s.W * (uint32_t)s.H;
  const float fr = g.random_float() * (float)s.H;
  const uint32_t rb = min((uint32_t)s.H - 1u, (uint32_t)fr);
  const uint32_t y = fr - (float)rb < __ldg(s.row_prob + rb) ? rb : __ldg(s.row_alias + rb);
  const float fc = g.random_float() * (float)s.W;
  const uint32_t cb = min((uint32_t)s.W - 1u, (uint32_t)fc);
  const size_t o = (size_t)y * (uint32_t)s.W;
  const uint32_t x = fc - (float)cb < __ldg(s.col_prob + o + cb) ? cb : __ldg(s.col_alias + o + cb);
  const uint32_t t = y * (uint32_t)s.W + x;
  const float u = ((float)x + g.random_float()) / (float)s.W;
  const float v = ((float)y + g.random_float()) / (float)s.H;
  const float theta = v * PI, phi = (u - 0.5f) * PI2;
  const float st = sinf(theta);
  const V3 dr = V3{st * cosf(phi), cosf(theta), st * sinf(phi)};
  pdf = st > 1e-7f ? __ldg(s.texel_pdf + t) * (float)n / (2.0f * PI * PI * st) : 0.0f;
  return mul_transpose(s.rot, dr);
}

__device__ __forceinline__ bool light_nee_ready(const DevScene& sc) {
  if (sc.light < 0) return false;
  const DevObject& ob = sc.objects[sc.light];
  const int type = ob.type == 6 ? ob.wrapped_type : ob.type;
  return type == 1 || type == 2;  // quads and spheres have a sampler and a pdf
}

// Samples lights[0] from p: unit direction, distance to the sampled point,
// solid-angle pdf and the radiance the light emits toward p.
template <typename MeshFn>
__device__ __forceinline__ bool light_sample_nee(const DevScene& sc, const V3& p, Rng& g, bool rtl,
                                                 V3& dir, float& dist, float& pdf, V3& Le,
                                                 TraceStats& st, uint32_t* err, MeshFn&& mesh_fn) {
  const V3 d = light_random(sc, p, g, rtl);
  const float len2 = length_squared(d);
  if (!(len2 > 0.0f)) return false;
  pdf = light_pdf_value(sc, p, d, st, err);
  if (!(pdf > 0.0f)) return false;
  const DevObject& ob = sc.objects[sc.light];
  const Ray wr = make_ray(p, d, 0.0f);
  const Ray r = to_object(ob, wr);
  Hit h;
  if (!object_hit_local_t(sc.cube_faces, ob, r, EPS, FMAX, h, mesh_fn)) return false;
  to_world(h, ob.R, ob.pos, ob.scale, ob.inv_s, r, wr, false);
  Le = mat_emitted(sc.materials[ob.material], h);
  if (Le.x <= 0.0f && Le.y <= 0.0f && Le.z <= 0.0f) return false;
  const float len = sqrtf(len2);
  dir = d / len;
  dist = h.t * len;
  return dist > 0.0f;
}

__device__ __forceinline__ float perf_bsdf_pdf(const Pdf& pdf, const V3& dir) {
  return pdf.kind == PDF_SPHERE ? 1.0f / (4.0f * PI) : pdf_value(pdf, dir);
}
__device__ __forceinline__ V3 perf_bsdf_eval(const DevMaterial& m, const Hit& rec, const V3& view,
                                             const V3& dir) {
  if (m.type == 5) return tex_sample(m.tex[0], rec.uv) * (1.0f / (4.0f * PI));
  return mat_evaluate(m, rec, view, dir);
}
__device__ __forceinline__ float power_heuristic(float a, float b) {
  const float a2 = a * a, b2 = b * b;
  return a2 + b2 > 0.0f ? a2 / (a2 + b2) : 0.0f;
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
