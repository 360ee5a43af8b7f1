// viewport.cu — interactive viewport kernels on the same scene and trees as
// the path tracer: the shaded preview (trace_viewport_kernel,
// nectar_render/csrc/engine/src/trace.cu:100-162, with the axis grid of
// nectar_render/csrc/engine/src/axis_grid.cu), the picking ray
// (hit_test_ray_kernel, trace.cu:168-188) and the selection outline
// (mask_selected_kernel + build_outline_kernel,
// nectar_render/csrc/scene/src/scene_interface.cu:3-81).
#include "viewport.cuh"

namespace nr {

namespace {

__device__ __forceinline__ float saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
// CG::smoothstep (core/cg_std.h:98-103)
__device__ __forceinline__ float smoothstep(float a, float b, float x) {
  float t = saturate((x - a) / (b - a));
  return t * t * (3.0f - (2.0f * t));
}
// CG::lerp (core/cg_std.h:91-93)
__device__ __forceinline__ V3 lerp3(const V3& x, const V3& y, float w) { return x + w * (y - x); }

// grid_mask (axis_grid.cu:4-9)
__device__ __forceinline__ float grid_mask(float u, float v, float spacing, float width) {
  float du = fabsf(fmodf(u + spacing * 0.5f, spacing) - spacing * 0.5f);
  float dv = fabsf(fmodf(v + spacing * 0.5f, spacing) - spacing * 0.5f);
  float d = fminf(du, dv);
  return 1.0f - smoothstep(0.0f, width, d);
}

__device__ __forceinline__ float axis_comp(const V3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// axis_grid (axis_grid.cu:11-53): the plane through the origin normal to
// `axis`, lines every power of ten chosen from the distance, faded by t.
__device__ bool axis_grid(const Ray& ray, float max_t, int axis, const V3& major, V3& color,
                          float& alpha) {
  const float line_width = 1e-3f;
  float dir_axis = axis_comp(ray.d, axis);
  if (fabsf(dir_axis) < 1e-6f) return false;
  float t = -axis_comp(ray.o, axis) / dir_axis;
  if (t <= 0.0f || t >= max_t) return false;
  V3 p = ray_at(ray, t);
  p = V3{fabsf(p.x), fabsf(p.y), fabsf(p.z)};
  int u_axis = (axis + 1) % 3, v_axis = (axis + 2) % 3;
  float u = axis_comp(p, u_axis), v = axis_comp(p, v_axis);
  float pixel_size = line_width * t;
  float level = fmaxf(log10f(fmaxf(pixel_size, 1e-5f)) + 1.0f, 0.0f);
  float level0 = floorf(level);
  float blend = level - level0;
  float spacing0 = powf(10.0f, level0);
  float spacing1 = spacing0 * 10.0f;
  float width = pixel_size * 1.5f;
  float g0 = grid_mask(u, v, spacing0, width);
  float g1 = grid_mask(u, v, spacing1, width);
  float mask = fmaxf(g0 * (1.0f - blend), g1);
  if (mask < 0.01f) return false;
  float fade = fmaxf(0.0f, 1.0f - t / 100.0f);
  color = lerp3(v3(0.35f), major, smoothstep(0.0f, 1.0f, g1));
  alpha = mask * fade;
  return true;
}

// triplanar_grid (axis_grid.cu:55-72): x, y, z planes in that order
__device__ bool triplanar_grid(const Ray& ray, float max_t, V3& color, float& alpha) {
  if (axis_grid(ray, max_t, 0, V3{1.0f, 0.3f, 0.3f}, color, alpha)) return true;
  if (axis_grid(ray, max_t, 1, V3{0.3f, 1.0f, 0.3f}, color, alpha)) return true;
  return axis_grid(ray, max_t, 2, V3{0.3f, 0.3f, 1.0f}, color, alpha);
}

// Material::viewport_color (material/material.h:43-45, 109-111, 218, 289-291, 335-337)
__device__ __forceinline__ V3 viewport_color(const DevMaterial& m, const Hit& h) {
  switch (m.type) {
    case 1:
    case 2:
    case 4:
    case 5:
      return tex_sample(m.tex[0], h.uv);
    case 3:
      return V3{m.tint[0], m.tint[1], m.tint[2]};
  }
  return V3{0.f, 0.f, 0.f};
}

// DeviceCamera::get_ray_center (camera.h:181-184): the focus point of sample
// 0 of pixel 0 with seed 0, i.e. every pixel shifted by the same offset.
__device__ __forceinline__ Ray center_ray(const DevCamera& c, uint32_t x, uint32_t y) {
  V2 base = c.pattern[0];
  V2 shift = pcg_vector2(0.0f, 0u);
  V2 off = V2{fmodf(base.x + shift.x, 1.0f) - 0.5f, fmodf(base.y + shift.y, 1.0f) - 0.5f};
  float u = ((float)x + off.x - (c.res_x - 1.0f) * 0.5f) * (c.uvw_x / c.res_x);
  float v = ((float)y + off.y - (c.res_y - 1.0f) * 0.5f) * (c.uvw_y / c.res_y);
  V3 center = mul(c.R, V3{u, v, -c.focal_length});
  float focus_scale = c.focus_distance / c.focal_length;
  V3 focus_point = c.position + center * focus_scale;
  return make_ray(c.position, normalize(focus_point - c.position), 0.0f);
}

// DeviceCamera::screen_space_ray (camera.h:215-227)
__device__ __forceinline__ Ray screen_ray(const DevCamera& c, float su, float sv) {
  float x = su * c.res_x;
  float y = sv * c.res_y;
  float u = (x - (c.res_x - 1.0f) * 0.5f) * (c.uvw_x / c.res_x);
  float v = (y - (c.res_y - 1.0f) * 0.5f) * (c.uvw_y / c.res_y);
  V3 d = normalize(mul(c.R, V3{u, v, -c.focal_length}));
  return make_ray(c.position, d, 0.0f);
}

__global__ void k_viewport(KernelParams P, int32_t show_axis_grid) {
  const uint32_t N = P.W * P.H;
  const size_t hw = N;
  TraceStats st{0u, 0u, 0u};
  for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < N; pix += gridDim.x * blockDim.x) {
    const uint32_t x = pix % P.W, y = pix / P.W;
    Ray ray = center_ray(P.cam, x, y);
    Hit rec;
    V3 beauty{0, 0, 0}, diffuse{0, 0, 0}, normal{0, 0, 0};
    if (!scene_hit(P.scene, ray, rec, true, st, P.err)) {
      V3 sky = sky_sample(P.scene.sky, ray);
      V3 gc;
      float ga;
      if (show_axis_grid && triplanar_grid(ray, FMAX, gc, ga)) beauty = lerp3(sky, gc, ga);
      else beauty = sky;
    } else {
      V3 light_vector = P.cam.position - rec.p;
      float light_dist = length(light_vector);
      V3 headlight_dir = normalize(light_vector);
      float headlight = dot(headlight_dir, rec.n) * 0.5f + 0.5f;
      headlight *= 1.0f / (light_dist * light_dist);
      headlight = fminf(0.75f, headlight);
      V3 directional_light_dir = V3{1.0f, 1.0f, 1.0f};
      float directional = (dot(directional_light_dir, rec.n) + 1.0f) * 0.5f;
      directional = fmaxf(0.1f, directional);
      const DevMaterial& m = P.scene.materials[P.scene.objects[rec.obj].material];
      V3 col = viewport_color(m, rec);
      beauty = col * fmaxf(headlight, directional);
      diffuse = col;
      normal = rec.n;
    }
    if (P.beauty) store3(P.beauty, hw, pix, beauty);
    if (P.diffuse) store3(P.diffuse, hw, pix, diffuse);
    if (P.normal) store3(P.normal, hw, pix, normal);
  }
}

__global__ void k_pick(KernelParams P, float su, float sv, PickOut* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  TraceStats st{0u, 0u, 0u};
  Ray ray = screen_ray(P.cam, su, sv);
  Hit rec;
  PickOut o{};
  o.hit = scene_hit(P.scene, ray, rec, true, st, P.err) ? 1 : 0;
  if (o.hit) {
    const DevObject& ob = P.scene.objects[rec.obj];
    o.object_id = ob.object_id;
    o.material_id = (uint32_t)ob.material;
    o.t = rec.t;
    o.p[0] = rec.p.x;
    o.p[1] = rec.p.y;
    o.p[2] = rec.p.z;
    o.n[0] = rec.n.x;
    o.n[1] = rec.n.y;
    o.n[2] = rec.n.z;
    o.uv[0] = rec.uv.x;
    o.uv[1] = rec.uv.y;
    o.front_face = rec.front_face ? 1 : 0;
  }
  *out = o;
}

// mask_selected_kernel (scene_interface.cu:3-24)
__global__ void k_mask(KernelParams P, uint32_t object_id, uint8_t* mask) {
  const uint32_t N = P.W * P.H;
  TraceStats st{0u, 0u, 0u};
  for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < N; pix += gridDim.x * blockDim.x) {
    const uint32_t x = pix % P.W, y = pix / P.W;
    float su = ((float)x + 0.5f) / (float)P.W;
    float sv = ((float)y + 0.5f) / (float)P.H;
    Ray ray = screen_ray(P.cam, su, sv);
    Hit rec;
    bool hit = scene_hit(P.scene, ray, rec, true, st, P.err);
    mask[pix] = (hit && P.scene.objects[rec.obj].object_id == object_id) ? 255u : 0u;
  }
}

// build_outline_kernel (scene_interface.cu:26-52)
__global__ void k_outline(const uint8_t* base, uint8_t* out, uint32_t W, uint32_t H, int radius) {
  const uint32_t N = W * H;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += gridDim.x * blockDim.x) {
    const int x = (int)(idx % W), y = (int)(idx / W);
    uint8_t v = 0u;
    if (base[idx] == 0) {
      for (int dy = -radius; dy <= radius && !v; ++dy)
        for (int dx = -radius; dx <= radius; ++dx) {
          int nx = x + dx, ny = y + dy;
          if (nx < 0 || ny < 0 || nx >= (int)W || ny >= (int)H) continue;
          if (base[ny * (int)W + nx] != 0) {
            v = 255u;
            break;
          }
        }
    }
    out[idx] = v;
  }
}

int grid_for(uint32_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<uint32_t>(1u, std::min<uint32_t>((n + 255) / 256, (uint32_t)sms * 8));
}

}  // namespace

cudaError_t launch_viewport(const KernelParams& P, int32_t show_axis_grid, cudaStream_t st) {
  k_viewport<<<grid_for(P.W * P.H), 256, 0, st>>>(P, show_axis_grid);
  return cudaGetLastError();
}

cudaError_t launch_pick(const KernelParams& P, float su, float sv, PickOut* d_out, cudaStream_t st) {
  k_pick<<<1, 32, 0, st>>>(P, su, sv, d_out);
  return cudaGetLastError();
}

cudaError_t launch_selection_mask(const KernelParams& P, uint32_t object_id, int radius,
                                  uint8_t* d_base, uint8_t* d_out, cudaStream_t st) {
  const uint32_t n = P.W * P.H;
  k_mask<<<grid_for(n), 256, 0, st>>>(P, object_id, d_base);
  k_outline<<<grid_for(n), 256, 0, st>>>(d_base, d_out, P.W, P.H, radius);
  return cudaGetLastError();
}

}  // namespace nr
