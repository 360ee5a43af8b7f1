// ref_cuda_harness.cu — drives the reference's CUDA path compiled for sm_100a
// (TEST INFRASTRUCTURE, built by oracle/Makefile into oracle/_ref/).
//
// The scene is assembled through the reference's own host API (Hittable,
// Material and Texture factories, Skylight::simple/hdri, Scene::build), the
// camera through Camera::__construct, and each sample runs the reference's
// trace_full launcher followed by RenderLayers::accumulate and clear, with a
// device synchronisation per sample: the loop body of RenderEngine::render
// (nectar_render/csrc/engine/src/engine.cpp:42-74) without its GUI polling.
// The only addition is clearing freshly allocated AOV buffers, which the
// reference leaves to whatever cudaMalloc returns (its fill kernel writes one
// element, core/src/cuda.cu:64-74).
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include "core/include/core.h"
#include "engine/include/engine/trace.h"
#include "engine/include/engine/camera.h"
#include "scene/include/scene.h"
#include "data/include/data.h"

#include "oracle.h"

// The reference's trace.cu compiled once more into this file, in its own
// namespace (its headers are included above, so only its own definitions
// land there): the per-bounce log below calls its trace_ray unchanged.
#include "engine/include/engine/pdf.h"
#include "engine/include/engine/ray.h"
namespace refsrc {
#include "engine/src/trace.cu"
}  // namespace refsrc

namespace {

// Texture::from_color, or an IMAGE texture set up as Texture::from_image
// does (texture.h:158-176) from CHW bytes already in memory instead of a
// file: device copy, channel count and size, scale.
std::shared_ptr<Texture> tex(const nr_texture_desc& t, const or_scene* s) {
  if (t.type == NR_TEXTURE_IMAGE && t.image >= 0 && (uint32_t)t.image < s->n_images) {
    const or_image& im = s->images[t.image];
    Texture tx(TextureType::IMAGE);
    tx.texture_scale = t.scale;
    tx.C = im.C;
    tx.H = im.H;
    tx.W = im.W;
    const size_t n = (size_t)im.C * im.H * im.W;
    uint8_t* d = nullptr;
    if (cudaMalloc(&d, n) != cudaSuccess || cudaMemcpy(d, im.chw, n, cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("image texture upload failed");
    tx.d_texture_ptr = d;
    return std::make_shared<Texture>(std::move(tx));
  }
  return Texture::from_color(Color(t.rgb[0], t.rgb[1], t.rgb[2]));
}

Material material(const nr_material_desc& d, const or_scene* s) {
  auto tex = [s](const nr_texture_desc& t) { return ::tex(t, s); };
  switch (d.type) {
    case NR_MATERIAL_LAMBERTIAN: return Material::lambertian(tex(d.tex[0]));
    case NR_MATERIAL_PBR:
      return Material::pbr(tex(d.tex[0]), tex(d.tex[1]), tex(d.tex[2]), tex(d.tex[3]), tex(d.tex[4]));
    case NR_MATERIAL_DIELECTRIC: return Material::dielectric(Color(d.tint[0], d.tint[1], d.tint[2]), d.ior);
    case NR_MATERIAL_EMISSIVE: return Material::emissive(tex(d.tex[0]), d.brightness);
    case NR_MATERIAL_ISOTROPIC: return Material::isotropic(tex(d.tex[0]));
  }
  return Material();
}

Hittable shape(int type, const nr_object_desc& d, const or_scene* s, Material m) {
  Vector3 p(d.position[0], d.position[1], d.position[2]);
  Vector3 r(d.rotation[0], d.rotation[1], d.rotation[2]);
  Vector3 sc(d.scale[0], d.scale[1], d.scale[2]);
  switch (type) {
    case NR_HITTABLE_QUAD: return Hittable::quad(p, r, sc, std::move(m));
    case NR_HITTABLE_CUBE: return Hittable::cube(p, r, sc, std::move(m));
    case NR_HITTABLE_SPHERE: return Hittable::sphere(p, d.radius, std::move(m));
    case NR_HITTABLE_MESH: return Hittable::mesh(s->meshes[d.mesh].obj_path, p, r, sc, std::move(m));
  }
  return Hittable();
}

__global__ void probe_kernel(float* out) {
  Generator g(7u, 11u);
  Vector3 v = Vector3::random(-1.0f, 1.0f, g);
  out[0] = v.x(); out[1] = v.y(); out[2] = v.z();
  Generator h(7u, 11u);
  Quad q;
  Transform xf;
  Vector3 p = q.random(Vector3(0.0f), h, xf);
  out[3] = p.x(); out[4] = p.y(); out[5] = p.z();
  Generator k(7u, 11u);
  for (int i = 0; i < 3; ++i) out[6 + i] = k.random_float(-1.0f, 1.0f);
  Generator k2(7u, 11u);
  for (int i = 0; i < 2; ++i) out[9 + i] = k2.random_float();
}

void clear(RenderLayers& L) {
  for (DataObject* o : L.get_data())
    if (o->is_enabled() && o->data_ptr()) cudaMemset(o->data_ptr(), 0, o->n_bytes());
}

void read3(DataObject& o, float* host) {
  if (host) cudaMemcpy(host, o.data_ptr(), o.n_bytes(), cudaMemcpyDeviceToHost);
}

// The reference's Scene for a checker scene description, built through its
// own host API (Hittable factories, Scene, Scene::build). `keep` owns the
// hittables the Scene points to.
std::unique_ptr<Scene> build_ref_scene(const or_scene* s, std::vector<std::unique_ptr<Hittable>>& keep) {
  std::vector<Hittable*> hittables, lights;
  for (uint32_t i = 0; i < s->n_objects; ++i) {
    const nr_object_desc& d = s->objects[i];
    const nr_material_desc& md = s->materials[d.material];
    if (d.type == NR_HITTABLE_OBJECT_LIGHT || d.type == NR_HITTABLE_CONSTANT_MEDIUM) {
      keep.emplace_back(new Hittable(shape(d.wrapped_type, d, s, Material())));
      Hittable& bound = *keep.back();
      if (d.type == NR_HITTABLE_OBJECT_LIGHT) {
        keep.emplace_back(new Hittable(Hittable::object_light(bound, md.brightness, tex(md.tex[0], s))));
        lights.push_back(keep.back().get());
      } else {
        keep.emplace_back(new Hittable(Hittable::constant_medium(bound, d.density, tex(md.tex[0], s))));
        hittables.push_back(keep.back().get());
      }
    } else {
      keep.emplace_back(new Hittable(shape(d.type, d, s, material(md, s))));
      hittables.push_back(keep.back().get());
    }
  }
  Skylight sky;
  if (s->sky_type == NR_SKY_SIMPLE)
    sky = Skylight::simple(Color(s->sky_start[0], s->sky_start[1], s->sky_start[2]),
                           Color(s->sky_end[0], s->sky_end[1], s->sky_end[2]));
  else if (s->sky_type == NR_SKY_HDRI) {
    // Skylight::hdri(path) copies an HDRISkylightConfig whose data_ptr is
    // never initialised and then frees that pointer before loading
    // (skylight.h:226-231, 205): whether that aborts depends on stale stack
    // contents. The same loader is reached without it through hdri() and
    // load_hdri_file once the pointer is cleared.
    sky = Skylight::hdri();
    sky.config_hdri().data_ptr = nullptr;
    sky.load_hdri_file(std::string(s->hdri_path));
    sky.config_hdri().rotation = s->hdri_rotation;
    sky.config_hdri().intensity = s->hdri_intensity;
  }
  auto scene = std::make_unique<Scene>(hittables, lights, std::move(sky));
  scene->build();
  return scene;
}

// Built on the heap: the reference's Camera copy re-creates it from its
// parameters only, so it is never copied once constructed.
std::unique_ptr<Camera> make_camera(const nr_camera_desc* c, uint32_t seed) {
  CameraParams params(Vector2(c->resolution[0], c->resolution[1]),
                      Vector3(c->position[0], c->position[1], c->position[2]),
                      Vector3(c->rotation[0], c->rotation[1], c->rotation[2]), c->samples_per_pixel,
                      c->focal_length, c->focus_distance, c->aperture, c->sensor_width, c->shutter_speed);
  auto cam = std::make_unique<Camera>(params);
  cam->__construct(seed);
  return cam;
}

// trace_full_kernel (trace.cu:47-79) with a record of every bounce: the ray
// before it, the hit's registry object id and world t (0xFFFFFFFF bits and 0
// on a miss), the throughput and the pixel's beauty after it, and whether the
// path goes on. 16 floats per pixel and bounce, the layout of
// nr_render_trace_log (the reference records no triangle index: 0xFFFFFFFF).
__global__ void trace_log_kernel(DeviceCamera* cam, SceneGraph* scene, AOVs* aovs, TraceConfig cfg,
                                 uint32_t max_bounces, float* log) {
  ProcessIndex p_idx = get_process_index();
  if (p_idx.x >= cam->W || p_idx.y >= cam->H) return;
  uint32_t pixel_idx = p_idx.y * cam->W + p_idx.x;
  Color atten = Color::white();
  Generator gen(cfg.seed, pixel_idx + cfg.sample_idx * (cam->W * cam->H));
  Ray ray = cam->get_ray(p_idx.x, p_idx.y, pixel_idx, cfg.sample_idx, cfg.seed, gen);
  ColorIndex ci(aovs->beauty.C, aovs->beauty.H, aovs->beauty.W);
  for (int bounce = 0; bounce < cfg.ray_depth; bounce++) {
    const Vector3 o = ray.origin(), d = ray.direction();
    HitRecord rec;
    rec.t = -1.0f;
    bool go = refsrc::trace_ray(scene, aovs, ray, rec, atten, gen);
    if (go) {
      if (bounce == 0) {
        aovs->diffuse += atten;
        aovs->world_normal += Color(rec.n);
      }
      if (cfg.do_rr_termination && bounce >= cfg.rr_start_bounce) {
        float survival = fmaxf(atten.r(), fmaxf(atten.g(), atten.b()));
        survival = fminf(survival, cfg.rr_survival_chance);
        if (gen.uniform() > survival) go = false;
        else atten *= 1.0f / survival;
      }
    }
    if ((uint32_t)bounce < max_bounces) {
      float* L = log + ((size_t)pixel_idx * max_bounces + bounce) * 16;
      const bool hit = rec.t >= 0.0f;
      const Color b = ci.get_color(aovs->beauty.ptr);
      L[0] = o.x(); L[1] = o.y(); L[2] = o.z();
      L[3] = d.x(); L[4] = d.y(); L[5] = d.z();
      L[6] = __uint_as_float(hit ? (uint32_t)rec.object_id : 0xffffffffu);
      L[7] = __uint_as_float(0xffffffffu);
      L[8] = hit ? rec.t : 0.0f;
      L[9] = atten.r(); L[10] = atten.g(); L[11] = atten.b();
      L[12] = b.r(); L[13] = b.g(); L[14] = b.b();
      L[15] = __uint_as_float(go && bounce + 1 < cfg.ray_depth ? 1u : 0u);
    }
    if (!go) break;
  }
}

}  // namespace

extern "C" {

// Draw order of Vector3::random and Quad::random in device code:
// 1 = right to left, 0 = left to right, -1 = neither.
int refcuda_probe_draw_order(int* vec3_order, int* quad_order) {
  float* d = nullptr;
  if (cudaMalloc(&d, 16 * sizeof(float)) != cudaSuccess) return -1;
  probe_kernel<<<1, 1>>>(d);
  float h[16];
  if (cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
  cudaFree(d);
  *vec3_order = (h[0] == h[6] && h[2] == h[8]) ? 0 : ((h[0] == h[8] && h[2] == h[6]) ? 1 : -1);
  float ra = h[3] + 0.5f;  // corner.x = -0.5, u = (1,0,0)
  *quad_order = (ra == h[9]) ? 0 : ((ra == h[10]) ? 1 : -1);
  return 0;
}

// The previous scene's teardown frees each image texture twice (the
// material registry's teardown frees it, material.h:572 via texture.h:181-183,
// then ~Texture frees the same pointer again, texture.h:109): the second
// cudaFree fails with cudaErrorInvalidValue after the entry point returned.
// That error is not sticky; clear it so that it is not reported as this
// call's.
void clear_stale_error() { (void)cudaGetLastError(); }

int refcuda_render(const or_scene* s, const nr_camera_desc* c, const nr_render_config* cfg,
                   const or_request* req, double* elapsed_ms) {
  clear_stale_error();
  cudaDeviceSetLimit(cudaLimitStackSize, CUDA_STACK_SIZE_LIMIT);
  std::vector<std::unique_ptr<Hittable>> keep;
  auto scene = build_ref_scene(s, keep);
  auto camp = make_camera(c, cfg->seed);
  Camera& cam = *camp;
  RenderLayers aovs(cam.resolution());
  RenderLayers sample_aovs(&aovs);
  clear(aovs);
  clear(sample_aovs);
  cudaDeviceSynchronize();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  uint32_t last = req->first + (req->mode == 0 ? 1 : req->count);
  for (uint32_t smp = req->first; smp < last; ++smp) {
    TraceConfig tc{smp, cfg->ray_depth, cfg->seed, cfg->rr_enabled != 0, cfg->rr_start_bounce,
                   cfg->rr_survival};
    trace_full(cam, scene->graph, sample_aovs.aovs(), tc);
    if (req->mode == 0) break;
    aovs.accumulate(sample_aovs, smp);
    sample_aovs.clear();
    cudaDeviceSynchronize();
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if (elapsed_ms) *elapsed_ms = ms;
  cudaError_t err = cudaGetLastError();
  RenderLayers& src = req->mode == 0 ? sample_aovs : aovs;
  read3(src.beauty, req->beauty);
  read3(src.diffuse, req->diffuse);
  read3(src.world_normal, req->normal);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  aovs.free_aovs();
  sample_aovs.free_aovs();
  return err == cudaSuccess ? 0 : (int)err;
}

// The reference's render loop (engine.cpp:42-74: trace_full, accumulate,
// clear, synchronise per sample) timed in steps of `spp_per_step` sample
// indices, after `warmup` untimed steps. A 256 MiB buffer is written between
// steps so that no step starts with the previous one's data in L2. step_ms
// receives each timed step's device time (CUDA events).
int refcuda_time_steps(const or_scene* s, const nr_camera_desc* c, const nr_render_config* cfg,
                       uint32_t first, uint32_t warmup, uint32_t steps, uint32_t spp_per_step,
                       double* step_ms) {
  clear_stale_error();
  cudaDeviceSetLimit(cudaLimitStackSize, CUDA_STACK_SIZE_LIMIT);
  std::vector<std::unique_ptr<Hittable>> keep;
  auto scene = build_ref_scene(s, keep);
  auto camp = make_camera(c, cfg->seed);
  Camera& cam = *camp;
  RenderLayers aovs(cam.resolution());
  RenderLayers sample_aovs(&aovs);
  clear(aovs);
  clear(sample_aovs);
  void* flush = nullptr;
  const size_t flush_bytes = size_t(256) << 20;
  if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) return -1;
  cudaDeviceSynchronize();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  uint32_t smp = first;
  for (uint32_t k = 0; k < warmup + steps; ++k) {
    cudaMemset(flush, k & 0xff, flush_bytes);
    cudaDeviceSynchronize();
    cudaEventRecord(e0);
    for (uint32_t i = 0; i < spp_per_step; ++i, ++smp) {
      TraceConfig tc{smp, cfg->ray_depth, cfg->seed, cfg->rr_enabled != 0, cfg->rr_start_bounce,
                     cfg->rr_survival};
      trace_full(cam, scene->graph, sample_aovs.aovs(), tc);
      aovs.accumulate(sample_aovs, smp);
      sample_aovs.clear();
      cudaDeviceSynchronize();
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (k >= warmup) step_ms[k - warmup] = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(flush);
  aovs.free_aovs();
  sample_aovs.free_aovs();
  return err == cudaSuccess ? 0 : (int)err;
}

// One sample index through trace_log_kernel: the per-bounce log (see the
// kernel) and the raw beauty of the sample (3*H*W floats, may be null), which
// equals what trace_full writes for that sample.
int refcuda_trace_log(const or_scene* s, const nr_camera_desc* c, const nr_render_config* cfg,
                      uint32_t sample, uint32_t max_bounces, float* host_log, float* beauty) {
  clear_stale_error();
  cudaDeviceSetLimit(cudaLimitStackSize, CUDA_STACK_SIZE_LIMIT);
  std::vector<std::unique_ptr<Hittable>> keep;
  auto scene = build_ref_scene(s, keep);
  auto camp = make_camera(c, cfg->seed);
  Camera& cam = *camp;
  RenderLayers aovs(cam.resolution());
  RenderLayers sample_aovs(&aovs);
  clear(sample_aovs);
  const size_t n = (size_t)cam.width() * cam.height() * max_bounces * 16;
  float* d_log = nullptr;
  if (cudaMalloc(&d_log, n * sizeof(float)) != cudaSuccess) return -1;
  cudaMemset(d_log, 0xff, n * sizeof(float));
  TraceConfig tc{sample, cfg->ray_depth, cfg->seed, cfg->rr_enabled != 0, cfg->rr_start_bounce,
                 cfg->rr_survival};
  dim3 block(BS2D, BS2D, 1);
  dim3 grid((cam.width() + BS2D - 1) / BS2D, (cam.height() + BS2D - 1) / BS2D, 1);
  trace_log_kernel<<<grid, block>>>(cam.device_camera(), scene->graph, sample_aovs.aovs(), tc,
                                    max_bounces, d_log);
  cudaDeviceSynchronize();
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) cudaMemcpy(host_log, d_log, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) read3(sample_aovs.beauty, beauty);
  cudaFree(d_log);
  aovs.free_aovs();
  sample_aovs.free_aovs();
  return err == cudaSuccess ? 0 : (int)err;
}

}  // extern "C"
