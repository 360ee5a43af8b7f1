// ref_cpu_harness.cpp — the reference's own integrator compiled for the host
// (TEST INFRASTRUCTURE, built by oracle/Makefile into oracle/_ref/).
//
// The reference's __device__ code (hittables, materials, PDFs, sky, camera,
// BVH, Philox through the cuRAND device header) compiles as ordinary host
// code under g++. This file supplies only what cannot come from those
// headers on a CPU:
//  * scene assembly with host pointers where the reference uses
//    device_build<T> placement-new kernels (registry.h:216-263,
//    scene.cpp:68-76, the device constructors of Hittable, Material, Mesh,
//    Cube);
//  * the per-pixel loop of trace_full_kernel and the body of trace_ray
//    (engine/src/trace.cu:11-41, 53-78), which live in a .cu kernel file,
//    with the AOV writes kept in registers;
//  * a traversal of the reference's mesh BVH that reports which triangle the
//    closest hit came from (Mesh::hit does not record it), for primary-hit
//    primitive ids;
//  * the per-pixel bodies of trace_viewport_kernel and hit_test_ray_kernel
//    (engine/src/trace.cu:100-188) and of mask_selected_kernel and
//    build_outline_kernel (scene/src/scene_interface.cu:3-52), around the
//    reference's own camera rays, scene traversal, viewport colours, sky and
//    axis grid.
// Access to private members is opened with a macro after all standard and
// pybind11 headers are included.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <optional>
#include <random>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <pybind11/functional.h>
#include <pybind11/pybind11.h>

#define private public
#include "core/include/core.h"
#include "engine/include/engine/pdf.h"
#include "scene/include/graph.h"
#include "engine/include/engine/camera.h"
#include "engine/src/brdf.cu"
#include "engine/src/axis_grid.cu"
#undef private

#include "oracle.h"

namespace {

struct RefScene {
  std::vector<std::unique_ptr<Material>> mats;
  std::vector<Material*> mat_ptrs;
  std::vector<std::unique_ptr<Hittable>> owned;
  std::vector<Hittable*> objects;  // leaf order
  std::vector<Hittable*> lights;
  std::vector<int> object_id;      // leaf slot -> registry id
  std::vector<int> object_mesh;    // leaf slot -> mesh index or -1
  BVH<int> tlas;
  Skylight sky;
  SceneGraph graph{};
  struct MeshData {
    MeshLoadResult data;
    BVH<TriangleRef> bvh;
    std::vector<uint32_t> tri_id;  // leaf slot -> original triangle index
    std::unique_ptr<Mesh> mesh;
  };
  std::vector<std::unique_ptr<MeshData>> meshes;
};

// A texture view as Texture::view() builds it (texture.h:187-191); an IMAGE
// texture points at the caller's host copy of the CHW bytes, which the
// reference's sample_image then reads as it reads device memory.
TextureView texture_view(const nr_texture_desc& t, const or_scene* in) {
  TextureView v{};
  v.type = TextureType::CONSTANT;
  v.d_tex_ptr = nullptr;
  v.constant_color = Color(t.rgb[0], t.rgb[1], t.rgb[2]);
  v.C = 3;
  v.H = 0;
  v.W = 0;
  v.scale = t.scale;
  if (t.type == NR_TEXTURE_IMAGE && t.image >= 0 && (uint32_t)t.image < in->n_images) {
    const or_image& im = in->images[t.image];
    v.type = TextureType::IMAGE;
    v.d_tex_ptr = const_cast<uint8_t*>(im.chw);
    v.C = im.C;
    v.H = im.H;
    v.W = im.W;
  }
  return v;
}

Material* make_material(const nr_material_desc& d, RefScene& S, const or_scene* in) {
  auto view_of = [in](const nr_texture_desc& t) { return texture_view(t, in); };
  void* core = nullptr;
  MaterialType type = (MaterialType)d.type;
  switch (d.type) {
    case NR_MATERIAL_LAMBERTIAN: core = new Lambertian(view_of(d.tex[0])); break;
    case NR_MATERIAL_PBR:
      core = new PBR(view_of(d.tex[0]), view_of(d.tex[1]), view_of(d.tex[2]), view_of(d.tex[3]),
                     view_of(d.tex[4]));
      break;
    case NR_MATERIAL_DIELECTRIC: core = new Dielectric(Color(d.tint[0], d.tint[1], d.tint[2]), d.ior); break;
    case NR_MATERIAL_EMISSIVE: core = new Emissive(view_of(d.tex[0]), d.brightness); break;
    case NR_MATERIAL_ISOTROPIC: core = new Isotropic(view_of(d.tex[0])); break;
    default: type = MaterialType::Null; break;
  }
  S.mats.emplace_back(new Material(type, core));
  return S.mats.back().get();
}

std::unique_ptr<RefScene::MeshData> load_mesh(const or_mesh& om) {
  auto md = std::make_unique<RefScene::MeshData>();
  md->data = parse_obj_file(om.obj_path);  // mesh.h:39-141 (tinyobjloader)
  auto& V = md->data.vertices;
  std::map<std::tuple<uint32_t, uint32_t, uint32_t>, uint32_t> index;
  for (size_t t = 0; t < md->data.triangles.size(); ++t) {
    const TriangleRef& r = md->data.triangles[t];
    index[std::make_tuple(r.v0, r.v1, r.v2)] = (uint32_t)t;
  }
  md->bvh.build(md->data.triangles, [&](const TriangleRef& t) {  // Mesh::build (mesh.h:177-216)
    return Mesh::triangle_bbox(V[t.v0].position, V[t.v1].position, V[t.v2].position);
  });
  md->tri_id.resize(md->bvh.items.size());
  for (size_t k = 0; k < md->bvh.items.size(); ++k) {
    const TriangleRef& r = md->bvh.items[k];
    md->tri_id[k] = index[std::make_tuple(r.v0, r.v1, r.v2)];
  }
  md->mesh.reset(new Mesh(V.data(), md->bvh.nodes.data(), md->bvh.items.data()));
  return md;
}

void* make_core(int type, const nr_object_desc& d, RefScene& S, int& mesh_index) {
  switch (type) {
    case NR_HITTABLE_QUAD: return new Quad();
    case NR_HITTABLE_SPHERE: return new Sphere(d.radius);
    case NR_HITTABLE_CUBE: {
      Quad** faces = new Quad*[6];
      for (int i = 0; i < 6; ++i) faces[i] = new Quad();
      return new Cube(faces);
    }
    case NR_HITTABLE_MESH: mesh_index = d.mesh; return S.meshes[d.mesh]->mesh.get();
  }
  return nullptr;
}

AABB local_box(int type, const nr_object_desc& d, RefScene& S) {
  switch (type) {
    case NR_HITTABLE_QUAD: return Quad().build_bbox();
    case NR_HITTABLE_SPHERE: return Sphere(d.radius).build_bbox();
    case NR_HITTABLE_CUBE: return AABB(Vector3(-0.5f), Vector3(0.5f));
    case NR_HITTABLE_MESH: {
      Mesh m;
      std::vector<MeshVertex> v = S.meshes[d.mesh]->data.vertices;
      m.set_geometry(v, {});
      return m.build_bbox();
    }
  }
  return AABB();
}

std::unique_ptr<RefScene> build(const or_scene* in) {
  auto S = std::make_unique<RefScene>();
  for (uint32_t i = 0; i < in->n_meshes; ++i) S->meshes.push_back(load_mesh(in->meshes[i]));
  for (uint32_t i = 0; i < in->n_materials; ++i) S->mat_ptrs.push_back(make_material(in->materials[i], *S, in));
  std::vector<Hittable*> reg(in->n_objects);
  std::vector<int> reg_mesh(in->n_objects, -1);
  std::vector<AABB> boxes(in->n_objects);
  for (uint32_t i = 0; i < in->n_objects; ++i) {
    const nr_object_desc& d = in->objects[i];
    bool wrapper = d.type == NR_HITTABLE_OBJECT_LIGHT || d.type == NR_HITTABLE_CONSTANT_MEDIUM;
    int bt = wrapper ? d.wrapped_type : d.type;
    Vector3 p(d.position[0], d.position[1], d.position[2]);
    Transform xf = bt == NR_HITTABLE_SPHERE
                       ? Transform(p)
                       : Transform(p, Vector3(d.rotation[0], d.rotation[1], d.rotation[2]),
                                   Vector3(d.scale[0], d.scale[1], d.scale[2]));
    int mi = -1;
    void* core = make_core(bt, d, *S, mi);
    Hittable* h;
    if (wrapper) {
      S->owned.emplace_back(new Hittable((HittableType)bt, xf, Transform(), 0, 0, nullptr, core));
      Hittable* wrapped = S->owned.back().get();
      void* wcore = d.type == NR_HITTABLE_OBJECT_LIGHT ? (void*)new ObjectLight()
                                                       : (void*)new ConstantMedium(d.density);
      S->owned.emplace_back(new Hittable((HittableType)d.type, xf, Transform(), i, d.material, wrapped, wcore));
    } else {
      S->owned.emplace_back(new Hittable((HittableType)bt, xf, Transform(), i, d.material, nullptr, core));
    }
    h = S->owned.back().get();
    h->bbox = local_box(bt, d, *S);
    reg[i] = h;
    reg_mesh[i] = mi;
    boxes[i] = h->bounding_box();
  }
  // HittablesRegistry::build_bvh / build_device_hittables (registry.h:216-263)
  std::vector<int> items(in->n_objects);
  std::iota(items.begin(), items.end(), 0);
  S->tlas.build(items, [&](int i) { return boxes[i]; });
  for (int i : S->tlas.items) {
    S->objects.push_back(reg[i]);
    S->object_id.push_back(i);
    S->object_mesh.push_back(reg_mesh[i]);
    if (in->objects[i].type == NR_HITTABLE_OBJECT_LIGHT) S->lights.push_back(reg[i]);
  }
  // Skylight (skylight.h:211-238); the HDRI is read with the reference's loader
  if (in->sky_type == NR_SKY_SIMPLE) {
    S->sky = Skylight::simple(Color(in->sky_start[0], in->sky_start[1], in->sky_start[2]),
                              Color(in->sky_end[0], in->sky_end[1], in->sky_end[2]));
  } else if (in->sky_type == NR_SKY_HDRI) {
    S->sky = Skylight(SkylightType::HDRI);
    S->sky.cfg_hdri = HDRISkylightConfig{};
    S->sky.cfg_hdri.rotation = in->hdri_rotation;
    S->sky.cfg_hdri.intensity = in->hdri_intensity;
    S->sky.cfg_hdri.data_ptr = const_cast<float*>(in->hdri);
    S->sky.cfg_hdri.C = (int)in->hdri_C;
    S->sky.cfg_hdri.H = (int)in->hdri_H;
    S->sky.cfg_hdri.W = (int)in->hdri_W;
  }
  S->graph.bvh_nodes = S->tlas.nodes.data();
  S->graph.objects = S->objects.data();
  S->graph.lights = S->lights.empty() ? nullptr : S->lights.data();
  S->graph.materials = S->mat_ptrs.data();
  S->graph.skylight = &S->sky;
  return S;
}

// Which leaf of the reference mesh BVH gave the closest hit (Mesh::hit order).
int mesh_hit_slot(const Mesh& m, const Ray& ray, Interval ray_t) {
  uint32_t stack[64];
  uint32_t sp = 0;
  stack[sp++] = 0u;
  int best = -1;
  while (sp > 0) {
    const BVHNode& node = m.tri_nodes[stack[--sp]];
    if (!node.bbox.hit(ray, ray_t)) continue;
    if (node.object != -1) {
      const TriangleRef& tri = m.triangles_ptr[node.object];
      float t, u, v;
      if (m.intersect_triangle(ray, m.vertices_ptr[tri.v0].position, m.vertices_ptr[tri.v1].position,
                               m.vertices_ptr[tri.v2].position, ray_t, t, u, v)) {
        ray_t.max = t;
        best = node.object;
      }
    } else {
      const BVHNode& L = m.tri_nodes[node.left];
      const BVHNode& R = m.tri_nodes[node.right];
      float tl = L.bbox.hit_t(ray, ray_t), tr = R.bbox.hit_t(ray, ray_t);
      bool ln = tl < tr;
      uint32_t ni = ln ? node.left : node.right, fi = ln ? node.right : node.left;
      float ft = ln ? tr : tl;
      if (ft < ray_t.max) stack[sp++] = fi;
      stack[sp++] = ni;
    }
  }
  return best;
}

struct Out {
  Color beauty{0.0f}, diffuse{0.0f}, normal{0.0f};
  uint32_t primary = 0xffffffffu;
};

// trace_full_kernel + trace_ray (trace.cu:11-41, 53-78) for one pixel sample
Out trace_pixel(RefScene& S, DeviceCamera& cam, const nr_render_config& cfg, int x, int y,
                uint32_t sample) {
  Out o;
  SceneGraph* scene = &S.graph;
  uint32_t pixel_idx = y * cam.W + x;
  Color atten = Color::white();
  Generator gen(cfg.seed, pixel_idx + sample * (cam.W * cam.H));
  Ray ray = cam.get_ray(x, y, pixel_idx, sample, cfg.seed, gen);
  for (int bounce = 0; bounce < (int)cfg.ray_depth; bounce++) {
    HitRecord rec;
    bool hit = scene->hit(ray, Interval(EPS, FMAX), rec);
    if (bounce == 0 && hit) {
      int slot = -1;
      for (size_t k = 0; k < S.objects.size(); ++k)
        if ((size_t)S.objects[k]->get_object_id() == rec.object_id) slot = (int)k;
      uint32_t prim = 0u;
      if (slot >= 0 && S.object_mesh[slot] >= 0 && S.objects[slot]->type == HittableType::Mesh) {
        Hittable* h = S.objects[slot];
        Ray r = ray.to_object_space(h->xform);
        int leaf = mesh_hit_slot(*h->d_mesh, r, Interval(EPS, FMAX));
        if (leaf >= 0) prim = S.meshes[S.object_mesh[slot]]->tri_id[leaf] + 1u;
      }
      o.primary = ((uint32_t)rec.object_id << 22) | (prim & 0x3fffffu);
    }
    if (!hit) {
      o.beauty += atten * scene->skylight->sample(ray);
      break;
    }
    ScatterRecord srec;
    Ray r_in = ray.clone();
    o.beauty += atten * rec.mat->emitted(ray, rec);
    if (!rec.mat->scatter(rec, ray, srec, gen)) break;
    if (srec.skip_pdf) {
      atten *= srec.atten;
      ray = srec.skip_pdf_ray;
    } else if (!sample_cosine_brdf(scene, ray, r_in, atten, rec, srec, gen)) {
      break;
    }
    if (bounce == 0) {
      o.diffuse += atten;
      o.normal += Color(rec.n);
    }
    if (cfg.rr_enabled && bounce >= (int)cfg.rr_start_bounce) {
      float survival = fmaxf(atten.r(), fmaxf(atten.g(), atten.b()));
      survival = fminf(survival, cfg.rr_survival);
      if (gen.uniform() > survival) break;
      atten *= 1.0f / survival;
    }
  }
  return o;
}

}  // namespace

extern "C" {

void* refcpu_scene_create(const or_scene* in, int32_t) { return build(in).release(); }

void refcpu_scene_destroy(void* h) { delete static_cast<RefScene*>(h); }

int refcpu_scene_render(void* handle, const nr_camera_desc* c, const nr_render_config* cfg,
                        const or_request* req) {
  RefScene* S = static_cast<RefScene*>(handle);
  CameraParams params(Vector2(c->resolution[0], c->resolution[1]),
                      Vector3(c->position[0], c->position[1], c->position[2]),
                      Vector3(c->rotation[0], c->rotation[1], c->rotation[2]), c->samples_per_pixel,
                      c->focal_length, c->focus_distance, c->aperture, c->sensor_width, c->shutter_speed);
  SampleGenerator sg;
  std::vector<Vector2> pattern = sg.generate_n_rooks(c->samples_per_pixel, cfg->seed);
  size_t H = (size_t)c->resolution[0], W = (size_t)c->resolution[1], hw = H * W;
  uint32_t r1 = std::min<uint32_t>(req->row_end, (uint32_t)H);
  int nt = req->threads > 0 ? req->threads : (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&, t]() {
      DeviceCamera cam(params, pattern.data());
      for (uint32_t y = req->row_begin + t; y < r1; y += nt)
        for (uint32_t x = 0; x < W; ++x) {
          size_t i = (size_t)y * W + x;
          auto put = [&](float* b, const Color& v) {
            if (!b) return;
            b[i] = v.r();
            b[hw + i] = v.g();
            b[2 * hw + i] = v.b();
          };
          auto get = [&](float* b) { return b ? Color(b[i], b[hw + i], b[2 * hw + i]) : Color(0.0f); };
          if (req->mode == 0) {
            Out o = trace_pixel(*S, cam, *cfg, x, y, req->first);
            put(req->beauty, o.beauty);
            put(req->diffuse, o.diffuse);
            put(req->normal, o.normal);
            if (req->primary) req->primary[i] = o.primary;
          } else {
            Color ab = get(req->beauty), ad = get(req->diffuse), an = get(req->normal);
            for (uint32_t k = 0; k < req->count; ++k) {
              uint32_t smp = req->first + k;
              Out o = trace_pixel(*S, cam, *cfg, x, y, smp);
              float fn = (float)smp;
              ab = ab * ((fn - 1.0f) / fn) + o.beauty * (1.0f / fn);
              ad = ad * ((fn - 1.0f) / fn) + o.diffuse * (1.0f / fn);
              an = an * ((fn - 1.0f) / fn) + o.normal * (1.0f / fn);
              if (req->beauty64) {
                req->beauty64[i] += (double)o.beauty.r();
                req->beauty64[hw + i] += (double)o.beauty.g();
                req->beauty64[2 * hw + i] += (double)o.beauty.b();
              }
            }
            put(req->beauty, ab);
            put(req->diffuse, ad);
            put(req->normal, an);
          }
        }
    });
  for (auto& th : pool) th.join();
  return 0;
}

static CameraParams ref_params(const nr_camera_desc* c) {
  return CameraParams(Vector2(c->resolution[0], c->resolution[1]),
                      Vector3(c->position[0], c->position[1], c->position[2]),
                      Vector3(c->rotation[0], c->rotation[1], c->rotation[2]), c->samples_per_pixel,
                      c->focal_length, c->focus_distance, c->aperture, c->sensor_width,
                      c->shutter_speed);
}

int refcpu_scene_viewport(void* handle, const nr_camera_desc* c, uint32_t seed,
                          int32_t show_axis_grid, float* beauty, float* diffuse, float* normal) {
  RefScene* S = static_cast<RefScene*>(handle);
  CameraParams params = ref_params(c);
  SampleGenerator sg;
  std::vector<Vector2> pattern = sg.generate_n_rooks(c->samples_per_pixel, seed);
  DeviceCamera cam(params, pattern.data());
  SceneGraph* scene = &S->graph;
  size_t H = cam.H, W = cam.W, hw = H * W;
  for (size_t y = 0; y < H; ++y)
    for (size_t x = 0; x < W; ++x) {
      size_t i = y * W + x;
      Color b(0.0f), d(0.0f), n(0.0f);
      HitRecord rec;
      Ray ray = cam.get_ray_center((uint32_t)x, (uint32_t)y);
      bool hit = scene->hit(ray, Interval(EPS, FMAX), rec);
      if (!hit) {
        Color grid_color;
        float grid_alpha;
        if (show_axis_grid && triplanar_grid(ray, FMAX, grid_color, grid_alpha))
          b = CG::lerp(scene->skylight->sample(ray), grid_color, grid_alpha);
        else
          b = scene->skylight->sample(ray);
      } else {
        Vector3 light_vector = cam.p.position - rec.p;
        float light_dist = light_vector.length();
        Vector3 headlight_dir = normalize(light_vector);
        float headlight = dot(headlight_dir, rec.n) * 0.5f + 0.5f;
        headlight *= 1.0f / (light_dist * light_dist);
        headlight = fminf(0.75f, headlight);
        Vector3 directional_light_dir = Vector3(1.0f, 1.0f, 1.0f);
        float directional = (dot(directional_light_dir, rec.n) + 1.0f) * 0.5f;
        directional = fmaxf(0.1f, directional);
        Color col = rec.mat->viewport_color(rec);
        b = col * fmaxf(headlight, directional);
        d = col;
        n = Color(rec.n);
      }
      auto put = [&](float* buf, const Color& v) {
        if (!buf) return;
        buf[i] = v.r();
        buf[hw + i] = v.g();
        buf[2 * hw + i] = v.b();
      };
      put(beauty, b);
      put(diffuse, d);
      put(normal, n);
    }
  return 0;
}

int refcpu_scene_pick(void* handle, const nr_camera_desc* c, uint32_t seed, float u, float v,
                      nr_pick_result* out) {
  RefScene* S = static_cast<RefScene*>(handle);
  CameraParams params = ref_params(c);
  SampleGenerator sg;
  std::vector<Vector2> pattern = sg.generate_n_rooks(c->samples_per_pixel, seed);
  DeviceCamera cam(params, pattern.data());
  HitRecord rec;
  Ray ray = cam.screen_space_ray(u, v);
  bool hit = S->graph.hit(ray, Interval(EPS, FMAX), rec);
  memset(out, 0, sizeof(*out));
  out->hit = hit ? 1 : 0;
  if (hit) {
    out->object_id = (uint32_t)rec.object_id;
    out->material_id = (uint32_t)rec.material_id;
    out->t = rec.t;
    for (int k = 0; k < 3; ++k) {
      out->p[k] = rec.p[k];
      out->n[k] = rec.n[k];
    }
    out->uv[0] = rec.uv.x();
    out->uv[1] = rec.uv.y();
    out->front_face = rec.front_face ? 1 : 0;
  }
  return 0;
}

int refcpu_scene_selection_mask(void* handle, const nr_camera_desc* c, uint32_t seed,
                                uint32_t object_id, int32_t radius, uint8_t* out) {
  RefScene* S = static_cast<RefScene*>(handle);
  CameraParams params = ref_params(c);
  SampleGenerator sg;
  std::vector<Vector2> pattern = sg.generate_n_rooks(c->samples_per_pixel, seed);
  DeviceCamera cam(params, pattern.data());
  const int H = (int)cam.H, W = (int)cam.W;
  std::vector<uint8_t> base((size_t)H * W);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      float su = (x + 0.5f) / (float)W;
      float sv = (y + 0.5f) / (float)H;
      Ray ray = cam.screen_space_ray(su, sv);
      HitRecord rec;
      bool hit = S->graph.hit(ray, Interval(EPS, FMAX), rec);
      base[(size_t)y * W + x] = (hit && rec.object_id == object_id) ? 255u : 0u;
    }
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      size_t idx = (size_t)y * W + x;
      out[idx] = 0u;
      if (base[idx] != 0) continue;
      for (int dy = -radius; dy <= radius && !out[idx]; dy++)
        for (int dx = -radius; dx <= radius; dx++) {
          int nx = x + dx, ny = y + dy;
          if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
          if (base[(size_t)ny * W + nx] != 0) {
            out[idx] = 255u;
            break;
          }
        }
    }
  return 0;
}

int refcpu_render(const or_scene* in, const nr_camera_desc* c, const nr_render_config* cfg,
                  const or_request* req) {
  void* h = refcpu_scene_create(in, 1);
  int rc = refcpu_scene_render(h, c, cfg, req);
  refcpu_scene_destroy(h);
  return rc;
}

double refcpu_mesh_sah(const or_mesh* om, uint64_t* n_nodes) {
  MeshLoadResult d = parse_obj_file(om->obj_path);
  BVH<TriangleRef> b;
  b.build(d.triangles, [&](const TriangleRef& t) {
    return Mesh::triangle_bbox(d.vertices[t.v0].position, d.vertices[t.v1].position,
                               d.vertices[t.v2].position);
  });
  if (n_nodes) *n_nodes = b.nodes.size();
  double root = b.nodes[0].bbox.surface_area(), acc = 0.0;
  for (const BVHNode& n : b.nodes) acc += (double)n.bbox.surface_area() / root;
  return acc;
}

int refcpu_n_rooks(uint32_t n, uint32_t seed, float* out) {
  SampleGenerator sg;
  std::vector<Vector2> p = sg.generate_n_rooks(n, seed);
  for (uint32_t i = 0; i < n; ++i) {
    out[2 * i] = p[i].x();
    out[2 * i + 1] = p[i].y();
  }
  return 0;
}

int refcpu_uniforms(uint32_t seed, uint32_t sub, uint32_t count, float* out) {
  Generator g(seed, sub);
  for (uint32_t i = 0; i < count; ++i) out[i] = g.uniform();
  return 0;
}

int refcpu_load_obj(const char* path, float* P, float* N, float* T, float* UV, uint32_t* tris,
                    uint32_t* nv, uint32_t* ntri, uint32_t cap_v, uint32_t cap_t) {
  MeshLoadResult d = parse_obj_file(path);
  *nv = (uint32_t)d.vertices.size();
  *ntri = (uint32_t)d.triangles.size();
  if (*nv > cap_v || *ntri > cap_t) return 1;
  for (size_t i = 0; i < d.vertices.size(); ++i) {
    const MeshVertex& v = d.vertices[i];
    for (int k = 0; k < 3; ++k) {
      P[3 * i + k] = v.position[k];
      N[3 * i + k] = v.normal[k];
      T[3 * i + k] = v.tangent[k];
    }
    UV[2 * i] = v.uv[0];
    UV[2 * i + 1] = v.uv[1];
  }
  for (size_t t = 0; t < d.triangles.size(); ++t) {
    tris[3 * t] = d.triangles[t].v0;
    tris[3 * t + 1] = d.triangles[t].v1;
    tris[3 * t + 2] = d.triangles[t].v2;
  }
  return 0;
}

int refcpu_load_hdr(const char* path, float* chw, uint32_t* C, uint32_t* H, uint32_t* W,
                    uint64_t cap) {
  int c, h, w;
  std::vector<float> d = load_image_float(path, c, h, w);  // texture.h:28-47 (stbi_loadf)
  *C = c;
  *H = h;
  *W = w;
  if (d.size() > cap) return 1;
  std::copy(d.begin(), d.end(), chw);
  return 0;
}

// The reference's image-texture loader (texture.h:8-26, stbi_load with the
// file's own channel count): its C planes as it builds them.
int refcpu_load_image_uint8(const char* path, uint8_t* chw, uint32_t* C, uint32_t* H, uint32_t* W,
                            uint64_t cap) {
  int c, h, w;
  std::vector<uint8_t> d;
  try {
    d = load_image_uint8(path, c, h, w);
  } catch (const std::exception&) {
    return -1;
  }
  *C = c;
  *H = h;
  *W = w;
  if (d.size() > cap) return 1;
  std::copy(d.begin(), d.end(), chw);
  return 0;
}

}  // extern "C"
