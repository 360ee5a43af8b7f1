// pathtracer_module.cpp — pybind11 module `_pathtracer`.
//
// Re-creates the Python surface of the reference's module of the same name
// (nectar_render/csrc/bindings/bindings.cpp:16-30 and bind_*.h) on top of the
// C ABI in include/nectar_b200.h, so that scripts and the reference's Python
// facade (nectar_render/python/*.py) can drive this back end unchanged:
//   core.vector.{Vector2, Vector3, Color}, core.matrix, core.Transform,
//   material.{Material, MaterialType}, material.texture.{Texture, TextureType},
//   hittable.{Hittable, HitRecord}, light.{Skylight, SkylightType, ...},
//   scene.Scene, engine.{RenderEngine, EngineState, EngineType, ...},
//   engine.camera.{Camera, CameraParams},
//   data.{RenderLayers, DataObject, LayerType, StreamConfig, TransferStream, ...},
//   cuda, host.memory.
// Errors from the C ABI surface as RuntimeError, where the reference throws
// std::runtime_error or aborts.
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/operators.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <atomic>
#include <cstring>
#include <cmath>
#include <fstream>
#include <chrono>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nectar_b200.h"

namespace py = pybind11;

namespace {

void check(int rc, const char* what) {
  if (rc != NR_OK) throw std::runtime_error(std::string(what) + ": " + nr_last_error());
}

// ---------------------------------------------------------------------------
// core (nectar_render/csrc/core/include/core/vector.h, matrix.h, transform.h)
struct Vector2 {
  float e[2];
  Vector2(float a = 0.f) : e{a, a} {}
  Vector2(float a, float b) : e{a, b} {}
};
struct Vector3 {
  float e[3];
  Vector3(float a = 0.f) : e{a, a, a} {}
  Vector3(float a, float b, float c) : e{a, b, c} {}
  float length() const { return std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]); }
};
struct Color : Vector3 {
  using Vector3::Vector3;
  static Color black() { return Color(0, 0, 0); }
  static Color white() { return Color(1, 1, 1); }
  static Color red() { return Color(1, 0, 0); }
  static Color green() { return Color(0, 1, 0); }
  static Color blue() { return Color(0, 0, 1); }
  static Color purple() { return Color(1, 0, 1); }
  static Color yellow() { return Color(1, 1, 0); }
  static Color teal() { return Color(0, 1, 1); }
};
struct Matrix3 {
  float m[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
};
Matrix3 rot_euler(const Vector3& r) {
  auto rx = [](float a) { Matrix3 M; float c = cosf(a), s = sinf(a); M.m[1][1] = c; M.m[1][2] = -s; M.m[2][1] = s; M.m[2][2] = c; return M; };
  auto ry = [](float a) { Matrix3 M; float c = cosf(a), s = sinf(a); M.m[0][0] = c; M.m[0][2] = s; M.m[2][0] = -s; M.m[2][2] = c; return M; };
  auto rz = [](float a) { Matrix3 M; float c = cosf(a), s = sinf(a); M.m[0][0] = c; M.m[0][1] = -s; M.m[1][0] = s; M.m[1][1] = c; return M; };
  auto mul = [](const Matrix3& a, const Matrix3& b) {
    Matrix3 o;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        o.m[i][j] = 0;
        for (int k = 0; k < 3; k++) o.m[i][j] += a.m[i][k] * b.m[k][j];
      }
    return o;
  };
  return mul(mul(rz(r.e[2]), ry(r.e[1])), rx(r.e[0]));
}
struct Transform {
  Vector3 position{0.f}, rotation{0.f}, scale{1.f};
};

// host/include/host/utils.h:34-38
struct CUDAMemInfo {
  size_t used = 0, free = 0, total = 0;
};
CUDAMemInfo cuda_meminfo() {
  uint64_t u = 0, f = 0, t = 0;
  check(nr_device_memory_info(&u, &f, &t), "get_cuda_meminfo");
  return CUDAMemInfo{(size_t)u, (size_t)f, (size_t)t};
}

// ---------------------------------------------------------------------------
// textures and materials (material.h:453-532, texture.h:93-192)
enum class TextureType { CONSTANT, IMAGE };
struct Texture {
  TextureType type = TextureType::CONSTANT;
  std::string filepath;
  Color constant_color = Color::black();
  size_t C = 3, H = 0, W = 0;
  float scale = 1.0f;
  std::vector<uint8_t> chw;
  static std::shared_ptr<Texture> from_color(const Color& c) {
    auto t = std::make_shared<Texture>();
    t->constant_color = c;
    return t;
  }
  static std::shared_ptr<Texture> from_image(const std::string& path, float scale) {
    // Decoded with Pillow into the file's own channels, as stb_image does
    // (req_comp 0). The reference then builds its planes as
    // chw[c * H * W + i] = data[i * 3 + c] whatever the channel count
    // (texture.h:17-22): RGB images come out right and RGBA images come out
    // shifted, which is kept here; grey images would be read past their
    // data, so those (and palette images) are expanded to RGB instead.
    py::gil_scoped_acquire gil;
    py::module_ np = py::module_::import("numpy");
    py::module_ image = py::module_::import("PIL.Image");
    py::object img = image.attr("open")(path);
    const std::string mode = py::str(img.attr("mode"));
    if (mode != "RGB" && mode != "RGBA") img = img.attr("convert")(mode == "P" || mode == "PA" ? "RGBA" : "RGB");
    if (mode == "P" && !py::bool_(img.attr("info").attr("__contains__")("transparency")))
      img = img.attr("convert")("RGB");
    py::array_t<uint8_t> hwc = np.attr("ascontiguousarray")(np.attr("asarray")(img));
    auto t = std::make_shared<Texture>();
    t->type = TextureType::IMAGE;
    t->filepath = path;
    t->scale = scale;
    t->H = hwc.shape(0);
    t->W = hwc.shape(1);
    t->C = hwc.ndim() == 3 ? hwc.shape(2) : 1;
    const size_t hw = t->H * t->W;
    const uint8_t* data = hwc.data();  // interleaved, C bytes per pixel
    t->chw.resize(t->C * hw);
    for (size_t c = 0; c < t->C; ++c)
      for (size_t i = 0; i < hw; ++i) t->chw[c * hw + i] = data[i * 3 + c];
    return t;
  }
};

enum class MaterialType { Null = 0, Lambertian = 1, PBR = 2, Dielectric = 3, Emissive = 4, Isotropic = 5 };
struct Material {
  MaterialType type = MaterialType::Null;
  std::shared_ptr<Texture> tex[5];
  float ior = 1.5f, brightness = 35.0f;
  Color tint = Color::white();
  uint8_t texture_count() const {
    uint8_t n = 0;
    for (auto& t : tex) n += t ? 1 : 0;
    return n;
  }
};
Material make_lambertian(std::shared_ptr<Texture> t) {
  Material m;
  m.type = MaterialType::Lambertian;
  m.tex[0] = t;
  return m;
}

// ---------------------------------------------------------------------------
// hittables (hittable.h:148-277)
struct Hittable {
  int type = NR_HITTABLE_NULL;
  int wrapped_type = NR_HITTABLE_NULL;
  Vector3 position{0.f}, rotation{0.f}, scale{1.f};
  float radius = 1.0f, density = 1.0f;
  Material mat;
  std::string mesh_path;
  int object_id = -1;
  bool is_light() const { return type == NR_HITTABLE_OBJECT_LIGHT; }
};
Hittable wrap(const Hittable& bound, int type, Material m) {
  if (bound.type == NR_HITTABLE_OBJECT_LIGHT || bound.type == NR_HITTABLE_CONSTANT_MEDIUM ||
      bound.type == NR_HITTABLE_NULL)
    throw std::runtime_error("a light or medium must bind a quad, sphere, cube or mesh");
  Hittable h = bound;
  h.type = type;
  h.wrapped_type = bound.type;
  h.mat = std::move(m);
  return h;
}

// ---------------------------------------------------------------------------
// sky (skylight.h:9-254)
struct SimpleSkylightConfig {
  Color start = Color(1.0f, 1.0f, 1.0f);
  Color end = Color(0.5f, 0.7f, 1.0f);
};
struct HDRISkylightConfig {
  float rotation = 0.0f;
  float intensity = 1.0f;
};
enum class SkylightType { Null, Simple, HDRI };
struct Skylight {
  SkylightType type = SkylightType::Null;
  SimpleSkylightConfig simple;
  HDRISkylightConfig hdri;
  std::string hdri_path;
};

// ---------------------------------------------------------------------------
// camera (camera.h:351-669)
struct CameraParams {
  Vector2 resolution{0.f};
  Vector3 position{0.f}, rotation{0.f};
  uint32_t samples_per_pixel = 0;
  float focal_length = 0, focus_distance = 0, aperture = 0, sensor_width = 0, shutter_speed = 0;
  nr_camera_desc desc() const {
    nr_camera_desc d{};
    d.resolution[0] = resolution.e[0];
    d.resolution[1] = resolution.e[1];
    for (int k = 0; k < 3; ++k) {
      d.position[k] = position.e[k];
      d.rotation[k] = rotation.e[k];
    }
    d.samples_per_pixel = samples_per_pixel;
    d.focal_length = focal_length;
    d.focus_distance = focus_distance;
    d.aperture = aperture;
    d.sensor_width = sensor_width;
    d.shutter_speed = shutter_speed;
    return d;
  }
};
struct Camera {
  CameraParams p;
  std::function<void(CameraParams)> on_updated = [](CameraParams) {};
};

// ---------------------------------------------------------------------------
// scene (scene.h:31-39): hittables followed by lights, one material each
struct Scene {
  std::vector<Hittable*> objects;
  Skylight sky;
};

// SceneNode / SceneOutline (scene/include/outliner.h:7-40): one node per
// registry entry in registration order; name and type_name are both the
// hittable type's name (registry.h:84), parent_id is never set (0).
struct SceneNode {
  size_t object_id = 0, parent_id = 0, material_id = 0;
  bool is_light = false;
  std::string name, type_name;
};
struct SceneOutline {
  std::vector<SceneNode> nodes;
};
constexpr size_t kMaxOutlinerItems = 512;  // outliner.h:5 MAX_OUTLINER_ITEMS

// hittabletype_to_string (hittable/include/hittable/hittable.h:17-28)
const char* hittable_type_name(int t) {
  switch (t) {
    case NR_HITTABLE_NULL: return "Null";
    case NR_HITTABLE_QUAD: return "Quad";
    case NR_HITTABLE_SPHERE: return "Sphere";
    case NR_HITTABLE_CUBE: return "Cube";
    case NR_HITTABLE_MESH: return "Mesh";
    case NR_HITTABLE_CONSTANT_MEDIUM: return "ConstantMedium";
    case NR_HITTABLE_OBJECT_LIGHT: return "ObjectLight";
  }
  return "UNKNOWN";
}

nr_texture_desc tex_desc(nr_scene* s, const std::shared_ptr<Texture>& t) {
  nr_texture_desc d{};
  d.scale = 1.0f;
  if (!t) return d;
  d.type = t->type == TextureType::IMAGE ? NR_TEXTURE_IMAGE : NR_TEXTURE_CONSTANT;
  d.scale = t->scale;
  for (int k = 0; k < 3; ++k) d.rgb[k] = t->constant_color.e[k];
  if (t->type == TextureType::IMAGE) {
    uint32_t id = 0;
    check(nr_scene_add_image(s, t->chw.data(), (uint32_t)t->C, (uint32_t)t->H, (uint32_t)t->W, &id),
          "Texture.from_image");
    d.image = (int32_t)id;
  }
  return d;
}

// Registers the objects (hittables, then lights) and the sky in a new
// nr_scene. `nodes` receives the outline entries and `materials` the
// registry's materials by id (id 0: the default material).
nr_scene* build_scene_desc(const std::vector<Hittable*>& objects, const Skylight& sky,
                           std::vector<SceneNode>* nodes = nullptr,
                           std::vector<Material>* materials = nullptr) {
  nr_scene* s = nullptr;
  check(nr_scene_create(&s), "Scene");
  if (nodes) nodes->clear();
  if (materials) {
    materials->clear();
    materials->push_back(make_lambertian(Texture::from_color(Color::purple())));
  }
  try {
    for (Hittable* h : objects) {
      nr_object_desc o{};
      o.type = h->type;
      o.wrapped_type = h->wrapped_type;
      for (int k = 0; k < 3; ++k) {
        o.position[k] = h->position.e[k];
        o.rotation[k] = h->rotation.e[k];
        o.scale[k] = h->scale.e[k];
      }
      o.radius = h->radius;
      o.density = h->density;
      o.mesh = -1;
      int bt = h->wrapped_type ? h->wrapped_type : h->type;
      if (bt == NR_HITTABLE_MESH) {
        uint32_t mid = 0;
        check(nr_scene_load_obj(s, h->mesh_path.c_str(), &mid), "Hittable.mesh");
        o.mesh = (int32_t)mid;
      }
      // MaterialRegisty::register_material (material/registry.h:30-44)
      if (h->mat.type == MaterialType::Null) {
        o.material = 0;
      } else {
        nr_material_desc m{};
        m.type = (int32_t)h->mat.type;
        m.ior = h->mat.ior;
        m.brightness = h->mat.brightness;
        for (int k = 0; k < 3; ++k) m.tint[k] = h->mat.tint.e[k];
        for (int k = 0; k < 5; ++k) m.tex[k] = tex_desc(s, h->mat.tex[k]);
        uint32_t id = 0;
        check(nr_scene_add_material(s, &m, &id), "material registry");
        o.material = (int32_t)id;
        if (materials) materials->push_back(h->mat);
      }
      uint32_t oid = 0;
      check(nr_scene_add_object(s, &o, &oid), "hittables registry");
      h->object_id = (int)oid;
      if (nodes) {
        SceneNode n;
        n.object_id = oid;
        n.material_id = (size_t)o.material;
        n.is_light = h->is_light();
        n.name = n.type_name = hittable_type_name(h->type);
        nodes->push_back(std::move(n));
      }
    }
    switch (sky.type) {
      case SkylightType::Null: check(nr_scene_set_sky_null(s), "Skylight"); break;
      case SkylightType::Simple:
        check(nr_scene_set_sky_simple(s, sky.simple.start.e, sky.simple.end.e), "Skylight");
        break;
      case SkylightType::HDRI:
        if (sky.hdri_path.empty())
          check(nr_scene_set_sky_hdri(s, nullptr, 0, 0, 0, sky.hdri.rotation, sky.hdri.intensity), "Skylight");
        else
          check(nr_scene_load_hdr(s, sky.hdri_path.c_str(), sky.hdri.rotation, sky.hdri.intensity),
                "Skylight.hdri");
        break;
    }
  } catch (...) {
    nr_scene_destroy(s);
    throw;
  }
  return s;
}

// ---------------------------------------------------------------------------
// data (render_layers.h, data_object.h, stream.h)
enum class LayerType { BEAUTY, DIFFUSE, SPECULAR, OBJECT_NORMAL, WORLD_NORMAL, SHADOW, DEPTH, EMISSION, OBJECT_ID };
enum class TonemapMethod { REINHARD, REINHARD_EXTENDED, ACES };
enum class DenoiseFilterQuality { DEFAULT, HIGH, BALANCED, FAST };
enum class StreamState { ACTIVE, INACTIVE, FROZEN };
struct StreamConfig {
  bool apply_denoising = true;
  bool denoise_clean_auxiliaries = true;
  DenoiseFilterQuality denoise_quality = DenoiseFilterQuality::FAST;
  float denoise_input_scale = 1.0f;
  bool linear_to_gamma = true;
  bool apply_white_balance = true;
  float wb_temperature = 6800.0f;
  float wb_tint = 1.0f;
  bool apply_tonemapping = true;
  TonemapMethod tm_method = TonemapMethod::REINHARD;
  float tm_white_point = 1.0f;
  float tm_alpha = 1.0f;
  nr_stream_config desc() const {
    nr_stream_config c{};
    c.linear_to_gamma = linear_to_gamma;
    c.apply_white_balance = apply_white_balance;
    c.wb_temperature = wb_temperature;
    c.wb_tint = wb_tint;
    c.apply_tonemapping = apply_tonemapping;
    c.tm_method = (int32_t)tm_method;
    c.tm_white_point = tm_white_point;
    c.tm_alpha = tm_alpha;
    return c;
  }
};
struct RenderLayersConfig {
  bool beauty = true, diffuse = true, world_normal = true, object_normal = false, specular = false,
       shadow = false, depth = false, emission = false, object_id = false;
};

struct EngineCore;  // forward

struct DataObject {
  EngineCore* eng = nullptr;
  int layer = 0;
  size_t C = 0, H = 0, W = 0;
  bool enabled = false;
  size_t n_pixels() const { return H * W; }
  size_t n_elements() const { return C * n_pixels(); }
  size_t n_bytes() const { return n_elements() * sizeof(float); }
  std::vector<size_t> shape() const { return {C, H, W}; }
  uintptr_t device_ptr() const;
  py::array numpy() const;
  bool is_enabled() const { return enabled; }
};

struct RenderLayers {
  DataObject beauty, diffuse, world_normal, object_normal, specular, shadow, depth, emission, object_id;
  DataObject* get(LayerType t) {
    switch (t) {
      case LayerType::BEAUTY: return &beauty;
      case LayerType::DIFFUSE: return &diffuse;
      case LayerType::WORLD_NORMAL: return &world_normal;
      case LayerType::OBJECT_NORMAL: return &object_normal;
      case LayerType::SPECULAR: return &specular;
      case LayerType::SHADOW: return &shadow;
      case LayerType::DEPTH: return &depth;
      case LayerType::EMISSION: return &emission;
      case LayerType::OBJECT_ID: return &object_id;
    }
    throw std::runtime_error("DataObject::get_layer() encountered invalid LayerType.");
  }
};

// Page-locked host bytes (nr_host_alloc), grown on demand.
struct PinnedBytes {
  uint8_t* p = nullptr;
  size_t n = 0;
  PinnedBytes() = default;
  PinnedBytes(const PinnedBytes&) = delete;
  PinnedBytes& operator=(const PinnedBytes&) = delete;
  ~PinnedBytes() { nr_host_free(p); }
  void resize(size_t bytes) {
    if (bytes == n) return;
    nr_host_free(p);
    p = nullptr;
    n = 0;
    void* q = nullptr;
    check(nr_host_alloc(bytes, &q), "TransferStream buffer");
    p = static_cast<uint8_t*>(q);
    n = bytes;
  }
  uint8_t* data() { return p; }
  const uint8_t* data() const { return p; }
  size_t size() const { return n; }
};

struct TransferStream {
  EngineCore* eng = nullptr;
  std::atomic<StreamState> state{StreamState::INACTIVE};
  StreamConfig cfg;
  int layer = (int)LayerType::BEAUTY;
  PinnedBytes buffer;  // page-locked, like the reference's readback buffer
  // the config the render's accumulate pass already applies (fused display)
  nr_render* fused_render = nullptr;
  nr_stream_config fused_cfg{};
  uintptr_t readback();
  uintptr_t buffer_ptr() { return reinterpret_cast<uintptr_t>(buffer.data()); }
  std::array<size_t, 3> shape() const;
};

// requests (engine/include/engine/requests.h:6-26)
struct EngineRequests {
  std::atomic<bool> start_{false}, stop_{false}, restart_{false}, shutdown_{false};
  void start() { start_ = true; }
  void stop() { stop_ = true; }
  void restart() { restart_ = true; }
  void shutdown() { shutdown_ = true; }
};

enum class EngineState { IDLE, RENDERING };
enum class EngineType { PATHTRACER, VIEWPORT };
struct EnginePollResponse {
  bool should_update_camera = false;
  CameraParams camera_params;
};

// HitRecord (hittable/include/hittable/hit_record.h:9-22) as a picking query
// returns it.
struct HitRecord {
  size_t object_id = 0;
  size_t material_id = 0;
  Vector3 p, n, tangent;
  Vector2 uv;
  float t = 0.f;
  bool front_face = false;
  bool hit = false;
};

// SceneInterface (scene/include/interface.h:36-200): picking and selection
// (query_scene casts the screen-space ray and keeps the hit), the scene
// outline, and edits of the selected object, the sky and the object list.
// Edits change the engine's copy of the scene and request a restart; the
// render loop rebuilds the device scene before its next sample, where the
// reference marks the registry entry dirty and rebuilds in its update step.
struct SceneInterface {
  EngineCore* eng = nullptr;
  HitRecord rec;
  std::atomic<bool> enabled{false};
  int outline_radius = 2;
  void query_scene(float u, float v);
  void select_scene_node(const SceneNode& n);
  SceneOutline get_scene_outline() const;
  Transform get_transform() const;
  void set_transform(const Transform& x);
  Material& get_material();
  void set_material(const Material& m);
  void add_object(const Hittable& h);
  Skylight& get_skylight();
  void request_skylight_update();
  void swap_skylight(const Skylight& sky);
  py::array selection_mask() const;
};

struct EngineCore {
  Camera cam;
  uint32_t ray_depth, seed;
  uint32_t sample_idx = 1;
  nr_scene* scene = nullptr;
  nr_render* render = nullptr;
  RenderLayers layers;
  TransferStream stream;
  EngineRequests requests;
  std::atomic<EngineState> state{EngineState::IDLE};
  std::atomic<EngineType> type{EngineType::PATHTRACER};
  std::atomic<bool> show_axis_grid{true};
  SceneInterface scene_interface;
  int mode = NR_MODE_REFERENCE;
  bool hooks_set = false;
  // the scene as last set or edited: objects (hittables, then lights), sky,
  // the outline and the material registry built from them
  std::mutex scene_mu;
  std::vector<Hittable> objects;
  Skylight sky;
  std::vector<SceneNode> nodes;
  std::vector<Material> materials;
  std::atomic<bool> scene_dirty{false};
  std::function<void()> on_render_started = [] {}, on_render_finished = [] {}, on_stopped = [] {},
                        on_restarted = [] {}, on_reset = [] {}, on_shutdown = [] {};
  std::function<void(uint32_t)> on_frame_finished = [](uint32_t) {};
  std::function<EnginePollResponse()> poll_updates = [] { return EnginePollResponse{}; };

  EngineCore(const Camera& c, uint32_t depth, uint32_t sd) : cam(c), ray_depth(depth), seed(sd) {
    stream.eng = this;
    scene_interface.eng = this;
    wire_layers(false);
  }
  ~EngineCore() {
    if (render) nr_render_destroy(render);
    if (scene) nr_scene_destroy(scene);
  }
  uint32_t H() const { return (uint32_t)cam.p.resolution.e[0]; }
  uint32_t W() const { return (uint32_t)cam.p.resolution.e[1]; }
  void wire_layers(bool live) {
    RenderLayers& L = layers;
    DataObject* all[9] = {&L.beauty, &L.diffuse, &L.specular, &L.object_normal, &L.world_normal,
                          &L.shadow, &L.depth, &L.emission, &L.object_id};
    for (int l = 0; l < 9; ++l) {
      DataObject& d = *all[l];
      d.eng = this;
      d.layer = l;
      bool on = l == 0 || l == 1 || l == 4;
      d.enabled = on;
      d.C = on ? 3 : 0;
      d.H = on ? H() : 0;
      d.W = on ? W() : 0;
    }
    (void)live;
  }
  void make_render() {
    if (render) {
      nr_render_destroy(render);
      render = nullptr;
    }
    if (!scene) return;
    nr_render_config cfg;
    nr_render_config_default(&cfg);
    cfg.ray_depth = ray_depth;
    cfg.seed = seed;
    cfg.mode = mode;
    nr_camera_desc d = cam.p.desc();
    check(nr_render_create(scene, &d, &cfg, &render), "RenderEngine");
    sample_idx = 1;
  }
  // Builds the device scene from `objects` and `sky` and replaces the
  // current one (and its render). Called with the GIL released.
  void rebuild_scene() {
    std::vector<Hittable*> ptrs;
    std::vector<SceneNode> new_nodes;
    std::vector<Material> new_mats;
    nr_scene* s = nullptr;
    {
      std::lock_guard<std::mutex> lk(scene_mu);
      for (Hittable& h : objects) ptrs.push_back(&h);
      s = build_scene_desc(ptrs, sky, &new_nodes, &new_mats);
    }
    int rc = nr_scene_build(s);
    if (rc != NR_OK) {
      std::string msg = nr_last_error();
      nr_scene_destroy(s);
      throw std::runtime_error("RenderEngine.set_scene: " + msg);
    }
    if (render) { nr_render_destroy(render); render = nullptr; }
    if (scene) nr_scene_destroy(scene);
    scene = s;
    {
      std::lock_guard<std::mutex> lk(scene_mu);
      nodes = std::move(new_nodes);
      materials = std::move(new_mats);
    }
    make_render();
  }
  // Scene edits made through the SceneInterface since the last sample.
  void apply_scene_edits() {
    if (scene_dirty.exchange(false)) rebuild_scene();
  }
  // RenderEngine::reset (engine.cpp:216-220): the next sample is 1, whose
  // running mean overwrites the layers; they are not cleared (a viewport
  // frame or a stopped render stays visible until then).
  void reset() {
    sample_idx = 1;
    py::gil_scoped_acquire gil;
    on_reset();
  }
  // RenderEngine::viewport (engine.cpp:77-95): one preview frame into the
  // layers; returns 3 (waiting for the next refresh), 1 stopped, 2 restarted.
  int run_viewport() {
    if (!render) throw std::runtime_error("RenderEngine.render() called before set_scene()");
    apply_scene_edits();
    EnginePollResponse resp;
    {
      py::gil_scoped_acquire gil;
      resp = poll_updates();
    }
    if (requests.stop_.exchange(false)) return 1;
    if (resp.should_update_camera) {
      cam.p = resp.camera_params;
      make_render();
    }
    check(nr_render_viewport(render, show_axis_grid.load() ? 1 : 0), "RenderEngine.viewport");
    if (requests.restart_.exchange(false)) return 2;
    return 3;
  }
  // RenderEngine::render (engine.cpp:42-74): samples sample_idx .. n-1
  int run() {
    if (!render) throw std::runtime_error("RenderEngine.render() called before set_scene()");
    apply_scene_edits();
    uint32_t n = cam.p.samples_per_pixel;
    if (!hooks_set && sample_idx < n) {
      int rc = nr_render_samples(render, sample_idx, n - sample_idx);
      check(rc, "RenderEngine.render");
      sample_idx = n;
      return 0;
    }
    for (; sample_idx < n;) {
      EnginePollResponse resp;
      {
        py::gil_scoped_acquire gil;
        resp = poll_updates();
      }
      if (requests.stop_.exchange(false)) return 1;
      if (resp.should_update_camera) {
        cam.p = resp.camera_params;
        make_render();
        requests.restart();
      }
      apply_scene_edits();
      check(nr_render_samples(render, sample_idx, 1), "RenderEngine.render");
      sample_idx++;
      {
        py::gil_scoped_acquire gil;
        on_frame_finished(sample_idx);
      }
      if (requests.restart_.exchange(false)) return 2;
    }
    return 0;
  }
};

void SceneInterface::query_scene(float u, float v) {
  if (!eng || !eng->render) throw std::runtime_error("query_scene() before set_scene()");
  nr_pick_result r;
  check(nr_render_pick(eng->render, u, v, &r), "SceneInterface.query_scene");
  rec = HitRecord{};
  rec.hit = r.hit != 0;
  if (rec.hit) {
    rec.object_id = r.object_id;
    rec.material_id = r.material_id;
    rec.p = Vector3(r.p[0], r.p[1], r.p[2]);
    rec.n = Vector3(r.n[0], r.n[1], r.n[2]);
    rec.uv = Vector2(r.uv[0], r.uv[1]);
    rec.t = r.t;
    rec.front_face = r.front_face != 0;
    enabled = true;
  }
}

void SceneInterface::select_scene_node(const SceneNode& n) {
  rec.object_id = n.object_id;
  rec.material_id = n.material_id;
  enabled = true;
}

// SceneOutliner::build_outline (outliner.h:48-66) with SceneOutline's limit
SceneOutline SceneInterface::get_scene_outline() const {
  if (!eng) throw std::runtime_error("get_scene_outline() before set_scene()");
  std::lock_guard<std::mutex> lk(eng->scene_mu);
  if (eng->nodes.size() > kMaxOutlinerItems)
    throw std::runtime_error("SceneOutline exceeded maximum node count [" +
                             std::to_string(kMaxOutlinerItems) + "].");
  return SceneOutline{eng->nodes};
}

static Hittable& selected_object(EngineCore* eng, size_t id) {
  if (!eng || id >= eng->objects.size()) throw std::runtime_error("Object index not valid.");
  return eng->objects[id];
}

Transform SceneInterface::get_transform() const {
  std::lock_guard<std::mutex> lk(eng->scene_mu);
  const Hittable& h = selected_object(eng, rec.object_id);
  Transform t;
  t.position = h.position;
  t.rotation = h.rotation;
  t.scale = h.scale;
  return t;
}

void SceneInterface::set_transform(const Transform& x) {
  {
    std::lock_guard<std::mutex> lk(eng->scene_mu);
    Hittable& h = selected_object(eng, rec.object_id);
    h.position = x.position;
    h.rotation = x.rotation;
    h.scale = x.scale;
  }
  eng->scene_dirty = true;
  eng->requests.restart();
}

Material& SceneInterface::get_material() {
  std::lock_guard<std::mutex> lk(eng->scene_mu);
  if (rec.material_id >= eng->materials.size()) throw std::runtime_error("Material index not valid.");
  return eng->materials[rec.material_id];
}

// The reference's set_material only requests a restart; its registry update
// is commented out (interface.h:154-159).
void SceneInterface::set_material(const Material&) { eng->requests.restart(); }

void SceneInterface::add_object(const Hittable& h) {
  {
    std::lock_guard<std::mutex> lk(eng->scene_mu);
    if (eng->objects.size() >= NR_MAX_OBJECTS)
      throw std::runtime_error("Hittables registry exceeded maximum registry entries [" +
                               std::to_string(NR_MAX_OBJECTS) + "]. Exiting...");
    eng->objects.push_back(h);
  }
  eng->scene_dirty = true;
  eng->requests.restart();
}

Skylight& SceneInterface::get_skylight() { return eng->sky; }

void SceneInterface::request_skylight_update() {
  eng->scene_dirty = true;
  eng->requests.restart();
}

void SceneInterface::swap_skylight(const Skylight& sky) {
  {
    std::lock_guard<std::mutex> lk(eng->scene_mu);
    eng->sky = sky;
  }
  eng->scene_dirty = true;
  eng->requests.restart();
}

py::array SceneInterface::selection_mask() const {
  if (!eng || !eng->render) throw std::runtime_error("selection mask before set_scene()");
  py::array_t<uint8_t> out({(size_t)eng->H(), (size_t)eng->W()});
  check(nr_render_selection_mask(eng->render, (uint32_t)rec.object_id, outline_radius,
                                 out.mutable_data()),
        "SceneInterface.selection_mask");
  return std::move(out);
}

uintptr_t DataObject::device_ptr() const {
  if (!eng || !eng->render || !enabled) return 0;
  uint64_t p = 0;
  check(nr_render_layer_device_ptr(eng->render, layer, &p), "DataObject.device_ptr");
  return (uintptr_t)p;
}

// DataObject::numpy (data_object.h:201-216): clamp(x,0,1)*255 truncated to uint8, CHW
py::array DataObject::numpy() const {
  py::array_t<uint8_t> out({C, H, W});
  if (!eng || !eng->render || !enabled) return std::move(out);
  nr_stream_config raw{};
  raw.tm_alpha = 1.0f;
  raw.tm_white_point = 1.0f;
  check(nr_render_readback(eng->render, layer, &raw, out.mutable_data()), "DataObject.numpy");
  return std::move(out);
}

uintptr_t TransferStream::readback() {
  if (!eng || !eng->render) throw std::runtime_error("TransferStream.readback() before set_scene()");
  if (state == StreamState::FROZEN) return buffer_ptr();
  buffer.resize((size_t)3 * eng->H() * eng->W());
  nr_stream_config c = cfg.desc();
  if (layer == (int)LayerType::BEAUTY &&
      (fused_render != eng->render || memcmp(&c, &fused_cfg, sizeof(c)) != 0)) {
    // later renders write this stream's bytes in their accumulate pass
    check(nr_render_set_fused_display(eng->render, &c), "TransferStream.readback");
    fused_render = eng->render;
    fused_cfg = c;
  }
  check(nr_render_readback(eng->render, layer, &c, buffer.data()), "TransferStream.readback");
  return buffer_ptr();
}
std::array<size_t, 3> TransferStream::shape() const {
  return {3, (size_t)eng->H(), (size_t)eng->W()};
}

// Not in the reference: a hittable's and a sky's settings as stored, for
// tools that convert a scene built through this API into another form.
py::tuple v3_tuple(const Vector3& v) { return py::make_tuple(v.e[0], v.e[1], v.e[2]); }

py::dict describe_hittable(const Hittable& h) {
  py::dict d, m;
  d["type"] = h.type;
  d["wrapped_type"] = h.wrapped_type;
  d["position"] = v3_tuple(h.position);
  d["rotation"] = v3_tuple(h.rotation);
  d["scale"] = v3_tuple(h.scale);
  d["radius"] = h.radius;
  d["density"] = h.density;
  d["mesh_path"] = h.mesh_path;
  m["type"] = (int)h.mat.type;
  m["ior"] = h.mat.ior;
  m["brightness"] = h.mat.brightness;
  m["tint"] = v3_tuple(h.mat.tint);
  py::list tex;
  for (auto& t : h.mat.tex) {
    if (!t) tex.append(py::make_tuple(0.f, 0.f, 0.f));
    else if (t->type == TextureType::IMAGE) tex.append(py::str(t->filepath));
    else tex.append(v3_tuple(t->constant_color));
  }
  m["tex"] = tex;
  d["material"] = m;
  return d;
}

py::dict describe_sky(const Skylight& s) {
  py::dict d;
  d["type"] = (int)s.type;
  d["start"] = v3_tuple(s.simple.start);
  d["end"] = v3_tuple(s.simple.end);
  d["path"] = s.hdri_path;
  d["rotation"] = s.hdri.rotation;
  d["intensity"] = s.hdri.intensity;
  return d;
}

}  // namespace

PYBIND11_MODULE(_pathtracer, m) {
  m.doc() = "NectarRender path-tracing back end for B200 (sm_100a)";
  m.def("abi_version", &nr_abi_version);
  m.def("device_count", &nr_device_count);

  // ---- core
  auto m_core = m.def_submodule("core", "Core module.");
  auto m_vec = m_core.def_submodule("vector", "Vector module.");
  py::class_<Vector2>(m_vec, "Vector2")
      .def(py::init<float>())
      .def(py::init<float, float>())
      .def("x", [](const Vector2& v) { return v.e[0]; })
      .def("y", [](const Vector2& v) { return v.e[1]; })
      .def("u", [](const Vector2& v) { return v.e[0]; })
      .def("v", [](const Vector2& v) { return v.e[1]; })
      .def("__repr__", [](const Vector2& v) {
        return "Vector2(" + std::to_string(v.e[0]) + ", " + std::to_string(v.e[1]) + ")";
      });
  py::class_<Vector3>(m_vec, "Vector3")
      .def(py::init<float>())
      .def(py::init<float, float, float>())
      .def("x", [](const Vector3& v) { return v.e[0]; })
      .def("y", [](const Vector3& v) { return v.e[1]; })
      .def("z", [](const Vector3& v) { return v.e[2]; })
      .def("u", [](const Vector3& v) { return v.e[0]; })
      .def("v", [](const Vector3& v) { return v.e[1]; })
      .def("w", [](const Vector3& v) { return v.e[2]; })
      .def("length", &Vector3::length)
      .def("as_array", [](const Vector3& v) { return std::array<float, 3>{v.e[0], v.e[1], v.e[2]}; })
      .def("__add__", [](const Vector3& a, const Vector3& b) { return Vector3(a.e[0] + b.e[0], a.e[1] + b.e[1], a.e[2] + b.e[2]); })
      .def("__sub__", [](const Vector3& a, const Vector3& b) { return Vector3(a.e[0] - b.e[0], a.e[1] - b.e[1], a.e[2] - b.e[2]); })
      .def("__mul__", [](const Vector3& a, float t) { return Vector3(a.e[0] * t, a.e[1] * t, a.e[2] * t); })
      .def("__repr__", [](const Vector3& v) {
        return "Vector3(" + std::to_string(v.e[0]) + ", " + std::to_string(v.e[1]) + ", " + std::to_string(v.e[2]) + ")";
      });
  py::class_<Color, Vector3>(m_vec, "Color")
      .def(py::init<float>())
      .def(py::init<float, float, float>())
      .def("r", [](const Color& v) { return v.e[0]; })
      .def("g", [](const Color& v) { return v.e[1]; })
      .def("b", [](const Color& v) { return v.e[2]; })
      .def_static("black", &Color::black)
      .def_static("white", &Color::white)
      .def_static("red", &Color::red)
      .def_static("green", &Color::green)
      .def_static("blue", &Color::blue)
      .def_static("purple", &Color::purple)
      .def_static("yellow", &Color::yellow)
      .def_static("teal", &Color::teal);
  py::implicitly_convertible<py::tuple, Vector3>();
  auto m_mat3 = m_core.def_submodule("matrix", "Matrix module.");
  py::class_<Matrix3>(m_mat3, "Matrix3")
      .def(py::init<>())
      .def("numpy", [](const Matrix3& a) {
        std::array<std::array<float, 3>, 3> o;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) o[i][j] = a.m[i][j];
        return o;
      });
  m_mat3.def("rotation_from_euler", &rot_euler);
  py::class_<Transform>(m_core, "Transform")
      .def(py::init<>())
      .def(py::init([](Vector3 p, Vector3 r, Vector3 s) { return Transform{p, r, s}; }),
           py::arg("position") = Vector3(0.f), py::arg("rotation") = Vector3(0.f),
           py::arg("scale") = Vector3(1.f))
      .def("position", [](const Transform& t) { return t.position; })
      .def("rotation", [](const Transform& t) { return rot_euler(Vector3(t.rotation.e[0] * 0.01745329f, t.rotation.e[1] * 0.01745329f, t.rotation.e[2] * 0.01745329f)); })
      .def("scale", [](const Transform& t) { return t.scale; });

  // ---- cuda / host utilities
  auto m_cuda = m.def_submodule("cuda", "CUDA utility module.");
  m_cuda.def("destroy_cublas_handle", []() {});
  m_cuda.def("cudaDeviceSynchronize", []() {});
  auto m_host = m.def_submodule("host", "Host module.");
  auto m_memory = m_host.def_submodule("memory", "Memory utils submodule.");
  m_host.def_submodule("devtools", "Devtools submodule.");
  // CUDAMemInfo and its getters (host/include/host/utils.h:34-42)
  py::class_<CUDAMemInfo>(m_memory, "CUDAMemInfo")
      .def_readonly("used", &CUDAMemInfo::used)
      .def_readonly("free", &CUDAMemInfo::free)
      .def_readonly("total", &CUDAMemInfo::total)
      .def("__repr__", [](const CUDAMemInfo& i) {
        return "CUDAMemInfo(used=" + std::to_string(i.used) + ", free=" + std::to_string(i.free) +
               ", total=" + std::to_string(i.total) + ")";
      });
  m_memory.def("get_cuda_meminfo", &cuda_meminfo);
  m_memory.def("get_cuda_memory_used", []() { return cuda_meminfo().used; });
  m_memory.def("get_cuda_memory_free", []() { return cuda_meminfo().free; });
  m_memory.def("get_cuda_memory_total", []() { return cuda_meminfo().total; });

  // ---- material
  auto m_material = m.def_submodule("material", "Material module.");
  auto m_texture = m_material.def_submodule("texture", "Texture submodule.");
  py::enum_<TextureType>(m_texture, "TextureType")
      .value("CONSTANT", TextureType::CONSTANT)
      .value("IMAGE", TextureType::IMAGE);
  py::class_<Texture, std::shared_ptr<Texture>>(m_texture, "Texture")
      .def_static("from_color", [](const Color& c) { return Texture::from_color(c); }, py::arg("color"))
      .def_static("from_color", [](float r, float g, float b) { return Texture::from_color(Color(r, g, b)); },
                  py::arg("r"), py::arg("g"), py::arg("b"))
      .def_static("from_image", &Texture::from_image, py::arg("filepath"), py::arg("scale") = 1.0f)
      .def_readonly("type", &Texture::type)
      .def_readonly("filepath", &Texture::filepath)
      .def_readonly("constant_color", &Texture::constant_color)
      .def_readonly("C", &Texture::C)
      .def_readonly("H", &Texture::H)
      .def_readonly("W", &Texture::W)
      .def_property_readonly("texels", [](const Texture& t) {
        // planar CHW uint8 copy of an IMAGE texture's planes (empty otherwise)
        py::array_t<uint8_t> a({(py::ssize_t)t.C, (py::ssize_t)t.H, (py::ssize_t)t.W});
        if (!t.chw.empty()) std::memcpy(a.mutable_data(), t.chw.data(), t.chw.size());
        return a;
      });
  py::enum_<MaterialType>(m_material, "MaterialType")
      .value("Lambertian", MaterialType::Lambertian)
      .value("PBR", MaterialType::PBR)
      .value("Dielectric", MaterialType::Dielectric)
      .value("Emissive", MaterialType::Emissive)
      .value("Isotropic", MaterialType::Isotropic);
  py::class_<Material>(m_material, "Material")
      .def(py::init<>())
      .def("material_type", [](const Material& m) { return m.type; })
      .def("texture_count", &Material::texture_count)
      .def("get_tracked_texture", [](Material& m, size_t i) { return m.tex[i]; })
      .def_static("lambertian", [](const Color& c) { return make_lambertian(Texture::from_color(c)); },
                  py::arg("color") = Color::white())
      .def_static("lambertian", [](std::shared_ptr<Texture> t) { return make_lambertian(t); },
                  py::arg("texture"))
      .def_static("pbr",
                  [](std::shared_ptr<Texture> a, std::shared_ptr<Texture> r, std::shared_ptr<Texture> mt,
                     std::shared_ptr<Texture> e, std::shared_ptr<Texture> n) {
                    Material m;
                    m.type = MaterialType::PBR;
                    m.tex[0] = a; m.tex[1] = r; m.tex[2] = mt; m.tex[3] = e; m.tex[4] = n;
                    return m;
                  },
                  py::arg("albedo") = Texture::from_color(Color::white()),
                  py::arg("roughness") = Texture::from_color(Color(0.8f)),
                  py::arg("metallic") = Texture::from_color(Color(0.0f)),
                  py::arg("emission") = Texture::from_color(Color::black()),
                  py::arg("normal") = Texture::from_color(Color(0.5f, 0.5f, 1.0f)))
      .def_static("dielectric",
                  [](const Color& tint, float ior) {
                    Material m;
                    m.type = MaterialType::Dielectric;
                    m.tint = tint;
                    m.ior = ior;
                    return m;
                  },
                  py::arg("tint") = Color::white(), py::arg("ior") = 1.5f)
      .def_static("emissive",
                  [](const Color& c, float b) {
                    Material m;
                    m.type = MaterialType::Emissive;
                    m.tex[0] = Texture::from_color(c);
                    m.brightness = b;
                    return m;
                  },
                  py::arg("albedo") = Color::white(), py::arg("brightness") = 35.0f)
      .def_static("emissive",
                  [](std::shared_ptr<Texture> t, float b) {
                    Material m;
                    m.type = MaterialType::Emissive;
                    m.tex[0] = t;
                    m.brightness = b;
                    return m;
                  },
                  py::arg("texture"), py::arg("brightness") = 35.0f)
      .def_static("isotropic",
                  [](const Color& c) {
                    Material m;
                    m.type = MaterialType::Isotropic;
                    m.tex[0] = Texture::from_color(c);
                    return m;
                  },
                  py::arg("albedo") = Color::white())
      .def_static("isotropic",
                  [](std::shared_ptr<Texture> t) {
                    Material m;
                    m.type = MaterialType::Isotropic;
                    m.tex[0] = t;
                    return m;
                  },
                  py::arg("texture"))
      .def("__repr__", [](const Material& m) {
        static const char* n[] = {"UNKNOWN", "Lambertian", "PBR", "Dielectric", "Emissive", "Isotropic"};
        return std::string("Material(type = ") + n[(int)m.type] + ")";
      });

  // ---- hittable
  auto m_hit = m.def_submodule("hittable", "Hittable module.");
  py::class_<HitRecord>(m_hit, "HitRecord")
      .def(py::init<>())
      .def_readonly("object_id", &HitRecord::object_id)
      .def_readonly("material_id", &HitRecord::material_id)
      .def_readonly("p", &HitRecord::p)
      .def_readonly("n", &HitRecord::n)
      .def_readonly("tangent", &HitRecord::tangent)
      .def_readonly("uv", &HitRecord::uv)
      .def_readonly("t", &HitRecord::t)
      .def_readonly("front_face", &HitRecord::front_face);
  auto default_mat = []() { return make_lambertian(Texture::from_color(Color::purple())); };
  py::class_<Hittable>(m_hit, "Hittable")
      .def(py::init<>())
      .def_static("quad",
                  [](Vector3 p, Vector3 r, Vector3 s, const Material& mat) {
                    Hittable h;
                    h.type = NR_HITTABLE_QUAD;
                    h.position = p; h.rotation = r; h.scale = s; h.mat = mat;
                    return h;
                  },
                  py::arg("position") = Vector3(0.f), py::arg("rotation") = Vector3(0.f),
                  py::arg("scale") = Vector3(0.f), py::arg("material") = default_mat())
      .def_static("cube",
                  [](Vector3 p, Vector3 r, Vector3 s, const Material& mat) {
                    Hittable h;
                    h.type = NR_HITTABLE_CUBE;
                    h.position = p; h.rotation = r; h.scale = s; h.mat = mat;
                    return h;
                  },
                  py::arg("position") = Vector3(0.f), py::arg("rotation") = Vector3(0.f),
                  py::arg("scale") = Vector3(0.f), py::arg("material") = default_mat())
      .def_static("sphere",
                  [](Vector3 p, float radius, const Material& mat) {
                    Hittable h;
                    h.type = NR_HITTABLE_SPHERE;
                    h.position = p; h.radius = radius; h.mat = mat;
                    return h;
                  },
                  py::arg("position") = Vector3(0.f), py::arg("radius") = 1.0f,
                  py::arg("material") = default_mat())
      .def_static("mesh",
                  [](const std::string& path, Vector3 p, Vector3 r, Vector3 s, const Material& mat) {
                    std::ifstream f(path);
                    if (!f) throw std::runtime_error("Failed to load OBJ '" + path + "': cannot open file");
                    Hittable h;
                    h.type = NR_HITTABLE_MESH;
                    h.mesh_path = path;
                    h.position = p; h.rotation = r; h.scale = s; h.mat = mat;
                    return h;
                  },
                  py::arg("path"), py::arg("position") = Vector3(0.f),
                  py::arg("rotation") = Vector3(0.f), py::arg("scale") = Vector3(0.f),
                  py::arg("material") = default_mat())
      .def_static("constant_medium",
                  [](const Hittable& b, float density, std::shared_ptr<Texture> t) {
                    Material m; m.type = MaterialType::Isotropic; m.tex[0] = t;
                    Hittable h = wrap(b, NR_HITTABLE_CONSTANT_MEDIUM, m);
                    h.density = density;
                    return h;
                  },
                  py::arg("bound_obj"), py::arg("density") = 1.0f, py::arg("texture"))
      .def_static("constant_medium",
                  [](const Hittable& b, float density, const Color& c) {
                    Material m; m.type = MaterialType::Isotropic; m.tex[0] = Texture::from_color(c);
                    Hittable h = wrap(b, NR_HITTABLE_CONSTANT_MEDIUM, m);
                    h.density = density;
                    return h;
                  },
                  py::arg("bound_obj"), py::arg("density") = 1.0f, py::arg("albedo") = Color(1.f, 1.f, 1.f))
      .def_static("object_light",
                  [](const Hittable& b, float brightness, std::shared_ptr<Texture> t) {
                    Material m; m.type = MaterialType::Emissive; m.tex[0] = t; m.brightness = brightness;
                    return wrap(b, NR_HITTABLE_OBJECT_LIGHT, m);
                  },
                  py::arg("bound_obj"), py::arg("brightness") = 1.0f, py::arg("texture"))
      .def_static("object_light",
                  [](const Hittable& b, float brightness, const Color& c) {
                    Material m; m.type = MaterialType::Emissive; m.tex[0] = Texture::from_color(c); m.brightness = brightness;
                    return wrap(b, NR_HITTABLE_OBJECT_LIGHT, m);
                  },
                  py::arg("bound_obj"), py::arg("brightness") = 1.0f, py::arg("albedo") = Color(1.f, 1.f, 1.f))
      .def("is_light", &Hittable::is_light)
      .def("get_object_id", [](const Hittable& h) { return h.object_id; })
      // not in the reference: the factory arguments as stored, for tools
      // that convert a scene built through this API into another form
      .def("describe", &describe_hittable);

  // ---- light
  auto m_light = m.def_submodule("light", "Lights module.");
  py::enum_<SkylightType>(m_light, "SkylightType")
      .value("Null", SkylightType::Null)
      .value("Simple", SkylightType::Simple)
      .value("HDRI", SkylightType::HDRI);
  py::class_<SimpleSkylightConfig>(m_light, "SimpleSkylightConfig")
      .def_readwrite("start", &SimpleSkylightConfig::start)
      .def_readwrite("end", &SimpleSkylightConfig::end);
  py::class_<HDRISkylightConfig>(m_light, "HDRISkylightConfig")
      .def_readwrite("rotation", &HDRISkylightConfig::rotation)
      .def_readwrite("intensity", &HDRISkylightConfig::intensity);
  py::class_<Skylight>(m_light, "Skylight")
      .def(py::init<>())
      .def_static("simple",
                  [](const Color& a, const Color& b) {
                    Skylight s;
                    s.type = SkylightType::Simple;
                    s.simple.start = a;
                    s.simple.end = b;
                    return s;
                  },
                  py::arg("start_color") = Color(1.f, 1.f, 1.f), py::arg("end_color") = Color(0.5f, 0.7f, 1.0f))
      .def_static("hdri", []() { Skylight s; s.type = SkylightType::HDRI; return s; })
      .def_static("hdri",
                  [](const std::string& path) {
                    std::ifstream f(path);
                    if (!f) throw std::runtime_error("Failed to load HDRI: cannot open '" + path + "'");
                    Skylight s;
                    s.type = SkylightType::HDRI;
                    s.hdri_path = path;
                    return s;
                  },
                  py::arg("filepath"))
      .def("load_hdri_file",
           [](Skylight& s, const std::string& path) {
             if (s.type != SkylightType::HDRI)
               throw std::runtime_error("Skylight::update_hdri is only valid on skylights with type SkylightType::HDRI.");
             s.hdri_path = path;
           })
      .def("config_simple", [](Skylight& s) -> SimpleSkylightConfig& { return s.simple; }, py::return_value_policy::reference_internal)
      .def("config_hdri", [](Skylight& s) -> HDRISkylightConfig& { return s.hdri; }, py::return_value_policy::reference_internal)
      // not in the reference: the sky's settings as stored
      .def("describe", &describe_sky);

  // ---- scene
  auto m_scene = m.def_submodule("scene", "Scene module.");
  py::class_<Scene>(m_scene, "Scene")
      .def(py::init([](py::list hittables, py::list lights, const Skylight& sky) {
             Scene s;
             for (auto& h : hittables) s.objects.push_back(h.cast<Hittable*>());
             for (auto& h : lights) s.objects.push_back(h.cast<Hittable*>());
             s.sky = sky;
             return s;
           }),
           py::arg("hittables"), py::arg("lights"), py::arg("skylight"), py::keep_alive<1, 2>(),
           py::keep_alive<1, 3>())
      // not in the reference: the registered objects (hittables, then
      // lights) and the sky, as describe() dicts
      .def("describe", [](const Scene& sc) {
        py::dict d;
        py::list objs;
        for (Hittable* h : sc.objects) objs.append(describe_hittable(*h));
        d["objects"] = objs;
        d["sky"] = describe_sky(sc.sky);
        return d;
      });

  py::class_<SceneNode>(m_scene, "SceneNode")
      .def_readonly("object_id", &SceneNode::object_id)
      .def_readonly("parent_id", &SceneNode::parent_id)
      .def_readonly("material_id", &SceneNode::material_id)
      .def_readonly("name", &SceneNode::name)
      .def_readonly("type_name", &SceneNode::type_name);
  py::class_<SceneOutline>(m_scene, "SceneOutline")
      .def_readonly("nodes", &SceneOutline::nodes);

  py::class_<SceneInterface>(m_scene, "SceneInterface")
      .def("set_material", &SceneInterface::set_material, py::arg("mat"))
      .def("add_object", &SceneInterface::add_object, py::arg("obj"))
      .def("query_scene", &SceneInterface::query_scene, py::arg("u"), py::arg("v"))
      .def("select_scene_node", &SceneInterface::select_scene_node, py::arg("node"))
      .def("enable", [](SceneInterface& si) { si.enabled = true; })
      .def("disable", [](SceneInterface& si) { si.enabled = false; })
      .def("is_enabled", [](SceneInterface& si) { return si.enabled.load(); })
      .def("is_disabled", [](SceneInterface& si) { return !si.enabled.load(); })
      .def("get_scene_outline", &SceneInterface::get_scene_outline)
      .def("get_transform", &SceneInterface::get_transform)
      .def("set_transform", &SceneInterface::set_transform)
      .def("get_material", &SceneInterface::get_material, py::return_value_policy::reference_internal)
      .def("get_hit_record", [](SceneInterface& si) -> HitRecord& { return si.rec; },
           py::return_value_policy::reference_internal)
      .def("request_skylight_update", &SceneInterface::request_skylight_update)
      .def("get_skylight", &SceneInterface::get_skylight, py::return_value_policy::reference_internal)
      .def("swap_skylight", &SceneInterface::swap_skylight, py::arg("new_skylight"))
      // not in the reference (its mask goes straight into the stream's
      // overlay): the selection outline as an H x W uint8 mask
      .def("selection_mask", &SceneInterface::selection_mask);

  // ---- data
  auto m_data = m.def_submodule("data", "Data module.");
  py::enum_<StreamState>(m_data, "StreamState")
      .value("ACTIVE", StreamState::ACTIVE)
      .value("INACTIVE", StreamState::INACTIVE)
      .value("FROZEN", StreamState::FROZEN);
  py::enum_<TonemapMethod>(m_data, "TonemapMethod")
      .value("REINHARD", TonemapMethod::REINHARD)
      .value("REINHARD_EXTENDED", TonemapMethod::REINHARD_EXTENDED)
      .value("ACES", TonemapMethod::ACES);
  py::enum_<DenoiseFilterQuality>(m_data, "DenoiseFilterQuality")
      .value("DEFAULT", DenoiseFilterQuality::DEFAULT)
      .value("HIGH", DenoiseFilterQuality::HIGH)
      .value("BALANCED", DenoiseFilterQuality::BALANCED)
      .value("FAST", DenoiseFilterQuality::FAST);
  py::class_<StreamConfig>(m_data, "StreamConfig")
      .def(py::init<>())
      .def_readwrite("apply_denoising", &StreamConfig::apply_denoising)
      .def_readwrite("denoise_clean_auxiliaries", &StreamConfig::denoise_clean_auxiliaries)
      .def_readwrite("denoise_quality", &StreamConfig::denoise_quality)
      .def_readwrite("denoise_input_scale", &StreamConfig::denoise_input_scale)
      .def_readwrite("linear_to_gamma", &StreamConfig::linear_to_gamma)
      .def_readwrite("apply_white_balance", &StreamConfig::apply_white_balance)
      .def_readwrite("wb_temperature", &StreamConfig::wb_temperature)
      .def_readwrite("wb_tint", &StreamConfig::wb_tint)
      .def_readwrite("apply_tonemapping", &StreamConfig::apply_tonemapping)
      .def_readwrite("tm_method", &StreamConfig::tm_method)
      .def_readwrite("tm_white_point", &StreamConfig::tm_white_point)
      .def_readwrite("tm_alpha", &StreamConfig::tm_alpha);
  py::enum_<LayerType>(m_data, "LayerType")
      .value("BEAUTY", LayerType::BEAUTY)
      .value("DIFFUSE", LayerType::DIFFUSE)
      .value("WORLD_NORMAL", LayerType::WORLD_NORMAL)
      .value("OBJECT_NORMAL", LayerType::OBJECT_NORMAL)
      .value("SPECULAR", LayerType::SPECULAR)
      .value("SHADOW", LayerType::SHADOW)
      .value("DEPTH", LayerType::DEPTH)
      .value("EMISSION", LayerType::EMISSION)
      .value("OBJECT_ID", LayerType::OBJECT_ID);
  py::class_<RenderLayersConfig>(m_data, "RenderLayersConfig")
      .def(py::init<>())
      .def_readwrite("beauty", &RenderLayersConfig::beauty)
      .def_readwrite("diffuse", &RenderLayersConfig::diffuse)
      .def_readwrite("world_normal", &RenderLayersConfig::world_normal)
      .def_readwrite("object_normal", &RenderLayersConfig::object_normal)
      .def_readwrite("specular", &RenderLayersConfig::specular)
      .def_readwrite("shadow", &RenderLayersConfig::shadow)
      .def_readwrite("depth", &RenderLayersConfig::depth)
      .def_readwrite("emission", &RenderLayersConfig::emission)
      .def_readwrite("object_id", &RenderLayersConfig::object_id);
  py::class_<DataObject>(m_data, "DataObject")
      .def("n_pixels", &DataObject::n_pixels)
      .def("n_elements", &DataObject::n_elements)
      .def("n_bytes", &DataObject::n_bytes)
      .def("shape", &DataObject::shape)
      .def("numpy", &DataObject::numpy)
      .def("is_enabled", &DataObject::is_enabled)
      .def("device_ptr", &DataObject::device_ptr)
      .def_readonly("C", &DataObject::C)
      .def_readonly("H", &DataObject::H)
      .def_readonly("W", &DataObject::W);
  py::class_<RenderLayers>(m_data, "RenderLayers")
      .def("get_layer", &RenderLayers::get, py::return_value_policy::reference_internal)
      .def_readonly("beauty", &RenderLayers::beauty)
      .def_readonly("diffuse", &RenderLayers::diffuse)
      .def_readonly("world_normal", &RenderLayers::world_normal)
      .def_readonly("object_normal", &RenderLayers::object_normal)
      .def_readonly("specular", &RenderLayers::specular)
      .def_readonly("shadow", &RenderLayers::shadow)
      .def_readonly("depth", &RenderLayers::depth)
      .def_readonly("emission", &RenderLayers::emission)
      .def_readonly("object_id", &RenderLayers::object_id);
  py::class_<TransferStream>(m_data, "TransferStream")
      .def("readback", [](TransferStream& s) { return s.readback(); })
      .def("update_config", [](TransferStream& s, const StreamConfig& c) { s.cfg = c; })
      .def("get_config", [](TransferStream& s) { return s.cfg; })
      .def("buffer_ptr", &TransferStream::buffer_ptr)
      .def("get_state", [](TransferStream& s) { return s.state.load(); })
      .def("is_active", [](TransferStream& s) { return s.state == StreamState::ACTIVE; })
      .def("is_inactive", [](TransferStream& s) { return s.state == StreamState::INACTIVE; })
      .def("is_linked", [](TransferStream& s) { return s.eng && s.eng->render; })
      .def("shape", &TransferStream::shape)
      .def("n_pixels", [](TransferStream& s) { return (size_t)s.eng->H() * s.eng->W(); })
      .def("n_elements", [](TransferStream& s) { return (size_t)3 * s.eng->H() * s.eng->W(); })
      .def("n_bytes", [](TransferStream& s) { return (size_t)3 * s.eng->H() * s.eng->W(); })
      .def("freeze", [](TransferStream& s) { if (s.state == StreamState::ACTIVE) s.state = StreamState::FROZEN; })
      .def("unfreeze", [](TransferStream& s) { if (s.state == StreamState::FROZEN) s.state = StreamState::ACTIVE; })
      .def("enable_denoising", [](TransferStream& s) { s.cfg.apply_denoising = true; })
      .def("disable_denoising", [](TransferStream& s) { s.cfg.apply_denoising = false; })
      .def("has_overlay", [](TransferStream&) { return false; })
      .def("remove_overlay", [](TransferStream&) {});

  // ---- engine
  auto m_engine = m.def_submodule("engine", "Engine module.");
  auto m_camera = m_engine.def_submodule("camera", "Camera submodule.");
  py::class_<CameraParams>(m_camera, "CameraParams")
      .def(py::init([](Vector2 res, Vector3 pos, Vector3 rot, uint32_t spp, float fl, float fd, float ap,
                       float sw, float ss) {
             CameraParams p;
             p.resolution = res; p.position = pos; p.rotation = rot; p.samples_per_pixel = spp;
             p.focal_length = fl; p.focus_distance = fd; p.aperture = ap; p.sensor_width = sw;
             p.shutter_speed = ss;
             return p;
           }),
           py::arg("resolution"), py::arg("position"), py::arg("rotation"), py::arg("samples_per_pixel"),
           py::arg("focal_length"), py::arg("focus_distance"), py::arg("aperture"),
           py::arg("sensor_width"), py::arg("shutter_speed"))
      .def_readwrite("resolution", &CameraParams::resolution)
      .def_readwrite("position", &CameraParams::position)
      .def_readwrite("rotation", &CameraParams::rotation)
      .def_readwrite("samples_per_pixel", &CameraParams::samples_per_pixel)
      .def_readwrite("focal_length", &CameraParams::focal_length)
      .def_readwrite("focus_distance", &CameraParams::focus_distance)
      .def_readwrite("aperture", &CameraParams::aperture)
      .def_readwrite("sensor_width", &CameraParams::sensor_width)
      .def_readwrite("shutter_speed", &CameraParams::shutter_speed);
  py::class_<Camera>(m_camera, "Camera")
      .def(py::init([](CameraParams p) { Camera c; c.p = p; return c; }), py::arg("params"))
      .def_readwrite("on_updated", &Camera::on_updated)
      .def("parameters", [](const Camera& c) { return c.p; });
  py::enum_<EngineState>(m_engine, "EngineState")
      .value("IDLE", EngineState::IDLE)
      .value("RENDERING", EngineState::RENDERING);
  py::enum_<EngineType>(m_engine, "EngineType")
      .value("PATHTRACER", EngineType::PATHTRACER)
      .value("VIEWPORT", EngineType::VIEWPORT);
  py::class_<EnginePollResponse>(m_engine, "EnginePollResponse")
      .def(py::init<>())
      .def_readwrite("should_update_camera", &EnginePollResponse::should_update_camera)
      .def_readwrite("camera_params", &EnginePollResponse::camera_params);
  py::class_<EngineRequests>(m_engine, "EngineRequests")
      .def("start", &EngineRequests::start)
      .def("stop", &EngineRequests::stop)
      .def("restart", &EngineRequests::restart)
      .def("shutdown", &EngineRequests::shutdown);

#define HOOK(name, type)                                                      \
  .def_property(#name, [](EngineCore& e) { return e.name; },                 \
                [](EngineCore& e, type f) { e.name = f; e.hooks_set = true; })
  py::class_<EngineCore>(m_engine, "RenderEngine")
      .def(py::init([](const Camera& c, uint32_t depth, uint32_t seed) {
             return std::make_unique<EngineCore>(c, depth, seed);
           }),
           py::arg("camera"), py::arg("ray_depth") = 8u, py::arg("seed") = 54321u)
      .def("set_scene",
           [](EngineCore& e, const Scene& sc) {
             {
               std::lock_guard<std::mutex> lk(e.scene_mu);
               e.objects.clear();
               for (Hittable* h : sc.objects) e.objects.push_back(*h);
               e.sky = sc.sky;
             }
             e.scene_dirty = false;
             {
               py::gil_scoped_release nogil;
               e.rebuild_scene();
             }
             // registry ids back onto the caller's objects (Hittable.get_object_id)
             for (size_t i = 0; i < sc.objects.size(); ++i) sc.objects[i]->object_id = (int)i;
             e.stream.state = StreamState::ACTIVE;
           })
      .def("render",
           [](EngineCore& e) {
             py::gil_scoped_release nogil;
             e.state = EngineState::RENDERING;
             int rc = e.run();
             e.state = EngineState::IDLE;
             return rc;
           })
      .def("idle",
           [](EngineCore& e) {
             py::gil_scoped_release nogil;
             while (!e.requests.shutdown_.load()) {
               if (e.requests.start_.exchange(false)) {
                 e.reset();
                 e.state = EngineState::RENDERING;
                 { py::gil_scoped_acquire gil; e.on_render_started(); }
                 int rs = e.type.load() == EngineType::VIEWPORT ? e.run_viewport() : e.run();
                 if (rs == 3) {  // WAITING: refresh the viewport again
                   e.requests.start();
                   std::this_thread::sleep_for(std::chrono::milliseconds(16));
                   continue;
                 }
                 e.state = EngineState::IDLE;
                 py::gil_scoped_acquire gil;
                 if (rs == 0) e.on_render_finished();
                 else if (rs == 1) e.on_stopped();
                 else { e.requests.start(); e.on_restarted(); }
                 continue;
               }
               std::this_thread::sleep_for(std::chrono::milliseconds(16));
             }
             py::gil_scoped_acquire gil;
             e.on_shutdown();
           })
      HOOK(on_render_started, std::function<void()>)
      HOOK(on_frame_finished, std::function<void(uint32_t)>)
      HOOK(on_render_finished, std::function<void()>)
      HOOK(on_stopped, std::function<void()>)
      HOOK(on_restarted, std::function<void()>)
      HOOK(on_reset, std::function<void()>)
      HOOK(on_shutdown, std::function<void()>)
      HOOK(poll_updates, std::function<EnginePollResponse()>)
      .def("camera", [](EngineCore& e) -> Camera& { return e.cam; }, py::return_value_policy::reference_internal)
      .def("layers", [](EngineCore& e) -> RenderLayers& { return e.layers; }, py::return_value_policy::reference_internal)
      .def("stream", [](EngineCore& e) -> TransferStream& { return e.stream; }, py::return_value_policy::reference_internal)
      .def("requests", [](EngineCore& e) -> EngineRequests& { return e.requests; }, py::return_value_policy::reference_internal)
      .def("get_state", [](EngineCore& e) { return e.state.load(); })
      .def("is_idle", [](EngineCore& e) { return e.state == EngineState::IDLE; })
      .def("is_rendering", [](EngineCore& e) { return e.state == EngineState::RENDERING; })
      .def("set_axis_grid_visible", [](EngineCore& e, bool v) { e.show_axis_grid = v; })
      .def("get_scene_interface", [](EngineCore& e) -> SceneInterface& { return e.scene_interface; },
           py::return_value_policy::reference_internal)
      .def("get_engine_type", [](EngineCore& e) { return e.type.load(); })
      .def("set_engine_type", [](EngineCore& e, EngineType t) { e.type = t; })
      .def("n_samples", [](EngineCore& e) { return e.cam.p.samples_per_pixel; })
      // RenderEngine::set_n_samples (engine.cpp:139-143) restarts at sample 1.
      // The sample pattern is rebuilt when n changes; the reference keeps the
      // pattern of the constructor's n and reads past it for larger n.
      .def("set_n_samples",
           [](EngineCore& e, uint32_t n) {
             if (e.render && n == e.cam.p.samples_per_pixel) {
               e.reset();
             } else {
               e.cam.p.samples_per_pixel = n;
               e.make_render();
             }
           })
      .def("max_depth", [](EngineCore& e) { return e.ray_depth; })
      .def("set_max_depth", [](EngineCore& e, uint32_t d) { e.ray_depth = d; e.make_render(); })
      .def("update_streaming_layer", [](EngineCore& e, LayerType t) { e.stream.layer = (int)t; })
      .def("set_integrator_mode", [](EngineCore& e, int mode) { e.mode = mode; e.make_render(); })
      .def("sample_index", [](EngineCore& e) { return e.sample_idx; })
      .def("last_render_ms", [](EngineCore& e) {
        double ms = 0;
        if (e.render) nr_render_last_ms(e.render, &ms);
        return ms;
      })
      .def("scene_stats", [](EngineCore& e) {
        nr_scene_stats st{};
        if (e.scene) check(nr_scene_get_stats(e.scene, &st), "scene_stats");
        py::dict d;
        d["n_objects"] = st.n_objects;
        d["n_materials"] = st.n_materials;
        d["n_lights"] = st.n_lights;
        d["n_triangles"] = st.n_triangles;
        d["binary_nodes"] = st.binary_nodes;
        d["wide_nodes"] = st.wide_nodes;
        d["sah_cost_binary"] = st.sah_cost_binary;
        d["build_ms"] = st.build_ms;
        d["device_bytes"] = st.device_bytes;
        return d;
      });
#undef HOOK
}
