// capi.cu — host side of the back end and its extern "C" entry points.
//
// Scene state mirrors the reference's registries (HittablesRegistry,
// MaterialRegisty, Skylight: nectar_render/csrc/hittable/include/hittable/
// registry.h:101-265, nectar_render/csrc/material/include/material/
// registry.h:8-103, nectar_render/csrc/light/include/skylight.h:138-254) but
// is uploaded as flat arrays (scene_device.cuh) and every BVH is built on the
// GPU (bvh_build.cu). Values the reference computes on the host (object
// transforms, camera parameters, the n-rooks sample pattern, the top-level
// leaf order that decides lights[0]) are computed here with the same host
// arithmetic; values it computes on the device (cube face transforms, the
// HDRI rotation, white-balance gains) are computed by device kernels.
#include <atomic>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/nectar_b200.h"
#include "bvh_build.cuh"
#include "host_io.h"
#include "mesh_ingest.cuh"
#include "sky_alias.cuh"
#include "image_ops.cuh"
#include "integrator.cuh"
#include "wavefront.cuh"
#include "viewport.cuh"
#include "conv_tc.cuh"
#include "denoiser.cuh"
#include "nrc.cuh"

using namespace nr;

// ---------------------------------------------------------------------------
// errors

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
static std::string hex_word(uint32_t w) {
  char b[16];
  snprintf(b, sizeof(b), "%x", w);
  return b;
}
static int cuda_fail(cudaError_t e, const char* what) {
  return fail(NR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CU(call, what)                                 \
  do {                                                 \
    cudaError_t e__ = (call);                          \
    if (e__ != cudaSuccess) return cuda_fail(e__, what); \
  } while (0)

// ---------------------------------------------------------------------------
// host math with the reference's expression order
// (core/matrix.h:64-96, core/utils.h:12-22, core/transform.h:125-134)

namespace {

struct HM3 {
  float m[3][3];
};
float h_deg2rad(float degrees) { return degrees * 0.01745329; }
HM3 h_rot_x(float a) {
  float c = cosf(a), s = sinf(a);
  return HM3{{{1, 0, 0}, {0, c, -s}, {0, s, c}}};
}
HM3 h_rot_y(float a) {
  float c = cosf(a), s = sinf(a);
  return HM3{{{c, 0, s}, {0, 1, 0}, {-s, 0, c}}};
}
HM3 h_rot_z(float a) {
  float c = cosf(a), s = sinf(a);
  return HM3{{{c, -s, 0}, {s, c, 0}, {0, 0, 1}}};
}
HM3 h_mul(const HM3& a, const HM3& b) {
  HM3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      r.m[i][j] = 0;
      for (int k = 0; k < 3; k++) r.m[i][j] += a.m[i][k] * b.m[k][j];
    }
  return r;
}
HM3 h_T(const HM3& a) {
  HM3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r.m[i][j] = a.m[j][i];
  return r;
}
HM3 h_euler_rad(float x, float y, float z) { return h_mul(h_mul(h_rot_z(z), h_rot_y(y)), h_rot_x(x)); }
HM3 h_euler_deg(const float r[3]) {
  return h_euler_rad(h_deg2rad(r[0]), h_deg2rad(r[1]), h_deg2rad(r[2]));
}

struct HXform {
  HM3 R, invR;
  float pos[3], scale[3], inv_s[3];
};
// Transform(position, rotation_deg, scale)
HXform h_xform(const float p[3], const float r[3], const float s[3]) {
  HXform x;
  x.R = h_euler_deg(r);
  x.invR = h_T(h_euler_deg(r));
  for (int k = 0; k < 3; ++k) {
    x.pos[k] = p[k];
    x.scale[k] = s[k];
    x.inv_s[k] = 1.0f / ((s[k] + 1e-8f) + 1e-8f);
  }
  return x;
}
// Transform(position): identity rotation from Euler zeros, unit scale
HXform h_xform_pos(const float p[3]) {
  HXform x;
  x.R = h_euler_rad(0.0f, 0.0f, 0.0f);
  x.invR = h_T(h_euler_rad(0.0f, 0.0f, 0.0f));
  for (int k = 0; k < 3; ++k) {
    x.pos[k] = p[k];
    x.scale[k] = 1.0f;
    x.inv_s[k] = 1.0f;
  }
  return x;
}

// AABB of the reference (hittable/include/bvh/aabb.h): intervals per axis.
struct HBox {
  float lo[3], hi[3];
};
// AABB::transformed(...).buffer() (aabb.h:60-91)
HBox h_transformed(const HBox& b, const HXform& x) {
  float c[8][3] = {{b.lo[0], b.lo[1], b.lo[2]}, {b.hi[0], b.lo[1], b.lo[2]},
                   {b.lo[0], b.hi[1], b.lo[2]}, {b.hi[0], b.hi[1], b.lo[2]},
                   {b.lo[0], b.lo[1], b.hi[2]}, {b.hi[0], b.lo[1], b.hi[2]},
                   {b.lo[0], b.hi[1], b.hi[2]}, {b.hi[0], b.hi[1], b.hi[2]}};
  float mn[3] = {1e32f, 1e32f, 1e32f}, mx[3] = {-1e32f, -1e32f, -1e32f};
  for (int i = 0; i < 8; ++i) {
    float s[3] = {c[i][0] * x.scale[0], c[i][1] * x.scale[1], c[i][2] * x.scale[2]};
    float w[3];
    for (int r = 0; r < 3; ++r)
      w[r] = x.R.m[r][0] * s[0] + x.R.m[r][1] * s[1] + x.R.m[r][2] * s[2] + x.pos[r];
    for (int k = 0; k < 3; ++k) {
      mn[k] = fminf(mn[k], w[k]);
      mx[k] = fmaxf(mx[k], w[k]);
    }
  }
  HBox o;
  for (int k = 0; k < 3; ++k) {
    float lo = mn[k] <= mx[k] ? mn[k] : mx[k];
    float hi = mn[k] <= mx[k] ? mx[k] : mn[k];
    if (hi - lo < 1e-4f) {
      float pad = 1e-4f / 2.0f;
      lo = lo - pad;
      hi = hi + pad;
    }
    o.lo[k] = lo;
    o.hi[k] = hi;
  }
  return o;
}

// Leaf order of the reference's top-level BVH<T>::build
// (hittable/include/bvh/bvh.h:35-320): 16 centroid bins, cost A_L*N_L +
// A_R*N_R, std::partition by bin, std::sort median split as fallback. Only
// the order is needed here: the reference's lights[0] is the first light in
// that order (registry.h:216-263).
struct RefOrder {
  const std::vector<HBox>& boxes;
  std::vector<int32_t> order;
  static constexpr int kB = 16;
  explicit RefOrder(const std::vector<HBox>& b) : boxes(b) {
    order.resize(b.size());
    std::iota(order.begin(), order.end(), 0);
    if (!order.empty()) rec(0, (int32_t)order.size());
  }
  static float area(const HBox& b) {
    float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
  }
  static HBox join(const HBox& a, const HBox& b) {
    HBox r;
    for (int k = 0; k < 3; ++k) {
      r.lo[k] = a.lo[k] <= b.lo[k] ? a.lo[k] : b.lo[k];
      r.hi[k] = a.hi[k] >= b.hi[k] ? a.hi[k] : b.hi[k];
    }
    return r;
  }
  void rec(int32_t start, int32_t end) {
    if (end - start == 1) return;
    float cmin[3] = {1e32f, 1e32f, 1e32f}, cmax[3] = {-1e32f, -1e32f, -1e32f};
    for (int32_t i = start; i < end; ++i) {
      const HBox& b = boxes[order[i]];
      for (int k = 0; k < 3; ++k) {
        float c = (b.lo[k] + b.hi[k]) * 0.5f;
        cmin[k] = fminf(cmin[k], c);
        cmax[k] = fmaxf(cmax[k], c);
      }
    }
    float best_cost = 1e32f;
    int32_t best_axis = -1, best_bin = -1;
    for (int a = 0; a < 3; ++a) {
      float extent = cmax[a] - cmin[a];
      if (extent < 1e-4f) continue;
      int32_t cnt[kB] = {0};
      HBox bb[kB];
      for (int32_t i = start; i < end; ++i) {
        const HBox& b = boxes[order[i]];
        float c = (b.lo[a] + b.hi[a]) * 0.5f;
        int32_t bin = (int32_t)(kB * (c - cmin[a]) / extent);
        bin = bin < 0 ? 0 : (bin >= kB ? kB - 1 : bin);
        cnt[bin]++;
        bb[bin] = cnt[bin] == 1 ? b : join(bb[bin], b);
      }
      HBox lb[kB], rb[kB];
      int32_t lc[kB], rc[kB];
      HBox run{};
      int32_t rcount = 0;
      bool started = false;
      for (int i = 0; i < kB; ++i) {
        if (cnt[i] > 0) {
          run = started ? join(run, bb[i]) : bb[i];
          started = true;
        }
        rcount += cnt[i];
        lb[i] = run;
        lc[i] = rcount;
      }
      rcount = 0;
      started = false;
      for (int i = kB - 1; i >= 0; --i) {
        if (cnt[i] > 0) {
          run = started ? join(run, bb[i]) : bb[i];
          started = true;
        }
        rcount += cnt[i];
        rb[i] = run;
        rc[i] = rcount;
      }
      for (int i = 0; i < kB - 1; ++i) {
        if (lc[i] == 0 || rc[i + 1] == 0) continue;
        float cost = area(lb[i]) * lc[i] + area(rb[i + 1]) * rc[i + 1];
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_bin = i;
        }
      }
    }
    if (best_axis == -1) {
      HBox comb = boxes[order[start]];
      for (int32_t i = start + 1; i < end; ++i) comb = join(comb, boxes[order[i]]);
      float lx = comb.hi[0] - comb.lo[0], ly = comb.hi[1] - comb.lo[1], lz = comb.hi[2] - comb.lo[2];
      best_axis = (lx > ly && lx > lz) ? 0 : (ly > lz ? 1 : 2);
    }
    if (best_bin == -1) {
      int a = best_axis;
      std::sort(order.begin() + start, order.begin() + end,
                [&](int32_t x, int32_t y) { return boxes[x].lo[a] < boxes[y].lo[a]; });
      int32_t mid = start + (end - start) / 2;
      rec(start, mid);
      rec(mid, end);
      return;
    }
    int a = best_axis;
    float c_min = cmin[a], extent = cmax[a] - c_min;
    auto it = std::partition(order.begin() + start, order.begin() + end, [&](int32_t i) {
      const HBox& b = boxes[i];
      float c = (b.lo[a] + b.hi[a]) * 0.5f;
      int32_t bin = (int32_t)(kB * (c - c_min) / extent);
      bin = bin < 0 ? 0 : (bin >= kB ? kB - 1 : bin);
      return bin <= best_bin;
    });
    int32_t mid = (int32_t)(it - order.begin());
    rec(start, mid);
    rec(mid, end);
  }
};

template <typename T>
cudaError_t upload(T*& d, const T* h, size_t n, cudaStream_t st) {
  cudaError_t e = cudaMalloc(&d, sizeof(T) * (n ? n : 1));
  if (e != cudaSuccess) return e;
  if (n) e = cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, st);
  return e;
}

struct MeshGpu {
  float* pos = nullptr;       // 3 per vertex
  float* nor = nullptr;
  float* tan = nullptr;
  float* uv = nullptr;
  uint32_t* vidx = nullptr;   // 3 per triangle
  TriRecord* tris2 = nullptr;
  TriRecord* tris8 = nullptr;
  BuildResult bvh;
  void release() {
    cudaFree(pos);
    cudaFree(nor);
    cudaFree(tan);
    cudaFree(uv);
    cudaFree(vidx);
    cudaFree(tris2);
    cudaFree(tris8);
    free_build(bvh);
    *this = MeshGpu{};
  }
};

// triangle boxes for the builder
__global__ void k_tri_boxes(const float* pos, const uint32_t* vidx, uint32_t n, float4* lo,
                            float4* hi) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float v[3][3];
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) v[k][c] = pos[3 * vidx[3 * t + k] + c];
  float mn[3], mx[3];
  for (int c = 0; c < 3; ++c) {
    mn[c] = fminf(v[0][c], fminf(v[1][c], v[2][c]));
    mx[c] = fmaxf(v[0][c], fmaxf(v[1][c], v[2][c]));
  }
  lo[t] = make_float4(mn[0], mn[1], mn[2], 0.f);
  hi[t] = make_float4(mx[0], mx[1], mx[2], 0.f);
}

// triangle records in a leaf order; .e1.w flags a zero-extent box (any axis)
__global__ void k_tri_records(const float* pos, const uint32_t* vidx, const uint32_t* order,
                              uint32_t n, TriRecord* out) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t t = order[s];
  float v[3][3];
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) v[k][c] = pos[3 * vidx[3 * t + k] + c];
  bool flat = false;
  for (int c = 0; c < 3; ++c) {
    float mn = fminf(v[0][c], fminf(v[1][c], v[2][c]));
    float mx = fmaxf(v[0][c], fmaxf(v[1][c], v[2][c]));
    if (mx == mn) flat = true;
  }
  TriRecord r;
  r.v0 = make_float4(v[0][0], v[0][1], v[0][2], __uint_as_float(t));
  r.e1 = make_float4(__fsub_rn(v[1][0], v[0][0]), __fsub_rn(v[1][1], v[0][1]),
                     __fsub_rn(v[1][2], v[0][2]), __uint_as_float(flat ? 1u : 0u));
  r.e2 = make_float4(__fsub_rn(v[2][0], v[0][0]), __fsub_rn(v[2][1], v[0][1]),
                     __fsub_rn(v[2][2], v[0][2]), 0.f);
  out[s] = r;
}

}  // namespace

// ---------------------------------------------------------------------------
// scene

struct HostImage8 {
  uint32_t C, H, W;
  std::vector<uint8_t> chw;
};

struct nr_scene {
  std::vector<nr_material_desc> materials;
  std::vector<HostImage8> images;
  std::vector<HostMesh> meshes;
  std::vector<nr_object_desc> objects;
  int32_t sky_type = NR_SKY_NULL;
  float sky_start[3] = {1.0f, 1.0f, 1.0f};
  float sky_end[3] = {0.5f, 0.7f, 1.0f};
  HostImageF hdri;
  float hdri_rotation = 0.0f;
  float hdri_intensity = 1.0f;

  // device state
  bool built = false;
  cudaStream_t stream = nullptr;
  std::vector<uint8_t*> d_images;
  std::vector<MeshGpu> d_meshes;
  DevMaterial* d_materials = nullptr;
  DevObject* d_objects = nullptr;
  DevMesh* d_mesh_table = nullptr;
  float* d_hdri = nullptr;
  SkyTables sky_tables;             // HDRI importance sampling (perf mode)
  CubeFace* d_cube_faces = nullptr;
  BuildResult tlas;
  DevScene dev{};
  nr_scene_stats stats{};
  std::vector<int32_t> ref_leaf_order;
  float world_lo[3] = {0.f, 0.f, 0.f}, world_hi[3] = {0.f, 0.f, 0.f};  // union of object boxes
  int32_t light = -1;
  uint32_t mesh_leaf_max = 1, tlas_leaf_max = 1;
  uint32_t mesh_width = 8, tlas_width = 8;

  void release_device() {
    for (auto p : d_images) cudaFree(p);
    d_images.clear();
    for (auto& m : d_meshes) m.release();
    d_meshes.clear();
    cudaFree(d_materials);
    cudaFree(d_objects);
    cudaFree(d_mesh_table);
    cudaFree(d_hdri);
    sky_tables.release();
    cudaFree(d_cube_faces);
    d_cube_faces = nullptr;
    d_materials = nullptr;
    d_objects = nullptr;
    d_mesh_table = nullptr;
    d_hdri = nullptr;
    free_build(tlas);
    built = false;
  }
  ~nr_scene() {
    release_device();
    if (stream) cudaStreamDestroy(stream);
  }
};

static nr_material_desc default_material() {
  // Material::lambertian(Color::purple()) (material.h:650-652)
  nr_material_desc m{};
  m.type = NR_MATERIAL_LAMBERTIAN;
  m.tex[0].type = NR_TEXTURE_CONSTANT;
  m.tex[0].rgb[0] = 1.0f;
  m.tex[0].rgb[1] = 0.0f;
  m.tex[0].rgb[2] = 1.0f;
  m.tex[0].scale = 1.0f;
  return m;
}

static bool device_available() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n > 0;
}

static int base_type(const nr_object_desc& o) {
  return (o.type == NR_HITTABLE_OBJECT_LIGHT || o.type == NR_HITTABLE_CONSTANT_MEDIUM)
             ? o.wrapped_type
             : o.type;
}

static HXform object_xform(const nr_object_desc& o) {
  return base_type(o) == NR_HITTABLE_SPHERE ? h_xform_pos(o.position)
                                            : h_xform(o.position, o.rotation, o.scale);
}

static HBox object_local_box(const nr_scene* s, const nr_object_desc& o) {
  HBox b;
  int t = base_type(o);
  if (t == NR_HITTABLE_SPHERE) {
    float r = o.radius + 1e-8f;
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = -r;
      b.hi[k] = r;
    }
  } else if (t == NR_HITTABLE_MESH) {
    const HostMesh& m = s->meshes[o.mesh];
    float mn[3] = {1e32f, 1e32f, 1e32f}, mx[3] = {-1e32f, -1e32f, -1e32f};
    for (size_t i = 0; i < m.positions.size() / 3; ++i)
      for (int k = 0; k < 3; ++k) {
        mn[k] = fminf(mn[k], m.positions[3 * i + k]);
        mx[k] = fmaxf(mx[k], m.positions[3 * i + k]);
      }
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = mn[k];
      b.hi[k] = mx[k];
    }
  } else {
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = -0.5f;
      b.hi[k] = 0.5f;
    }
  }
  return b;
}

static DevTexture make_tex(const nr_scene* s, const nr_texture_desc& t) {
  DevTexture d{};
  d.type = t.type;
  d.r = t.rgb[0];
  d.g = t.rgb[1];
  d.b = t.rgb[2];
  d.scale = t.scale;
  if (t.type == NR_TEXTURE_IMAGE && t.image >= 0 && (size_t)t.image < s->images.size()) {
    d.data = s->d_images[t.image];
    d.C = s->images[t.image].C;
    d.H = s->images[t.image].H;
    d.W = s->images[t.image].W;
  }
  return d;
}

extern "C" {

int nr_abi_version(void) { return NR_ABI_VERSION; }
const char* nr_last_error(void) { return g_last_error.c_str(); }
int nr_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int nr_device_memory_info(uint64_t* used, uint64_t* free_bytes, uint64_t* total) {
  if (!used || !free_bytes || !total) return fail(NR_ERR_INVALID, "nr_device_memory_info: null output");
  if (!device_available()) return fail(NR_ERR_NO_DEVICE, "no CUDA device is available");
  size_t f = 0, t = 0;
  CU(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
  *used = t - f;
  *free_bytes = f;
  *total = t;
  return NR_OK;
}

int nr_scene_create(nr_scene** out) {
  if (!out) return fail(NR_ERR_INVALID, "nr_scene_create: null output");
  nr_scene* s = new nr_scene();
  s->materials.push_back(default_material());
  *out = s;
  return NR_OK;
}

int nr_scene_destroy(nr_scene* scene) {
  delete scene;
  return NR_OK;
}

int nr_scene_add_material(nr_scene* s, const nr_material_desc* d, uint32_t* out_id) {
  if (!s || !d) return fail(NR_ERR_INVALID, "nr_scene_add_material: null argument");
  if (d->type < NR_MATERIAL_NULL || d->type > NR_MATERIAL_ISOTROPIC)
    return fail(NR_ERR_INVALID, "nr_scene_add_material: unknown material type");
  if (s->materials.size() >= NR_MAX_MATERIALS)
    return fail(NR_ERR_LIMIT,
                "Maximum material count reached. Unable to register additional materials.");
  for (int k = 0; k < 5; ++k)
    if (d->tex[k].type == NR_TEXTURE_IMAGE &&
        (d->tex[k].image < 0 || (size_t)d->tex[k].image >= s->images.size()))
      return fail(NR_ERR_INVALID, "nr_scene_add_material: texture references an unknown image");
  s->materials.push_back(*d);
  if (out_id) *out_id = (uint32_t)(s->materials.size() - 1);
  s->built = false;
  return NR_OK;
}

int nr_scene_add_image(nr_scene* s, const uint8_t* chw, uint32_t C, uint32_t H, uint32_t W,
                       uint32_t* out_id) {
  if (!s || !chw || C < 3 || H == 0 || W == 0)
    return fail(NR_ERR_INVALID, "nr_scene_add_image: need a CHW image with at least 3 channels");
  HostImage8 im{C, H, W, std::vector<uint8_t>(chw, chw + (size_t)C * H * W)};
  s->images.push_back(std::move(im));
  if (out_id) *out_id = (uint32_t)(s->images.size() - 1);
  s->built = false;
  return NR_OK;
}

// Vertex positions and transforms must be finite: the reference renders
// NaN geometry as undefined results, and the GPU builder's Morton codes and
// SAH bins are only defined for finite boxes, so such input is refused on
// the host before anything reaches the device.
static bool all_finite(const float* v, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return false;
  return true;
}

int nr_scene_add_mesh(nr_scene* s, const float* positions, const float* normals,
                      const float* tangents, const float* uvs, uint32_t n_vertices,
                      const uint32_t* triangles, uint32_t n_triangles, uint32_t* out_id) {
  if (!s || !positions || !triangles || n_vertices == 0 || n_triangles == 0)
    return fail(NR_ERR_INVALID, "nr_scene_add_mesh: empty mesh");
  if (n_triangles >= (1u << 22))
    return fail(NR_ERR_LIMIT, "nr_scene_add_mesh: at most 4194303 triangles per mesh");
  for (size_t i = 0; i < (size_t)n_triangles * 3; ++i)
    if (triangles[i] >= n_vertices)
      return fail(NR_ERR_INVALID, "nr_scene_add_mesh: triangle index out of range");
  if (!all_finite(positions, 3 * (size_t)n_vertices))
    return fail(NR_ERR_INVALID, "nr_scene_add_mesh: non-finite vertex position");
  HostMesh m;
  m.positions.assign(positions, positions + 3 * (size_t)n_vertices);
  m.normals = normals ? std::vector<float>(normals, normals + 3 * (size_t)n_vertices)
                      : std::vector<float>(3 * (size_t)n_vertices, 0.0f);
  m.tangents = tangents ? std::vector<float>(tangents, tangents + 3 * (size_t)n_vertices)
                        : std::vector<float>(3 * (size_t)n_vertices, 0.0f);
  m.uvs = uvs ? std::vector<float>(uvs, uvs + 2 * (size_t)n_vertices)
              : std::vector<float>(2 * (size_t)n_vertices, 0.0f);
  m.triangles.assign(triangles, triangles + 3 * (size_t)n_triangles);
  s->meshes.push_back(std::move(m));
  if (out_id) *out_id = (uint32_t)(s->meshes.size() - 1);
  s->built = false;
  return NR_OK;
}

int nr_scene_load_obj(nr_scene* s, const char* path, uint32_t* out_id) {
  if (!s || !path) return fail(NR_ERR_INVALID, "nr_scene_load_obj: null argument");
  HostMesh m;
  std::string err;
  if (!load_obj(path, m, err)) return fail(NR_ERR_IO, err);
  if (m.triangles.empty()) return fail(NR_ERR_INVALID, std::string("OBJ has no faces: ") + path);
  if (m.triangles.size() / 3 >= (1u << 22))
    return fail(NR_ERR_LIMIT, "nr_scene_load_obj: at most 4194303 triangles per mesh");
  if (!all_finite(m.positions.data(), m.positions.size()))
    return fail(NR_ERR_INVALID, std::string("OBJ has a non-finite vertex position: ") + path);
  s->meshes.push_back(std::move(m));
  if (out_id) *out_id = (uint32_t)(s->meshes.size() - 1);
  s->built = false;
  return NR_OK;
}

int nr_scene_load_obj_device(nr_scene* s, const char* path, uint32_t* out_id) {
  if (!s || !path) return fail(NR_ERR_INVALID, "nr_scene_load_obj_device: null argument");
  ObjRaw raw;
  std::string err;
  if (!parse_obj(path, raw, err)) return fail(NR_ERR_IO, err);
  if (raw.corners.empty()) return fail(NR_ERR_INVALID, std::string("OBJ has no faces: ") + path);
  if (raw.corners.size() / 9 >= (1u << 22))
    return fail(NR_ERR_LIMIT, "nr_scene_load_obj_device: at most 4194303 triangles per mesh");
  if (!all_finite(raw.vpos.data(), raw.vpos.size()))
    return fail(NR_ERR_INVALID, std::string("OBJ has a non-finite vertex position: ") + path);
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    return fail(NR_ERR_NO_DEVICE, "nr_scene_load_obj_device: no CUDA device");
  HostMesh m;
  err = assemble_obj_device(raw, m, nullptr);
  if (!err.empty())
    return fail(err.find("key bits") != std::string::npos ? NR_ERR_LIMIT : NR_ERR_CUDA, err);
  s->meshes.push_back(std::move(m));
  if (out_id) *out_id = (uint32_t)(s->meshes.size() - 1);
  s->built = false;
  return NR_OK;
}

int nr_scene_get_mesh(const nr_scene* s, uint32_t id, float* P, float* N, float* T, float* UV,
                      uint32_t* tris, uint32_t* nv, uint32_t* nt) {
  if (!s || !nv || !nt) return fail(NR_ERR_INVALID, "nr_scene_get_mesh: null argument");
  if (id >= s->meshes.size()) return fail(NR_ERR_INVALID, "nr_scene_get_mesh: unknown mesh id");
  const HostMesh& m = s->meshes[id];
  *nv = (uint32_t)(m.positions.size() / 3);
  *nt = (uint32_t)(m.triangles.size() / 3);
  if (P) std::copy(m.positions.begin(), m.positions.end(), P);
  if (N) std::copy(m.normals.begin(), m.normals.end(), N);
  if (T) std::copy(m.tangents.begin(), m.tangents.end(), T);
  if (UV) std::copy(m.uvs.begin(), m.uvs.end(), UV);
  if (tris) std::copy(m.triangles.begin(), m.triangles.end(), tris);
  return NR_OK;
}

int nr_scene_add_object(nr_scene* s, const nr_object_desc* d, uint32_t* out_id) {
  if (!s || !d) return fail(NR_ERR_INVALID, "nr_scene_add_object: null argument");
  if (s->objects.size() >= NR_MAX_OBJECTS)
    return fail(NR_ERR_LIMIT, "Hittables registry exceeded maximum registry entries [1024].");
  int bt = base_type(*d);
  if (d->type < NR_HITTABLE_QUAD || d->type > NR_HITTABLE_OBJECT_LIGHT)
    return fail(NR_ERR_INVALID, "nr_scene_add_object: unknown hittable type");
  if (bt < NR_HITTABLE_QUAD || bt > NR_HITTABLE_MESH)
    return fail(NR_ERR_INVALID, "nr_scene_add_object: a wrapper must bind a quad, sphere, cube or mesh");
  if (bt == NR_HITTABLE_MESH && (d->mesh < 0 || (size_t)d->mesh >= s->meshes.size()))
    return fail(NR_ERR_INVALID, "nr_scene_add_object: unknown mesh id");
  if (d->material < 0 || (size_t)d->material >= s->materials.size())
    return fail(NR_ERR_INVALID, "nr_scene_add_object: unknown material id");
  if (!all_finite(d->position, 3) || !all_finite(d->rotation, 3) || !all_finite(d->scale, 3) ||
      !std::isfinite(d->radius) || !std::isfinite(d->density))
    return fail(NR_ERR_INVALID, "nr_scene_add_object: non-finite transform, radius or density");
  s->objects.push_back(*d);
  if (out_id) *out_id = (uint32_t)(s->objects.size() - 1);
  s->built = false;
  return NR_OK;
}

int nr_scene_set_sky_null(nr_scene* s) {
  if (!s) return fail(NR_ERR_INVALID, "null scene");
  s->sky_type = NR_SKY_NULL;
  s->built = false;
  return NR_OK;
}

int nr_scene_set_sky_simple(nr_scene* s, const float a[3], const float b[3]) {
  if (!s || !a || !b) return fail(NR_ERR_INVALID, "null argument");
  s->sky_type = NR_SKY_SIMPLE;
  for (int k = 0; k < 3; ++k) {
    s->sky_start[k] = a[k];
    s->sky_end[k] = b[k];
  }
  s->built = false;
  return NR_OK;
}

int nr_scene_set_sky_hdri(nr_scene* s, const float* chw, uint32_t C, uint32_t H, uint32_t W,
                          float rotation, float intensity) {
  if (!s) return fail(NR_ERR_INVALID, "null scene");
  s->sky_type = NR_SKY_HDRI;
  s->hdri = HostImageF{};
  if (chw) {
    if (C < 3 || H == 0 || W == 0)
      return fail(NR_ERR_INVALID, "nr_scene_set_sky_hdri: need at least 3 channels");
    s->hdri.C = C;
    s->hdri.H = H;
    s->hdri.W = W;
    s->hdri.chw.assign(chw, chw + (size_t)C * H * W);
  }
  s->hdri_rotation = rotation;
  s->hdri_intensity = intensity;
  s->built = false;
  return NR_OK;
}

int nr_scene_load_hdr(nr_scene* s, const char* path, float rotation, float intensity) {
  if (!s || !path) return fail(NR_ERR_INVALID, "null argument");
  HostImageF im;
  std::string err;
  if (!load_hdr(path, im, err)) return fail(NR_ERR_IO, err);
  s->sky_type = NR_SKY_HDRI;
  s->hdri = std::move(im);
  s->hdri_rotation = rotation;
  s->hdri_intensity = intensity;
  s->built = false;
  return NR_OK;
}

int nr_scene_set_hdri_params(nr_scene* s, float rotation, float intensity) {
  if (!s) return fail(NR_ERR_INVALID, "null scene");
  s->hdri_rotation = rotation;
  s->hdri_intensity = intensity;
  s->built = false;
  return NR_OK;
}

int nr_scene_set_bvh_width(nr_scene* s, uint32_t mesh_width, uint32_t tlas_width) {
  // narrower trees are deeper: below 4 children their depth could outgrow
  // the traversal kernels' fixed stacks
  if (!s || mesh_width < 4 || mesh_width > 8 || tlas_width < 4 || tlas_width > 8)
    return fail(NR_ERR_INVALID, "nr_scene_set_bvh_width: widths must be 4..8");
  s->mesh_width = mesh_width;
  s->tlas_width = tlas_width;
  s->built = false;
  return NR_OK;
}

int nr_scene_set_tuning(nr_scene* s, uint32_t mesh_leaf_max, uint32_t tlas_leaf_max) {
  if (!s || mesh_leaf_max < 1 || mesh_leaf_max > 3 || tlas_leaf_max < 1 || tlas_leaf_max > 3)
    return fail(NR_ERR_INVALID, "nr_scene_set_tuning: leaf sizes must be 1..3");
  s->mesh_leaf_max = mesh_leaf_max;
  s->tlas_leaf_max = tlas_leaf_max;
  s->built = false;
  return NR_OK;
}

int nr_scene_build(nr_scene* s) {
  if (!s) return fail(NR_ERR_INVALID, "null scene");
  if (s->objects.empty()) return fail(NR_ERR_INVALID, "Hittables list cannot be empty.");
  if (!device_available()) return fail(NR_ERR_NO_DEVICE, "no CUDA device is available");
  s->release_device();
  if (!s->stream) CU(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
  cudaStream_t st = s->stream;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0), "event");
  CU(cudaEventCreate(&e1), "event");
  CU(cudaEventRecord(e0, st), "event");

  // device-built constants: cube faces and the HDRI rotation
  M3 hdri_rot;
  CU(cudaMalloc(&s->d_cube_faces, sizeof(CubeFace) * 6), "alloc cube faces");
  CU(launch_init_constants(s->hdri_rotation, s->d_cube_faces, &hdri_rot, st), "init constants");

  // images and materials
  for (auto& im : s->images) {
    uint8_t* d = nullptr;
    CU(upload(d, im.chw.data(), im.chw.size(), st), "upload image");
    s->d_images.push_back(d);
  }
  std::vector<DevMaterial> mats(s->materials.size());
  for (size_t i = 0; i < s->materials.size(); ++i) {
    const nr_material_desc& m = s->materials[i];
    DevMaterial& d = mats[i];
    d.type = m.type;
    d.ior = m.ior;
    d.brightness = m.brightness;
    for (int k = 0; k < 3; ++k) d.tint[k] = m.tint[k];
    for (int k = 0; k < 5; ++k) d.tex[k] = make_tex(s, m.tex[k]);
  }
  CU(upload(s->d_materials, mats.data(), mats.size(), st), "upload materials");

  // meshes: GPU BVH per mesh
  uint64_t n_tris_total = 0, bin_nodes = 0, wide_nodes = 0, dev_bytes = 0;
  double largest_sah = 0.0;
  uint32_t largest_n = 0;
  std::vector<DevMesh> table(s->meshes.size());
  s->d_meshes.resize(s->meshes.size());
  for (size_t mi = 0; mi < s->meshes.size(); ++mi) {
    const HostMesh& hm = s->meshes[mi];
    MeshGpu& g = s->d_meshes[mi];
    uint32_t nv = (uint32_t)(hm.positions.size() / 3), nt = (uint32_t)(hm.triangles.size() / 3);
    CU(upload(g.pos, hm.positions.data(), hm.positions.size(), st), "upload mesh");
    CU(upload(g.nor, hm.normals.data(), hm.normals.size(), st), "upload mesh");
    CU(upload(g.tan, hm.tangents.data(), hm.tangents.size(), st), "upload mesh");
    CU(upload(g.uv, hm.uvs.data(), hm.uvs.size(), st), "upload mesh");
    CU(upload(g.vidx, hm.triangles.data(), hm.triangles.size(), st), "upload mesh");
    float4 *lo = nullptr, *hi = nullptr;
    CU(cudaMalloc(&lo, sizeof(float4) * nt), "alloc boxes");
    CU(cudaMalloc(&hi, sizeof(float4) * nt), "alloc boxes");
    k_tri_boxes<<<(nt + 255) / 256, 256, 0, st>>>(g.pos, g.vidx, nt, lo, hi);
    int be = build_bvh(lo, hi, nt, true, g.bvh, st, s->mesh_leaf_max, s->mesh_width);
    cudaFree(lo);
    cudaFree(hi);
    if (be != 0) return cuda_fail((cudaError_t)be, "mesh BVH build");
    CU(cudaMalloc(&g.tris2, sizeof(TriRecord) * nt), "alloc tris");
    CU(cudaMalloc(&g.tris8, sizeof(TriRecord) * nt), "alloc tris");
    k_tri_records<<<(nt + 255) / 256, 256, 0, st>>>(g.pos, g.vidx, g.bvh.d_order, nt, g.tris2);
    k_tri_records<<<(nt + 255) / 256, 256, 0, st>>>(g.pos, g.vidx, g.bvh.d_order8, nt, g.tris8);
    CU(cudaGetLastError(), "triangle records");
    DevMesh& d = table[mi];
    d.tris2 = g.tris2;
    d.tris8 = g.tris8;
    d.bvh2 = g.bvh.d_bvh2;
    d.bvh8 = g.bvh.d_bvh8;
    d.tri_vidx = g.vidx;
    d.vnormal = g.nor;
    d.vtangent = g.tan;
    d.vuv = g.uv;
    d.n_tris = nt;
    d.n_bvh2 = g.bvh.n_bvh2;
    d.n_bvh8 = g.bvh.n_bvh8;
    n_tris_total += nt;
    bin_nodes += g.bvh.n_nodes;
    wide_nodes += g.bvh.n_bvh8;
    dev_bytes += (uint64_t)nt * (2 * sizeof(TriRecord) + 12) + (uint64_t)nv * 44 +
                 (uint64_t)g.bvh.n_bvh2 * sizeof(Bvh2Node) + (uint64_t)g.bvh.n_bvh8 * sizeof(Bvh8Node);
    if (nt >= largest_n) {
      largest_n = nt;
      largest_sah = g.bvh.sah_cost;
    }
  }
  CU(upload(s->d_mesh_table, table.data(), table.size(), st), "upload mesh table");

  // objects (registry order) and their world boxes
  std::vector<DevObject> objs(s->objects.size());
  std::vector<HBox> boxes(s->objects.size());
  std::vector<float4> blo(s->objects.size()), bhi(s->objects.size());
  for (size_t i = 0; i < s->objects.size(); ++i) {
    const nr_object_desc& o = s->objects[i];
    HXform x = object_xform(o);
    DevObject& d = objs[i];
    memset(&d, 0, sizeof(d));
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        d.R.m[r][c] = x.R.m[r][c];
        d.invR.m[r][c] = x.invR.m[r][c];
      }
    d.pos = V3{x.pos[0], x.pos[1], x.pos[2]};
    d.scale = V3{x.scale[0], x.scale[1], x.scale[2]};
    d.inv_s = V3{x.inv_s[0], x.inv_s[1], x.inv_s[2]};
    d.type = o.type;
    d.wrapped_type = o.wrapped_type;
    d.material = (uint32_t)o.material;
    d.mesh = (uint32_t)std::max(0, o.mesh);
    d.radius = o.radius + 1e-8f;
    d.neg_inv_density = -1.0f / (o.density + 1e-8f);
    d.object_id = (uint32_t)i;
    boxes[i] = h_transformed(object_local_box(s, o), x);
    blo[i] = make_float4(boxes[i].lo[0], boxes[i].lo[1], boxes[i].lo[2], 0.f);
    bhi[i] = make_float4(boxes[i].hi[0], boxes[i].hi[1], boxes[i].hi[2], 0.f);
    for (int k = 0; k < 3; ++k) {
      s->world_lo[k] = i ? std::min(s->world_lo[k], boxes[i].lo[k]) : boxes[i].lo[k];
      s->world_hi[k] = i ? std::max(s->world_hi[k], boxes[i].hi[k]) : boxes[i].hi[k];
    }
  }
  CU(upload(s->d_objects, objs.data(), objs.size(), st), "upload objects");
  float4 *dlo = nullptr, *dhi = nullptr;
  CU(upload(dlo, blo.data(), blo.size(), st), "upload boxes");
  CU(upload(dhi, bhi.data(), bhi.size(), st), "upload boxes");
  int be = build_bvh(dlo, dhi, (uint32_t)objs.size(), true, s->tlas, st, s->tlas_leaf_max,
                     s->tlas_width);
  cudaFree(dlo);
  cudaFree(dhi);
  if (be != 0) return cuda_fail((cudaError_t)be, "top-level BVH build");

  // lights[0]: first OBJECT_LIGHT in the reference's top-level leaf order
  RefOrder ro(boxes);
  s->ref_leaf_order = ro.order;
  s->light = -1;
  uint32_t n_lights = 0;
  for (int32_t idx : ro.order)
    if (s->objects[idx].type == NR_HITTABLE_OBJECT_LIGHT) {
      if (s->light < 0) s->light = idx;
      n_lights++;
    }

  // sky
  DevSky sky{};
  sky.type = s->sky_type;
  for (int k = 0; k < 3; ++k) {
    sky.start[k] = s->sky_start[k];
    sky.end[k] = s->sky_end[k];
  }
  sky.rotation = s->hdri_rotation;
  sky.intensity = s->hdri_intensity;
  sky.rot = hdri_rot;
  if (s->sky_type == NR_SKY_HDRI && !s->hdri.chw.empty()) {
    CU(upload(s->d_hdri, s->hdri.chw.data(), s->hdri.chw.size(), st), "upload hdri");
    sky.data = s->d_hdri;
    sky.C = (int)s->hdri.C;
    sky.H = (int)s->hdri.H;
    sky.W = (int)s->hdri.W;
    dev_bytes += s->hdri.chw.size() * 4;
    bool has_energy = false;
    CU(build_sky_tables(s->d_hdri, sky.W, sky.H, s->sky_tables, has_energy, st),
       "build sky sampling tables");
    if (has_energy) {
      sky.row_prob = s->sky_tables.row_prob;
      sky.row_alias = s->sky_tables.row_alias;
      sky.col_prob = s->sky_tables.col_prob;
      sky.col_alias = s->sky_tables.col_alias;
      sky.texel_pdf = s->sky_tables.texel_pdf;
      dev_bytes += (size_t)sky.W * sky.H * 12 + (size_t)sky.H * 8;
    }
  }

  DevScene& ds = s->dev;
  ds = DevScene{};
  ds.max_steps = kMaxTraversalSteps;  // renders set their own bounds (make_params)
  ds.stack_limit = 0xffffffffu;
  ds.objects = s->d_objects;
  ds.n_objects = (uint32_t)objs.size();
  ds.materials = s->d_materials;
  ds.n_materials = (uint32_t)mats.size();
  ds.meshes = s->d_mesh_table;
  ds.n_meshes = (uint32_t)table.size();
  ds.tlas2 = s->tlas.d_bvh2;
  ds.tlas8 = s->tlas.d_bvh8;
  ds.tlas_prims = s->tlas.d_order;
  ds.tlas_prims8 = s->tlas.d_order8;
  ds.n_tlas2 = s->tlas.n_bvh2;
  ds.n_tlas8 = s->tlas.n_bvh8;
  ds.light = s->light;
  ds.use_bvh8 = 1;
  ds.cube_faces = s->d_cube_faces;
  ds.sky = sky;

  CU(cudaEventRecord(e1, st), "event");
  CU(cudaEventSynchronize(e1), "build");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);

  nr_scene_stats& S = s->stats;
  S.n_objects = (uint32_t)objs.size();
  S.n_materials = (uint32_t)mats.size();
  S.n_lights = n_lights;
  S.n_triangles = n_tris_total;
  S.binary_nodes = bin_nodes + s->tlas.n_nodes;
  S.wide_nodes = wide_nodes + s->tlas.n_bvh8;
  S.sah_cost_binary = largest_sah;
  S.build_ms = ms;
  S.device_bytes = dev_bytes;
  s->built = true;
  return NR_OK;
}

int nr_scene_get_sky_tables(const nr_scene* s, float* texel_pdf, float* row_prob,
                            uint32_t* row_alias, float* col_prob, uint32_t* col_alias,
                            int32_t* W, int32_t* H) {
  if (!s) return fail(NR_ERR_INVALID, "nr_scene_get_sky_tables: null scene");
  if (!s->built) return fail(NR_ERR_STATE, "nr_scene_get_sky_tables: scene not built");
  const SkyTables& t = s->sky_tables;
  if (W) *W = t.W;
  if (H) *H = t.H;
  if (!t.texel_pdf) return NR_OK;
  const size_t hw = (size_t)t.W * t.H;
  auto rd = [&](void* dst, const void* src, size_t bytes) {
    return dst ? cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) : cudaSuccess;
  };
  CU(rd(texel_pdf, t.texel_pdf, hw * 4), "read sky tables");
  CU(rd(row_prob, t.row_prob, (size_t)t.H * 4), "read sky tables");
  CU(rd(row_alias, t.row_alias, (size_t)t.H * 4), "read sky tables");
  CU(rd(col_prob, t.col_prob, hw * 4), "read sky tables");
  CU(rd(col_alias, t.col_alias, hw * 4), "read sky tables");
  return NR_OK;
}

int nr_scene_get_bounds(const nr_scene* s, float lo[3], float hi[3]) {
  if (!s || !lo || !hi) return fail(NR_ERR_INVALID, "nr_scene_get_bounds: null argument");
  if (!s->built) return fail(NR_ERR_STATE, "nr_scene_get_bounds: scene not built");
  for (int k = 0; k < 3; ++k) {
    lo[k] = s->world_lo[k];
    hi[k] = s->world_hi[k];
  }
  return NR_OK;
}

int nr_scene_get_stats(const nr_scene* s, nr_scene_stats* out) {
  if (!s || !out) return fail(NR_ERR_INVALID, "null argument");
  if (!s->built) return fail(NR_ERR_STATE, "scene is not built");
  *out = s->stats;
  return NR_OK;
}

int nr_scene_get_binary_bvh(const nr_scene* s, uint32_t mesh_id, float* nodes8, uint64_t* n_nodes,
                            uint32_t* prim_order) {
  if (!s || !n_nodes) return fail(NR_ERR_INVALID, "null argument");
  if (!s->built) return fail(NR_ERR_STATE, "scene is not built");
  if (mesh_id >= s->d_meshes.size()) return fail(NR_ERR_INVALID, "unknown mesh id");
  const BuildResult& b = s->d_meshes[mesh_id].bvh;
  *n_nodes = b.n_nodes;
  if (nodes8) {
    std::vector<BinNode> h(b.n_nodes);
    CU(cudaMemcpy(h.data(), b.d_nodes, sizeof(BinNode) * b.n_nodes, cudaMemcpyDeviceToHost),
       "read nodes");
    for (size_t i = 0; i < h.size(); ++i) {
      float* o = nodes8 + 8 * i;
      for (int k = 0; k < 3; ++k) {
        o[k] = h[i].lo[k];
        o[3 + k] = h[i].hi[k];
      }
      int32_t a = h[i].left >= 0 ? h[i].left : (int32_t)h[i].start;
      int32_t c = h[i].left >= 0 ? h[i].right : -(int32_t)h[i].count;
      memcpy(o + 6, &a, 4);
      memcpy(o + 7, &c, 4);
    }
  }
  if (prim_order) {
    uint32_t nt = s->d_meshes[mesh_id].bvh.n_nodes ? (uint32_t)(s->meshes[mesh_id].triangles.size() / 3) : 0;
    CU(cudaMemcpy(prim_order, b.d_order, sizeof(uint32_t) * nt, cudaMemcpyDeviceToHost), "read order");
  }
  return NR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// render

struct nr_render {
  nr_scene* scene = nullptr;
  nr_camera_desc cam{};
  nr_render_config cfg{};
  uint32_t W = 0, H = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float* layer[9] = {nullptr};
  uint32_t layer_c[9] = {0};
  double* beauty64 = nullptr;
  uint64_t n64 = 0;  // samples in the FP64 sum since the last reset
  float* raw[3] = {nullptr, nullptr, nullptr};
  float* trace_log = nullptr;  // set only during nr_render_trace_log
  uint32_t log_bounces = 0;
  uint32_t* raw_primary = nullptr;
  uint32_t* work = nullptr;
  uint32_t* err = nullptr;
  unsigned long long* counters = nullptr;
  V2* pattern = nullptr;
  uint8_t* disp8 = nullptr;
  float* dispf = nullptr;
  V3* wb_scratch = nullptr;
  DevCamera dcam{};
  WfParams wf{};
  uint32_t samples_per_wave = 0;
  int rtl = 0;
  bool counters_on = false;
  bool profile_on = false;
  std::vector<cudaEvent_t> pev;  // profiling: one event per launch boundary
  std::vector<uint8_t> pkind;
  nr_kernel_profile prof{};
  // captured waves: the wave's launches with everything but its first sample
  // index baked in (that one is read from device memory)
  struct WaveGraph {
    WfParams key;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<WaveGraph> graphs;
  // radiance cache attached with nr_render_set_nrc (perf mode)
  nr_nrc* nrc = nullptr;
  uint32_t nrc_bounce = 2, nrc_one_in = 32, nrc_batch = 16384, nrc_min_steps = 4;
  float nrc_lr = 0.0f;
  float4 *nrc_q = nullptr, *nrc_q_beta = nullptr, *nrc_t = nullptr, *nrc_t_beta = nullptr,
         *nrc_t_before = nullptr, *nrc_t_perm = nullptr;
  float *nrc_radiance = nullptr, *nrc_target = nullptr;
  uint32_t nrc_cap = 0;
  uint64_t nrc_queries = 0, nrc_records = 0;  // totals since attached
  std::string nrc_error;                       // set by the wave hook
  // fused display of the beauty layer (nr_render_set_fused_display)
  bool fused_on = false, fused_valid = false;
  nr_stream_config fused_cfg{};
  DisplayParams fused_p{};
  PickOut* d_pick = nullptr;        // viewport queries (allocated on first use)
  uint8_t* d_mask = nullptr;        // 2 x W*H selection masks
  uint32_t graphs_captured = 0;
  uint64_t graph_replays = 0;
  nr_trace_counters last{};
  double last_ms = 0.0;
  ~nr_render() {
    if (wf.capacity) wf_free(wf);
    for (auto p : layer) cudaFree(p);
    cudaFree(beauty64);
    for (auto p : raw) cudaFree(p);
    cudaFree(raw_primary);
    cudaFree(work);
    cudaFree(err);
    cudaFree(counters);
    cudaFree(pattern);
    cudaFree(disp8);
    cudaFree(dispf);
    cudaFree(wb_scratch);
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto e : pev) cudaEventDestroy(e);
    cudaFree(d_pick);
    cudaFree(d_mask);
    for (void* q : {(void*)nrc_q, (void*)nrc_q_beta, (void*)nrc_t, (void*)nrc_t_beta,
                    (void*)nrc_t_before, (void*)nrc_t_perm, (void*)nrc_radiance,
                    (void*)nrc_target})
      cudaFree(q);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

// Order of the draws taken by multi-draw constructor arguments: the
// reference's CUDA build evaluates them left to right (probed on sm_100a).
static int g_device_rtl = 0;

extern "C" {

int nr_device_draw_order(void) { return g_device_rtl; }
int nr_set_draw_order(int rtl) {
  g_device_rtl = rtl ? 1 : 0;
  return NR_OK;
}

int nr_render_config_default(nr_render_config* c) {
  if (!c) return fail(NR_ERR_INVALID, "null config");
  memset(c, 0, sizeof(*c));
  c->ray_depth = 8;
  c->seed = 54321;
  c->rr_enabled = 1;
  c->rr_start_bounce = 3;
  c->rr_survival = 0.95f;
  c->mode = NR_MODE_REFERENCE;
  c->schedule = NR_SCHEDULE_WAVEFRONT;
  c->fp64_accumulate = 0;
  c->layer_mask = (1u << NR_LAYER_BEAUTY) | (1u << NR_LAYER_DIFFUSE) | (1u << NR_LAYER_WORLD_NORMAL);
  c->extend_variant = 0;
  c->samples_per_wave = 0;
  c->use_graphs = 1;
  return NR_OK;
}

// n-rooks pattern of SampleGenerator::generate_n_rooks (camera.h:45-61). The
// two jitter draws of each Vector2(...) are evaluated right to left by the
// reference's host compiler, so the y jitter is drawn first.
static std::vector<V2> n_rooks(uint32_t n, uint32_t seed) {
  std::vector<uint32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937 rng(seed);
  std::shuffle(perm.begin(), perm.end(), rng);
  std::uniform_real_distribution<float> jitter(0.0f, 1.0f);
  std::vector<V2> out(n);
  for (uint32_t i = 0; i < n; ++i) {
    float jy = jitter(rng);
    float jx = jitter(rng);
    out[i] = V2{(i + jx) / (float)n, (perm[i] + jy) / (float)n};
  }
  return out;
}

int nr_render_create(nr_scene* s, const nr_camera_desc* c, const nr_render_config* cfg,
                     nr_render** out) {
  if (!s || !c || !cfg || !out) return fail(NR_ERR_INVALID, "nr_render_create: null argument");
  if (!s->built) return fail(NR_ERR_STATE, "nr_render_create: scene is not built");
  if (c->samples_per_pixel == 0) return fail(NR_ERR_INVALID, "samples_per_pixel must be > 0");
  if (c->resolution[0] < 1.0f || c->resolution[1] < 1.0f)
    return fail(NR_ERR_INVALID, "resolution must be at least 1x1");
  std::unique_ptr<nr_render> r(new nr_render());
  r->scene = s;
  r->cam = *c;
  r->cfg = *cfg;
  r->H = (uint32_t)c->resolution[0];
  r->W = (uint32_t)c->resolution[1];
  if ((uint64_t)r->W * r->H * (uint64_t)c->samples_per_pixel > 0xffffffffull)
    return fail(NR_ERR_LIMIT, "pixel count x samples exceeds the 32-bit sample stream");
  r->rtl = g_device_rtl;
  CU(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking), "stream");
  CU(cudaEventCreate(&r->ev0), "event");
  CU(cudaEventCreate(&r->ev1), "event");
  size_t hw = (size_t)r->W * r->H;
  static const uint32_t kC[9] = {3, 3, 3, 3, 3, 1, 1, 3, 3};
  for (int l = 0; l < 9; ++l) {
    if (!(cfg->layer_mask & (1u << l))) continue;
    r->layer_c[l] = kC[l];
    CU(cudaMalloc(&r->layer[l], sizeof(float) * kC[l] * hw), "alloc layer");
    CU(cudaMemsetAsync(r->layer[l], 0, sizeof(float) * kC[l] * hw, r->stream), "clear layer");
  }
  if (cfg->fp64_accumulate) {
    CU(cudaMalloc(&r->beauty64, sizeof(double) * 3 * hw), "alloc fp64");
    CU(cudaMemsetAsync(r->beauty64, 0, sizeof(double) * 3 * hw, r->stream), "clear fp64");
  }
  CU(cudaMalloc(&r->work, 4), "alloc");
  CU(cudaMalloc(&r->err, 4), "alloc");
  CU(cudaMemsetAsync(r->err, 0, 4, r->stream), "clear");
  CU(cudaMalloc(&r->counters, 8 * 5), "alloc");
  CU(cudaMalloc(&r->wb_scratch, sizeof(V3)), "alloc");
  std::vector<V2> pat = n_rooks(c->samples_per_pixel, cfg->seed);
  CU(upload(r->pattern, pat.data(), pat.size(), r->stream), "upload pattern");
  // CameraParams::build (camera.h:124-136)
  HM3 R = h_euler_deg(c->rotation);
  DevCamera& d = r->dcam;
  d.res_x = c->resolution[0];
  d.res_y = c->resolution[1];
  d.position = V3{c->position[0], c->position[1], c->position[2]};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) d.R.m[i][j] = R.m[i][j];
  d.shutter_time = 1.0f / (c->shutter_speed + 1e-8f);
  float aperture_radius = c->aperture / 2.0f;
  d.defocus_angle = 2.0f * atanf(aperture_radius / (c->focus_distance + 1e-8f));
  d.defocus_radius = c->focus_distance * tanf(d.defocus_angle / 2.0f);
  float aspect = c->resolution[1] / c->resolution[0];
  d.uvw_x = c->sensor_width;
  d.uvw_y = -c->sensor_width * aspect;
  d.focal_length = c->focal_length;
  d.focus_distance = c->focus_distance;
  d.W = r->W;
  d.H = r->H;
  d.pattern = r->pattern;
  CU(cudaStreamSynchronize(r->stream), "render create");
  *out = r.release();
  return NR_OK;
}

int nr_render_destroy(nr_render* r) {
  if (r) cudaStreamSynchronize(r->stream);
  delete r;
  return NR_OK;
}

int nr_render_reset(nr_render* r) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  r->fused_valid = false;
  size_t hw = (size_t)r->W * r->H;
  for (int l = 0; l < 9; ++l)
    if (r->layer[l]) CU(cudaMemsetAsync(r->layer[l], 0, sizeof(float) * r->layer_c[l] * hw, r->stream), "clear");
  if (r->beauty64) CU(cudaMemsetAsync(r->beauty64, 0, sizeof(double) * 3 * hw, r->stream), "clear");
  r->n64 = 0;
  CU(cudaStreamSynchronize(r->stream), "reset");
  return NR_OK;
}

static KernelParams make_params(nr_render* r, uint32_t first, uint32_t count, bool raw) {
  KernelParams P;
  memset(&P, 0, sizeof(P));
  P.scene = r->scene->dev;
  P.scene.use_bvh8 = 1;
  P.scene.max_steps = r->cfg.max_traversal_steps ? r->cfg.max_traversal_steps : kMaxTraversalSteps;
  P.scene.stack_limit = r->cfg.traversal_stack_limit ? r->cfg.traversal_stack_limit : 0xffffffffu;
  P.cam = r->dcam;
  P.W = r->W;
  P.H = r->H;
  P.first_sample = first;
  P.n_samples = count;
  P.seed = r->cfg.seed;
  P.depth = r->cfg.ray_depth;
  P.rr_enabled = r->cfg.rr_enabled;
  P.rr_start = r->cfg.rr_start_bounce;
  P.rr_survival = r->cfg.rr_survival;
  P.mode = r->cfg.mode;
  P.rtl = r->rtl;
  P.write_raw = raw ? 1 : 0;
  if (raw) {
    P.beauty = r->raw[0];
    P.diffuse = r->raw[1];
    P.normal = r->raw[2];
    P.primary = r->raw_primary;
  } else {
    P.beauty = r->layer[NR_LAYER_BEAUTY];
    P.diffuse = r->layer[NR_LAYER_DIFFUSE];
    P.normal = r->layer[NR_LAYER_WORLD_NORMAL];
    P.depth_layer = r->cfg.schedule == NR_SCHEDULE_WAVEFRONT ? r->layer[NR_LAYER_DEPTH] : nullptr;
    P.beauty64 = r->beauty64;
  }
  P.work_counter = r->work;
  P.err = r->err;
  P.counters = r->counters;
  return P;
}

// Waves of the wavefront schedule hold up to ~8M paths (about 1 GB of state).
// Traversal kernels: the nested two-level traversal (5 CTAs per SM) for the
// coherent camera rays of bounce 0, the flattened traversal with lane refill
// (4 CTAs per SM) for the later bounces, each iteration running primitive
// tests when at least half as many lanes have one next as have other work
// (vote 2); on the 1.31 M-triangle mesh scene at 1920x1080 the traversal
// takes 7.76 ms per 4-spp step against 8.32 without the vote (same hits).
constexpr int32_t kDefaultExtendVariant = 574;
// Queue length below which the last bounces of a wave run as one per-path
// launch (wavefront.cu, k_wf_tail).
constexpr uint32_t kDefaultTailPaths = 131072;
// Shading kernel register budget for 6 CTAs of 128 threads per SM: spills a
// little, but the occupancy gain hides more memory latency (9% less time per
// sample than 128 registers on the 1.31 M-triangle scene).
constexpr int32_t kDefaultShadeVariant = 6;

static uint32_t waves_of(nr_render* r) {
  if (r->cfg.samples_per_wave > 0) return std::min(16u, r->cfg.samples_per_wave);
  uint32_t N = r->W * r->H;
  uint32_t s = std::max(1u, std::min(8u, (8u << 20) / std::max(1u, N)));
  return s;
}

// Launches one wave through a CUDA graph. A wave configuration (all launch
// parameters except the first sample index) is launched directly the first
// time it is seen, captured the second time and replayed from then on.
static cudaError_t launch_wave_graph(nr_render* r, const WfParams& W) {
  WfParams key;
  memcpy(&key, &W, sizeof(key));
  key.base = 0;
  key.kp.first_sample = 0;
  key.kp.n_samples = 0;
  for (auto& g : r->graphs) {
    if (memcmp(&g.key, &key, sizeof(key)) != 0) continue;
    if (g.exec) {
      r->graph_replays++;
      return cudaGraphLaunch(g.exec, r->stream);
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t el = wf_launch_wave(W, false, r->stream, nullptr);
    e = cudaStreamEndCapture(r->stream, &graph);
    if (el != cudaSuccess || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return el != cudaSuccess ? el : e;
    }
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      g.exec = nullptr;
      return e;
    }
    r->graphs_captured++;
    r->graph_replays++;
    return cudaGraphLaunch(g.exec, r->stream);
  }
  if (r->graphs.size() >= 8) {
    if (r->graphs.front().exec) cudaGraphExecDestroy(r->graphs.front().exec);
    r->graphs.erase(r->graphs.begin());
  }
  nr_render::WaveGraph g;
  memset(&g.key, 0, sizeof(g.key));
  g.key = key;
  r->graphs.push_back(g);
  return wf_launch_wave(W, false, r->stream, nullptr);
}

struct nr_nrc {
  Nrc n;
};

constexpr uint32_t kNrcMaxGroups = 4096;  // Adam steps per wave at most

// After the bounces of a wave: the cache answers the queries of the paths
// that stopped at the cache bounce, then trains on the training paths.
static cudaError_t nrc_hook(void* ctx, const WfParams& W, cudaStream_t st) {
  nr_render* r = static_cast<nr_render*>(ctx);
  uint32_t n_q = 0, n_t = 0;
  cudaError_t e = wf_nrc_counts(W, &n_q, &n_t, st);  // synchronises the stream
  if (e != cudaSuccess) return e;
  Nrc& cache = r->nrc->n;
  std::string msg = nrc_poll_error(cache, st);  // waits of the previous wave's cache launches
  const uint32_t chunk = std::max(1u, nrc_max_queries(cache));
  for (uint32_t o = 0; o < n_q && msg.empty(); o += chunk) {
    const uint32_t c = std::min(chunk, n_q - o);
    WfParams Wo = W;
    Wo.nrc_q_beta = W.nrc_q_beta + o;
    msg = nrc_infer(cache, reinterpret_cast<const NrcQuery*>(W.nrc_q + 4 * (size_t)o), c,
                    r->nrc_radiance, st);
    if (msg.empty() && (e = wf_nrc_apply(Wo, r->nrc_radiance, c, st)) != cudaSuccess) return e;
  }
  r->nrc_queries += n_q;
  if (msg.empty() && n_t && r->nrc_lr > 0.0f) {
    // one Adam step per batch; batch g holds records g, g + groups, ...
    const uint32_t batch = std::min(r->nrc_batch, chunk);
    const uint32_t groups =
        std::min(std::max((n_t + batch - 1) / batch, std::min(r->nrc_min_steps, n_t)),
                 kNrcMaxGroups);
    const uint32_t per = (n_t + groups - 1) / groups;
    if ((e = wf_nrc_targets(W, r->nrc_target, r->nrc_t_perm, n_t, groups, st)) != cudaSuccess)
      return e;
    for (uint32_t g = 0; g < groups && msg.empty(); ++g) {
      const uint32_t c = std::min(n_t / groups + (g < n_t % groups ? 1u : 0u), chunk);
      msg = nrc_train(cache, reinterpret_cast<const NrcQuery*>(r->nrc_t_perm + 4 * (size_t)g * per),
                      r->nrc_target + 3 * (size_t)g * per, c, r->nrc_lr, nullptr, st);
      r->nrc_records += c;
    }
  }
  if (!msg.empty()) {
    r->nrc_error = msg;
    return cudaErrorUnknown;
  }
  return cudaSuccess;
}

static int launch(nr_render* r, const KernelParams& P, WaveTimer* tm) {
  // NR_MODE_PERF runs on the wavefront schedule only
  if (r->cfg.schedule != NR_SCHEDULE_WAVEFRONT && r->cfg.mode != NR_MODE_PERF) {
    CU(cudaMemsetAsync(r->work, 0, 4, r->stream), "clear work counter");
    CU(launch_megakernel(P, r->counters_on, r->stream), "launch integrator");
    if (tm) tm->mark(NR_KERNEL_MEGAKERNEL, r->stream);
    return NR_OK;
  }
  uint32_t N = r->W * r->H;
  if (!r->wf.capacity) {
    r->samples_per_wave = waves_of(r);
    CU(wf_alloc(r->wf, r->samples_per_wave * N, r->cfg.mode == NR_MODE_PERF,
                r->cfg.sort_materials >= 0),
       "allocate wavefront state");
  }
  uint32_t per = P.write_raw ? 1u : r->samples_per_wave;
  WfParams W = r->wf;
  W.kp = P;
  W.extend_variant = r->cfg.extend_variant > 0 ? r->cfg.extend_variant : kDefaultExtendVariant;
  W.shade_variant = r->cfg.shade_variant > 0 ? r->cfg.shade_variant : kDefaultShadeVariant;
  W.tail_max_paths = r->cfg.tail_max_paths == 0 ? kDefaultTailPaths
                     : (r->cfg.tail_max_paths == UINT32_MAX ? 0u : r->cfg.tail_max_paths);
  if (r->trace_log) {
    // per-bounce log: every bounce in k_wf_shade, so no hand-off to the tail
    W.trace_log = r->trace_log;
    W.log_bounces = r->log_bounces;
    W.tail_max_paths = 0;
  }
  const bool fused = r->fused_on && r->disp8 && !P.write_raw && P.beauty;
  if (fused) {
    W.disp8 = r->disp8;
    W.disp_p = r->fused_p;
  }
  WaveHook hook;
  const bool nrc = r->nrc && r->cfg.mode == NR_MODE_PERF && !P.write_raw;
  if (nrc) {
    const uint32_t cap = r->wf.capacity;
    if (r->nrc_cap < cap) {
      for (void* q : {(void*)r->nrc_q, (void*)r->nrc_q_beta, (void*)r->nrc_t, (void*)r->nrc_t_beta,
                      (void*)r->nrc_t_before, (void*)r->nrc_t_perm, (void*)r->nrc_radiance,
                      (void*)r->nrc_target})
        cudaFree(q);
      CU(cudaMalloc(&r->nrc_q, sizeof(float4) * 4 * (size_t)cap), "alloc cache queries");
      CU(cudaMalloc(&r->nrc_q_beta, sizeof(float4) * (size_t)cap), "alloc cache queries");
      CU(cudaMalloc(&r->nrc_t, sizeof(float4) * 4 * (size_t)cap), "alloc cache records");
      CU(cudaMalloc(&r->nrc_t_beta, sizeof(float4) * (size_t)cap), "alloc cache records");
      CU(cudaMalloc(&r->nrc_t_before, sizeof(float4) * (size_t)cap), "alloc cache records");
      // regrouped records: n + groups - 1 slots at most
      const size_t slots = (size_t)cap + kNrcMaxGroups;
      CU(cudaMalloc(&r->nrc_t_perm, sizeof(float4) * 4 * slots), "alloc cache records");
      CU(cudaMalloc(&r->nrc_radiance, sizeof(float) * 3 * (size_t)cap), "alloc cache output");
      CU(cudaMalloc(&r->nrc_target, sizeof(float) * 3 * slots), "alloc cache targets");
      r->nrc_cap = cap;
    }
    W.nrc_bounce = r->nrc_bounce;
    W.nrc_train_one_in = r->nrc_one_in;
    W.nrc_q_cap = W.nrc_t_cap = r->nrc_cap;
    W.nrc_q = r->nrc_q;
    W.nrc_q_beta = r->nrc_q_beta;
    W.nrc_t = r->nrc_t;
    W.nrc_t_beta = r->nrc_t_beta;
    W.nrc_t_before = r->nrc_t_before;
    hook.fn = nrc_hook;
    hook.ctx = r;
  }
  CU(wf_set_base(W, P.first_sample, r->stream), "set wave base");
  if (tm) tm->mark(NR_KERNEL_ROTATE, r->stream);
  for (uint32_t s = 0; s < P.n_samples; s += per) {
    W.base = P.first_sample + s;
    W.count = std::min(per, P.n_samples - s);
    if (!r->counters_on && !tm && r->cfg.use_graphs && !nrc && !r->trace_log)
      CU(launch_wave_graph(r, W), "launch wavefront graph");
    else {
      cudaError_t e = wf_launch_wave(W, r->counters_on, r->stream, tm, nrc ? &hook : nullptr);
      if (!r->nrc_error.empty()) {
        const std::string m = r->nrc_error;
        r->nrc_error.clear();
        return fail(m.find("timed out") != std::string::npos ? NR_ERR_DEVICE : NR_ERR_CUDA, m);
      }
      CU(e, "launch wavefront");
    }
  }
  if (nrc) {
    const std::string m = nrc_poll_error(r->nrc->n, r->stream);  // the last wave's cache launches
    if (!m.empty()) return fail(NR_ERR_DEVICE, m);
  }
  r->fused_valid = fused;
  return NR_OK;
}

// Enqueues a render call on the render's stream (events around it).
static int enqueue_kernel(nr_render* r, const KernelParams& P, WaveTimer& tm) {
  r->fused_valid = false;  // set again when the wavefront's accumulate writes the display
  if (r->counters_on) CU(cudaMemsetAsync(r->counters, 0, 8 * 5, r->stream), "clear counters");
  CU(cudaEventRecord(r->ev0, r->stream), "event");
  if (r->profile_on) {
    CU(cudaEventRecord(r->pev[0], r->stream), "event");
    tm.ev = r->pev.data() + 1;
    tm.kind = r->pkind.data() + 1;
    tm.cap = (int)r->pev.size() - 1;
  }
  int rc = launch(r, P, r->profile_on ? &tm : nullptr);
  if (rc != NR_OK) return rc;
  CU(cudaEventRecord(r->ev1, r->stream), "event");
  return NR_OK;
}

// Waits for an enqueued call and reads its timing, error word and counters.
static int finish_kernel(nr_render* r, const KernelParams& P, const WaveTimer& tm) {
  CU(cudaEventSynchronize(r->ev1), "integrator");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, r->ev0, r->ev1);
  r->last_ms = ms;
  if (r->profile_on) {
    r->prof = nr_kernel_profile{};
    for (int i = 0; i < tm.n; ++i) {
      float d = 0.f;
      cudaEventElapsedTime(&d, i ? tm.ev[i - 1] : r->pev[0], tm.ev[i]);
      r->prof.ms[tm.kind[i]] += d;
      r->prof.launches[tm.kind[i]] += 1;
    }
  }
  uint32_t herr = 0;
  CU(cudaMemcpy(&herr, r->err, 4, cudaMemcpyDeviceToHost), "read error word");
  if (herr) {
    cudaMemset(r->err, 0, 4);
    return fail(NR_ERR_DEVICE, "integrator error word 0x" + hex_word(herr) +
                                   " (1: traversal stack overflow, 8: traversal step bound)");
  }
  if (r->counters_on) {
    unsigned long long c[5];
    CU(cudaMemcpy(c, r->counters, sizeof(c), cudaMemcpyDeviceToHost), "read counters");
    r->last.rays = c[0];
    r->last.node_visits = c[1];
    r->last.tri_tests = c[2];
    r->last.obj_tests = c[3];
    r->last.paths = r->cfg.schedule == NR_SCHEDULE_WAVEFRONT
                        ? (unsigned long long)P.n_samples * r->W * r->H
                        : c[4];
  }
  return NR_OK;
}

static int run_kernel(nr_render* r, const KernelParams& P) {
  WaveTimer tm;
  int rc = enqueue_kernel(r, P, tm);
  if (rc != NR_OK) return rc;
  return finish_kernel(r, P, tm);
}

int nr_render_samples(nr_render* r, uint32_t first, uint32_t count) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (count == 0) return NR_OK;
  if (first == 0) return fail(NR_ERR_INVALID, "sample indices start at 1");
  if ((uint64_t)first + count > r->cam.samples_per_pixel)
    return fail(NR_ERR_INVALID, "sample index beyond samples_per_pixel");
  KernelParams P = make_params(r, first, count, false);
  int rc = run_kernel(r, P);
  if (rc == NR_OK) r->n64 += count;
  return rc;
}

int nr_render_samples_batch(nr_render* const* renders, uint32_t n, const uint32_t* first,
                            const uint32_t* count) {
  if (!renders || (n && (!first || !count))) return fail(NR_ERR_INVALID, "null argument");
  for (uint32_t i = 0; i < n; ++i) {
    nr_render* r = renders[i];
    if (!r) return fail(NR_ERR_INVALID, "null render in batch");
    if (first[i] == 0) return fail(NR_ERR_INVALID, "sample indices start at 1");
    if ((uint64_t)first[i] + count[i] > r->cam.samples_per_pixel)
      return fail(NR_ERR_INVALID, "sample index beyond samples_per_pixel");
    for (uint32_t j = 0; j < i; ++j)
      if (renders[j] == r) return fail(NR_ERR_INVALID, "a render appears twice in the batch");
  }
  std::vector<KernelParams> ps(n);
  std::vector<WaveTimer> tms(n);
  int rc = NR_OK;
  uint32_t queued = 0;
  for (; queued < n && rc == NR_OK; ++queued) {
    if (count[queued] == 0) continue;
    ps[queued] = make_params(renders[queued], first[queued], count[queued], false);
    rc = enqueue_kernel(renders[queued], ps[queued], tms[queued]);
  }
  // every enqueued call is waited for, also after a failure
  for (uint32_t i = 0; i < queued; ++i) {
    if (count[i] == 0) continue;
    int ri = finish_kernel(renders[i], ps[i], tms[i]);
    if (ri == NR_OK) renders[i]->n64 += count[i];
    else if (rc == NR_OK) rc = ri;
  }
  return rc;
}

// nr_render_samples_static: the wave state lives in static_wave.cu's
// file-scope device buffer, looked up once per device.
static std::atomic<uintptr_t> g_static_wave_addr[64];

int nr_render_samples_static(nr_render* r, uint32_t first, uint32_t count) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  // set-up on this device (also for count == 0): the buffer's address, whose
  // first lookup makes the driver load the module that holds the buffer
  int dev = 0;
  CU(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(NR_ERR_LIMIT, "device ordinal beyond 63");
  uintptr_t addr = g_static_wave_addr[dev].load(std::memory_order_acquire);
  if (!addr) {
    void* p = nullptr;
    CU(static_wave_address(&p), "cudaGetSymbolAddress(static wave buffer)");
    addr = (uintptr_t)p;
    g_static_wave_addr[dev].store(addr, std::memory_order_release);
  }
  if (first == 0) return fail(NR_ERR_INVALID, "sample indices start at 1");
  if ((uint64_t)first + count > r->cam.samples_per_pixel)
    return fail(NR_ERR_INVALID, "sample index beyond samples_per_pixel");
  const uint32_t N = r->W * r->H;
  if (r->cfg.mode != NR_MODE_REFERENCE)
    return fail(NR_ERR_STATE, "nr_render_samples_static renders NR_MODE_REFERENCE only");
  if ((uint64_t)r->W * r->H > NR_STATIC_WAVE_PATHS)
    return fail(NR_ERR_LIMIT, "nr_render_samples_static: " + std::to_string(r->W) + "x" +
                                  std::to_string(r->H) + " = " + std::to_string(N) +
                                  " pixels exceeds the static wave buffer's " +
                                  std::to_string(NR_STATIC_WAVE_PATHS) + " paths");
  if (count == 0) return NR_OK;
  r->fused_valid = false;  // this path leaves the fused display untouched
  WfParams W{};
  static_wave_carve((void*)addr, W);
  KernelParams P = make_params(r, first, count, false);
  uint32_t per = std::max(1u, std::min(waves_of(r), NR_STATIC_WAVE_PATHS / N));

  if (r->counters_on) CU(cudaMemsetAsync(r->counters, 0, 8 * 5, r->stream), "clear counters");
  CU(cudaEventRecord(r->ev0, r->stream), "event");
  CU(wf_set_base(W, first, r->stream), "set wave base");
  for (uint32_t s = 0; s < count; s += per) {
    WfParams w = W;
    w.kp = P;
    w.extend_variant = r->cfg.extend_variant > 0 ? r->cfg.extend_variant : kDefaultExtendVariant;
    w.shade_variant = r->cfg.shade_variant > 0 ? r->cfg.shade_variant : kDefaultShadeVariant;
    w.tail_max_paths = 0;  // the tail kernel's per-thread stack could make the driver grow its
                           // local-memory reservation, an allocation this entry point avoids
    w.base = first + s;
    w.count = std::min(per, count - s);
    CU(wf_launch_wave(w, r->counters_on, r->stream), "launch wavefront");
  }
  CU(cudaEventRecord(r->ev1, r->stream), "event");
  CU(cudaEventSynchronize(r->ev1), "integrator");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, r->ev0, r->ev1);
  r->last_ms = ms;
  uint32_t herr = 0;
  CU(cudaMemcpy(&herr, r->err, 4, cudaMemcpyDeviceToHost), "read error word");
  if (herr) {
    cudaMemset(r->err, 0, 4);
    return fail(NR_ERR_DEVICE, "integrator error word 0x" + hex_word(herr));
  }
  if (r->counters_on) {
    unsigned long long c[5];
    CU(cudaMemcpy(c, r->counters, sizeof(c), cudaMemcpyDeviceToHost), "read counters");
    r->last.rays = c[0];
    r->last.node_visits = c[1];
    r->last.tri_tests = c[2];
    r->last.obj_tests = c[3];
    r->last.paths = (unsigned long long)count * N;
  }
  r->n64 += count;
  return NR_OK;
}

int nr_render_viewport(nr_render* r, int32_t show_axis_grid) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  KernelParams P = make_params(r, 0, 0, false);
  P.beauty64 = nullptr;
  CU(launch_viewport(P, show_axis_grid, r->stream), "viewport");
  CU(cudaStreamSynchronize(r->stream), "viewport");
  uint32_t herr = 0;
  CU(cudaMemcpy(&herr, r->err, 4, cudaMemcpyDeviceToHost), "read error word");
  if (herr) {
    cudaMemset(r->err, 0, 4);
    return fail(NR_ERR_DEVICE, "viewport error word 0x" + hex_word(herr));
  }
  return NR_OK;
}

int nr_render_pick(nr_render* r, float u, float v, nr_pick_result* out) {
  if (!r || !out) return fail(NR_ERR_INVALID, "null argument");
  if (!r->d_pick) CU(cudaMalloc(&r->d_pick, sizeof(PickOut)), "alloc pick");
  KernelParams P = make_params(r, 0, 0, false);
  CU(launch_pick(P, u, v, r->d_pick, r->stream), "pick");
  PickOut h;
  CU(cudaMemcpyAsync(&h, r->d_pick, sizeof(h), cudaMemcpyDeviceToHost, r->stream), "read pick");
  CU(cudaStreamSynchronize(r->stream), "pick");
  static_assert(sizeof(PickOut) == sizeof(nr_pick_result), "pick result layout");
  memcpy(out, &h, sizeof(h));
  return NR_OK;
}

int nr_render_selection_mask(nr_render* r, uint32_t object_id, int32_t outline_radius,
                             uint8_t* host_hw) {
  if (!r || !host_hw || outline_radius < 0 || outline_radius > 64)
    return fail(NR_ERR_INVALID, "bad argument (outline radius 0..64)");
  size_t hw = (size_t)r->W * r->H;
  if (!r->d_mask) CU(cudaMalloc(&r->d_mask, 2 * hw), "alloc mask");
  KernelParams P = make_params(r, 0, 0, false);
  CU(launch_selection_mask(P, object_id, outline_radius, r->d_mask, r->d_mask + hw, r->stream),
     "selection mask");
  CU(cudaMemcpyAsync(host_hw, r->d_mask + hw, hw, cudaMemcpyDeviceToHost, r->stream), "read mask");
  CU(cudaStreamSynchronize(r->stream), "selection mask");
  return NR_OK;
}

int nr_render_set_nrc(nr_render* r, nr_nrc* cache, uint32_t terminate_bounce,
                      uint32_t train_one_in, float lr, uint32_t batch, uint32_t min_steps) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (cache && r->cfg.mode != NR_MODE_PERF)
    return fail(NR_ERR_STATE, "the radiance cache needs NR_MODE_PERF");
  if (cache && (terminate_bounce < 1 || terminate_bounce >= r->cfg.ray_depth))
    return fail(NR_ERR_INVALID, "terminate_bounce must be in [1, ray_depth)");
  r->nrc = cache;
  r->nrc_bounce = terminate_bounce;
  r->nrc_one_in = std::max(1u, train_one_in);
  r->nrc_lr = lr;
  r->nrc_batch = batch ? batch : 16384u;
  r->nrc_min_steps = min_steps ? std::min(min_steps, kNrcMaxGroups) : 4u;
  return NR_OK;
}

int nr_render_nrc_stats(const nr_render* r, uint64_t* queries, uint64_t* records) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (queries) *queries = r->nrc_queries;
  if (records) *records = r->nrc_records;
  return NR_OK;
}

int nr_render_sample_layers(nr_render* r, uint32_t sample_idx, float* beauty, float* diffuse,
                            float* normal, uint32_t* primary) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (sample_idx >= r->cam.samples_per_pixel)
    return fail(NR_ERR_INVALID, "sample index beyond samples_per_pixel");
  size_t hw = (size_t)r->W * r->H;
  for (int k = 0; k < 3; ++k)
    if (!r->raw[k]) CU(cudaMalloc(&r->raw[k], sizeof(float) * 3 * hw), "alloc raw");
  if (!r->raw_primary) CU(cudaMalloc(&r->raw_primary, sizeof(uint32_t) * hw), "alloc raw");
  KernelParams P = make_params(r, sample_idx, 1, true);
  int rc = run_kernel(r, P);
  if (rc != NR_OK) return rc;
  if (beauty) CU(cudaMemcpy(beauty, r->raw[0], sizeof(float) * 3 * hw, cudaMemcpyDeviceToHost), "read");
  if (diffuse) CU(cudaMemcpy(diffuse, r->raw[1], sizeof(float) * 3 * hw, cudaMemcpyDeviceToHost), "read");
  if (normal) CU(cudaMemcpy(normal, r->raw[2], sizeof(float) * 3 * hw, cudaMemcpyDeviceToHost), "read");
  if (primary) CU(cudaMemcpy(primary, r->raw_primary, sizeof(uint32_t) * hw, cudaMemcpyDeviceToHost), "read");
  return NR_OK;
}

int nr_render_trace_log(nr_render* r, uint32_t sample_idx, uint32_t max_bounces, float* host_log,
                        float* beauty) {
  if (!r || !host_log) return fail(NR_ERR_INVALID, "null argument");
  if (sample_idx == 0 || sample_idx >= r->cam.samples_per_pixel)
    return fail(NR_ERR_INVALID, "sample index outside 1 .. samples_per_pixel - 1");
  if (max_bounces == 0 || max_bounces > 64) return fail(NR_ERR_INVALID, "max_bounces outside 1 .. 64");
  if (r->cfg.mode != NR_MODE_REFERENCE || r->cfg.schedule != NR_SCHEDULE_WAVEFRONT)
    return fail(NR_ERR_STATE, "the trace log covers the wavefront schedule in NR_MODE_REFERENCE");
  size_t hw = (size_t)r->W * r->H;
  for (int k = 0; k < 3; ++k)
    if (!r->raw[k]) CU(cudaMalloc(&r->raw[k], sizeof(float) * 3 * hw), "alloc raw");
  if (!r->raw_primary) CU(cudaMalloc(&r->raw_primary, sizeof(uint32_t) * hw), "alloc raw");
  const size_t n = hw * max_bounces * kTraceLogFloats;
  float* d = nullptr;
  CU(cudaMalloc(&d, sizeof(float) * n), "alloc trace log");
  // entries of bounces a path never reaches stay all-ones bits
  cudaError_t e = cudaMemsetAsync(d, 0xff, sizeof(float) * n, r->stream);
  int rc = NR_OK;
  if (e != cudaSuccess) rc = cuda_fail(e, "clear trace log");
  if (rc == NR_OK) {
    r->trace_log = d;
    r->log_bounces = max_bounces;
    rc = run_kernel(r, make_params(r, sample_idx, 1, true));
    r->trace_log = nullptr;
    r->log_bounces = 0;
  }
  if (rc == NR_OK && (e = cudaMemcpy(host_log, d, sizeof(float) * n, cudaMemcpyDeviceToHost)) != cudaSuccess)
    rc = cuda_fail(e, "read trace log");
  if (rc == NR_OK && beauty &&
      (e = cudaMemcpy(beauty, r->raw[0], sizeof(float) * 3 * hw, cudaMemcpyDeviceToHost)) != cudaSuccess)
    rc = cuda_fail(e, "read beauty");
  cudaFree(d);
  return rc;
}

int nr_render_layer_device_ptr(nr_render* r, int32_t layer, uint64_t* out) {
  if (!r || !out || layer < 0 || layer > 8) return fail(NR_ERR_INVALID, "bad layer");
  *out = (uint64_t)(uintptr_t)r->layer[layer];
  return NR_OK;
}

int nr_render_read_layer(nr_render* r, int32_t layer, float* host) {
  if (!r || !host || layer < 0 || layer > 8) return fail(NR_ERR_INVALID, "bad layer");
  if (!r->layer[layer]) return fail(NR_ERR_STATE, "layer is not enabled");
  size_t n = (size_t)r->layer_c[layer] * r->W * r->H;
  CU(cudaMemcpy(host, r->layer[layer], sizeof(float) * n, cudaMemcpyDeviceToHost), "read layer");
  return NR_OK;
}

int nr_render_read_beauty_fp64(nr_render* r, double* host) {
  if (!r || !host) return fail(NR_ERR_INVALID, "null argument");
  if (!r->beauty64) return fail(NR_ERR_STATE, "fp64 accumulation is not enabled");
  size_t n = (size_t)3 * r->W * r->H;
  CU(cudaMemcpy(host, r->beauty64, sizeof(double) * n, cudaMemcpyDeviceToHost), "read fp64");
  double inv = r->n64 ? 1.0 / (double)r->n64 : 0.0;
  for (size_t i = 0; i < n; ++i) host[i] *= inv;
  return NR_OK;
}

int nr_render_read_beauty_fp64_sum(nr_render* r, double* host, uint64_t* n_samples) {
  if (!r || !host || !n_samples) return fail(NR_ERR_INVALID, "null argument");
  if (!r->beauty64) return fail(NR_ERR_STATE, "fp64 accumulation is not enabled");
  size_t n = (size_t)3 * r->W * r->H;
  CU(cudaMemcpy(host, r->beauty64, sizeof(double) * n, cudaMemcpyDeviceToHost), "read fp64");
  *n_samples = r->n64;
  return NR_OK;
}

static DisplayParams display_params(const nr_stream_config* c) {
  DisplayParams p{};
  p.linear_to_gamma = c->linear_to_gamma;
  p.apply_white_balance = c->apply_white_balance;
  p.wb_tint = c->wb_tint;
  p.apply_tonemapping = c->apply_tonemapping;
  p.tm_method = c->tm_method;
  p.tm_white_point = c->tm_white_point;
  p.tm_alpha = c->tm_alpha;
  return p;
}

static int display(nr_render* r, int32_t layer, const nr_stream_config* c, uint8_t* h8, float* hf) {
  if (!r || !c || layer < 0 || layer > 8) return fail(NR_ERR_INVALID, "bad argument");
  if (!r->layer[layer] || r->layer_c[layer] != 3)
    return fail(NR_ERR_STATE, "display needs an enabled 3-channel layer");
  size_t hw = (size_t)r->W * r->H;
  if (h8 && !hf && layer == NR_LAYER_BEAUTY && r->fused_on && r->fused_valid &&
      memcmp(c, &r->fused_cfg, sizeof(*c)) == 0) {
    // the last render call's accumulate pass already wrote these bytes
    CU(cudaMemcpyAsync(h8, r->disp8, 3 * hw, cudaMemcpyDeviceToHost, r->stream), "read");
    CU(cudaStreamSynchronize(r->stream), "display");
    return NR_OK;
  }
  if (h8 && !r->disp8) CU(cudaMalloc(&r->disp8, 3 * hw), "alloc");
  if (hf && !r->dispf) CU(cudaMalloc(&r->dispf, sizeof(float) * 3 * hw), "alloc");
  DisplayParams p = display_params(c);
  CU(display_params_resolve(p, c->wb_temperature, r->wb_scratch, r->stream), "white balance");
  CU(launch_display(r->layer[layer], h8 ? r->disp8 : nullptr, hf ? r->dispf : nullptr, hw, p,
                    r->stream),
     "display");
  if (h8) CU(cudaMemcpyAsync(h8, r->disp8, 3 * hw, cudaMemcpyDeviceToHost, r->stream), "read");
  if (hf) CU(cudaMemcpyAsync(hf, r->dispf, sizeof(float) * 3 * hw, cudaMemcpyDeviceToHost, r->stream), "read");
  CU(cudaStreamSynchronize(r->stream), "display");
  return NR_OK;
}

int nr_render_set_fused_display(nr_render* r, const nr_stream_config* c) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  r->fused_valid = false;
  if (!c) {
    r->fused_on = false;
    return NR_OK;
  }
  if (!r->layer[NR_LAYER_BEAUTY]) return fail(NR_ERR_STATE, "the beauty layer is not enabled");
  const size_t hw = (size_t)r->W * r->H;
  if (!r->disp8) CU(cudaMalloc(&r->disp8, 3 * hw), "alloc");
  DisplayParams p = display_params(c);
  CU(display_params_resolve(p, c->wb_temperature, r->wb_scratch, r->stream), "white balance");
  r->fused_p = p;
  r->fused_cfg = *c;
  r->fused_on = true;
  return NR_OK;
}

int nr_host_alloc(uint64_t bytes, void** out) {
  if (!out) return fail(NR_ERR_INVALID, "nr_host_alloc: null output");
  *out = nullptr;
  if (bytes == 0) return NR_OK;
  CU(cudaMallocHost(out, bytes), "nr_host_alloc");
  return NR_OK;
}

int nr_host_free(void* p) {
  if (p) CU(cudaFreeHost(p), "nr_host_free");
  return NR_OK;
}

int nr_render_readback(nr_render* r, int32_t layer, const nr_stream_config* c, uint8_t* h8) {
  if (!h8) return fail(NR_ERR_INVALID, "null output");
  return display(r, layer, c, h8, nullptr);
}

int nr_render_display_float(nr_render* r, int32_t layer, const nr_stream_config* c, float* hf) {
  if (!hf) return fail(NR_ERR_INVALID, "null output");
  return display(r, layer, c, nullptr, hf);
}

int nr_render_dims(const nr_render* r, uint32_t* C, uint32_t* H, uint32_t* W) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (C) *C = 3;
  if (H) *H = r->H;
  if (W) *W = r->W;
  return NR_OK;
}

int nr_render_set_counters(nr_render* r, int32_t on) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  r->counters_on = on != 0;
  return NR_OK;
}

int nr_render_set_profiling(nr_render* r, int32_t on) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (on && r->pev.empty()) {
    // up to 4095 launches per call are timed (a wave is 2 + 3 * depth launches)
    r->pev.resize(4096, nullptr);
    r->pkind.resize(4096, 0);
    for (auto& e : r->pev) CU(cudaEventCreate(&e), "event");
  }
  r->profile_on = on != 0;
  return NR_OK;
}

int nr_render_graph_stats(const nr_render* r, uint32_t* captured, uint64_t* replays) {
  if (!r) return fail(NR_ERR_INVALID, "null render");
  if (captured) *captured = r->graphs_captured;
  if (replays) *replays = r->graph_replays;
  return NR_OK;
}

int nr_render_get_profile(const nr_render* r, nr_kernel_profile* out) {
  if (!r || !out) return fail(NR_ERR_INVALID, "null argument");
  *out = r->prof;
  return NR_OK;
}

int nr_render_get_counters(const nr_render* r, nr_trace_counters* out) {
  if (!r || !out) return fail(NR_ERR_INVALID, "null argument");
  *out = r->last;
  return NR_OK;
}

int nr_render_last_ms(const nr_render* r, double* out) {
  if (!r || !out) return fail(NR_ERR_INVALID, "null argument");
  *out = r->last_ms;
  return NR_OK;
}

int nr_render_stream(const nr_render* r, uint64_t* out) {
  if (!r || !out) return fail(NR_ERR_INVALID, "null argument");
  *out = (uint64_t)(uintptr_t)r->stream;
  return NR_OK;
}

static uint32_t* conv_err_word() {
  static uint32_t* d = nullptr;
  if (!d && cudaMalloc(&d, 4) == cudaSuccess) cudaMemset(d, 0, 4);
  return d;
}

int nr_conv3x3_forward_device(const void* x, int32_t x_stride, int32_t x_off, const void* w,
                              const float* bias, void* y, int32_t y_stride, int32_t y_off,
                              int32_t cin, int32_t cout, int32_t B, int32_t H, int32_t W,
                              int32_t relu, uint64_t stream) {
  if (!x || !w || !y || B < 1 || H < 1 || W < 1) return fail(NR_ERR_INVALID, "bad argument");
  ConvFwdArgs a{static_cast<const __nv_bfloat16*>(x), x_stride, x_off,
                static_cast<const __nv_bfloat16*>(w), bias, static_cast<__nv_bfloat16*>(y),
                y_stride, y_off, cin, cout, B, H, W, relu, conv_err_word()};
  if (!a.err) return fail(NR_ERR_CUDA, "alloc error word");
  cudaError_t e = launch_conv_fwd(a, (cudaStream_t)(uintptr_t)stream);
  if (e == cudaErrorInvalidValue)
    return fail(NR_ERR_INVALID, "conv3x3: channels must be multiples of 16 (<= 256), strides and "
                                "offsets multiples of 8");
  CU(e, "conv3x3 forward");
  return NR_OK;
}

int nr_conv3x3_wgrad_device(const void* dy, int32_t dy_stride, int32_t dy_off, const void* x,
                            int32_t x_stride, int32_t x_off, float* dw, int32_t cin,
                            int32_t cout, int32_t B, int32_t H, int32_t W, uint64_t stream) {
  if (!dy || !x || !dw || B < 1 || H < 1 || W < 1) return fail(NR_ERR_INVALID, "bad argument");
  const int P = B * H * W;
  const int chunks = (P + 127) / 128;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // about two CTAs per SM over the 9 taps
  int per = std::max(1, (chunks * 9 + 2 * sms - 1) / (2 * sms));
  ConvWgradArgs a{static_cast<const __nv_bfloat16*>(dy), dy_stride, dy_off,
                  static_cast<const __nv_bfloat16*>(x), x_stride, x_off, dw, cin, cout, B, H, W,
                  per, conv_err_word()};
  if (!a.err) return fail(NR_ERR_CUDA, "alloc error word");
  cudaError_t e = launch_conv_wgrad(a, (cudaStream_t)(uintptr_t)stream);
  if (e == cudaErrorInvalidValue)
    return fail(NR_ERR_INVALID, "conv3x3 wgrad: cin multiple of 16 (<= 256), cout multiple of 16 "
                                "(<= 128), strides and offsets multiples of 8");
  CU(e, "conv3x3 wgrad");
  return NR_OK;
}

}  // extern "C"

struct nr_denoiser {
  Denoiser d;
};

extern "C" {

int nr_denoiser_create(uint32_t max_pixels, uint32_t seed, nr_denoiser** out) {
  if (!out) return fail(NR_ERR_INVALID, "null argument");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(NR_ERR_NO_DEVICE, "no CUDA device");
  auto d = std::make_unique<nr_denoiser>();
  std::string e = denoiser_create(d->d, max_pixels, seed);
  if (!e.empty()) return fail(e.find("must") != std::string::npos ? NR_ERR_INVALID : NR_ERR_CUDA, e);
  *out = d.release();
  return NR_OK;
}

int nr_denoiser_destroy(nr_denoiser* d) {
  delete d;
  return NR_OK;
}

static int den_status(const std::string& e) {
  if (e.empty()) return NR_OK;
  if (e.find("must") != std::string::npos || e.find("exceeds") != std::string::npos ||
      e.find("more queries") != std::string::npos)
    return fail(NR_ERR_INVALID, e);
  if (e.find("timed out") != std::string::npos) return fail(NR_ERR_DEVICE, e);
  return fail(NR_ERR_CUDA, e);
}

int nr_denoiser_set_loss(nr_denoiser* d, int32_t kind) {
  if (!d) return fail(NR_ERR_INVALID, "null argument");
  return den_status(denoiser_set_loss(d->d, kind));
}

int nr_denoiser_train_step(nr_denoiser* d, const float* beauty, const float* diffuse,
                           const float* normal, const float* depth, const float* target,
                           int32_t B, int32_t H, int32_t W, float lr, double* loss,
                           uint64_t stream) {
  if (!d || !beauty || !target) return fail(NR_ERR_INVALID, "null argument");
  cudaStream_t st = (cudaStream_t)(uintptr_t)stream;
  int rc = den_status(denoiser_forward_backward(d->d, beauty, diffuse, normal, depth, target, B,
                                                H, W, loss, st));
  if (rc != NR_OK || lr <= 0.0f) return rc;
  return den_status(denoiser_adam(d->d, lr, st));
}

int nr_denoiser_infer(nr_denoiser* d, const float* beauty, const float* diffuse,
                      const float* normal, const float* depth, float* out, int32_t B, int32_t H,
                      int32_t W, uint64_t stream) {
  if (!d || !beauty || !out) return fail(NR_ERR_INVALID, "null argument");
  return den_status(denoiser_infer(d->d, beauty, diffuse, normal, depth, out, B, H, W,
                                   (cudaStream_t)(uintptr_t)stream));
}

int nr_denoiser_param_count(const nr_denoiser* d, uint64_t* out) {
  if (!d || !out) return fail(NR_ERR_INVALID, "null argument");
  *out = denoiser_param_count(d->d);
  return NR_OK;
}

int nr_denoiser_get_params(const nr_denoiser* d, int32_t what, float* host) {
  if (!d || !host || what < 0 || what > 1) return fail(NR_ERR_INVALID, "bad argument");
  return den_status(denoiser_get(d->d, what, host));
}

int nr_denoiser_set_params(nr_denoiser* d, const float* host) {
  if (!d || !host) return fail(NR_ERR_INVALID, "null argument");
  return den_status(denoiser_set_weights(d->d, host));
}

int nr_denoiser_layers(const nr_denoiser* d, int32_t* count, int32_t* cin_cout) {
  if (!d || !count) return fail(NR_ERR_INVALID, "null argument");
  *count = denoiser_layer_count(d->d);
  if (cin_cout)
    for (int i = 0; i < *count; ++i) denoiser_layer_shape(d->d, i, cin_cout + 2 * i, cin_cout + 2 * i + 1);
  return NR_OK;
}

int nr_nrc_create(uint32_t max_queries, const float lo[3], const float hi[3], uint32_t seed,
                  nr_nrc** out) {
  if (!out || !lo || !hi) return fail(NR_ERR_INVALID, "null argument");
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) return fail(NR_ERR_NO_DEVICE, "no CUDA device");
  auto n = std::make_unique<nr_nrc>();
  std::string e = nrc_create(n->n, max_queries, lo, hi, seed);
  if (!e.empty()) return fail(e.find("must") != std::string::npos ? NR_ERR_INVALID : NR_ERR_CUDA, e);
  *out = n.release();
  return NR_OK;
}

int nr_nrc_destroy(nr_nrc* n) {
  delete n;
  return NR_OK;
}

int nr_nrc_infer(nr_nrc* n, const float* queries, uint32_t count, float* radiance,
                 uint64_t stream) {
  if (!n || (count && (!queries || !radiance))) return fail(NR_ERR_INVALID, "null argument");
  return den_status(nrc_infer(n->n, reinterpret_cast<const NrcQuery*>(queries), count, radiance,
                              (cudaStream_t)(uintptr_t)stream));
}

int nr_nrc_train(nr_nrc* n, const float* queries, const float* target, uint32_t count,
                 float lr, double* loss, uint64_t stream) {
  if (!n || (count && (!queries || !target))) return fail(NR_ERR_INVALID, "null argument");
  return den_status(nrc_train(n->n, reinterpret_cast<const NrcQuery*>(queries), target, count, lr,
                              loss, (cudaStream_t)(uintptr_t)stream));
}

int nr_nrc_count(const nr_nrc* n, int32_t what, uint64_t* out) {
  if (!n || !out || what < 0 || what > 4) return fail(NR_ERR_INVALID, "bad argument");
  *out = nrc_count(n->n, what);
  return NR_OK;
}

int nr_nrc_get(const nr_nrc* n, int32_t what, float* host) {
  if (!n || !host || what < 0 || what > 4) return fail(NR_ERR_INVALID, "bad argument");
  return den_status(nrc_get(n->n, what, host));
}

int nr_nrc_set(nr_nrc* n, const float* mlp, const float* grid) {
  if (!n) return fail(NR_ERR_INVALID, "null argument");
  return den_status(nrc_set_weights(n->n, mlp, grid));
}

int nr_accumulate_device(float* avg, const float* smp, uint32_t C, uint32_t H, uint32_t W,
                         uint32_t sample_idx, uint64_t stream) {
  if (!avg || !smp || sample_idx == 0) return fail(NR_ERR_INVALID, "bad argument");
  CU(launch_accumulate(avg, smp, (size_t)C * H * W, sample_idx, (cudaStream_t)(uintptr_t)stream),
     "accumulate");
  return NR_OK;
}

int nr_display_device(const float* src, uint8_t* dst, uint32_t C, uint32_t H, uint32_t W,
                      const nr_stream_config* c, uint64_t stream) {
  if (!src || !dst || !c || C != 3) return fail(NR_ERR_INVALID, "bad argument");
  cudaStream_t st = (cudaStream_t)(uintptr_t)stream;
  DisplayParams p{};
  p.linear_to_gamma = c->linear_to_gamma;
  p.apply_white_balance = c->apply_white_balance;
  p.wb_tint = c->wb_tint;
  p.apply_tonemapping = c->apply_tonemapping;
  p.tm_method = c->tm_method;
  p.tm_white_point = c->tm_white_point;
  p.tm_alpha = c->tm_alpha;
  V3* scratch = nullptr;
  if (p.apply_white_balance) {
    CU(cudaMalloc(&scratch, sizeof(V3)), "alloc");
    cudaError_t e = display_params_resolve(p, c->wb_temperature, scratch, st);
    cudaFree(scratch);
    if (e != cudaSuccess) return cuda_fail(e, "white balance");
  }
  CU(launch_display(src, dst, nullptr, (size_t)H * W, p, st), "display");
  return NR_OK;
}

}  // extern "C"
