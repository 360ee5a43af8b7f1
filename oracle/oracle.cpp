// oracle.cpp — CPU restatement of the reference path tracer (TEST
// INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline as the checker; never linked into the product).
//
// Scalar C++ that follows the reference's algorithm step by step, in the same
// floating-point operation order, compiled without fast-math or FMA so that
// it reproduces the reference's own integrator compiled for the host
// (oracle/ref_cpu_harness.cpp) bit for bit. It includes the reference's host
// BVH builder (16-bin SAH, std::partition, std::sort median fallback, leaf
// size 1), so traversal order and closest-hit tie breaking match too.
//
// Per function, the reference file:line it restates is cited (paths relative
// to nectar_render/csrc/).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <unordered_map>
#include <numeric>
#include <random>
#include <thread>
#include <tuple>
#include <vector>

namespace {

constexpr float EPS = 1e-4f;   // core/constants.h:7-13
constexpr float FMIN = 1e-8f;
constexpr float FMAX = 1e32f;
constexpr float PI = 3.1415926535897932385f;
constexpr float PI2 = PI * 2.0f;
constexpr float PI4 = PI2 * PI2;

// ---- vectors (core/vector.h) ------------------------------------------------
struct V {
  float x, y, z;
};
struct V2 {
  float x, y;
};
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(V a, V b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V operator*(V a, float t) { return {a.x * t, a.y * t, a.z * t}; }
inline V operator*(float t, V a) { return {a.x * t, a.y * t, a.z * t}; }
inline V operator+(V a, float t) { return {a.x + t, a.y + t, a.z + t}; }
inline V operator-(V a) { return {-a.x, -a.y, -a.z}; }
inline V operator/(V a, float t) { return (1.0f / t) * a; }
inline V operator/(V a, V b) { return {a.x / (b.x + FMIN), a.y / (b.y + FMIN), a.z / (b.z + FMIN)}; }
inline float lsq(V v) {
  float o = v.x * v.x + v.y * v.y;
  o += v.z * v.z;
  return o;
}
inline float len(V v) { return sqrtf(lsq(v)); }
inline V normalize(V v) { return v / len(v); }
inline bool near_zero(V v) { return len(v) < 1e-8f; }
inline float dot(V u, V v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
inline V cross(V u, V v) {
  return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
inline V reflect(V v, V n) { return v - 2.0f * dot(v, n) * n; }
inline V refract(V uv, V n, float ior) {
  float ct = fminf(dot(-uv, n), 1.0f);
  V perp = ior * (uv + ct * n);
  V par = -sqrtf(fabsf((float)(1.0 - (double)lsq(perp)))) * n;
  return perp + par;
}
inline float comp(V v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// ---- matrices and transforms (core/matrix.h:6-96, core/transform.h) --------
struct M {
  float m[3][3];
};
inline V mul(const M& a, V v) {
  return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
          a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
          a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
M mmul(const M& a, const M& b) {
  M r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      r.m[i][j] = 0;
      for (int k = 0; k < 3; k++) r.m[i][j] += a.m[i][k] * b.m[k][j];
    }
  return r;
}
M mT(const M& a) {
  M r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r.m[i][j] = a.m[j][i];
  return r;
}
M rx(float a) { float c = cosf(a), s = sinf(a); return M{{{1, 0, 0}, {0, c, -s}, {0, s, c}}}; }
M ry(float a) { float c = cosf(a), s = sinf(a); return M{{{c, 0, s}, {0, 1, 0}, {-s, 0, c}}}; }
M rz(float a) { float c = cosf(a), s = sinf(a); return M{{{c, -s, 0}, {s, c, 0}, {0, 0, 1}}}; }
float deg2rad(float d) { return d * 0.01745329; }
M euler_rad(V r) { return mmul(mmul(rz(r.z), ry(r.y)), rx(r.x)); }
M euler_deg(V r) { return euler_rad(V{deg2rad(r.x), deg2rad(r.y), deg2rad(r.z)}); }

struct Xf {
  V pos, scale, inv_s;
  M R, invR;
};
Xf xform(V p, V rdeg, V s) {
  Xf x;
  x.pos = p;
  x.R = euler_deg(rdeg);
  x.scale = s;
  x.invR = mT(euler_deg(rdeg));
  x.inv_s = V{1.0f, 1.0f, 1.0f} / (s + FMIN);
  return x;
}
Xf xform_pos(V p) {
  Xf x;
  x.pos = p;
  x.R = euler_rad(V{0.0f, 0.0f, 0.0f});
  x.scale = V{1.0f, 1.0f, 1.0f};
  x.invR = mT(euler_rad(V{0.0f, 0.0f, 0.0f}));
  x.inv_s = V{1.0f, 1.0f, 1.0f};
  return x;
}

// ---- random numbers (core/random.h:11-77; random/include/hash.h) -----------
// Philox4x32-10 (Salmon et al., SC'11) with curand_init's counter layout.
struct Rng {
  uint32_t seed, sub, draw = 0;
  float uniform() {
    uint32_t c[4] = {draw >> 2, 0u, sub, 0u}, k0 = seed, k1 = 0u;
    for (int r = 0; r < 10; ++r) {
      uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
      uint32_t h0 = (uint32_t)(p0 >> 32), l0 = (uint32_t)p0, h1 = (uint32_t)(p1 >> 32), l1 = (uint32_t)p1;
      uint32_t n0 = h1 ^ c[1] ^ k0, n2 = h0 ^ c[3] ^ k1;
      c[0] = n0;
      c[1] = l1;
      c[2] = n2;
      c[3] = l0;
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t v = c[draw & 3u];
    draw++;
    return (float)v * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
  }
  float random_float() { return uniform() * (1.0f - 0.0f) + 0.0f; }
  float random_float(float mn, float mx) { return uniform() * (mx - mn) + mn; }
};

inline uint32_t f2u(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}
inline uint32_t hmix(uint32_t v, uint32_t mult) {
  v ^= (v >> 16u) * mult;
  return v ^ (v >> 13u);
}
inline uint32_t pcg_int(uint32_t i, uint32_t seed) {  // hash.h:48-62 (stream 0)
  uint32_t s = seed * 1759274928u;
  s = i ^ s;
  s = hmix(s, 0x9E3779B9u);
  s = hmix(s, 0x85EBCA6Bu);
  s = hmix(s, 0xC2B2AE35u);
  uint32_t state = s * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
inline float pcg_f(float f, uint32_t seed) { return (float)pcg_int(f2u(f), seed) * (1.0f / (float)0xFFFFFFFF); }
inline float pcg_v(V a, uint32_t seed) {  // hash.h:98-106
  uint32_t s = seed * 1759274928u;
  s ^= pcg_int(f2u(a.x), (seed + 0u) * 2654435761u) ^ 668265263u;
  s ^= pcg_int(f2u(a.y), (seed + 1u) * 2246822519u) ^ 374761393u;
  s ^= pcg_int(f2u(a.z), (seed + 2u) * 3266489917u) ^ 2654435761u;
  uint32_t state = s * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (float)((word >> 22u) ^ word) * (1.0f / (float)0xFFFFFFFF);
}
inline float pcg_ray(V o, V d) {  // hash.h:108-125
  float a = pcg_v(o, (0u + 0u) * 2654435761u);
  float b = pcg_v(d, (0u + 1u) * 3266489917u);
  return (a + b) * 0.5f;
}
inline V2 pcg_vector2(float f, uint32_t seed) {  // hash.h:182-191
  float x = pcg_f(f, seed);
  uint32_t s = seed ^ (uint32_t)(x * 4294967296.0f);
  uint32_t i = s * 747796405u + 2891336453u;
  float y = pcg_f((float)i, 0u);
  return V2{x, y};
}

// ---- rays and hit records (engine/ray.h, hittable/hit_record.h) -------------
struct Ray {
  V o, d, inv;
  float tm;
};
Ray mkray(V o, V d, float tm = 0.0f) { return Ray{o, d, V{1.0f / d.x, 1.0f / d.y, 1.0f / d.z}, tm}; }
Ray to_object(const Xf& x, const Ray& r) {
  V o = mul(x.invR, r.o - x.pos) * x.inv_s;
  V d = mul(x.invR, r.d) * x.inv_s;
  return mkray(o, d, r.tm);
}
inline V at(const Ray& r, float t) { return r.o + t * r.d; }

struct Hit {
  int obj = 0;
  int mat = 0;
  V p{0, 0, 0}, n{0, 0, 0}, tangent{0, 0, 0};
  V2 uv{0, 0};
  float t = 0.0f;
  bool front_face = false;
  uint32_t prim = 0xffffffffu;
};

void to_world(Hit& h, const Xf& x, const Ray& oray, const Ray& wray, bool bias) {
  h.p = mul(x.R, h.p * x.scale) + x.pos;
  h.tangent = normalize(mul(x.R, h.tangent * x.scale));
  h.front_face = dot(oray.d, h.n) < 0.0f;
  h.n = h.front_face ? h.n : -h.n;
  h.n = normalize(mul(x.R, h.n * x.inv_s));
  h.front_face = dot(wray.d, h.n) < 0.0f;
  h.n = h.front_face ? h.n : -h.n;
  h.tangent = normalize(h.tangent - h.n * dot(h.tangent, h.n));
  if (near_zero(h.tangent))
    h.tangent = normalize(cross(h.n, fabsf(h.n.x) > 0.9f ? V{0.0f, 1.0f, 0.0f} : V{1.0f, 0.0f, 0.0f}));
  if (bias) h.p = h.p + h.n * EPS;
  h.t = dot(h.p - wray.o, wray.d) / lsq(wray.d);
}

// ---- AABB and BVH (hittable/include/bvh/aabb.h, bvh.h) ----------------------
struct Box {
  float lo[3], hi[3];
};
bool box_hit(const Box& b, const Ray& r, float tmin, float tmax) {  // aabb.h:111-133
  for (int a = 0; a < 3; ++a) {
    float t0 = (b.lo[a] - comp(r.o, a)) * comp(r.inv, a);
    float t1 = (b.hi[a] - comp(r.o, a)) * comp(r.inv, a);
    if (t0 < t1) {
      if (t0 > tmin) tmin = t0;
      if (t1 < tmax) tmax = t1;
    } else {
      if (t1 > tmin) tmin = t1;
      if (t0 < tmax) tmax = t0;
    }
    if (tmax <= tmin) return false;
  }
  return true;
}
float box_hit_t(const Box& b, const Ray& r, float tmin, float tmax) {  // aabb.h:135-157
  for (int a = 0; a < 3; ++a) {
    float t0 = (b.lo[a] - comp(r.o, a)) * comp(r.inv, a);
    float t1 = (b.hi[a] - comp(r.o, a)) * comp(r.inv, a);
    if (t0 < t1) {
      if (t0 > tmin) tmin = t0;
      if (t1 < tmax) tmax = t1;
    } else {
      if (t1 > tmin) tmin = t1;
      if (t0 < tmax) tmax = t0;
    }
    if (tmax <= tmin) return FMAX;
  }
  return tmin;
}
Box join(const Box& a, const Box& b) {  // AABB(box0, box1) via Interval(a, b)
  Box r;
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = a.lo[k] <= b.lo[k] ? a.lo[k] : b.lo[k];
    r.hi[k] = a.hi[k] >= b.hi[k] ? a.hi[k] : b.hi[k];
  }
  return r;
}
float area(const Box& b) {
  float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}
Box make_box(V a, V b) {  // AABB(const Vector3&, const Vector3&)
  Box r;
  for (int k = 0; k < 3; ++k) {
    float x = comp(a, k), y = comp(b, k);
    r.lo[k] = x <= y ? x : y;
    r.hi[k] = x <= y ? y : x;
  }
  return r;
}
Box transformed(const Box& b, const Xf& x) {  // aabb.h:60-91
  V c[8] = {{b.lo[0], b.lo[1], b.lo[2]}, {b.hi[0], b.lo[1], b.lo[2]}, {b.lo[0], b.hi[1], b.lo[2]},
            {b.hi[0], b.hi[1], b.lo[2]}, {b.lo[0], b.lo[1], b.hi[2]}, {b.hi[0], b.lo[1], b.hi[2]},
            {b.lo[0], b.hi[1], b.hi[2]}, {b.hi[0], b.hi[1], b.hi[2]}};
  V mn{FMAX, FMAX, FMAX}, mx{-FMAX, -FMAX, -FMAX};
  for (auto& k : c) {
    V w = mul(x.R, k * x.scale) + x.pos;
    mn = V{fminf(mn.x, w.x), fminf(mn.y, w.y), fminf(mn.z, w.z)};
    mx = V{fmaxf(mx.x, w.x), fmaxf(mx.y, w.y), fmaxf(mx.z, w.z)};
  }
  Box r = make_box(mn, mx);
  for (int k = 0; k < 3; ++k)
    if (r.hi[k] - r.lo[k] < EPS) {
      float pad = EPS / 2.0f;
      float lo = r.lo[k] - pad, hi = r.hi[k] + pad;
      r.lo[k] = lo;
      r.hi[k] = hi;
    }
  return r;
}

struct Node {
  Box bbox;
  int32_t left, right, object;
};

// BVH<T>::build (bvh.h:35-320): returns nodes and the item order
struct Bvh {
  std::vector<Node> nodes;
  std::vector<int32_t> order;
  const std::vector<Box>* boxes = nullptr;
  static constexpr int kB = 16;
  void build(const std::vector<Box>& b) {
    boxes = &b;
    nodes.clear();
    order.resize(b.size());
    std::iota(order.begin(), order.end(), 0);
    if (b.empty()) return;
    nodes.reserve(b.size() * 2);
    rec(0, (int32_t)b.size());
  }
  int32_t rec(int32_t start, int32_t end) {
    const std::vector<Box>& B = *boxes;
    int32_t span = end - start;
    size_t idx = nodes.size();
    nodes.push_back(Node{});
    if (span == 1) {
      nodes[idx].object = start;
      nodes[idx].left = -1;
      nodes[idx].right = -1;
      nodes[idx].bbox = B[order[start]];
      return (int32_t)idx;
    }
    V cmin{FMAX, FMAX, FMAX}, cmax{-FMAX, -FMAX, -FMAX};
    for (int32_t i = start; i < end; ++i) {
      const Box& b = B[order[i]];
      V c{(b.lo[0] + b.hi[0]) * 0.5f, (b.lo[1] + b.hi[1]) * 0.5f, (b.lo[2] + b.hi[2]) * 0.5f};
      cmin = V{fminf(cmin.x, c.x), fminf(cmin.y, c.y), fminf(cmin.z, c.z)};
      cmax = V{fmaxf(cmax.x, c.x), fmaxf(cmax.y, c.y), fmaxf(cmax.z, c.z)};
    }
    float best_cost = FMAX;
    int32_t best_axis = -1, best_bin = -1;
    for (int a = 0; a < 3; ++a) {
      float c_min = comp(cmin, a), extent = comp(cmax, a) - c_min;
      if (extent < EPS) continue;
      int32_t cnt[kB] = {0};
      Box bb[kB];
      for (int32_t i = start; i < end; ++i) {
        const Box& b = B[order[i]];
        float c = (b.lo[a] + b.hi[a]) * 0.5f;
        int32_t bin = (int32_t)(kB * (c - c_min) / extent);
        bin = bin < 0 ? 0 : (bin >= kB ? kB - 1 : bin);
        cnt[bin]++;
        bb[bin] = cnt[bin] == 1 ? b : join(bb[bin], b);
      }
      Box lb[kB], rb[kB], run{};
      int32_t lc[kB], rc[kB], rcount = 0;
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
      Box comb = B[order[start]];
      for (int32_t i = start + 1; i < end; ++i) comb = join(comb, B[order[i]]);
      float lx = comb.hi[0] - comb.lo[0], ly = comb.hi[1] - comb.lo[1], lz = comb.hi[2] - comb.lo[2];
      best_axis = (lx > ly && lx > lz) ? 0 : (ly > lz ? 1 : 2);
    }
    int32_t mid;
    if (best_bin == -1) {
      int a = best_axis;
      std::sort(order.begin() + start, order.begin() + end,
                [&](int32_t x, int32_t y) { return B[x].lo[a] < B[y].lo[a]; });
      mid = start + (end - start) / 2;
    } else {
      int a = best_axis;
      float c_min = comp(cmin, a), extent = comp(cmax, a) - c_min;
      auto it = std::partition(order.begin() + start, order.begin() + end, [&](int32_t i) {
        const Box& b = B[i];
        float c = (b.lo[a] + b.hi[a]) * 0.5f;
        int32_t bin = (int32_t)(kB * (c - c_min) / extent);
        bin = bin < 0 ? 0 : (bin >= kB ? kB - 1 : bin);
        return bin <= best_bin;
      });
      mid = (int32_t)(it - order.begin());
    }
    nodes[idx].object = -1;
    int32_t l = rec(start, mid);
    nodes[idx].left = l;
    int32_t r = rec(mid, end);
    nodes[idx].right = r;
    nodes[idx].bbox = join(nodes[nodes[idx].left].bbox, nodes[nodes[idx].right].bbox);
    return (int32_t)idx;
  }
};

// ---- scene objects ------------------------------------------------------------
struct Mesh {
  std::vector<V> pos, nor, tan;
  std::vector<V2> uv;
  std::vector<uint32_t> tri;  // leaf-ordered triangle (v0, v1, v2) triples
  std::vector<uint32_t> tri_id;
  Bvh bvh;
};

struct Obj {
  int type, wtype;
  Xf x;
  int mat;
  int mesh;
  float radius;           // + FMIN
  float neg_inv_density;
  int id;
};

struct Tex {
  int type;
  V rgb;
  const uint8_t* img = nullptr;  // IMAGE: planar CHW, 3 channels read
  uint32_t H = 0, W = 0;
  float scale = 1.0f;
};
struct Mat {
  int type;
  float ior, brightness;
  V tint;
  Tex tex[5];
};

struct Scene {
  std::vector<Obj> objs;  // in the reference's leaf order
  std::vector<Mat> mats;
  std::vector<Mesh> meshes;
  Bvh tlas;
  int light = -1;
  int sky_type;
  V sky_start, sky_end;
  const float* hdri = nullptr;
  int hC = 0, hH = 0, hW = 0;
  float hrot = 0.f, hint = 1.f;
  Xf cube[6];
  bool rtl = true;
};

// Quad (hittable/primitives.h:3-88): members built by Quad()
struct QuadC {
  V u{1.0f, 0.0f, 0.0f}, v{0.0f, 0.0f, -1.0f}, w, normal;
  float area;
  QuadC() {
    V n = cross(u, v);
    normal = normalize(n);
    w = n / dot(n, n);
    area = len(n);
  }
};
const QuadC& quadc() {
  static QuadC q;
  return q;
}

bool quad_hit(const Ray& r, float tmin, float tmax, Hit& h) {
  const QuadC& q = quadc();
  float denom = dot(q.normal, r.d);
  if (fabsf(denom) < FMIN) return false;
  float t = -dot(q.normal, r.o) / denom;
  if (!(tmin <= t && t <= tmax)) return false;
  h.t = t;
  h.p = at(r, t);
  h.n = q.normal;
  h.tangent = q.u;
  float a = dot(q.w, cross(h.p, q.v));
  float b = dot(q.w, cross(q.u, h.p));
  h.uv = V2{a + 0.5f, b + 0.5f};
  return (-0.5f < a && a < 0.5f) & (-0.5f < b && b < 0.5f);
}

bool sphere_hit(const Ray& r, float tmin, float tmax, float radius, V scale, Hit& h) {  // shapes.h:25-58
  V oc = -r.o;
  float a = lsq(r.d);
  float hh = dot(r.d, oc);
  float c = lsq(oc) - radius * radius;
  float disc = hh * hh - a * c;
  if (disc < 0) return false;
  float sq = sqrtf(disc);
  float root = (hh - sq) / a;
  if (!(tmin < root && root < tmax)) {
    root = (hh + sq) / a;
    if (!(tmin < root && root < tmax)) return false;
  }
  h.t = root;
  h.p = at(r, root);
  V norm = h.p / ((radius * scale) + FMIN);
  h.n = norm;
  h.tangent = normalize(V{-h.p.z, 0.0f, h.p.x});
  float theta = acosf(-norm.y);
  float phi = atan2f(-norm.z, norm.x) + PI;
  h.uv = V2{phi / PI2, theta / PI};
  return true;
}

bool cube_hit(const Scene& S, const Ray& r, float tmin, float tmax, Hit& h) {  // shapes.h:142-173
  bool any = false;
  int face = -1;
  Ray fray;
  for (int i = 0; i < 6; ++i) {
    Ray fr = to_object(S.cube[i], r);
    Hit fh;
    if (quad_hit(fr, tmin, tmax, fh)) {
      any = true;
      face = i;
      fray = fr;
      h = fh;
      tmax = fh.t;
    }
  }
  if (any) to_world(h, S.cube[face], fray, r, false);
  return any;
}

// Moller-Trumbore (mesh.h:338-365)
bool tri_hit(const Ray& r, V v0, V v1, V v2, float tmin, float tmax, float& ot, float& ou, float& ov) {
  V e1 = v1 - v0, e2 = v2 - v0;
  V hv = cross(r.d, e2);
  float a = dot(e1, hv);
  if (fabsf(a) < FMIN) return false;
  float f = 1.0f / a;
  V s = r.o - v0;
  float u = f * dot(s, hv);
  if (u < 0.0f || u > 1.0f) return false;
  V q = cross(s, e1);
  float v = f * dot(r.d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = f * dot(e2, q);
  if (!(tmin <= t && t <= tmax)) return false;
  ot = t;
  ou = u;
  ov = v;
  return true;
}

bool mesh_hit(const Mesh& m, const Ray& r, float tmin, float tmax, Hit& h) {  // mesh.h:239-292
  uint32_t stack[64];
  uint32_t sp = 0;
  stack[sp++] = 0u;
  bool any = false;
  while (sp > 0) {
    const Node& nd = m.bvh.nodes[stack[--sp]];
    if (!box_hit(nd.bbox, r, tmin, tmax)) continue;
    if (nd.object != -1) {
      uint32_t k = (uint32_t)nd.object;
      V v0 = m.pos[m.tri[3 * k]], v1 = m.pos[m.tri[3 * k + 1]], v2 = m.pos[m.tri[3 * k + 2]];
      float t, u, v;
      if (tri_hit(r, v0, v1, v2, tmin, tmax, t, u, v)) {
        any = true;
        tmax = t;
        h.t = t;
        h.p = at(r, t);
        uint32_t a = m.tri[3 * k], b = m.tri[3 * k + 1], c = m.tri[3 * k + 2];
        float w = 1.0f - u - v;
        h.uv = V2{m.uv[a].x * w + m.uv[b].x * u + m.uv[c].x * v, m.uv[a].y * w + m.uv[b].y * u + m.uv[c].y * v};
        h.n = normalize(m.nor[a] * w + m.nor[b] * u + m.nor[c] * v);
        h.tangent = normalize(m.tan[a] * w + m.tan[b] * u + m.tan[c] * v);
        h.prim = m.tri_id[k];
      }
    } else {
      const Node& L = m.bvh.nodes[nd.left];
      const Node& R = m.bvh.nodes[nd.right];
      float tl = box_hit_t(L.bbox, r, tmin, tmax), tr = box_hit_t(R.bbox, r, tmin, tmax);
      bool left_near = tl < tr;
      uint32_t near_i = left_near ? nd.left : nd.right, far_i = left_near ? nd.right : nd.left;
      float far_t = left_near ? tr : tl;
      if (far_t < tmax) stack[sp++] = far_i;
      stack[sp++] = near_i;
    }
  }
  return any;
}

bool shape_hit(const Scene& S, const Obj& o, int type, const Ray& r, float tmin, float tmax, Hit& h) {
  switch (type) {
    case NR_HITTABLE_QUAD: return quad_hit(r, tmin, tmax, h);
    case NR_HITTABLE_SPHERE: return sphere_hit(r, tmin, tmax, o.radius, o.x.scale, h);
    case NR_HITTABLE_CUBE: return cube_hit(S, r, tmin, tmax, h);
    case NR_HITTABLE_MESH: return mesh_hit(S.meshes[o.mesh], r, tmin, tmax, h);
  }
  return false;
}

bool medium_hit(const Scene& S, const Obj& o, const Ray& r, float tmin, float tmax, Hit& h) {  // volumes.h:10-45
  Hit h1, h2;
  if (!shape_hit(S, o, o.wtype, r, -FMAX, FMAX, h1)) return false;
  if (!shape_hit(S, o, o.wtype, r, h1.t + EPS, FMAX, h2)) return false;
  if (h1.t < tmin) h1.t = tmin;
  if (h2.t > tmax) h2.t = tmax;
  if (h1.t >= h2.t) return false;
  if (h1.t < 0.0f) h1.t = 0.0f;
  float rl = len(r.d);
  float inside = (h2.t - h1.t) * rl;
  float dist = o.neg_inv_density * logf(pcg_ray(r.o, r.d));
  if (dist > inside) return false;
  h.p = at(r, h1.t + dist / rl);
  h.n = V{1.0f, 0.0f, 0.0f};
  h.front_face = true;
  return true;
}

bool object_hit(const Scene& S, const Obj& o, const Ray& r, float tmin, float tmax, Hit& h) {  // hittable.h:332-352
  switch (o.type) {
    case NR_HITTABLE_OBJECT_LIGHT: return shape_hit(S, o, o.wtype, r, -FMAX, FMAX, h);
    case NR_HITTABLE_CONSTANT_MEDIUM: return medium_hit(S, o, r, tmin, tmax, h);
    default: return shape_hit(S, o, o.type, r, tmin, tmax, h);
  }
}

bool hit_test(const Scene& S, const Obj& o, const Ray& wr, Hit& h) {  // hittable.h:324-330
  Ray r = to_object(o.x, wr);
  bool hit = object_hit(S, o, r, EPS, FMAX, h);
  to_world(h, o.x, r, wr, true);
  return hit;
}

bool scene_hit(const Scene& S, const Ray& ray, Hit& rec) {  // scene/include/graph.h:16-66
  float tmin = EPS, tmax = FMAX;
  uint32_t stack[64];
  uint32_t sp = 0;
  stack[sp++] = 0u;
  bool any = false;
  while (sp > 0) {
    const Node& nd = S.tlas.nodes[stack[--sp]];
    if (!box_hit(nd.bbox, ray, tmin, tmax)) continue;
    if (nd.object != -1) {
      Hit tmp;
      const Obj& o = S.objs[nd.object];
      if (hit_test(S, o, ray, tmp)) {
        if (tmin < tmp.t && tmp.t < tmax) {
          any = true;
          rec = tmp;
          rec.obj = nd.object;
          rec.mat = o.mat;
          tmax = tmp.t;
        }
      }
    } else {
      const Node& L = S.tlas.nodes[nd.left];
      const Node& R = S.tlas.nodes[nd.right];
      float tl = box_hit_t(L.bbox, ray, tmin, tmax), tr = box_hit_t(R.bbox, ray, tmin, tmax);
      bool left_near = tl < tr;
      uint32_t near_i = left_near ? nd.left : nd.right, far_i = left_near ? nd.right : nd.left;
      float far_t = left_near ? tr : tl;
      if (far_t < tmax) stack[sp++] = far_i;
      stack[sp++] = near_i;
    }
  }
  return any;
}

// ---- textures, materials, PDFs -----------------------------------------------
// TextureView::sample (texture.h:58-90): constant colour, or the image texel
// at the scaled, wrapped and clamped uv (nearest texel, v flipped), / 255.
V tex(const Tex& t, V2 uv) {
  if (t.type != NR_TEXTURE_IMAGE) return t.rgb;
  const float inv = 1.0f / fmaxf(1e-8f, t.scale);  // FMIN (core/constants.h:9)
  float su = fmodf(uv.x * inv, 1.0f), sv = fmodf(uv.y * inv, 1.0f);
  float u = su < 0.0f ? 0.0f : (su > 1.0f ? 1.0f : su);
  float v = 1.0f - (sv < 0.0f ? 0.0f : (sv > 1.0f ? 1.0f : sv));
  int i = (int)(u * (float)t.W);
  if (i >= (int)t.W) i = (int)t.W - 1;
  int j = (int)(v * (float)t.H);
  if (j >= (int)t.H) j = (int)t.H - 1;
  const size_t px = (size_t)j * t.W + i, hw = (size_t)t.H * t.W;
  const float k = 1.0f / 255.0f;  // Color / 255.0f multiplies by the reciprocal (core/vector.h:251-253)
  return V{(float)t.img[px] * k, (float)t.img[hw + px] * k, (float)t.img[2 * hw + px] * k};
}

struct ONB {
  V u, v, w;
};
ONB onb(V n) {  // core/onb.h
  ONB b;
  b.w = normalize(n);
  V a = (fabsf(b.w.x) > 0.9f) ? V{0.0f, 1.0f, 0.0f} : V{1.0f, 0.0f, 0.0f};
  b.v = normalize(cross(b.w, a));
  b.u = cross(b.w, b.v);
  return b;
}
inline V onb_t(const ONB& b, V v) { return (v.x * b.u) + (v.y * b.v) + (v.z * b.w); }

float ggx_d(float ndh, float alpha) {
  float a2 = alpha * alpha;
  float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
  return a2 / fmaxf(PI * d * d, 1e-8f);
}
float g1(float ndx, float alpha) {
  float a2 = alpha * alpha;
  return 2.0f * ndx / (ndx + sqrtf(a2 + (1.0f - a2) * ndx * ndx));
}

V cosine_dir(Rng& g) {  // vector.h:509-519
  float r1 = g.random_float();
  float r2 = g.random_float();
  float phi = PI2 * r1;
  float x = cosf(phi) * sqrtf(r2);
  float y = sinf(phi) * sqrtf(r2);
  float z = sqrtf(1.0f - r2);
  return V{x, y, z};
}
V unit_vector(Rng& g, bool rtl) {  // vector.h:489-496
  while (true) {
    float a = g.random_float(-1.0f, 1.0f);
    float b = g.random_float(-1.0f, 1.0f);
    float c = g.random_float(-1.0f, 1.0f);
    V p = rtl ? V{c, b, a} : V{a, b, c};
    float l = lsq(p);
    if (1e-160 < (double)l && l <= 1) return p / sqrtf(l);
  }
}

struct Pdf {
  int kind = 1;  // 0 cosine, 1 sphere, 5 pbr
  ONB uvw;
  V view;
  float alpha = 0, spec = 0;
};
float pdf_value(const Pdf& p, V d) {
  if (p.kind == 0) return fmaxf(0.0f, dot(normalize(d), p.uvw.w) / PI);
  if (p.kind == 1) return 1.0f / PI4;
  float diffuse = fmaxf(0.0f, dot(normalize(d), p.uvw.w) / PI);
  V hv = normalize(p.view + d);
  float ndh = fmaxf(dot(p.uvw.w, hv), 0.0f);
  float vdh = fmaxf(dot(p.view, hv), 1e-4f);
  float specular = (ggx_d(ndh, p.alpha) * ndh) / (4.0f * vdh);
  return (1.0f - p.spec) * diffuse + p.spec * specular;
}
V pdf_gen(const Pdf& p, Rng& g, bool rtl) {
  if (p.kind == 0) return onb_t(p.uvw, cosine_dir(g));
  if (p.kind == 1) return unit_vector(g, rtl);
  if (g.random_float() < p.spec) {
    float u1 = g.random_float();
    float u2 = g.random_float();
    float ct = sqrtf((1.0f - u1) / (1.0f + (p.alpha * p.alpha - 1.0f) * u1));
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float phi = PI2 * u2;
    V hv = onb_t(p.uvw, V{st * cosf(phi), st * sinf(phi), ct});
    return normalize(2.0f * dot(p.view, hv) * hv - p.view);
  }
  return onb_t(p.uvw, cosine_dir(g));
}

float light_pdf(const Scene& S, V origin, V dir) {  // primitives.h:44-59, shapes.h:60-70
  const Obj& o = S.objs[S.light];
  int t = o.type == NR_HITTABLE_OBJECT_LIGHT ? o.wtype : o.type;
  if (t == NR_HITTABLE_QUAD) {
    Hit h;
    Ray wr = mkray(origin, dir);
    Ray r = to_object(o.x, wr);
    bool hit = quad_hit(r, EPS, FMAX, h);
    to_world(h, o.x, r, wr, true);
    if (!hit) return 0.0f;
    float d2 = h.t * h.t * lsq(dir);
    float cosine = fabsf(dot(dir, h.n) / len(dir));
    if (cosine < 1e-8f) return 0.0f;
    float world_area = quadc().area * o.x.scale.x * o.x.scale.z;
    return d2 / (cosine * world_area);
  }
  if (t == NR_HITTABLE_SPHERE) {
    Hit h;
    if (!sphere_hit(mkray(origin, dir), EPS, FMAX, o.radius, o.x.scale, h)) return 0.0f;
    float rad_sq = o.radius * o.radius;
    float d2 = lsq(o.x.pos - origin);
    float ctm = sqrtf(1.0f - rad_sq / d2);
    float solid = PI2 * (1.0f - ctm);
    return 1.0f / solid;
  }
  return 0.0f;
}
V light_random(const Scene& S, V origin, Rng& g, bool rtl) {  // primitives.h:61-70, shapes.h:72-84
  const Obj& o = S.objs[S.light];
  int t = o.type == NR_HITTABLE_OBJECT_LIGHT ? o.wtype : o.type;
  if (t == NR_HITTABLE_QUAD) {
    const QuadC& q = quadc();
    float first = g.random_float();
    float second = g.random_float();
    float ra = rtl ? second : first, rb = rtl ? first : second;
    V corner = (-0.5f * q.u) - (0.5f * q.v);
    V p = corner + (ra * q.u) + (rb * q.v);
    p = mul(o.x.R, p * o.x.scale) + o.x.pos;
    return p - origin;
  }
  if (t == NR_HITTABLE_SPHERE) {
    V dir = o.x.pos - origin;
    float d2 = lsq(dir);
    ONB b = onb(dir);
    float r1 = g.random_float();
    float r2 = g.random_float();
    float rad_sq = o.radius * o.radius;
    float z = 1.0f + r2 * (sqrtf(1.0f - rad_sq / d2) - 1.0f);
    float phi = PI2 * r1;
    float x = cosf(phi) * sqrtf(1.0f - z * z);
    float y = sinf(phi) * sqrtf(1.0f - z * z);
    return onb_t(b, V{x, y, z});
  }
  if (t == NR_HITTABLE_MESH) return V{0.0f, 0.0f, 0.0f};
  return V{1.0f, 0.0f, 0.0f};
}

V pbr_normal(const Mat& m, const Hit& h) {  // material.h:113-125
  V tn = tex(m.tex[4], h.uv);
  V map = normalize(V{tn.x * 2.0f - 1.0f, tn.y * 2.0f - 1.0f, tn.z * 2.0f - 1.0f});
  V t = normalize(h.tangent - h.n * dot(h.tangent, h.n));
  V b = cross(h.n, t);
  return normalize(t * map.x + b * map.y + h.n * map.z);
}
V emitted(const Mat& m, const Hit& h) {
  if (m.type == NR_MATERIAL_PBR) return h.front_face ? tex(m.tex[3], h.uv) : V{0, 0, 0};
  if (m.type == NR_MATERIAL_EMISSIVE) return h.front_face ? tex(m.tex[0], h.uv) * m.brightness : V{0, 0, 0};
  return V{0, 0, 0};
}
float reflectance(float c, float ri) {
  float r0 = (1.0f - ri) / (1.0f + ri);
  r0 = r0 * r0;
  return r0 + (1.0f - r0) * powf((1.0f - c), 5.0f);
}
struct Scat {
  V atten;
  Pdf pdf;
  bool skip;
  V dir;
};
bool scatter(const Mat& m, const Hit& h, const Ray& ray, Scat& s, Rng& g) {
  switch (m.type) {
    case NR_MATERIAL_LAMBERTIAN:
      s.atten = tex(m.tex[0], h.uv);
      s.pdf.kind = 0;
      s.pdf.uvw = onb(h.n);
      s.skip = false;
      return true;
    case NR_MATERIAL_PBR: {
      V n = pbr_normal(m, h);
      V albedo = tex(m.tex[0], h.uv);
      float metallic = tex(m.tex[2], h.uv).x;
      V F0 = V{0.04f, 0.04f, 0.04f} * (1.0f - metallic) + albedo * metallic;
      float spec = fminf(0.9f, fmaxf(0.1f, fmaxf(F0.x, fmaxf(F0.y, F0.z))));
      s.atten = V{1, 1, 1};
      s.skip = false;
      s.pdf.kind = 5;
      s.pdf.uvw = onb(n);
      s.pdf.view = normalize(-ray.d);
      float rough = tex(m.tex[1], h.uv).x;
      s.pdf.alpha = fmaxf(rough * rough, 1e-3f);
      s.pdf.spec = spec;
      return true;
    }
    case NR_MATERIAL_DIELECTRIC: {
      s.atten = m.tint;
      s.skip = true;
      float ri = h.front_face ? (1.0f / m.ior) : m.ior;
      V unit = normalize(ray.d);
      float ct = fminf(dot(-unit, h.n), 1.0f);
      float st = sqrtf(1.0f - ct * ct);
      bool cannot = (double)(ri * st) > 1.0;
      if (cannot || reflectance(ct, ri) > g.uniform())
        s.dir = reflect(unit, h.n);
      else
        s.dir = refract(unit, h.n, ri);
      return true;
    }
    case NR_MATERIAL_ISOTROPIC:
      s.atten = tex(m.tex[0], h.uv);
      s.pdf.kind = 1;
      s.skip = false;
      return true;
  }
  return false;
}
V evaluate(const Mat& m, const Hit& h, V view, V light) {
  if (m.type == NR_MATERIAL_LAMBERTIAN) {
    float ct = dot(h.n, normalize(light));
    if (ct <= 0.0f) return V{0, 0, 0};
    return tex(m.tex[0], h.uv) * (ct / PI);
  }
  if (m.type == NR_MATERIAL_PBR) {
    V n = pbr_normal(m, h);
    float ndl = dot(n, light), ndv = dot(n, view);
    if (ndl <= 0.0f || ndv <= 0.0f) return V{0, 0, 0};
    V albedo = tex(m.tex[0], h.uv);
    float rough = tex(m.tex[1], h.uv).x, metallic = tex(m.tex[2], h.uv).x;
    float alpha = fmaxf(rough * rough, 1e-3f);
    V hv = normalize(view + light);
    float ndh = fmaxf(dot(n, hv), 0.0f), vdh = fmaxf(dot(view, hv), 0.0f);
    V F0 = V{0.04f, 0.04f, 0.04f} * (1.0f - metallic) + albedo * metallic;
    V F = F0 + (V{1, 1, 1} - F0) * powf(1.0f - vdh, 5.0f);
    float D = ggx_d(ndh, alpha);
    float G = g1(ndl, alpha) * g1(ndv, alpha);
    V spec = F * (D * G / fmaxf(4.0f * ndv * ndl, 1e-4f));
    V diff = albedo * (1.0f - metallic) * (1.0f / PI);
    return (diff + spec) * ndl;
  }
  if (m.type == NR_MATERIAL_ISOTROPIC) return tex(m.tex[0], h.uv) * (1.0f / PI4);
  return V{0, 0, 0};
}

// ---- sky (light/include/skylight.h) ------------------------------------------
V sky(const Scene& S, const Ray& r) {
  if (S.sky_type == NR_SKY_SIMPLE) {
    float a = 0.5 * (r.d.y + 1.0);
    return (1.0 - a) * S.sky_start + a * S.sky_end;
  }
  if (S.sky_type == NR_SKY_HDRI) {
    if (!S.hdri) return V{0, 0, 0};
    M rot = ry(deg2rad(S.hrot));
    V d = mul(rot, normalize(r.d));
    float u = atan2f(d.z, d.x) / PI2 + 0.5f;
    float v = acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) / PI;
    float fx = u * (float)S.hW - 0.5f, fy = v * (float)S.hH - 0.5f;
    int x0 = (int)floorf(fx), y0 = (int)floorf(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    float tx = fx - (float)x0, ty = fy - (float)y0;
    x0 = ((x0 % S.hW) + S.hW) % S.hW;
    x1 = ((x1 % S.hW) + S.hW) % S.hW;
    y0 = (int)fmaxf(0, fminf(S.hH - 1, y0));
    y1 = (int)fmaxf(0, fminf(S.hH - 1, y1));
    size_t hw = (size_t)S.hH * S.hW;
    auto texel = [&](int x, int y) {
      size_t i = (size_t)y * S.hW + x;
      return V{S.hdri[i], S.hdri[hw + i], S.hdri[2 * hw + i]};
    };
    V c00 = texel(x0, y0), c10 = texel(x1, y0), c01 = texel(x0, y1), c11 = texel(x1, y1);
    V top = c00 * (1.0f - tx) + c10 * tx;
    V bottom = c01 * (1.0f - tx) + c11 * tx;
    return (top * (1.0f - ty) + bottom * ty) * S.hint;
  }
  return V{0, 0, 0};
}

// ---- camera (engine/include/engine/camera.h) ---------------------------------
struct Cam {
  float rx, ry;
  V pos;
  M R;
  float uvw_x, uvw_y, focal, focus, shutter, dangle, dradius;
  uint32_t W, H;
  std::vector<V2> pattern;
};

std::vector<V2> n_rooks(uint32_t n, uint32_t seed, bool rtl) {  // camera.h:45-61
  std::vector<uint32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937 rng(seed);
  std::shuffle(perm.begin(), perm.end(), rng);
  std::uniform_real_distribution<float> jitter(0.0f, 1.0f);
  std::vector<V2> out(n);
  for (uint32_t i = 0; i < n; ++i) {
    float ja = jitter(rng);
    float jb = jitter(rng);
    float jx = rtl ? jb : ja, jy = rtl ? ja : jb;
    out[i] = V2{(i + jx) / (float)n, (perm[i] + jy) / (float)n};
  }
  return out;
}

Cam make_cam(const nr_camera_desc& c, uint32_t seed) {  // camera.h:124-136, 176-178
  Cam k;
  k.rx = c.resolution[0];
  k.ry = c.resolution[1];
  k.pos = V{c.position[0], c.position[1], c.position[2]};
  k.R = euler_deg(V{c.rotation[0], c.rotation[1], c.rotation[2]});
  k.shutter = 1.0f / (c.shutter_speed + FMIN);
  float ar = c.aperture / 2.0f;
  k.dangle = 2.0f * atanf(ar / (c.focus_distance + FMIN));
  k.dradius = c.focus_distance * tanf(k.dangle / 2.0f);
  float aspect = c.resolution[1] / c.resolution[0];
  k.uvw_x = c.sensor_width;
  k.uvw_y = -c.sensor_width * aspect;
  k.focal = c.focal_length;
  k.focus = c.focus_distance;
  k.H = (uint32_t)c.resolution[0];
  k.W = (uint32_t)c.resolution[1];
  k.pattern = n_rooks(c.samples_per_pixel, seed, true);
  return k;
}

Ray cam_ray(const Cam& c, uint32_t x, uint32_t y, uint32_t pix, uint32_t s, uint32_t seed, Rng& g, bool rtl) {
  V2 base = c.pattern[s];
  V2 shift = pcg_vector2((float)pix, seed);
  V2 off{fmodf(base.x + shift.x, 1.0f) - 0.5f, fmodf(base.y + shift.y, 1.0f) - 0.5f};
  float u = ((float)x + off.x - (c.rx - 1.0f) * 0.5f) * (c.uvw_x / c.rx);
  float v = ((float)y + off.y - (c.ry - 1.0f) * 0.5f) * (c.uvw_y / c.ry);
  float w = -c.focal;
  V center = mul(c.R, V{u, v, w});
  float fs = c.focus / c.focal;
  V focus_point = c.pos + center * fs;
  V origin;
  if (c.dangle <= 0.0f) {
    origin = c.pos;
  } else {
    V du = V{c.R.m[0][0], c.R.m[1][0], c.R.m[2][0]} * c.dradius;
    V dv = V{c.R.m[0][1], c.R.m[1][1], c.R.m[2][1]} * c.dradius;
    V2 loc;
    while (true) {
      float a = g.random_float(-1.0f, 1.0f);
      float b = g.random_float(-1.0f, 1.0f);
      loc = rtl ? V2{b, a} : V2{a, b};
      if (loc.x * loc.x + loc.y * loc.y < 1.0f) break;
    }
    origin = c.pos + (loc.x * du + loc.y * dv);
  }
  float time = c.shutter > 0.0f ? g.uniform() * c.shutter : 0.0f;
  return mkray(origin, normalize(focus_point - origin), time);
}


// ---- file readers (mesh.h:39-141 via tinyobjloader; texture.h:28-47 via
// stbi_loadf). Triangles and quads only for OBJ; Radiance RGBE for HDR.
struct ObjOut {
  std::vector<float> P, N, T, UV;
  std::vector<uint32_t> tris;
};
bool read_obj(const char* path, ObjOut& o) {
  std::ifstream f(path);
  if (!f) return false;
  std::vector<float> vp, vn, vt;
  struct C3 {
    int v, t, n;
  };
  std::vector<C3> corners;
  std::string line;
  while (std::getline(f, line)) {
    const char* s = line.c_str();
    while (*s == ' ' || *s == '\t') ++s;
    char* e;
    if (s[0] == 'v' && s[1] == ' ') {
      float a = strtof(s + 2, &e), b = strtof(e, &e), c = strtof(e, &e);
      vp.insert(vp.end(), {a, b, c});
    } else if (s[0] == 'v' && s[1] == 'n' && s[2] == ' ') {
      float a = strtof(s + 3, &e), b = strtof(e, &e), c = strtof(e, &e);
      vn.insert(vn.end(), {a, b, c});
    } else if (s[0] == 'v' && s[1] == 't' && s[2] == ' ') {
      float a = strtof(s + 3, &e), b = strtof(e, &e);
      vt.insert(vt.end(), {a, b});
    } else if (s[0] == 'f' && s[1] == ' ') {
      std::vector<C3> poly;
      const char* p = s + 2;
      while (*p) {
        while (*p == ' ' || *p == '\t') ++p;
        if (!*p || *p == '\r') break;
        long a = strtol(p, &e, 10), b = 0, c = 0;
        p = e;
        if (*p == '/') {
          ++p;
          if (*p != '/') { b = strtol(p, &e, 10); p = e; }
          if (*p == '/') { ++p; c = strtol(p, &e, 10); p = e; }
        }
        auto res = [](long i, size_t n) { return i > 0 ? (int)(i - 1) : (i < 0 ? (int)((long)n + i) : -1); };
        poly.push_back(C3{res(a, vp.size() / 3), b ? res(b, vt.size() / 2) : -1, c ? res(c, vn.size() / 3) : -1});
        while (*p && *p != ' ' && *p != '\t') ++p;
      }
      if (poly.size() == 4) {
        auto q = [&](int i, int k) { return vp[3 * (size_t)poly[i].v + k]; };
        float a0 = q(2, 0) - q(0, 0), a1 = q(2, 1) - q(0, 1), a2 = q(2, 2) - q(0, 2);
        float b0 = q(3, 0) - q(1, 0), b1 = q(3, 1) - q(1, 1), b2 = q(3, 2) - q(1, 2);
        float s02 = a0 * a0 + a1 * a1 + a2 * a2, s13 = b0 * b0 + b1 * b1 + b2 * b2;
        const int A[6] = {0, 1, 2, 0, 2, 3}, B[6] = {0, 1, 3, 1, 2, 3};
        for (int k = 0; k < 6; ++k) corners.push_back(poly[s02 < s13 ? A[k] : B[k]]);
      } else {
        for (size_t k = 2; k < poly.size(); ++k) corners.insert(corners.end(), {poly[0], poly[k - 1], poly[k]});
      }
    }
  }
  struct KH {
    size_t operator()(const std::tuple<int, int, int>& k) const {
      return std::get<0>(k) * 73856093u ^ std::get<1>(k) * 19349663u ^ std::get<2>(k) * 83492791u;
    }
  };
  std::unordered_map<std::tuple<int, int, int>, uint32_t, KH> uniq;
  std::vector<V> P, N, T;
  std::vector<V2> UV;
  for (const C3& c : corners) {
    auto key = std::make_tuple(c.v, c.t, c.n);
    auto it = uniq.find(key);
    if (it != uniq.end()) { o.tris.push_back(it->second); continue; }
    uint32_t id = (uint32_t)P.size();
    P.push_back(V{vp[3 * c.v], vp[3 * c.v + 1], vp[3 * c.v + 2]});
    N.push_back(c.n >= 0 ? V{vn[3 * c.n], vn[3 * c.n + 1], vn[3 * c.n + 2]} : V{0, 0, 0});
    UV.push_back(c.t >= 0 ? V2{vt[2 * c.t], vt[2 * c.t + 1]} : V2{0, 0});
    T.push_back(V{0, 0, 0});
    uniq.emplace(key, id);
    o.tris.push_back(id);
  }
  size_t nt = o.tris.size() / 3;
  if (vn.empty()) {
    for (size_t t = 0; t < nt; ++t) {
      uint32_t a = o.tris[3 * t], b = o.tris[3 * t + 1], c = o.tris[3 * t + 2];
      V fn = normalize(cross(P[b] - P[a], P[c] - P[a]));
      N[a] = N[a] + fn; N[b] = N[b] + fn; N[c] = N[c] + fn;
    }
    for (V& n : N) n = near_zero(n) ? V{0, 1, 0} : normalize(n);
  }
  for (size_t t = 0; t < nt; ++t) {
    uint32_t a = o.tris[3 * t], b = o.tris[3 * t + 1], c = o.tris[3 * t + 2];
    V e1 = P[b] - P[a], e2 = P[c] - P[a];
    V2 d1{UV[b].x - UV[a].x, UV[b].y - UV[a].y}, d2{UV[c].x - UV[a].x, UV[c].y - UV[a].y};
    float den = d1.x * d2.y - d2.x * d1.y;
    V tg = fabsf(den) < FMIN ? V{1, 0, 0} : (e1 * d2.y - e2 * d1.y) * (1.0f / den);
    T[a] = T[a] + tg; T[b] = T[b] + tg; T[c] = T[c] + tg;
  }
  for (size_t i = 0; i < T.size(); ++i) {
    V t = T[i] - N[i] * dot(T[i], N[i]);
    T[i] = near_zero(t) ? V{1, 0, 0} : normalize(t);
  }
  for (size_t i = 0; i < P.size(); ++i) {
    o.P.insert(o.P.end(), {P[i].x, P[i].y, P[i].z});
    o.N.insert(o.N.end(), {N[i].x, N[i].y, N[i].z});
    o.T.insert(o.T.end(), {T[i].x, T[i].y, T[i].z});
    o.UV.insert(o.UV.end(), {UV[i].x, UV[i].y});
  }
  return true;
}

bool read_hdr(const char* path, std::vector<float>& chw, uint32_t& H, uint32_t& W) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  std::vector<uint8_t> d;
  uint8_t buf[65536];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) d.insert(d.end(), buf, buf + n);
  fclose(f);
  size_t pos = 0;
  auto line = [&]() {
    std::string l;
    while (pos < d.size() && d[pos] != '\n') l.push_back((char)d[pos++]);
    ++pos;
    return l;
  };
  if (line().compare(0, 2, "#?") != 0) return false;
  while (pos < d.size() && !line().empty()) {}
  int h = 0, w = 0;
  if (sscanf(line().c_str(), "-Y %d +X %d", &h, &w) != 2) return false;
  H = (uint32_t)h;
  W = (uint32_t)w;
  size_t hw = (size_t)h * w;
  chw.assign(3 * hw, 0.0f);
  std::vector<uint8_t> sc((size_t)w * 4);
  auto put = [&](size_t i, const uint8_t* e) {
    float f1 = e[3] ? (float)ldexp(1.0f, (int)e[3] - 136) : 0.0f;
    chw[i] = e[3] ? e[0] * f1 : 0.0f;
    chw[hw + i] = e[3] ? e[1] * f1 : 0.0f;
    chw[2 * hw + i] = e[3] ? e[2] * f1 : 0.0f;
  };
  for (int y = 0; y < h; ++y) {
    bool rle = w >= 8 && w < 32768 && pos + 4 <= d.size() && d[pos] == 2 && d[pos + 1] == 2 &&
               ((d[pos + 2] << 8) | d[pos + 3]) == w;
    if (!rle) {
      for (; y < h; ++y)
        for (int x = 0; x < w; ++x, pos += 4) put((size_t)y * w + x, &d[pos]);
      break;
    }
    pos += 4;
    for (int c = 0; c < 4; ++c)
      for (int x = 0; x < w;) {
        int cnt = d[pos++];
        if (cnt > 128) {
          cnt -= 128;
          uint8_t v = d[pos++];
          while (cnt--) sc[(size_t)(x++) * 4 + c] = v;
        } else {
          while (cnt--) sc[(size_t)(x++) * 4 + c] = d[pos++];
        }
      }
    for (int x = 0; x < w; ++x) put((size_t)y * w + x, &sc[(size_t)x * 4]);
  }
  return true;
}


// display transform (data/src/stream.cu:7-159): white balance, tonemap,
// sqrt gamma, then NaN->0, clamp, *255 and truncation to uint8
V kelvin_rgb(float kelvin) {
  float temp = kelvin / 100.0f, r, g, b;
  if (temp <= 66.0f) {
    r = 255.0f;
    g = 99.4708025861f * logf(temp) - 161.1195681661f;
  } else {
    r = 329.698727446f * powf(temp - 60.0f, -0.1332047592f);
    g = 288.1221695283f * powf(temp - 60.0f, -0.0755148492f);
  }
  if (temp >= 66.0f) b = 255.0f;
  else if (temp <= 19.0f) b = 0.0f;
  else b = 138.5177312231f * logf(temp - 10.0f) - 305.0447927307f;
  return V{fminf(1.0f, fmaxf(0.0f, r / 255.0f)), fminf(1.0f, fmaxf(0.0f, g / 255.0f)),
           fminf(1.0f, fmaxf(0.0f, b / 255.0f))};
}
V display_pixel(V c, const nr_stream_config& cfg) {
  if (cfg.apply_white_balance) {
    V ref = kelvin_rgb(6500.0f);
    V tgt = kelvin_rgb(fmaxf(1000.0f, fminf(cfg.wb_temperature, 40000.0f)));
    V ratio{tgt.x / fmaxf(ref.x, 1e-4f), tgt.y / fmaxf(ref.y, 1e-4f), tgt.z / fmaxf(ref.z, 1e-4f)};
    c = c * ratio;
    float tint = cfg.wb_tint * 0.0025f;
    c = V{c.x * (1.0f + tint * 0.5f), c.y * (1.0f - tint), c.z * (1.0f + tint * 0.5f)};
  }
  if (cfg.apply_tonemapping) {
    V col = c;
    if (cfg.tm_method == 1) {
      float iw2 = 1.0f / (cfg.tm_white_point * cfg.tm_white_point);
      V num = col * (V{1, 1, 1} + col * iw2);
      col = num / (V{1, 1, 1} + col);
    } else if (cfg.tm_method == 2) {
      V num = col * (col * 2.51f + 0.03f);
      V den = col * (col * 2.43f + 0.59f) + 0.14f;
      col = V{fminf(1.0f, fmaxf(0.0f, num.x / den.x)), fminf(1.0f, fmaxf(0.0f, num.y / den.y)),
              fminf(1.0f, fmaxf(0.0f, num.z / den.z))};
    }
    float a = cfg.tm_alpha;
    c = ((1.0f - a) * c + a * col);
    c = V{fminf(1.0f, fmaxf(0.0f, c.x)), fminf(1.0f, fmaxf(0.0f, c.y)), fminf(1.0f, fmaxf(0.0f, c.z))};
  }
  if (cfg.linear_to_gamma)
    c = V{c.x > 0.0f ? sqrtf(c.x) : 0.0f, c.y > 0.0f ? sqrtf(c.y) : 0.0f, c.z > 0.0f ? sqrtf(c.z) : 0.0f};
  return c;
}

// ---- integrator (engine/src/trace.cu:11-79, engine/src/brdf.cu:4-35) --------
struct Sample {
  V beauty{0, 0, 0}, diffuse{0, 0, 0}, normal{0, 0, 0};
  uint32_t primary = 0xffffffffu;
};

Sample trace(const Scene& S, const Cam& c, const nr_render_config& cfg, uint32_t x, uint32_t y,
             uint32_t sample) {
  Sample out;
  uint32_t pix = y * c.W + x;
  V atten{1, 1, 1};
  Rng g{cfg.seed, pix + sample * (c.W * c.H)};
  Ray ray = cam_ray(c, x, y, pix, sample, cfg.seed, g, S.rtl);
  for (uint32_t bounce = 0; bounce < cfg.ray_depth; ++bounce) {
    Hit rec;
    bool hit = scene_hit(S, ray, rec);
    if (bounce == 0 && hit) {
      uint32_t oid = (uint32_t)S.objs[rec.obj].id;
      out.primary = (oid << 22) | (rec.prim == 0xffffffffu ? 0u : ((rec.prim + 1u) & 0x3fffffu));
    }
    if (!hit) {
      out.beauty = out.beauty + atten * sky(S, ray);
      break;
    }
    const Mat& m = S.mats[rec.mat];
    Ray r_in = ray;
    out.beauty = out.beauty + atten * emitted(m, rec);
    Scat s;
    if (!scatter(m, rec, ray, s, g)) break;
    if (s.skip) {
      atten = atten * s.atten;
      ray = mkray(rec.p, s.dir, ray.tm);
    } else {
      V dir;
      float pv;
      if (S.light >= 0) {
        if (g.random_float() < 0.5f) dir = pdf_gen(s.pdf, g, S.rtl);
        else dir = light_random(S, rec.p, g, S.rtl);
        pv = 0.5f * pdf_value(s.pdf, dir) + 0.5f * light_pdf(S, rec.p, dir);
      } else {
        dir = pdf_gen(s.pdf, g, S.rtl);
        pv = pdf_value(s.pdf, dir);
      }
      if (pv <= 0.0f) break;
      ray = mkray(rec.p, dir, r_in.tm);
      V brdf = evaluate(m, rec, normalize(-r_in.d), dir);
      atten = atten * (brdf / pv);
    }
    if (bounce == 0) {
      out.diffuse = out.diffuse + atten;
      out.normal = out.normal + rec.n;
    }
    if (cfg.rr_enabled && bounce >= cfg.rr_start_bounce) {
      float surv = fmaxf(atten.x, fmaxf(atten.y, atten.z));
      surv = fminf(surv, cfg.rr_survival);
      if (g.uniform() > surv) break;
      atten = atten * V{1.0f / surv, 1.0f / surv, 1.0f / surv};
    }
  }
  return out;
}

// ---- scene assembly (scene.cpp:68-76, registry.h:216-263) --------------------
bool build_scene(const or_scene* in, bool rtl, Scene& S) {
  S.rtl = rtl;
  S.mats.resize(in->n_materials);
  for (uint32_t i = 0; i < in->n_materials; ++i) {
    const nr_material_desc& d = in->materials[i];
    Mat& m = S.mats[i];
    m.type = d.type;
    m.ior = d.ior;
    m.brightness = d.brightness;
    m.tint = V{d.tint[0], d.tint[1], d.tint[2]};
    for (int k = 0; k < 5; ++k) {
      m.tex[k].type = d.tex[k].type;
      m.tex[k].rgb = V{d.tex[k].rgb[0], d.tex[k].rgb[1], d.tex[k].rgb[2]};
      if (d.tex[k].type == NR_TEXTURE_IMAGE) {
        if (d.tex[k].image < 0 || (uint32_t)d.tex[k].image >= in->n_images) return false;
        const or_image& im = in->images[d.tex[k].image];
        if (!im.chw || im.C < 3) return false;
        m.tex[k].img = im.chw;
        m.tex[k].H = im.H;
        m.tex[k].W = im.W;
        m.tex[k].scale = d.tex[k].scale;
      } else if (d.tex[k].type != NR_TEXTURE_CONSTANT) {
        return false;
      }
    }
  }
  const float P[6][3] = {{0, 0, 0.5f}, {0, 0, -0.5f}, {0.5f, 0, 0}, {-0.5f, 0, 0}, {0, 0.5f, 0}, {0, -0.5f, 0}};
  const float E[6][3] = {{90, 0, 0}, {-90, 0, 0}, {0, 0, -90}, {0, 0, 90}, {0, 0, 0}, {180, 0, 0}};
  for (int i = 0; i < 6; ++i)
    S.cube[i] = xform(V{P[i][0], P[i][1], P[i][2]}, V{E[i][0], E[i][1], E[i][2]}, V{1.0f, 1.0f, 1.0f});
  S.meshes.resize(in->n_meshes);
  for (uint32_t mi = 0; mi < in->n_meshes; ++mi) {
    const or_mesh& om = in->meshes[mi];
    Mesh& m = S.meshes[mi];
    m.pos.resize(om.n_vertices);
    m.nor.resize(om.n_vertices);
    m.tan.resize(om.n_vertices);
    m.uv.resize(om.n_vertices);
    for (uint32_t v = 0; v < om.n_vertices; ++v) {
      m.pos[v] = V{om.positions[3 * v], om.positions[3 * v + 1], om.positions[3 * v + 2]};
      m.nor[v] = V{om.normals[3 * v], om.normals[3 * v + 1], om.normals[3 * v + 2]};
      m.tan[v] = V{om.tangents[3 * v], om.tangents[3 * v + 1], om.tangents[3 * v + 2]};
      m.uv[v] = om.uvs ? V2{om.uvs[2 * v], om.uvs[2 * v + 1]} : V2{0, 0};
    }
    std::vector<Box> boxes(om.n_triangles);
    for (uint32_t t = 0; t < om.n_triangles; ++t) {  // Mesh::triangle_bbox (mesh.h:320-336)
      V a = m.pos[om.triangles[3 * t]], b = m.pos[om.triangles[3 * t + 1]], c = m.pos[om.triangles[3 * t + 2]];
      V mn{fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z))};
      V mx{fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z))};
      boxes[t] = make_box(mn, mx);
    }
    m.bvh.build(boxes);
    m.tri.resize(3 * (size_t)om.n_triangles);
    m.tri_id.resize(om.n_triangles);
    for (uint32_t k = 0; k < om.n_triangles; ++k) {
      uint32_t t = (uint32_t)m.bvh.order[k];
      m.tri_id[k] = t;
      for (int j = 0; j < 3; ++j) m.tri[3 * k + j] = om.triangles[3 * t + j];
    }
  }
  // objects in registry order, then reordered to the top-level leaf order
  std::vector<Obj> objs(in->n_objects);
  std::vector<Box> boxes(in->n_objects);
  for (uint32_t i = 0; i < in->n_objects; ++i) {
    const nr_object_desc& d = in->objects[i];
    Obj& o = objs[i];
    o.type = d.type;
    o.wtype = d.wrapped_type;
    int bt = (d.type == NR_HITTABLE_OBJECT_LIGHT || d.type == NR_HITTABLE_CONSTANT_MEDIUM) ? d.wrapped_type : d.type;
    V p{d.position[0], d.position[1], d.position[2]};
    o.x = bt == NR_HITTABLE_SPHERE ? xform_pos(p)
                                   : xform(p, V{d.rotation[0], d.rotation[1], d.rotation[2]},
                                           V{d.scale[0], d.scale[1], d.scale[2]});
    o.mat = d.material;
    o.mesh = d.mesh;
    o.radius = d.radius + FMIN;
    o.neg_inv_density = -1.0f / (d.density + FMIN);
    o.id = (int)i;
    Box lb;
    if (bt == NR_HITTABLE_SPHERE) {
      lb = make_box(V{-o.radius, -o.radius, -o.radius}, V{o.radius, o.radius, o.radius});
    } else if (bt == NR_HITTABLE_MESH) {  // Mesh::build_bbox (mesh.h:218-237)
      V mn{FMAX, FMAX, FMAX}, mx{-FMAX, -FMAX, -FMAX};
      for (const V& v : S.meshes[d.mesh].pos) {
        mn = V{fminf(mn.x, v.x), fminf(mn.y, v.y), fminf(mn.z, v.z)};
        mx = V{fmaxf(mx.x, v.x), fmaxf(mx.y, v.y), fmaxf(mx.z, v.z)};
      }
      lb = make_box(mn, mx);
    } else {
      lb = make_box(V{-0.5f, -0.5f, -0.5f}, V{0.5f, 0.5f, 0.5f});
    }
    boxes[i] = transformed(lb, o.x);
  }
  S.tlas.build(boxes);
  S.objs.resize(in->n_objects);
  for (uint32_t k = 0; k < in->n_objects; ++k) S.objs[k] = objs[S.tlas.order[k]];
  S.light = -1;
  for (uint32_t k = 0; k < in->n_objects; ++k)
    if (S.objs[k].type == NR_HITTABLE_OBJECT_LIGHT) {
      S.light = (int)k;
      break;
    }
  S.sky_type = in->sky_type;
  S.sky_start = V{in->sky_start[0], in->sky_start[1], in->sky_start[2]};
  S.sky_end = V{in->sky_end[0], in->sky_end[1], in->sky_end[2]};
  S.hdri = in->hdri;
  S.hC = (int)in->hdri_C;
  S.hH = (int)in->hdri_H;
  S.hW = (int)in->hdri_W;
  S.hrot = in->hdri_rotation;
  S.hint = in->hdri_intensity;
  return true;
}

void store(float* buf, size_t hw, size_t i, V v) {
  if (!buf) return;
  buf[i] = v.x;
  buf[hw + i] = v.y;
  buf[2 * hw + i] = v.z;
}
V load(const float* buf, size_t hw, size_t i) { return V{buf[i], buf[hw + i], buf[2 * hw + i]}; }
V running_mean(V avg, V s, uint32_t n) {  // data.cu:28-50
  float fn = (float)n;
  return avg * ((fn - 1.0f) / fn) + s * (1.0f / fn);
}

}  // namespace

// ---- viewport (engine/src/trace.cu:100-188, engine/src/axis_grid.cu,
// scene/src/scene_interface.cu:3-81) ---------------------------------------
float vp_saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
float vp_smoothstep(float a, float b, float x) {  // core/cg_std.h:98-103
  float t = vp_saturate((x - a) / (b - a));
  return t * t * (3.0f - (2.0f * t));
}
V vp_lerp(V x, V y, float w) { return x + w * (y - x); }  // core/cg_std.h:91-93
float vp_comp(V v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
float vp_grid_mask(float u, float v, float spacing, float width) {  // axis_grid.cu:4-9
  float du = fabsf(fmodf(u + spacing * 0.5f, spacing) - spacing * 0.5f);
  float dv = fabsf(fmodf(v + spacing * 0.5f, spacing) - spacing * 0.5f);
  return 1.0f - vp_smoothstep(0.0f, width, fminf(du, dv));
}
bool vp_axis_grid(const Ray& r, float max_t, int axis, V major, V& color, float& alpha) {
  float da = vp_comp(r.d, axis);  // axis_grid.cu:11-53
  if (fabsf(da) < 1e-6f) return false;
  float t = -vp_comp(r.o, axis) / da;
  if (t <= 0.0f || t >= max_t) return false;
  V p = r.o + t * r.d;
  p = V{fabsf(p.x), fabsf(p.y), fabsf(p.z)};
  float u = vp_comp(p, (axis + 1) % 3), v = vp_comp(p, (axis + 2) % 3);
  float pixel_size = 1e-3f * t;
  float level = fmaxf(log10f(fmaxf(pixel_size, 1e-5f)) + 1.0f, 0.0f);
  float level0 = floorf(level);
  float blend = level - level0;
  float s0 = powf(10.0f, level0), s1 = s0 * 10.0f;
  float width = pixel_size * 1.5f;
  float g0 = vp_grid_mask(u, v, s0, width), g1 = vp_grid_mask(u, v, s1, width);
  float mask = fmaxf(g0 * (1.0f - blend), g1);
  if (mask < 0.01f) return false;
  float fade = fmaxf(0.0f, 1.0f - t / 100.0f);
  color = vp_lerp(V{0.35f, 0.35f, 0.35f}, major, vp_smoothstep(0.0f, 1.0f, g1));
  alpha = mask * fade;
  return true;
}
bool vp_triplanar(const Ray& r, V& color, float& alpha) {  // axis_grid.cu:55-72
  return vp_axis_grid(r, FMAX, 0, V{1.0f, 0.3f, 0.3f}, color, alpha) ||
         vp_axis_grid(r, FMAX, 1, V{0.3f, 1.0f, 0.3f}, color, alpha) ||
         vp_axis_grid(r, FMAX, 2, V{0.3f, 0.3f, 1.0f}, color, alpha);
}
V vp_color(const Mat& m, V2 uv) {  // material.h viewport_color
  if (m.type == NR_MATERIAL_DIELECTRIC) return m.tint;
  if (m.type >= 1 && m.type <= 5) return tex(m.tex[0], uv);
  return V{0, 0, 0};
}
Ray vp_center_ray(const Cam& c, uint32_t x, uint32_t y) {  // camera.h:181-184
  V2 base = c.pattern[0];
  V2 shift = pcg_vector2(0.0f, 0u);
  V2 off{fmodf(base.x + shift.x, 1.0f) - 0.5f, fmodf(base.y + shift.y, 1.0f) - 0.5f};
  float u = ((float)x + off.x - (c.rx - 1.0f) * 0.5f) * (c.uvw_x / c.rx);
  float v = ((float)y + off.y - (c.ry - 1.0f) * 0.5f) * (c.uvw_y / c.ry);
  V center = mul(c.R, V{u, v, -c.focal});
  V focus_point = c.pos + center * (c.focus / c.focal);
  return mkray(c.pos, normalize(focus_point - c.pos));
}
Ray vp_screen_ray(const Cam& c, float su, float sv) {  // camera.h:215-227
  float x = su * c.rx, y = sv * c.ry;
  float u = (x - (c.rx - 1.0f) * 0.5f) * (c.uvw_x / c.rx);
  float v = (y - (c.ry - 1.0f) * 0.5f) * (c.uvw_y / c.ry);
  return mkray(c.pos, normalize(mul(c.R, V{u, v, -c.focal})));
}

extern "C" {

struct OracleHandle {
  Scene S;
};

void* oracle_scene_create(const or_scene* in, int32_t draw_rtl) {
  if (!in) return nullptr;
  OracleHandle* h = new OracleHandle();
  if (!build_scene(in, draw_rtl != 0, h->S)) {
    delete h;
    return nullptr;
  }
  return h;
}

void oracle_scene_destroy(void* h) { delete static_cast<OracleHandle*>(h); }

int oracle_scene_render(void* handle, const nr_camera_desc* cam, const nr_render_config* cfg,
                        const or_request* req) {
  if (!handle || !cam || !cfg || !req) return -1;
  const Scene& S = static_cast<OracleHandle*>(handle)->S;
  Cam c = make_cam(*cam, cfg->seed);
  uint32_t r0 = req->row_begin, r1 = std::min(req->row_end, c.H);
  size_t hw = (size_t)c.W * c.H;
  int nt = req->threads > 0 ? req->threads : (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) {
    pool.emplace_back([&, t]() {
      for (uint32_t y = r0 + t; y < r1; y += nt)
        for (uint32_t x = 0; x < c.W; ++x) {
          size_t i = (size_t)y * c.W + x;
          if (req->mode == 0) {
            Sample s = trace(S, c, *cfg, x, y, req->first);
            store(req->beauty, hw, i, s.beauty);
            store(req->diffuse, hw, i, s.diffuse);
            store(req->normal, hw, i, s.normal);
            if (req->primary) req->primary[i] = s.primary;
          } else {
            V ab = req->beauty ? load(req->beauty, hw, i) : V{0, 0, 0};
            V ad = req->diffuse ? load(req->diffuse, hw, i) : V{0, 0, 0};
            V an = req->normal ? load(req->normal, hw, i) : V{0, 0, 0};
            for (uint32_t k = 0; k < req->count; ++k) {
              uint32_t smp = req->first + k;
              Sample s = trace(S, c, *cfg, x, y, smp);
              ab = running_mean(ab, s.beauty, smp);
              ad = running_mean(ad, s.diffuse, smp);
              an = running_mean(an, s.normal, smp);
              if (req->beauty64) {
                req->beauty64[i] += (double)s.beauty.x;
                req->beauty64[hw + i] += (double)s.beauty.y;
                req->beauty64[2 * hw + i] += (double)s.beauty.z;
              }
            }
            store(req->beauty, hw, i, ab);
            store(req->diffuse, hw, i, ad);
            store(req->normal, hw, i, an);
          }
        }
    });
  }
  for (auto& th : pool) th.join();
  return 0;
}

// trace_viewport_kernel (trace.cu:100-162) into float CHW layers.
int oracle_scene_viewport(void* handle, const nr_camera_desc* cam, uint32_t seed,
                          int32_t show_axis_grid, float* beauty, float* diffuse, float* normal) {
  if (!handle || !cam) return -1;
  const Scene& S = static_cast<OracleHandle*>(handle)->S;
  Cam c = make_cam(*cam, seed);
  size_t hw = (size_t)c.W * c.H;
  for (uint32_t y = 0; y < c.H; ++y)
    for (uint32_t x = 0; x < c.W; ++x) {
      size_t i = (size_t)y * c.W + x;
      Ray ray = vp_center_ray(c, x, y);
      Hit rec;
      V b{0, 0, 0}, d{0, 0, 0}, n{0, 0, 0};
      if (!scene_hit(S, ray, rec)) {
        V sk = sky(S, ray), gc;
        float ga;
        b = (show_axis_grid && vp_triplanar(ray, gc, ga)) ? vp_lerp(sk, gc, ga) : sk;
      } else {
        V lv = c.pos - rec.p;
        float ld = len(lv);
        float head = dot(normalize(lv), rec.n) * 0.5f + 0.5f;
        head *= 1.0f / (ld * ld);
        head = fminf(0.75f, head);
        float dir = (dot(V{1.0f, 1.0f, 1.0f}, rec.n) + 1.0f) * 0.5f;
        dir = fmaxf(0.1f, dir);
        V col = vp_color(S.mats[S.objs[rec.obj].mat], rec.uv);
        b = col * fmaxf(head, dir);
        d = col;
        n = rec.n;
      }
      if (beauty) store(beauty, hw, i, b);
      if (diffuse) store(diffuse, hw, i, d);
      if (normal) store(normal, hw, i, n);
    }
  return 0;
}

// hit_test_ray_kernel (trace.cu:168-188)
int oracle_scene_pick(void* handle, const nr_camera_desc* cam, uint32_t seed, float u, float v,
                      nr_pick_result* out) {
  if (!handle || !cam || !out) return -1;
  const Scene& S = static_cast<OracleHandle*>(handle)->S;
  Cam c = make_cam(*cam, seed);
  Hit rec;
  memset(out, 0, sizeof(*out));
  out->hit = scene_hit(S, vp_screen_ray(c, u, v), rec) ? 1 : 0;
  if (out->hit) {
    out->object_id = (uint32_t)S.objs[rec.obj].id;
    out->material_id = (uint32_t)S.objs[rec.obj].mat;
    out->t = rec.t;
    out->p[0] = rec.p.x;
    out->p[1] = rec.p.y;
    out->p[2] = rec.p.z;
    out->n[0] = rec.n.x;
    out->n[1] = rec.n.y;
    out->n[2] = rec.n.z;
    out->uv[0] = rec.uv.x;
    out->uv[1] = rec.uv.y;
    out->front_face = rec.front_face ? 1 : 0;
  }
  return 0;
}

// mask_selected_kernel + build_outline_kernel (scene_interface.cu:3-52)
int oracle_scene_selection_mask(void* handle, const nr_camera_desc* cam, uint32_t seed,
                                uint32_t object_id, int32_t radius, uint8_t* out) {
  if (!handle || !cam || !out) return -1;
  const Scene& S = static_cast<OracleHandle*>(handle)->S;
  Cam c = make_cam(*cam, seed);
  const int W = (int)c.W, H = (int)c.H;
  std::vector<uint8_t> base((size_t)W * H);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      Hit rec;
      float su = ((float)x + 0.5f) / (float)W, sv = ((float)y + 0.5f) / (float)H;
      bool hit = scene_hit(S, vp_screen_ray(c, su, sv), rec);
      base[(size_t)y * W + x] = (hit && (uint32_t)S.objs[rec.obj].id == object_id) ? 255u : 0u;
    }
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      uint8_t v = 0;
      if (base[(size_t)y * W + x] == 0)
        for (int dy = -radius; dy <= radius && !v; ++dy)
          for (int dx = -radius; dx <= radius; ++dx) {
            int nx = x + dx, ny = y + dy;
            if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
            if (base[(size_t)ny * W + nx]) {
              v = 255u;
              break;
            }
          }
      out[(size_t)y * W + x] = v;
    }
  return 0;
}

int oracle_render(const or_scene* in, const nr_camera_desc* cam, const nr_render_config* cfg,
                  const or_request* req) {
  if (!in || !req) return -1;
  void* h = oracle_scene_create(in, req->draw_rtl);
  if (!h) return -2;
  int rc = oracle_scene_render(h, cam, cfg, req);
  oracle_scene_destroy(h);
  return rc;
}

double oracle_mesh_sah(const or_mesh* om, uint64_t* n_nodes) {
  std::vector<Box> boxes(om->n_triangles);
  for (uint32_t t = 0; t < om->n_triangles; ++t) {
    const float* p = om->positions;
    const uint32_t* tr = om->triangles + 3 * t;
    V a{p[3 * tr[0]], p[3 * tr[0] + 1], p[3 * tr[0] + 2]};
    V b{p[3 * tr[1]], p[3 * tr[1] + 1], p[3 * tr[1] + 2]};
    V c{p[3 * tr[2]], p[3 * tr[2] + 1], p[3 * tr[2] + 2]};
    V mn{fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z))};
    V mx{fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z))};
    boxes[t] = make_box(mn, mx);
  }
  Bvh b;
  b.build(boxes);
  if (n_nodes) *n_nodes = b.nodes.size();
  double root = area(b.nodes[0].bbox), acc = 0.0;
  for (const Node& n : b.nodes) acc += (n.object != -1 ? 1.0 : 1.0) * (double)area(n.bbox) / root;
  return acc;
}

int oracle_n_rooks(uint32_t n, uint32_t seed, int32_t rtl, float* out) {
  std::vector<V2> p = n_rooks(n, seed, rtl != 0);
  for (uint32_t i = 0; i < n; ++i) {
    out[2 * i] = p[i].x;
    out[2 * i + 1] = p[i].y;
  }
  return 0;
}

int oracle_uniforms(uint32_t seed, uint32_t sub, uint32_t count, float* out) {
  Rng g{seed, sub};
  for (uint32_t i = 0; i < count; ++i) out[i] = g.uniform();
  return 0;
}

int oracle_load_obj(const char* path, float* P, float* N, float* T, float* UV, uint32_t* tris,
                    uint32_t* nv, uint32_t* ntri, uint32_t cap_v, uint32_t cap_t) {
  ObjOut o;
  if (!read_obj(path, o)) return -1;
  *nv = (uint32_t)(o.P.size() / 3);
  *ntri = (uint32_t)(o.tris.size() / 3);
  if (*nv > cap_v || *ntri > cap_t) return 1;
  std::copy(o.P.begin(), o.P.end(), P);
  std::copy(o.N.begin(), o.N.end(), N);
  std::copy(o.T.begin(), o.T.end(), T);
  std::copy(o.UV.begin(), o.UV.end(), UV);
  std::copy(o.tris.begin(), o.tris.end(), tris);
  return 0;
}

int oracle_load_hdr(const char* path, float* chw, uint32_t* C, uint32_t* H, uint32_t* W, uint64_t cap) {
  std::vector<float> d;
  uint32_t h = 0, w = 0;
  if (!read_hdr(path, d, h, w)) return -1;
  *C = 3;
  *H = h;
  *W = w;
  if (d.size() > cap) return 1;
  std::copy(d.begin(), d.end(), chw);
  return 0;
}

int oracle_display(const float* chw, uint32_t hw, const nr_stream_config* cfg, uint8_t* out8,
                   float* outf) {
  for (size_t i = 0; i < hw; ++i) {
    V c = display_pixel(V{chw[i], chw[hw + i], chw[2 * hw + i]}, *cfg);
    if (outf) {
      outf[i] = c.x;
      outf[hw + i] = c.y;
      outf[2 * hw + i] = c.z;
    }
    float v[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) {
      float x = std::isnan(v[k]) ? 0.0f : v[k];
      x = fmaxf(0.0f, fminf(1.0f, x)) * 255.0f;
      if (out8) out8[k * (size_t)hw + i] = (uint8_t)x;
    }
  }
  return 0;
}

}  // extern "C"
