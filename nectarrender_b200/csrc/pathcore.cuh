// pathcore.cuh — device functions of the path tracer: rays, object
// intersection, the two-level BVH traversal, textures, materials, PDFs, sky
// and camera. Every function restates the reference's arithmetic in the same
// order (file:line cited per function) so that NR_MODE_REFERENCE reproduces
// its samples; the data they read is the flat layout of scene_device.cuh.
#pragma once
#include "rng.cuh"
#include "scene_device.cuh"

namespace nr {

// ---------------------------------------------------------------------------
// rays (nectar_render/csrc/engine/include/engine/ray.h:5-49)
struct Ray {
  V3 o, d, inv;
  float tm;
};
__device__ __forceinline__ Ray make_ray(const V3& o, const V3& d, float tm) {
  Ray r;
  r.o = o;
  r.d = d;
  r.inv = V3{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  r.tm = tm;
  return r;
}
// Ray::to_object_space (ray.h:33-37)
__device__ __forceinline__ Ray to_object(const DevObject& ob, const Ray& r) {
  V3 o = mul(ob.invR, r.o - ob.pos) * ob.inv_s;
  V3 d = mul(ob.invR, r.d) * ob.inv_s;
  return make_ray(o, d, r.tm);
}
__device__ __forceinline__ V3 ray_at(const Ray& r, float t) { return r.o + t * r.d; }

// Hit record (nectar_render/csrc/hittable/include/hittable/hit_record.h:9-22)
struct Hit {
  V3 p, n, tangent;
  V2 uv;
  float t;
  bool front_face;
  uint32_t obj;   // object slot (top-level leaf order)
  uint32_t prim;  // original triangle index or 0xffffffff
};

// HitRecord::to_world_space (hit_record.h:24-51)
__device__ __forceinline__ void to_world(Hit& h, const M3& R, const V3& pos, const V3& scale,
                                         const V3& inv_s, const Ray& object_ray,
                                         const Ray& world_ray, bool apply_bias) {
  h.p = mul(R, h.p * scale) + pos;
  h.tangent = normalize(mul(R, h.tangent * scale));
  h.front_face = dot(object_ray.d, h.n) < 0.0f;
  h.n = h.front_face ? h.n : -h.n;
  h.n = normalize(mul(R, h.n * inv_s));
  h.front_face = dot(world_ray.d, h.n) < 0.0f;
  h.n = h.front_face ? h.n : -h.n;
  h.tangent = normalize(h.tangent - h.n * dot(h.tangent, h.n));
  if (near_zero(h.tangent))
    h.tangent = normalize(cross(h.n, fabsf(h.n.x) > 0.9f ? V3{0.0f, 1.0f, 0.0f}
                                                          : V3{1.0f, 0.0f, 0.0f}));
  if (apply_bias) h.p += h.n * EPS;
  h.t = dot(h.p - world_ray.o, world_ray.d) / length_squared(world_ray.d);
}

// ---------------------------------------------------------------------------
// Quad: unit square in the y=0 plane, u=(1,0,0), v=(0,0,-1), normal (0,1,0)
// (nectar_render/csrc/hittable/include/hittable/primitives.h:3-88). With
// these constant vectors dot(normal, d) = d.y, dot(w, cross(p, v)) = p.x and
// dot(w, cross(u, p)) = -p.z exactly for finite inputs.
__device__ __forceinline__ bool quad_hit(const Ray& r, float tmin, float tmax, Hit& h) {
  float denom = r.d.y;
  if (fabsf(denom) < FMIN) return false;
  float t = -r.o.y / denom;
  if (!(tmin <= t && t <= tmax)) return false;  // Interval::contains
  h.t = t;
  h.p = ray_at(r, t);
  h.n = V3{0.0f, 1.0f, 0.0f};
  h.tangent = V3{1.0f, 0.0f, 0.0f};
  float a = h.p.x;
  float b = -h.p.z;
  h.uv = V2{a + 0.5f, b + 0.5f};
  return (-0.5f < a && a < 0.5f) & (-0.5f < b && b < 0.5f);  // surrounds
}

// Sphere centred at the object origin (shapes.h:5-58).
__device__ __forceinline__ bool sphere_hit(const Ray& r, float tmin, float tmax, float radius,
                                           const V3& scale, Hit& h) {
  V3 oc = -r.o;
  float a = length_squared(r.d);
  float hh = dot(r.d, oc);
  float c = length_squared(oc) - radius * radius;
  float disc = hh * hh - a * c;
  if (disc < 0) return false;
  float sq = sqrtf(disc);
  float root = (hh - sq) / a;
  if (!(tmin < root && root < tmax)) {
    root = (hh + sq) / a;
    if (!(tmin < root && root < tmax)) return false;
  }
  h.t = root;
  h.p = ray_at(r, root);
  V3 norm = h.p / ((scale * radius) + FMIN);
  h.n = norm;
  h.tangent = normalize(V3{-h.p.z, 0.0f, h.p.x});
  float theta = acosf(-norm.y);
  float phi = atan2f(-norm.z, norm.x) + PI;
  h.uv = V2{phi / PI2, theta / PI};
  return true;
}

// Cube = six quads with fixed face transforms (shapes.h:60-173). The face
// transforms are built on the device exactly as the reference's device-side
// Cube constructor does (init_device_constants in integrator.cu) and stored
// once per scene (DevScene::cube_faces).
__device__ __forceinline__ bool cube_hit(const CubeFace* faces, const Ray& r, float tmin,
                                         float tmax, Hit& h) {
  bool any = false;
  int hit_face = -1;
  Ray hit_ray;
  const V3 one = V3{1.0f, 1.0f, 1.0f};
  for (int i = 0; i < 6; ++i) {
    const CubeFace& f = faces[i];
    // to_object_space with unit scale (inv_s = 1/(1+FMIN+FMIN) = 1 in float)
    V3 o = mul(f.invR, r.o - f.pos) * one;
    V3 d = mul(f.invR, r.d) * one;
    Ray fr = make_ray(o, d, r.tm);
    Hit fh;
    if (quad_hit(fr, tmin, tmax, fh)) {
      any = true;
      hit_face = i;
      hit_ray = fr;
      h = fh;
      tmax = fh.t;
    }
  }
  if (any) {
    const CubeFace& f = faces[hit_face];
    to_world(h, f.R, f.pos, one, one, hit_ray, r, false);
  }
  return any;
}

// ---------------------------------------------------------------------------
// BVH box tests
__device__ __forceinline__ bool slab(float lox, float hix, float loy, float hiy, float loz,
                                     float hiz, const V3& oinv, const V3& inv, float tmin,
                                     float tmax, float& tnear) {
  float tx0 = fmaf(lox, inv.x, -oinv.x), tx1 = fmaf(hix, inv.x, -oinv.x);
  float ty0 = fmaf(loy, inv.y, -oinv.y), ty1 = fmaf(hiy, inv.y, -oinv.y);
  float tz0 = fmaf(loz, inv.z, -oinv.z), tz1 = fmaf(hiz, inv.z, -oinv.z);
  float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
  float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
  tnear = tn;
  return tn <= tf;
}

// Moller-Trumbore exactly as Mesh::intersect_triangle (mesh.h:338-365),
// with the edges precomputed in float (the same rounding as v1 - v0).
__device__ __forceinline__ bool tri_hit(const Ray& r, const V3& v0, const V3& e1, const V3& e2,
                                        float tmin, float tmax, float& ot, float& ou,
                                        float& ov) {
  V3 hv = cross(r.d, e2);
  float a = dot(e1, hv);
  if (fabsf(a) < FMIN) return false;
  float f = 1.0f / a;
  V3 s = r.o - v0;
  float u = f * dot(s, hv);
  if (u < 0.0f || u > 1.0f) return false;
  V3 q = cross(s, e1);
  float v = f * dot(r.d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = f * dot(e2, q);
  if (!(tmin <= t && t <= tmax)) return false;
  ot = t;
  ou = u;
  ov = v;
  return true;
}

struct TraceStats {
  uint32_t nodes, tris, objs;
};

#ifndef NR_STACK
#define NR_STACK 64
#endif
// Upper bound on traversal steps of one query; a well-formed tree needs far
// fewer. Reaching it sets error bit 8 and ends the query, so a corrupted tree
// can never keep a kernel spinning.
constexpr uint32_t kMaxTraversalSteps = 1u << 20;

// Closest triangle of a mesh in object space with Interval(tmin, tmax) and
// inclusive acceptance (mesh.h:239-292): returns the leaf-order triangle slot.
// Triangles flagged flat (an axis of zero extent) are skipped in reference
// mode: the reference's leaf box test can never pass for them (aabb.h:111-133).
__device__ __forceinline__ int mesh_closest_bvh2(const DevMesh& m, const Ray& r, float tmin,
                                                 float& tmax, float& bu, float& bv,
                                                 bool skip_flat, TraceStats& st,
                                                 uint32_t* err, uint32_t max_steps,
                                                 uint32_t stack_limit) {
  int best = -1;
  V3 oinv = r.o * r.inv;
  uint32_t stack[NR_STACK];
  const int cap = stack_limit < (uint32_t)NR_STACK ? (int)stack_limit : NR_STACK;
  int sp = 0;
  int cur = 0;
  if (m.n_bvh2 == 0) return -1;
  for (uint32_t steps = 0;; ++steps) {
    if (steps >= max_steps || (uint32_t)cur >= m.n_bvh2) {
      atomicOr(err, 8u);
      break;
    }
    const Bvh2Node* nd = m.bvh2 + cur;
    float4 A = __ldg(&nd->a), B = __ldg(&nd->b), C = __ldg(&nd->c);
    int4 D = __ldg(&nd->d);
    st.nodes++;
    float tn0, tn1;
    bool h0 = slab(A.x, A.y, A.z, A.w, C.x, C.y, oinv, r.inv, tmin, tmax, tn0);
    bool h1 = slab(B.x, B.y, B.z, B.w, C.z, C.w, oinv, r.inv, tmin, tmax, tn1);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      bool hc = c == 0 ? h0 : h1;
      int link = c == 0 ? D.x : D.y;
      int cnt = c == 0 ? D.z : D.w;
      if (hc && link < 0) {
        int first = ~link;
        for (int k = 0; k < cnt; ++k) {
          const TriRecord* tr = m.tris2 + first + k;
          float4 p0 = __ldg(&tr->v0), p1 = __ldg(&tr->e1), p2 = __ldg(&tr->e2);
          st.tris++;
          if (skip_flat && __float_as_uint(p1.w) != 0u) continue;
          float t, u, v;
          if (tri_hit(r, V3{p0.x, p0.y, p0.z}, V3{p1.x, p1.y, p1.z}, V3{p2.x, p2.y, p2.z}, tmin,
                      tmax, t, u, v)) {
            tmax = t;
            bu = u;
            bv = v;
            best = first + k;
          }
        }
        if (c == 0) h0 = false; else h1 = false;
      }
    }
    if (h0 && h1) {
      bool near0 = tn0 <= tn1;
      int nearl = near0 ? D.x : D.y, farl = near0 ? D.y : D.x;
      if (sp < cap) stack[sp++] = (uint32_t)farl;
      else atomicOr(err, 1u);
      cur = nearl;
    } else if (h0) {
      cur = D.x;
    } else if (h1) {
      cur = D.y;
    } else {
      if (sp == 0) break;
      cur = (int)stack[--sp];
    }
  }
  return best;
}

// ---- compressed 8-wide traversal (Ylitie, Karras, Laine 2017) ------------
__device__ __forceinline__ uint32_t extract_byte(uint32_t x, uint32_t i) {
  return (x >> (i * 8u)) & 0xffu;
}
// Byte i of x as a float, exactly (float)byte: the byte is placed in the
// mantissa of 2^23 (0x4B0000bb = 2^23 + b) and 2^23 is subtracted, which is
// exact for b < 2^23. One byte permute (integer pipe) and one add (FMA pipe)
// instead of a conversion (the narrow XU pipe). The box test converts the
// near-plane bytes one way and the far-plane bytes the other, so neither the
// XU nor the integer pipe saturates.
__device__ __forceinline__ float byte_to_float(uint32_t x, uint32_t i) {
  return __uint_as_float(__byte_perm(x, 0x4Bu, 0x4550u | i)) - 8388608.0f;
}
__device__ __forceinline__ uint32_t s8x4_mask(uint32_t x) {
  // x has only bit 7 of each byte possibly set; spread it to the whole byte
  uint32_t m = x & 0x80808080u;
  return (m >> 7) * 0xffu;
}

// Intersects the 8 children of a wide node; returns the hit mask in the
// compressed-BVH convention: bits 24..31 inner children (slot order xor the
// ray octant), bits 0..23 leaf primitives relative to the node's prim base.
__device__ __forceinline__ uint32_t bvh8_intersect(const Bvh8Node* nd, const V3& o,
                                                   const V3& inv, uint32_t oct_inv4,
                                                   float tmin, float tmax, float4& n0out,
                                                   uint4& n1out) {
  float4 n0 = __ldg(&nd->n0);
  uint4 n1 = __ldg(&nd->n1), n2 = __ldg(&nd->n2), n3 = __ldg(&nd->n3), n4 = __ldg(&nd->n4);
  n0out = n0;
  n1out = n1;
  uint32_t e = __float_as_uint(n0.w);
  float sx = __uint_as_float((e & 0xffu) << 23);
  float sy = __uint_as_float(((e >> 8) & 0xffu) << 23);
  float sz = __uint_as_float(((e >> 16) & 0xffu) << 23);
  float adx = sx * inv.x, ady = sy * inv.y, adz = sz * inv.z;
  float aox = (n0.x - o.x) * inv.x, aoy = (n0.y - o.y) * inv.y, aoz = (n0.z - o.z) * inv.z;
  uint32_t hitmask = 0u;
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    uint32_t meta4 = g == 0 ? n1.z : n1.w;
    uint32_t is_inner4 = (meta4 & (meta4 << 1)) & 0x10101010u;
    uint32_t inner_mask4 = s8x4_mask(is_inner4 << 3);
    uint32_t bit_index4 = (meta4 ^ (oct_inv4 & inner_mask4)) & 0x1f1f1f1fu;
    uint32_t child_bits4 = (meta4 >> 5) & 0x07070707u;
    uint32_t qlox = g == 0 ? n2.x : n2.y, qloy = g == 0 ? n2.z : n2.w;
    uint32_t qloz = g == 0 ? n3.x : n3.y, qhix = g == 0 ? n3.z : n3.w;
    uint32_t qhiy = g == 0 ? n4.x : n4.y, qhiz = g == 0 ? n4.z : n4.w;
    // swap lo/hi by ray direction sign
    uint32_t sxlo = inv.x < 0.0f ? qhix : qlox, sxhi = inv.x < 0.0f ? qlox : qhix;
    uint32_t sylo = inv.y < 0.0f ? qhiy : qloy, syhi = inv.y < 0.0f ? qloy : qhiy;
    uint32_t szlo = inv.z < 0.0f ? qhiz : qloz, szhi = inv.z < 0.0f ? qloz : qhiz;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float tx0 = fmaf((float)extract_byte(sxlo, j), adx, aox);
      float ty0 = fmaf((float)extract_byte(sylo, j), ady, aoy);
      float tz0 = fmaf((float)extract_byte(szlo, j), adz, aoz);
      float tx1 = fmaf(byte_to_float(sxhi, j), adx, aox);
      float ty1 = fmaf(byte_to_float(syhi, j), ady, aoy);
      float tz1 = fmaf(byte_to_float(szhi, j), adz, aoz);
      float tn = fmaxf(fmaxf(tx0, ty0), fmaxf(tz0, tmin));
      float tf = fminf(fminf(tx1, ty1), fminf(tz1, tmax));
      if (tn <= tf) {
        uint32_t cb = extract_byte(child_bits4, j);
        uint32_t bi = extract_byte(bit_index4, j);
        hitmask |= cb << bi;
      }
    }
  }
  return hitmask;
}

// Closest triangle using the compressed 8-wide BVH.
__device__ __forceinline__ int mesh_closest_bvh8(const DevMesh& m, const Ray& r, float tmin,
                                                 float& tmax, float& bu, float& bv,
                                                 bool skip_flat, TraceStats& st,
                                                 uint32_t* err, uint32_t max_steps,
                                                 uint32_t stack_limit) {
  if (m.n_bvh8 == 0) return -1;
  int best = -1;
  uint32_t oct = (r.d.x < 0.0f ? 4u : 0u) | (r.d.y < 0.0f ? 2u : 0u) | (r.d.z < 0.0f ? 1u : 0u);
  uint32_t oct_inv4 = (7u - oct) * 0x01010101u;
  uint2 stack[NR_STACK];
  const int cap = stack_limit < (uint32_t)NR_STACK ? (int)stack_limit : NR_STACK;
  int sp = 0;
  // The root is the single inner child (bit 31) of a virtual group whose
  // child base is 0 and whose inner mask (low byte) is empty, so it resolves
  // to node 0.
  uint2 ngroup = make_uint2(0u, 0x80000000u);
  const uint32_t oct_inv = 7u - oct;
  for (uint32_t steps = 0;; ++steps) {
    if (steps >= max_steps) {
      atomicOr(err, 8u);
      break;
    }
    if (ngroup.y > 0x00ffffffu) {
      uint32_t hits = ngroup.y;
      uint32_t child_bit = 31u - __clz(hits);
      ngroup.y &= ~(1u << child_bit);
      uint32_t slot = (child_bit - 24u) ^ oct_inv;
      uint32_t imask = hits & 0xffu;
      uint32_t node_index = ngroup.x + __popc(imask & ~(0xffffffffu << slot));
      if (node_index >= m.n_bvh8) {
        atomicOr(err, 8u);
        break;
      }
      if (ngroup.y > 0x00ffffffu) {
        if (sp < cap) stack[sp++] = ngroup;
        else atomicOr(err, 1u);
      }
      float4 n0;
      uint4 n1;
      uint32_t hm = bvh8_intersect(m.bvh8 + node_index, r.o, r.inv, oct_inv4, tmin, tmax, n0, n1);
      st.nodes++;
      uint32_t child_imask = __float_as_uint(n0.w) >> 24;
      ngroup = make_uint2(n1.x, (hm & 0xff000000u) | child_imask);
      uint32_t tbits = hm & 0x00ffffffu;
      while (tbits != 0u) {
        uint32_t b = __ffs(tbits) - 1u;
        tbits &= tbits - 1u;
        uint32_t slot_i = n1.y + b;
        const TriRecord* tr = m.tris8 + slot_i;
        float4 p0 = __ldg(&tr->v0), p1 = __ldg(&tr->e1), p2 = __ldg(&tr->e2);
        st.tris++;
        if (skip_flat && __float_as_uint(p1.w) != 0u) continue;
        float t, u, v;
        if (tri_hit(r, V3{p0.x, p0.y, p0.z}, V3{p1.x, p1.y, p1.z}, V3{p2.x, p2.y, p2.z}, tmin,
                    tmax, t, u, v)) {
          tmax = t;
          bu = u;
          bv = v;
          best = (int)slot_i;
        }
      }
    }
    if (ngroup.y <= 0x00ffffffu) {
      if (sp == 0) break;
      ngroup = stack[--sp];
    }
  }
  return best;
}

// Mesh::hit + interpolate_hit (mesh.h:239-292, 367-383).
__device__ __forceinline__ bool mesh_hit(const DevScene& sc, const DevObject& ob, const Ray& r,
                                         float tmin, float tmax, Hit& h, bool ref_mode,
                                         TraceStats& st, uint32_t* err) {
  const DevMesh& m = sc.meshes[ob.mesh];
  float u = 0.f, v = 0.f;
  int slot = sc.use_bvh8 ? mesh_closest_bvh8(m, r, tmin, tmax, u, v, ref_mode, st, err,
                                             sc.max_steps, sc.stack_limit)
                         : mesh_closest_bvh2(m, r, tmin, tmax, u, v, ref_mode, st, err,
                                             sc.max_steps, sc.stack_limit);
  if (slot < 0) return false;
  const TriRecord* tr = (sc.use_bvh8 ? m.tris8 : m.tris2) + slot;
  uint32_t tri = __float_as_uint(__ldg(&tr->v0.w));
  uint32_t i0 = __ldg(m.tri_vidx + 3 * tri), i1 = __ldg(m.tri_vidx + 3 * tri + 1),
           i2 = __ldg(m.tri_vidx + 3 * tri + 2);
  h.t = tmax;
  h.p = ray_at(r, tmax);
  float w = 1.0f - u - v;
  V2 uv0 = V2{__ldg(m.vuv + 2 * i0), __ldg(m.vuv + 2 * i0 + 1)};
  V2 uv1 = V2{__ldg(m.vuv + 2 * i1), __ldg(m.vuv + 2 * i1 + 1)};
  V2 uv2 = V2{__ldg(m.vuv + 2 * i2), __ldg(m.vuv + 2 * i2 + 1)};
  h.uv = V2{uv0.x * w + uv1.x * u + uv2.x * v, uv0.y * w + uv1.y * u + uv2.y * v};
  V3 n0 = V3{__ldg(m.vnormal + 3 * i0), __ldg(m.vnormal + 3 * i0 + 1), __ldg(m.vnormal + 3 * i0 + 2)};
  V3 n1 = V3{__ldg(m.vnormal + 3 * i1), __ldg(m.vnormal + 3 * i1 + 1), __ldg(m.vnormal + 3 * i1 + 2)};
  V3 n2 = V3{__ldg(m.vnormal + 3 * i2), __ldg(m.vnormal + 3 * i2 + 1), __ldg(m.vnormal + 3 * i2 + 2)};
  h.n = normalize(n0 * w + n1 * u + n2 * v);
  V3 t0 = V3{__ldg(m.vtangent + 3 * i0), __ldg(m.vtangent + 3 * i0 + 1), __ldg(m.vtangent + 3 * i0 + 2)};
  V3 t1 = V3{__ldg(m.vtangent + 3 * i1), __ldg(m.vtangent + 3 * i1 + 1), __ldg(m.vtangent + 3 * i1 + 2)};
  V3 t2 = V3{__ldg(m.vtangent + 3 * i2), __ldg(m.vtangent + 3 * i2 + 1), __ldg(m.vtangent + 3 * i2 + 2)};
  h.tangent = normalize(t0 * w + t1 * u + t2 * v);
  h.prim = tri;
  return true;
}

// Hittable::hit dispatch on an object-space ray for the primitive kinds a
// wrapper can hold (hittable.h:332-352). `mesh_fn(ob, r, tmin, tmax, h)`
// intersects the object's mesh; callers choose its traversal.
template <typename MeshFn>
__device__ __forceinline__ bool shape_hit_t(const CubeFace* faces, const DevObject& ob, int type,
                                            const Ray& r, float tmin, float tmax, Hit& h,
                                            MeshFn&& mesh_fn) {
  switch (type) {
    case 1: return quad_hit(r, tmin, tmax, h);
    case 2: return sphere_hit(r, tmin, tmax, ob.radius, ob.scale, h);
    case 3: return cube_hit(faces, r, tmin, tmax, h);
    case 4: return mesh_fn(ob, r, tmin, tmax, h);
  }
  return false;
}

// ConstantMedium::hit (volumes.h:10-45): two boundary hits of the wrapped
// shape, free flight from a hash of the object-space ray.
template <typename MeshFn>
__device__ __forceinline__ bool medium_hit_t(const CubeFace* faces, const DevObject& ob,
                                             const Ray& r, float tmin, float tmax, Hit& h,
                                             MeshFn&& mesh_fn) {
  Hit h1, h2;
  if (!shape_hit_t(faces, ob, ob.wrapped_type, r, -FMAX, FMAX, h1, mesh_fn)) return false;
  if (!shape_hit_t(faces, ob, ob.wrapped_type, r, h1.t + EPS, FMAX, h2, mesh_fn)) return false;
  if (h1.t < tmin) h1.t = tmin;
  if (h2.t > tmax) h2.t = tmax;
  if (h1.t >= h2.t) return false;
  if (h1.t < 0.0f) h1.t = 0.0f;
  float ray_length = length(r.d);
  float inside = (h2.t - h1.t) * ray_length;
  float hit_distance = ob.neg_inv_density * logf(pcg_float_ray(r.o, r.d));
  if (hit_distance > inside) return false;
  h.p = ray_at(r, h1.t + hit_distance / ray_length);
  h.n = V3{1.0f, 0.0f, 0.0f};
  h.front_face = true;
  // The reference leaves t, tangent and uv of this record at their defaults.
  h.t = 0.0f;
  h.tangent = V3{0.0f, 0.0f, 0.0f};
  h.uv = V2{0.0f, 0.0f};
  h.prim = 0xffffffffu;
  return true;
}

// Hittable::hit on an object-space ray (hittable.h:332-352).
template <typename MeshFn>
__device__ __forceinline__ bool object_hit_local_t(const CubeFace* faces, const DevObject& ob,
                                                   const Ray& r, float tmin, float tmax, Hit& h,
                                                   MeshFn&& mesh_fn) {
  h.prim = 0xffffffffu;
  h.uv = V2{0.0f, 0.0f};
  h.tangent = V3{0.0f, 0.0f, 0.0f};
  h.n = V3{0.0f, 0.0f, 0.0f};
  h.p = V3{0.0f, 0.0f, 0.0f};
  h.t = 0.0f;
  switch (ob.type) {
    case 6:  // ObjectLight: wrapped->hit(ray, Interval(-FMAX, FMAX)) (lights.h:10-18)
      return shape_hit_t(faces, ob, ob.wrapped_type, r, -FMAX, FMAX, h, mesh_fn);
    case 5:
      return medium_hit_t(faces, ob, r, tmin, tmax, h, mesh_fn);
    default:
      return shape_hit_t(faces, ob, ob.type, r, tmin, tmax, h, mesh_fn);
  }
}

// The same with the local-stack mesh traversal of the megakernel.
__device__ __forceinline__ bool object_hit_local(const DevScene& sc, const DevObject& ob,
                                                 const Ray& r, float tmin, float tmax, Hit& h,
                                                 bool ref_mode, TraceStats& st,
                                                 uint32_t* err) {
  auto mesh_fn = [&](const DevObject& o, const Ray& rr, float t0, float t1, Hit& hh) {
    return mesh_hit(sc, o, rr, t0, t1, hh, ref_mode, st, err);
  };
  return object_hit_local_t(sc.cube_faces, ob, r, tmin, tmax, h, mesh_fn);
}

// Hittable::hit_test (hittable.h:324-330): object space, Interval(EPS, FMAX),
// back to world space with the EPS bias. `prune` is an upper bound on the
// object-space ray parameter that can still win at the top level; it only
// skips candidates whose world t would be rejected anyway.
__device__ __forceinline__ bool object_hit_test(const DevScene& sc, uint32_t slot, const Ray& wr,
                                                float prune, Hit& h, bool ref_mode,
                                                TraceStats& st, uint32_t* err) {
  const DevObject& ob = sc.objects[slot];
  Ray r = to_object(ob, wr);
  float tmax = (ob.type == 4) ? prune : FMAX;
  bool hit = object_hit_local(sc, ob, r, EPS, tmax, h, ref_mode, st, err);
  st.objs++;
  if (!hit) return false;
  to_world(h, ob.R, ob.pos, ob.scale, ob.inv_s, r, wr, true);
  h.obj = slot;
  return true;
}

// SceneGraph::hit (nectar_render/csrc/scene/include/graph.h:16-66): closest
// object by world t with the strict `surrounds` test; the top-level tree is
// traversed near-first with the current closest t as the far bound.
__device__ __forceinline__ bool scene_hit(const DevScene& sc, const Ray& wr, Hit& rec,
                                          bool ref_mode, TraceStats& st, uint32_t* err) {
  float best = FMAX;
  bool any = false;
  V3 oinv = wr.o * wr.inv;
  float inv_len = 1.0f / length(wr.d);
  float slack_base = (2.0f * EPS + 1e-4f * (fabsf(wr.o.x) + fabsf(wr.o.y) + fabsf(wr.o.z) + 1.0f));
  uint32_t stack[NR_STACK];
  const int cap = sc.stack_limit < (uint32_t)NR_STACK ? (int)sc.stack_limit : NR_STACK;
  int sp = 0;
  int cur = 0;
  for (uint32_t steps = 0;; ++steps) {
    if (steps >= sc.max_steps || (uint32_t)cur >= sc.n_tlas2) {
      atomicOr(err, 8u);
      break;
    }
    const Bvh2Node* nd = sc.tlas2 + cur;
    float4 A = __ldg(&nd->a), B = __ldg(&nd->b), C = __ldg(&nd->c);
    int4 D = __ldg(&nd->d);
    float tn0, tn1;
    bool h0 = slab(A.x, A.y, A.z, A.w, C.x, C.y, oinv, wr.inv, EPS, best, tn0);
    bool h1 = slab(B.x, B.y, B.z, B.w, C.z, C.w, oinv, wr.inv, EPS, best, tn1);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      bool hc = c == 0 ? h0 : h1;
      int link = c == 0 ? D.x : D.y;
      int cnt = c == 0 ? D.z : D.w;
      if (hc && link < 0) {
        int first = ~link;
        for (int k = 0; k < cnt; ++k) {
          uint32_t slot = __ldg(sc.tlas_prims + first + k);
          float prune = fminf(FMAX, best * 1.0011f + slack_base * inv_len);
          Hit tmp;
          if (object_hit_test(sc, slot, wr, prune, tmp, ref_mode, st, err)) {
            if (EPS < tmp.t && tmp.t < best) {
              any = true;
              rec = tmp;
              best = tmp.t;
            }
          }
        }
        if (c == 0) h0 = false; else h1 = false;
      }
    }
    if (h0 && h1) {
      bool near0 = tn0 <= tn1;
      int nearl = near0 ? D.x : D.y, farl = near0 ? D.y : D.x;
      if (sp < cap) stack[sp++] = (uint32_t)farl;
      else atomicOr(err, 1u);
      cur = nearl;
    } else if (h0) {
      cur = D.x;
    } else if (h1) {
      cur = D.y;
    } else {
      if (sp == 0) break;
      cur = (int)stack[--sp];
    }
  }
  return any;
}

// ---------------------------------------------------------------------------
// textures (nectar_render/csrc/material/include/material/texture.h:49-91)
struct C3 {
  float r, g, b;
};
__device__ __forceinline__ V3 tex_sample(const DevTexture& t, const V2& uv) {
  if (t.type == 0) return V3{t.r, t.g, t.b};
  float sc = 1.0f / fmaxf(FMIN, t.scale);
  float su = fmodf(uv.x * sc, 1.0f);
  float sv = fmodf(uv.y * sc, 1.0f);
  float u = su < 0.0f ? 0.0f : (su > 1.0f ? 1.0f : su);
  float v = 1.0f - (sv < 0.0f ? 0.0f : (sv > 1.0f ? 1.0f : sv));
  int i = (int)(u * t.W);
  if (i >= (int)t.W) i = (int)t.W - 1;
  int j = (int)(v * t.H);
  if (j >= (int)t.H) j = (int)t.H - 1;
  size_t px = (size_t)j * t.W + i;
  size_t hw = (size_t)t.H * t.W;
  V3 c = V3{(float)t.data[px], (float)t.data[hw + px], (float)t.data[2 * hw + px]};
  return c / 255.0f;
}

// ---------------------------------------------------------------------------
// PDFs (nectar_render/csrc/engine/include/engine/pdf.h:5-283)
enum PdfKind : int { PDF_COSINE = 0, PDF_SPHERE = 1, PDF_PBR = 5 };
struct Pdf {
  int kind;
  ONB uvw;
  V3 view;
  float alpha;
  float spec_prob;
};

// GGX helpers (pdf.h:100-119)
__device__ __forceinline__ float ggx_d(float ndh, float alpha) {
  float a2 = alpha * alpha;
  float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
  return a2 / fmaxf(PI * d * d, 1e-8f);
}
__device__ __forceinline__ float smith_g1(float ndx, float alpha) {
  float a2 = alpha * alpha;
  return 2.0f * ndx / (ndx + sqrtf(a2 + (1.0f - a2) * ndx * ndx));
}

// random_cosine_direction (vector.h:509-519)
__device__ __forceinline__ V3 random_cosine_direction(Rng& g) {
  float r1 = g.random_float();
  float r2 = g.random_float();
  float phi = PI2 * r1;
  float x = cosf(phi) * sqrtf(r2);
  float y = sinf(phi) * sqrtf(r2);
  float z = sqrtf(1.0f - r2);
  return V3{x, y, z};
}
// random_unit_vector (vector.h:489-496); `rtl` selects the order in which the
// three coordinates of Vector3::random consume draws (unspecified in C++).
__device__ __forceinline__ V3 random_unit_vector(Rng& g, bool rtl) {
  while (true) {
    float a = g.random_float(-1.0f, 1.0f);
    float b = g.random_float(-1.0f, 1.0f);
    float c = g.random_float(-1.0f, 1.0f);
    V3 p = rtl ? V3{c, b, a} : V3{a, b, c};
    float lensq = length_squared(p);
    if (1e-160 < (double)lensq && lensq <= 1) return p / sqrtf(lensq);
  }
}

__device__ __forceinline__ float pdf_value(const Pdf& p, const V3& dir) {
  switch (p.kind) {
    case PDF_COSINE: {
      float ct = dot(normalize(dir), p.uvw.w);
      return fmaxf(0.0f, ct / PI);
    }
    case PDF_SPHERE:
      return 1.0f / PI4;
    case PDF_PBR: {
      float diffuse_pdf = fmaxf(0.0f, dot(normalize(dir), p.uvw.w) / PI);
      V3 hv = normalize(p.view + dir);
      float ndh = fmaxf(dot(p.uvw.w, hv), 0.0f);
      float vdh = fmaxf(dot(p.view, hv), 1e-4f);
      float spec_pdf = (ggx_d(ndh, p.alpha) * ndh) / (4.0f * vdh);
      return (1.0f - p.spec_prob) * diffuse_pdf + p.spec_prob * spec_pdf;
    }
  }
  return 0.0f;
}

__device__ __forceinline__ V3 pdf_generate(const Pdf& p, Rng& g, bool rtl) {
  switch (p.kind) {
    case PDF_COSINE:
      return onb_transform(p.uvw, random_cosine_direction(g));
    case PDF_SPHERE:
      return random_unit_vector(g, rtl);
    case PDF_PBR: {
      if (g.random_float() < p.spec_prob) {
        float u1 = g.random_float();
        float u2 = g.random_float();
        float ct = sqrtf((1.0f - u1) / (1.0f + (p.alpha * p.alpha - 1.0f) * u1));
        float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float phi = PI2 * u2;
        V3 hv = onb_transform(p.uvw, V3{st * cosf(phi), st * sinf(phi), ct});
        return normalize(2.0f * dot(p.view, hv) * hv - p.view);
      }
      return onb_transform(p.uvw, random_cosine_direction(g));
    }
  }
  return V3{0.0f, 0.0f, 1.0f};
}

// ---------------------------------------------------------------------------
// lights[0] as a sampling target (HittablePDF, pdf.h:45-67; Quad, Sphere,
// Cube and Mesh pdf_value/random, primitives.h:44-70, shapes.h:60-84,
// 175-185, mesh.h:294-304; ObjectLight forwarding, lights.h:20-34).
__device__ __forceinline__ float light_pdf_value(const DevScene& sc, const V3& origin,
                                                 const V3& dir, TraceStats& st, uint32_t* err) {
  const DevObject& ob = sc.objects[sc.light];
  int type = ob.type == 6 ? ob.wrapped_type : ob.type;
  if (type == 1) {
    // Quad::pdf_value -> Quad::hit_test with the object transform
    Ray wr = make_ray(origin, dir, 0.0f);
    Ray r = to_object(ob, wr);
    Hit h;
    bool hit = quad_hit(r, EPS, FMAX, h);
    to_world(h, ob.R, ob.pos, ob.scale, ob.inv_s, r, wr, true);
    if (!hit) return 0.0f;
    float dist2 = h.t * h.t * length_squared(dir);
    float cosine = fabsf(dot(dir, h.n) / length(dir));
    if (cosine < 1e-8f) return 0.0f;
    float world_area = 1.0f * ob.scale.x * ob.scale.z;
    return dist2 / (cosine * world_area);
  }
  if (type == 2) {
    // Sphere::pdf_value tests the world-space ray against a sphere at the
    // origin, as the reference does.
    Hit h;
    Ray wr = make_ray(origin, dir, 0.0f);
    if (!sphere_hit(wr, EPS, FMAX, ob.radius, ob.scale, h)) return 0.0f;
    float rad_sq = ob.radius * ob.radius;
    float dist2 = length_squared(ob.pos - origin);
    float ctm = sqrtf(1.0f - rad_sq / dist2);
    float solid = PI2 * (1.0f - ctm);
    return 1.0f / solid;
  }
  return 0.0f;
}

__device__ __forceinline__ V3 light_random(const DevScene& sc, const V3& origin, Rng& g,
                                           bool rtl) {
  const DevObject& ob = sc.objects[sc.light];
  int type = ob.type == 6 ? ob.wrapped_type : ob.type;
  if (type == 1) {
    // corner + (r_a*u) + (r_b*v), u=(1,0,0), v=(0,0,-1); draw order of r_a, r_b
    // is the compiler's argument order.
    float first = g.random_float();
    float second = g.random_float();
    float ra = rtl ? second : first;
    float rb = rtl ? first : second;
    const V3 u = V3{1.0f, 0.0f, 0.0f}, v = V3{0.0f, 0.0f, -1.0f};
    V3 corner = (-0.5f * u) - (0.5f * v);
    V3 p = corner + (ra * u) + (rb * v);
    p = mul(ob.R, p * ob.scale) + ob.pos;
    return p - origin;
  }
  if (type == 2) {
    V3 direction = ob.pos - origin;
    float d2 = length_squared(direction);
    ONB b = make_onb(direction);
    float r1 = g.random_float();
    float r2 = g.random_float();
    float rad_sq = ob.radius * ob.radius;
    float z = 1.0f + r2 * (sqrtf(1.0f - rad_sq / d2) - 1.0f);
    float phi = PI2 * r1;
    float x = cosf(phi) * sqrtf(1.0f - z * z);
    float y = sinf(phi) * sqrtf(1.0f - z * z);
    return onb_transform(b, V3{x, y, z});
  }
  if (type == 3) return V3{1.0f, 0.0f, 0.0f};
  if (type == 4) return V3{0.0f, 0.0f, 0.0f};
  return V3{1.0f, 0.0f, 0.0f};
}

// ---------------------------------------------------------------------------
// materials (nectar_render/csrc/material/include/material/material.h:33-646)
__device__ __forceinline__ V3 pbr_shading_normal(const DevMaterial& m, const Hit& h) {
  V3 tn = tex_sample(m.tex[4], h.uv);
  V3 map_n = normalize(V3{tn.x * 2.0f - 1.0f, tn.y * 2.0f - 1.0f, tn.z * 2.0f - 1.0f});
  V3 t = normalize(h.tangent - h.n * dot(h.tangent, h.n));
  V3 b = cross(h.n, t);
  return normalize(t * map_n.x + b * map_n.y + h.n * map_n.z);
}

__device__ __forceinline__ V3 mat_emitted(const DevMaterial& m, const Hit& h) {
  switch (m.type) {
    case 2:
      if (!h.front_face) return V3{0.f, 0.f, 0.f};
      return tex_sample(m.tex[3], h.uv);
    case 4:
      if (!h.front_face) return V3{0.f, 0.f, 0.f};
      return tex_sample(m.tex[0], h.uv) * m.brightness;
  }
  return V3{0.f, 0.f, 0.f};
}

struct Scatter {
  V3 atten;
  Pdf pdf;
  bool skip_pdf;
  V3 skip_dir;
};

// Dielectric::reflectance (material.h:262-269)
__device__ __forceinline__ float reflectance(float cosine, float ri) {
  float r0 = (1.0f - ri) / (1.0f + ri);
  r0 = r0 * r0;
  return r0 + (1.0f - r0) * powf((1.0f - cosine), 5.0f);
}

__device__ __forceinline__ bool mat_scatter(const DevMaterial& m, const Hit& h, const Ray& ray,
                                            Scatter& s, Rng& g) {
  switch (m.type) {
    case 1:  // Lambertian (material.h:47-57)
      s.atten = tex_sample(m.tex[0], h.uv);
      s.pdf.kind = PDF_COSINE;
      s.pdf.uvw = make_onb(h.n);
      s.skip_pdf = false;
      return true;
    case 2: {  // PBR (material.h:127-150)
      V3 n = pbr_shading_normal(m, h);
      V3 albedo = tex_sample(m.tex[0], h.uv);
      float metallic = tex_sample(m.tex[2], h.uv).x;
      V3 F0 = v3(0.04f) * (1.0f - metallic) + albedo * metallic;
      float spec_prob = fminf(0.9f, fmaxf(0.1f, fmaxf(F0.x, fmaxf(F0.y, F0.z))));
      s.atten = V3{1.f, 1.f, 1.f};
      s.skip_pdf = false;
      s.pdf.kind = PDF_PBR;
      s.pdf.uvw = make_onb(n);
      s.pdf.view = normalize(-ray.d);
      float roughness = tex_sample(m.tex[1], h.uv).x;
      s.pdf.alpha = fmaxf(roughness * roughness, 1e-3f);
      s.pdf.spec_prob = spec_prob;
      return true;
    }
    case 3: {  // Dielectric (material.h:220-244)
      s.atten = V3{m.tint[0], m.tint[1], m.tint[2]};
      s.skip_pdf = true;
      float ri = h.front_face ? (1.0f / m.ior) : m.ior;
      V3 unit = normalize(ray.d);
      float cos_theta = fminf(dot(-unit, h.n), 1.0f);
      float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
      bool cannot_refract = (double)(ri * sin_theta) > 1.0;
      if (cannot_refract || reflectance(cos_theta, ri) > g.uniform())
        s.skip_dir = reflect(unit, h.n);
      else
        s.skip_dir = refract(unit, h.n, ri);
      return true;
    }
    case 5:  // Isotropic (material.h:339-349)
      s.atten = tex_sample(m.tex[0], h.uv);
      s.pdf.kind = PDF_SPHERE;
      s.skip_pdf = false;
      return true;
  }
  return false;  // Emissive, Null
}

__device__ __forceinline__ V3 mat_evaluate(const DevMaterial& m, const Hit& h, const V3& view,
                                           const V3& light) {
  switch (m.type) {
    case 1: {  // material.h:59-67
      float ct = dot(h.n, normalize(light));
      if (ct <= 0.0f) return V3{0.f, 0.f, 0.f};
      return tex_sample(m.tex[0], h.uv) * (ct / PI);
    }
    case 2: {  // material.h:152-180
      V3 n = pbr_shading_normal(m, h);
      float ndl = dot(n, light);
      float ndv = dot(n, view);
      if (ndl <= 0.0f || ndv <= 0.0f) return V3{0.f, 0.f, 0.f};
      V3 albedo = tex_sample(m.tex[0], h.uv);
      float roughness = tex_sample(m.tex[1], h.uv).x;
      float metallic = tex_sample(m.tex[2], h.uv).x;
      float alpha = fmaxf(roughness * roughness, 1e-3f);
      V3 hv = normalize(view + light);
      float ndh = fmaxf(dot(n, hv), 0.0f);
      float vdh = fmaxf(dot(view, hv), 0.0f);
      V3 F0 = v3(0.04f) * (1.0f - metallic) + albedo * metallic;
      V3 F = F0 + (V3{1.f, 1.f, 1.f} - F0) * powf(1.0f - vdh, 5.0f);
      float D = ggx_d(ndh, alpha);
      float G = smith_g1(ndl, alpha) * smith_g1(ndv, alpha);
      V3 spec = F * (D * G / fmaxf(4.0f * ndv * ndl, 1e-4f));
      V3 diff = albedo * (1.0f - metallic) * (1.0f / PI);
      return (diff + spec) * ndl;
    }
    case 5:  // material.h:351-357
      return tex_sample(m.tex[0], h.uv) * (1.0f / PI4);
  }
  return V3{0.f, 0.f, 0.f};
}

// ---------------------------------------------------------------------------
// sky (nectar_render/csrc/light/include/skylight.h:30-123, 243-252)
__device__ __forceinline__ V3 sky_texel(const DevSky& s, int x, int y) {
  size_t hw = (size_t)s.H * s.W;
  size_t idx = (size_t)y * s.W + (size_t)x;
  return V3{__ldg(s.data + idx), __ldg(s.data + hw + idx), __ldg(s.data + 2 * hw + idx)};
}
__device__ __forceinline__ V3 hdri_lookup(const DevSky& s, const V3& dir_rot) {
  float u = atan2f(dir_rot.z, dir_rot.x) / PI2 + 0.5f;
  float v = acosf(fminf(fmaxf(dir_rot.y, -1.0f), 1.0f)) / PI;
  float fx = u * (float)s.W - 0.5f;
  float fy = v * (float)s.H - 0.5f;
  int x0 = (int)floorf(fx), y0 = (int)floorf(fy);
  int x1 = x0 + 1, y1 = y0 + 1;
  float tx = fx - (float)x0, ty = fy - (float)y0;
  x0 = ((x0 % s.W) + s.W) % s.W;
  x1 = ((x1 % s.W) + s.W) % s.W;
  y0 = (int)fmaxf(0, fminf(s.H - 1, y0));
  y1 = (int)fmaxf(0, fminf(s.H - 1, y1));
  V3 c00 = sky_texel(s, x0, y0), c10 = sky_texel(s, x1, y0);
  V3 c01 = sky_texel(s, x0, y1), c11 = sky_texel(s, x1, y1);
  V3 top = c00 * (1.0f - tx) + c10 * tx;
  V3 bottom = c01 * (1.0f - tx) + c11 * tx;
  return top * (1.0f - ty) + bottom * ty;
}
__device__ __forceinline__ V3 sky_sample(const DevSky& s, const Ray& ray) {
  if (s.type == 1) {
    float a = (float)(0.5 * ((double)ray.d.y + 1.0));
    float one_minus = (float)(1.0 - (double)a);
    return V3{s.start[0], s.start[1], s.start[2]} * one_minus +
           V3{s.end[0], s.end[1], s.end[2]} * a;
  }
  if (s.type == 2) {
    if (!s.data) return V3{0.f, 0.f, 0.f};
    V3 dir = mul(s.rot, normalize(ray.d));
    return hdri_lookup(s, dir) * s.intensity;
  }
  return V3{0.f, 0.f, 0.f};
}

// ---------------------------------------------------------------------------
// camera (nectar_render/csrc/engine/include/engine/camera.h:124-278)
struct DevCamera {
  float res_x, res_y;  // resolution[0], resolution[1]
  V3 position;
  M3 R;
  float uvw_x, uvw_y;
  float focal_length, focus_distance;
  float shutter_time;
  float defocus_angle, defocus_radius;
  uint32_t W, H;
  const V2* pattern;  // n-rooks pattern, one entry per sample index
};

__device__ __forceinline__ Ray camera_ray(const DevCamera& c, uint32_t x, uint32_t y,
                                          uint32_t pixel_idx, uint32_t sample_idx,
                                          uint32_t seed, Rng& g, bool rtl) {
  V2 base = c.pattern[sample_idx];
  V2 shift = pcg_vector2((float)pixel_idx, seed);
  V2 off = V2{fmodf(base.x + shift.x, 1.0f) - 0.5f, fmodf(base.y + shift.y, 1.0f) - 0.5f};
  float u = ((float)x + off.x - (c.res_x - 1.0f) * 0.5f) * (c.uvw_x / c.res_x);
  float v = ((float)y + off.y - (c.res_y - 1.0f) * 0.5f) * (c.uvw_y / c.res_y);
  float w = -c.focal_length;
  V3 center = mul(c.R, V3{u, v, w});
  float focus_scale = c.focus_distance / c.focal_length;
  V3 focus_point = c.position + center * focus_scale;
  V3 origin;
  if (c.defocus_angle <= 0.0f) {
    origin = c.position;
  } else {
    V3 du = V3{c.R.m[0][0], c.R.m[1][0], c.R.m[2][0]} * c.defocus_radius;
    V3 dv = V3{c.R.m[0][1], c.R.m[1][1], c.R.m[2][1]} * c.defocus_radius;
    V2 loc;
    while (true) {
      float a = g.random_float(-1.0f, 1.0f);
      float b = g.random_float(-1.0f, 1.0f);
      loc = rtl ? V2{b, a} : V2{a, b};
      float l2 = loc.x * loc.x + loc.y * loc.y;
      if (l2 < 1.0f) break;
    }
    origin = c.position + (loc.x * du + loc.y * dv);
  }
  float time = c.shutter_time > 0.0f ? g.uniform() * c.shutter_time : 0.0f;
  return make_ray(origin, normalize(focus_point - origin), time);
}

}  // namespace nr
