// wavefront.cu — wavefront path tracer: generate / extend / shade /
// accumulate kernels over path state kept in HBM.
//
// A wave renders `count` consecutive sample indices of every pixel: path
// p = k*N + pixel (N = W*H) carries sample index base + k. Each bounce runs
//   extend  — persistent traversal kernel: warps take 32 queued paths at a
//             time, walk the 8-wide top-level tree and, for mesh instances,
//             the 8-wide bottom-level tree in object space, with per-thread
//             stacks in shared memory; writes a 20-byte hit record;
//   shade   — rebuilds the closest hit exactly as the reference's hit_test
//             would return it, runs emission / scatter / BSDF sampling /
//             Russian roulette (nectar_render/csrc/engine/src/trace.cu:11-79,
//             brdf.cu:4-35) and appends surviving paths to the next queue
//             with one atomic per warp;
// and after the last bounce
//   accumulate — folds the wave's samples of each pixel into the running mean
//             in sample order (data.cu:28-50) and the FP64 sums.
// Path state per path: ray origin+time, direction, throughput + draw counter,
// beauty + primary id, diffuse + bounce, normal (six 16-byte records) plus
// the hit record. Queue lengths live in device memory, so the sequence of
// launches of a wave is fixed and is captured once as a CUDA graph.
#include "pathstep.cuh"
#include "wavefront.cuh"

namespace nr {

constexpr int kExtThreads = 128;
constexpr int kTlasStack = 8;
constexpr int kBlasStack = 24;
constexpr int kShadeThreads = 128;

enum : uint32_t {
  CTR_N0 = 0,      // paths in queue 0
  CTR_N1 = 1,      // paths in queue 1
  CTR_WORK = 2,    // extend work counter
  CTR_ERR = 3,
  CTR_BASE = 4,    // first sample index of the current wave
  CTR_SH = 5,      // shadow rays queued by this bounce's shade (perf mode)
  CTR_SHWORK = 6,  // shadow kernel work counter
  CTR_TAIL = 7,    // set once the tail kernel has finished the wave's paths
  CTR_NQ = 8,      // radiance-cache queries of the wave
  CTR_NT = 9,      // radiance-cache training records of the wave
};

constexpr int kSortKeys = 8;  // shade_key values

// Shading key of a hit: 0 for a miss, else its material type (1..7), so
// that a warp of the binned queue runs one branch of the BSDF dispatch.
__device__ __forceinline__ uint32_t shade_key(const DevScene& sc, uint32_t obj) {
  if (obj == 0xffffffffu) return 0u;
  const int32_t t = sc.materials[sc.objects[obj].material].type;
  return (uint32_t)min(max(t, 1), (int32_t)kSortKeys - 1);
}

// Material sort of a bounce's queue, pass 1 inside the extend kernels: the
// kernel that writes a path's hit also stores its shading key (skey, one
// byte per path: 8 MB for 8 M paths, resident in L2) and counts the keys
// in a shared-memory histogram that is added to sort_ctr[0..7] at exit.
// Pass 2 (k_wf_bin_scatter) moves the queue into key order.
struct KeyHist {
  uint32_t* h;  // shared memory, kSortKeys counters
  __device__ void init() {
    if (threadIdx.x < kSortKeys) h[threadIdx.x] = 0u;
    __syncthreads();
  }
  __device__ void add(const WfParams& W, const DevScene& sc, uint32_t p, uint32_t obj) {
    const uint32_t key = shade_key(sc, obj);
    W.skey[p] = (uint8_t)key;
    atomicAdd(h + key, 1u);
  }
  __device__ void flush(const WfParams& W) {  // every thread of the block
    __syncthreads();
    if (threadIdx.x < kSortKeys && h[threadIdx.x]) atomicAdd(&W.sort_ctr[threadIdx.x], h[threadIdx.x]);
  }
};

// Features of a hit for the radiance cache (NrcQuery layout, nrc.cuh).
__device__ __forceinline__ void nrc_features(const DevMaterial& m, const Hit& rec, const V3& wo,
                                             float4* out) {
  V3 albedo{0.f, 0.f, 0.f};
  float rough = 1.0f;
  switch (m.type) {
    case 2:
      albedo = tex_sample(m.tex[0], rec.uv);
      rough = tex_sample(m.tex[1], rec.uv).x;
      break;
    case 3:
      albedo = V3{m.tint[0], m.tint[1], m.tint[2]};
      rough = 0.0f;
      break;
    default:
      albedo = tex_sample(m.tex[0], rec.uv);
  }
  out[0] = make_float4(rec.p.x, rec.p.y, rec.p.z, rough);
  out[1] = make_float4(wo.x, wo.y, wo.z, 0.f);
  out[2] = make_float4(rec.n.x, rec.n.y, rec.n.z, 0.f);
  out[3] = make_float4(albedo.x, albedo.y, albedo.z, 0.f);
}

// One path in nrc_train_one_in trains the cache (a hash of pixel and sample).
__device__ __forceinline__ bool nrc_training_path(uint32_t pix, uint32_t sample, uint32_t one_in) {
  uint32_t h = pix * 0x9E3779B9u ^ (sample + 0x632BE5ABu) * 0x85EBCA6Bu;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  return one_in <= 1u || h % one_in == 0u;
}

// Tail hand-off (reference mode): once a wave's queue has shrunk to at most
// kTailMaxPaths paths after bounce kTailFrom or later, one launch finishes
// every remaining path to its end, one path per thread, instead of one
// extend and one shade launch per remaining bounce. The last bounces carry
// few, long paths (glass and mirror chains): as separate launches each costs
// the latency of its slowest ray; in one launch those latencies overlap.
constexpr uint32_t kTailFrom = 3;

// The wave's first sample index is read from device memory, so that the
// launches of a wave do not depend on it and one captured graph serves every
// wave of the same size.
__device__ __forceinline__ uint32_t wave_base(const WfParams& W) { return W.ctr[CTR_BASE]; }

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// One aligned 32-byte sector of a path record (two float4) in one 256-bit
// global load or store (sm_100), so that a lane moves a whole sector.
__device__ __forceinline__ void ld8(const float4* p, float4& a, float4& b) {
  asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z),
                 "=f"(b.w)
               : "l"(p)
               : "memory");
}
__device__ __forceinline__ void st8(float4* p, const float4& a, const float4& b) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x),
               "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

// ---------------------------------------------------------------------------
// compressed 8-wide traversal with a shared-memory stack; `leaf(slot, tmax)`
// is called for every primitive slot whose leaf box the ray enters.
// `depth` bounds the stack entries and `max_steps` the loop (error bits 1 and 8).
template <typename Leaf>
__device__ __forceinline__ void cwbvh_trace(const Bvh8Node* __restrict__ nodes, uint32_t n_nodes,
                                            const V3& o, const V3& d, const V3& inv, float tmin,
                                            float& tmax, uint2* stk, uint32_t stride, int depth,
                                            uint32_t max_steps, Leaf&& leaf, uint32_t& node_count,
                                            uint32_t* err) {
  if (n_nodes == 0) return;
  uint32_t oct = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
  const uint32_t oct_inv = 7u - oct;
  const uint32_t oct_inv4 = oct_inv * 0x01010101u;
  uint2 ngroup = make_uint2(0u, 0x80000000u);
  int sp = 0;
  for (uint32_t steps = 0;; ++steps) {
    if (steps >= max_steps) {
      atomicOr(err, 8u);
      return;
    }
    if (ngroup.y > 0x00ffffffu) {
      uint32_t hits = ngroup.y;
      uint32_t child_bit = 31u - __clz(hits);
      ngroup.y &= ~(1u << child_bit);
      uint32_t slot = (child_bit - 24u) ^ oct_inv;
      uint32_t imask = hits & 0xffu;
      uint32_t node_index = ngroup.x + __popc(imask & ~(0xffffffffu << slot));
      if (node_index >= n_nodes) {
        atomicOr(err, 8u);
        return;
      }
      if (ngroup.y > 0x00ffffffu) {
        if (sp < depth) stk[(sp++) * stride] = ngroup;
        else atomicOr(err, 1u);
      }
      float4 n0;
      uint4 n1;
      uint32_t hm = bvh8_intersect(nodes + node_index, o, inv, oct_inv4, tmin, tmax, n0, n1);
      node_count++;
      ngroup = make_uint2(n1.x, (hm & 0xff000000u) | (__float_as_uint(n0.w) >> 24));
      uint32_t tbits = hm & 0x00ffffffu;
      while (tbits) {
        uint32_t b = __ffs(tbits) - 1u;
        tbits &= tbits - 1u;
        leaf(n1.y + b, tmax);
      }
    }
    if (ngroup.y <= 0x00ffffffu) {
      if (sp == 0) return;
      ngroup = stk[(--sp) * stride];
    }
  }
}

// World-space t of an object-space hit as HitRecord::to_world_space computes
// it with the bias (hit_record.h:24-51), without the tangent frame.
__device__ __forceinline__ float world_t(V3 p, V3 n, const DevObject& ob, const Ray& r_obj,
                                         const Ray& wr) {
  p = mul(ob.R, p * ob.scale) + ob.pos;
  bool front = dot(r_obj.d, n) < 0.0f;
  n = front ? n : -n;
  n = normalize(mul(ob.R, n * ob.inv_s));
  bool front2 = dot(wr.d, n) < 0.0f;
  n = front2 ? n : -n;
  p += n * EPS;
  return dot(p - wr.o, wr.d) / length_squared(wr.d);
}

__device__ __forceinline__ V3 mesh_normal(const DevMesh& m, uint32_t tri, float u, float v) {
  uint32_t i0 = __ldg(m.tri_vidx + 3 * tri), i1 = __ldg(m.tri_vidx + 3 * tri + 1),
           i2 = __ldg(m.tri_vidx + 3 * tri + 2);
  float w = 1.0f - u - v;
  V3 n0 = V3{__ldg(m.vnormal + 3 * i0), __ldg(m.vnormal + 3 * i0 + 1), __ldg(m.vnormal + 3 * i0 + 2)};
  V3 n1 = V3{__ldg(m.vnormal + 3 * i1), __ldg(m.vnormal + 3 * i1 + 1), __ldg(m.vnormal + 3 * i1 + 2)};
  V3 n2 = V3{__ldg(m.vnormal + 3 * i2), __ldg(m.vnormal + 3 * i2 + 1), __ldg(m.vnormal + 3 * i2 + 2)};
  return normalize(n0 * w + n1 * u + n2 * v);
}

// A kernel's traversal stack depth under the render's stack limit.
__device__ __forceinline__ int stack_cap(int depth, const DevScene& sc) {
  return sc.stack_limit < (uint32_t)depth ? (int)sc.stack_limit : depth;
}

// Mesh::hit + interpolate_hit (mesh.h:239-292, 367-383) with the 8-wide tree
// and a shared-memory stack.
__device__ __forceinline__ bool mesh_hit8(const DevScene& sc, const DevObject& ob, const Ray& r,
                                          float tmin, float tmax, Hit& h, uint2* stk,
                                          uint32_t stride, uint32_t* err) {
  const DevMesh& m = sc.meshes[ob.mesh];
  int best = -1;
  float bu = 0.f, bv = 0.f;
  uint32_t nodes = 0;
  auto tri_leaf = [&](uint32_t ts, float& tm) {
    const TriRecord* tr = m.tris8 + ts;
    float4 p0 = ld4(&tr->v0), p1 = ld4(&tr->e1), p2 = ld4(&tr->e2);
    if (__float_as_uint(p1.w) != 0u) return;
    float t, u, v;
    if (tri_hit(r, V3{p0.x, p0.y, p0.z}, V3{p1.x, p1.y, p1.z}, V3{p2.x, p2.y, p2.z}, tmin, tm, t,
                u, v)) {
      tm = t;
      bu = u;
      bv = v;
      best = (int)ts;
    }
  };
  cwbvh_trace(m.bvh8, m.n_bvh8, r.o, r.d, r.inv, tmin, tmax, stk, stride,
              stack_cap(kBlasStack, sc), sc.max_steps, tri_leaf, nodes, err);
  if (best < 0) return false;
  uint32_t tri = __float_as_uint(__ldg(&m.tris8[best].v0.w));
  uint32_t i0 = __ldg(m.tri_vidx + 3 * tri), i1 = __ldg(m.tri_vidx + 3 * tri + 1),
           i2 = __ldg(m.tri_vidx + 3 * tri + 2);
  h.t = tmax;
  h.p = ray_at(r, tmax);
  float w = 1.0f - bu - bv;
  V2 uv0 = V2{__ldg(m.vuv + 2 * i0), __ldg(m.vuv + 2 * i0 + 1)};
  V2 uv1 = V2{__ldg(m.vuv + 2 * i1), __ldg(m.vuv + 2 * i1 + 1)};
  V2 uv2 = V2{__ldg(m.vuv + 2 * i2), __ldg(m.vuv + 2 * i2 + 1)};
  h.uv = V2{uv0.x * w + uv1.x * bu + uv2.x * bv, uv0.y * w + uv1.y * bu + uv2.y * bv};
  h.n = mesh_normal(m, tri, bu, bv);
  V3 t0 = V3{__ldg(m.vtangent + 3 * i0), __ldg(m.vtangent + 3 * i0 + 1), __ldg(m.vtangent + 3 * i0 + 2)};
  V3 t1 = V3{__ldg(m.vtangent + 3 * i1), __ldg(m.vtangent + 3 * i1 + 1), __ldg(m.vtangent + 3 * i1 + 2)};
  V3 t2 = V3{__ldg(m.vtangent + 3 * i2), __ldg(m.vtangent + 3 * i2 + 1), __ldg(m.vtangent + 3 * i2 + 2)};
  h.tangent = normalize(t0 * w + t1 * bu + t2 * bv);
  h.prim = tri;
  return true;
}

// Closest hit of a world ray over the whole scene: the object with the
// smallest biased world t in (EPS, best), as SceneGraph::hit selects it
// (scene/include/graph.h:16-66). Returns obj = 0xffffffff on a miss.
template <bool kCount>
__device__ __forceinline__ void trace_closest(const DevScene& sc, const Ray& wr, uint2* tlas_stk,
                                              uint2* blas_stk, uint32_t stride, uint32_t& out_obj,
                                              uint32_t& out_slot, float& out_t, float& out_u,
                                              float& out_v, TraceStats& st, uint32_t* err,
                                              float best0 = FMAX) {
  float best = best0;
  out_obj = 0xffffffffu;
  out_slot = 0xffffffffu;
  out_t = 0.0f;
  out_u = out_v = 0.0f;
  const float slack = (2.0f * EPS + 1e-4f * (fabsf(wr.o.x) + fabsf(wr.o.y) + fabsf(wr.o.z) + 1.0f)) /
                      length(wr.d);
  uint32_t nodes = 0;
  auto object_leaf = [&](uint32_t slot, float& tlas_tmax) {
    uint32_t oi = __ldg(sc.tlas_prims8 + slot);
    const DevObject& ob = sc.objects[oi];
    Ray r = to_object(ob, wr);
    if (kCount) st.objs++;
    if (ob.type == 4) {
      const DevMesh& m = sc.meshes[ob.mesh];
      float tmax = fminf(FMAX, best * 1.0011f + slack);
      int best_slot = -1;
      float bu = 0.f, bv = 0.f;
      auto tri_leaf = [&](uint32_t ts, float& tm) {
        const TriRecord* tr = m.tris8 + ts;
        float4 p0 = ld4(&tr->v0), p1 = ld4(&tr->e1), p2 = ld4(&tr->e2);
        if (kCount) st.tris++;
        if (__float_as_uint(p1.w) != 0u) return;  // zero-extent box: never hit in the reference
        float t, u, v;
        if (tri_hit(r, V3{p0.x, p0.y, p0.z}, V3{p1.x, p1.y, p1.z}, V3{p2.x, p2.y, p2.z}, EPS, tm,
                    t, u, v)) {
          tm = t;
          bu = u;
          bv = v;
          best_slot = (int)ts;
        }
      };
      cwbvh_trace(m.bvh8, m.n_bvh8, r.o, r.d, r.inv, EPS, tmax, blas_stk, stride,
                  stack_cap(kBlasStack, sc), sc.max_steps, tri_leaf, nodes, err);
      if (best_slot >= 0) {
        uint32_t tri = __float_as_uint(__ldg(&m.tris8[best_slot].v0.w));
        V3 p = ray_at(r, tmax);
        V3 n = mesh_normal(m, tri, bu, bv);
        float tw = world_t(p, n, ob, r, wr);
        if (EPS < tw && tw < best) {
          best = tw;
          tlas_tmax = best;
          out_obj = oi;
          out_slot = (uint32_t)best_slot;
          out_t = tmax;
          out_u = bu;
          out_v = bv;
        }
      }
    } else {
      Hit h;
      auto mesh_fn = [&](const DevObject& o, const Ray& rr, float t0, float t1, Hit& hh) {
        return mesh_hit8(sc, o, rr, t0, t1, hh, blas_stk, stride, err);
      };
      if (object_hit_local_t(sc.cube_faces, ob, r, EPS, FMAX, h, mesh_fn)) {
        float tw = world_t(h.p, h.n, ob, r, wr);
        if (EPS < tw && tw < best) {
          best = tw;
          tlas_tmax = best;
          out_obj = oi;
          out_slot = 0xffffffffu;
          out_t = h.t;
        }
      }
    }
  };
  float tlas_tmax = best0;
  cwbvh_trace(sc.tlas8, sc.n_tlas8, wr.o, wr.d, wr.inv, EPS, tlas_tmax, tlas_stk, stride,
              stack_cap(kTlasStack, sc), sc.max_steps, object_leaf, nodes, err);
  if (kCount) st.nodes += nodes;
}

// Rebuilds the hit record of the closest object (Hittable::hit_test).
__device__ __forceinline__ void rebuild_hit(const DevScene& sc, uint32_t oi, uint32_t slot, float t,
                                            float u, float v, const Ray& wr, Hit& h, uint2* stk,
                                            uint32_t stride, uint32_t* err) {
  const DevObject& ob = sc.objects[oi];
  Ray r = to_object(ob, wr);
  h.prim = 0xffffffffu;
  if (ob.type == 4) {
    const DevMesh& m = sc.meshes[ob.mesh];
    uint32_t tri = __float_as_uint(__ldg(&m.tris8[slot].v0.w));
    uint32_t i0 = __ldg(m.tri_vidx + 3 * tri), i1 = __ldg(m.tri_vidx + 3 * tri + 1),
             i2 = __ldg(m.tri_vidx + 3 * tri + 2);
    h.t = t;
    h.p = ray_at(r, t);
    float w = 1.0f - u - v;
    V2 uv0 = V2{__ldg(m.vuv + 2 * i0), __ldg(m.vuv + 2 * i0 + 1)};
    V2 uv1 = V2{__ldg(m.vuv + 2 * i1), __ldg(m.vuv + 2 * i1 + 1)};
    V2 uv2 = V2{__ldg(m.vuv + 2 * i2), __ldg(m.vuv + 2 * i2 + 1)};
    h.uv = V2{uv0.x * w + uv1.x * u + uv2.x * v, uv0.y * w + uv1.y * u + uv2.y * v};
    h.n = mesh_normal(m, tri, u, v);
    V3 t0 = V3{__ldg(m.vtangent + 3 * i0), __ldg(m.vtangent + 3 * i0 + 1), __ldg(m.vtangent + 3 * i0 + 2)};
    V3 t1 = V3{__ldg(m.vtangent + 3 * i1), __ldg(m.vtangent + 3 * i1 + 1), __ldg(m.vtangent + 3 * i1 + 2)};
    V3 t2 = V3{__ldg(m.vtangent + 3 * i2), __ldg(m.vtangent + 3 * i2 + 1), __ldg(m.vtangent + 3 * i2 + 2)};
    h.tangent = normalize(t0 * w + t1 * u + t2 * v);
    h.prim = tri;
  } else {
    auto mesh_fn = [&](const DevObject& o, const Ray& rr, float t0, float t1, Hit& hh) {
      return mesh_hit8(sc, o, rr, t0, t1, hh, stk, stride, err);
    };
    object_hit_local_t(sc.cube_faces, ob, r, EPS, FMAX, h, mesh_fn);
  }
  to_world(h, ob.R, ob.pos, ob.scale, ob.inv_s, r, wr, true);
  h.obj = oi;
}

// ---------------------------------------------------------------------------
// kernels

__global__ void k_wf_generate(WfParams W) {
  const KernelParams& P = W.kp;
  const uint32_t N = P.W * P.H;
  uint32_t total = N * W.count;
  const uint32_t base = wave_base(W);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    uint32_t k = p / N, pix = p - k * N;
    uint32_t x = pix % P.W, y = pix / P.W;
    uint32_t sample = base + k;
    Rng g;
    g.init(P.seed, pix + sample * (P.W * P.H));
    Ray r = camera_ray(P.cam, x, y, pix, sample, P.seed, g, P.rtl != 0);
    float4* rp = W.path + path_at(p, 0);
    st8(rp + kRecO, make_float4(r.o.x, r.o.y, r.o.z, r.tm),
        make_float4(r.d.x, r.d.y, r.d.z, __uint_as_float(0u)));
    st8(rp + kRecAtten, make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(g.draw)),
        make_float4(0.f, 0.f, 0.f, __uint_as_float(0xffffffffu)));
    // acc_d / acc_n are written by the shading of bounce 0, which every
    // path of the wave reaches
    if (W.mis_pdf) W.mis_pdf[p] = 0.0f;  // camera rays: emission is not MIS-weighted
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    W.ctr[CTR_N0] = total;
    W.ctr[CTR_N1] = 0u;
    W.ctr[CTR_WORK] = 0u;
    W.ctr[CTR_SH] = 0u;
    W.ctr[CTR_SHWORK] = 0u;
    W.ctr[CTR_TAIL] = 0u;
    W.ctr[CTR_NQ] = 0u;
    W.ctr[CTR_NT] = 0u;
  }
}

// kMinBlocks bounds registers so that kMinBlocks CTAs of 128 threads fit per
// SM (4: 128 registers, 5: 96, 6: 80, 8: 64); the autotuner picks the variant.
template <bool kCount, int kMinBlocks>
__global__ void __launch_bounds__(kExtThreads, kMinBlocks) k_wf_extend(WfParams W, int qsel,
                                                                       int identity) {
  if (W.ctr[CTR_TAIL]) return;
  extern __shared__ uint2 wf_smem[];
  const KernelParams& P = W.kp;
  const uint32_t n = W.ctr[qsel];
  const uint32_t* queue = qsel == 0 ? W.queue0 : W.queue1;
  const uint32_t lane = threadIdx.x & 31u;
  uint2* tlas_stk = wf_smem + threadIdx.x;
  uint2* blas_stk = wf_smem + kTlasStack * kExtThreads + threadIdx.x;
  TraceStats st{0u, 0u, 0u};
  uint32_t rays = 0;
  const bool binned = W.queue_s != nullptr;  // block-uniform
  __shared__ uint32_t key_hist[kSortKeys];
  KeyHist kh{key_hist};
  if (binned) kh.init();
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&W.ctr[CTR_WORK], 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    uint32_t i = base + lane;
    if (i < n) {
      const uint32_t p = identity ? i : __ldg(queue + i);
      float4 o = ld4(W.path + path_at(p, kRecO)), d = ld4(W.path + path_at(p, kRecD));
      Ray r = make_ray(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, o.w);
      uint32_t obj, slot;
      float t, u, v;
      trace_closest<kCount>(P.scene, r, tlas_stk, blas_stk, kExtThreads, obj, slot, t, u, v, st, P.err);
      W.hit[p] = make_uint4(obj, slot, __float_as_uint(u), __float_as_uint(v));
      W.hit_t[p] = t;
      if (binned) kh.add(W, P.scene, p, obj);
      rays++;
    }
  }
  if (binned) kh.flush(W);
  if (kCount) {
    unsigned long long vals[4] = {rays, st.nodes, st.tris, st.objs};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      unsigned long long a = vals[k];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) atomicAdd(P.counters + k, a);
    }
  }
}

// ---------------------------------------------------------------------------
// Flattened two-level traversal with lane refill.
//
// One loop iteration does one unit of work per lane: a primitive of the
// current leaf group, a wide node, a stack pop, a switch between the top-level
// tree and a mesh tree, or the end of a ray. Lanes whose ray has ended take
// new rays from the queue whenever at least kRefill lanes of the warp are idle,
// so a warp no longer waits for its slowest ray. The order in which nodes and
// primitives are visited per ray is the one of trace_closest, so the closest
// hit (ties included) is the same.
// (kRefill: a template parameter of the kernel, 12 by default.)

__device__ __forceinline__ uint32_t octant_inv4(const V3& d) {
  uint32_t oct = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
  return (7u - oct) * 0x01010101u;
}

// Per-thread state the flat loop touches only when a ray starts, enters or
// leaves a mesh, or records a hit lives in shared memory (one word per field
// per thread, field-major), which keeps the loop within 96 registers.
enum : uint32_t {
  FS_WO = 0,        // world origin x, y, z
  FS_WD = 3,        // world direction x, y, z
  FS_WTM = 6,       // ray time
  FS_SLACK = 7,     // world-t slack of the instance prune
  FS_OUT_OBJ = 8,   // closest object so far
  FS_OUT_SLOT = 9,  // its triangle slot (meshes)
  FS_OUT_T = 10,    // its object-space t
  FS_OUT_U = 11,
  FS_OUT_V = 12,
  FS_TL_NG = 13,    // saved top-level node group (2 words)
  FS_TL_TG = 15,    // saved top-level leaf group (2 words)
  FS_TL_SP = 17,    // saved top-level stack depth
  FS_TL_TMAX = 18,  // saved top-level t bound
  FS_MESH_OI = 19,  // mesh instance being traversed
  FS_PATH = 20,     // path index of the ray
  FS_COUNT = 21
};
constexpr size_t kExtStackBytes = sizeof(uint2) * (kTlasStack + kBlasStack) * kExtThreads;
constexpr size_t kFlatSmemBytes = kExtStackBytes + sizeof(uint32_t) * FS_COUNT * kExtThreads;

// kVote (1-3): each iteration a warp runs one kind of work, primitive tests
// or the rest (nodes, mesh exits, ends of rays); the other lanes wait an
// iteration. Primitive tests run when p lanes have one next and n lanes the
// rest with p >= n (1), 2p >= n (2) or p >= 2n (3). (Telling triangle tests
// from object tests as a third kind was slower: 8.26 against 7.76 ms per
// step.) Every ray still takes
// the same steps in the same order, so the hits are the same.
template <bool kCount, int kMinBlocks, uint32_t kRefill = 12, int kVote = 0>
__global__ void __launch_bounds__(kExtThreads, kMinBlocks) k_wf_extend_flat(WfParams W, int qsel,
                                                                            int identity) {
  if (W.ctr[CTR_TAIL]) return;
  extern __shared__ uint2 wf_smem[];
  const KernelParams& P = W.kp;
  const DevScene& sc = P.scene;
  const uint32_t n = W.ctr[qsel];
  const uint32_t* queue = qsel == 0 ? W.queue0 : W.queue1;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint2* const tstk = wf_smem + threadIdx.x;
  uint2* const bstk = wf_smem + kTlasStack * kExtThreads + threadIdx.x;
  uint32_t* const cold = reinterpret_cast<uint32_t*>(wf_smem + (kTlasStack + kBlasStack) * kExtThreads) +
                         threadIdx.x;
  auto cf = [&](uint32_t f) -> float& { return reinterpret_cast<float*>(cold)[f * kExtThreads]; };
  auto cu = [&](uint32_t f) -> uint32_t& { return cold[f * kExtThreads]; };
  uint32_t rays = 0, nodes = 0, tris = 0, objs = 0;

  bool active = false, exhausted = false, in_mesh = false;
  uint32_t steps = 0, oct4 = 0, cur_n = 0;
  V3 o{0, 0, 0}, d{0, 0, 1}, inv{0, 0, 1};
  float tmax = FMAX, best = FMAX, bu = 0.f, bv = 0.f;
  uint2 ng = make_uint2(0u, 0u), tg = make_uint2(0u, 0u);
  int sp = 0, best_slot = -1;
  const Bvh8Node* cur_nodes = sc.tlas8;
  const TriRecord* cur_tris = nullptr;
  const bool binned = W.queue_s != nullptr;  // block-uniform
  __shared__ uint32_t key_hist[kSortKeys];
  KeyHist kh{key_hist};
  if (binned) kh.init();

  while (true) {
    if (!exhausted) {
      const uint32_t idle = __ballot_sync(0xffffffffu, !active);
      const uint32_t nidle = __popc(idle);
      if (nidle >= kRefill || nidle == 32u) {
        const uint32_t leader = __ffs(idle) - 1u;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&W.ctr[CTR_WORK], nidle);
        base = __shfl_sync(0xffffffffu, base, leader);
        if (base + nidle >= n) exhausted = true;
        if (!active) {
          const uint32_t i = base + __popc(idle & lt_mask);
          if (i < n) {
            const uint32_t p = identity ? i : __ldg(queue + i);
            const float4 ro = ld4(W.path + path_at(p, kRecO));
            const float4 rd = ld4(W.path + path_at(p, kRecD));
            o = V3{ro.x, ro.y, ro.z};
            d = V3{rd.x, rd.y, rd.z};
            inv = V3{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
            oct4 = octant_inv4(d);
            cf(FS_WO) = o.x;
            cf(FS_WO + 1) = o.y;
            cf(FS_WO + 2) = o.z;
            cf(FS_WD) = d.x;
            cf(FS_WD + 1) = d.y;
            cf(FS_WD + 2) = d.z;
            cf(FS_WTM) = ro.w;
            cf(FS_SLACK) = (2.0f * EPS + 1e-4f * (fabsf(o.x) + fabsf(o.y) + fabsf(o.z) + 1.0f)) /
                           length(d);
            cu(FS_OUT_OBJ) = 0xffffffffu;
            cu(FS_OUT_SLOT) = 0xffffffffu;
            cf(FS_OUT_T) = 0.f;
            cf(FS_OUT_U) = 0.f;
            cf(FS_OUT_V) = 0.f;
            cu(FS_PATH) = p;
            best = FMAX;
            tmax = FMAX;
            ng = make_uint2(0u, sc.n_tlas8 ? 0x80000000u : 0u);
            tg = make_uint2(0u, 0u);
            sp = 0;
            in_mesh = false;
            cur_nodes = sc.tlas8;
            cur_n = sc.n_tlas8;
            steps = 0;
            active = true;
            rays++;
          }
        }
      }
    }
    const uint32_t act_mask = __ballot_sync(0xffffffffu, active);
    if (act_mask == 0u) break;
    if (kVote) {
      const uint32_t prim_mask = __ballot_sync(0xffffffffu, active && tg.y != 0u);
      const int np = __popc(prim_mask), nn = __popc(act_mask & ~prim_mask);
      const bool run_prims = np > 0 && (kVote == 1   ? np >= nn
                                        : kVote == 2 ? 2 * np >= nn
                                                     : np >= 2 * nn || nn == 0);
      if (active && (tg.y != 0u) != run_prims) continue;
    }
    if (!active) continue;

    if (++steps > sc.max_steps) {
      atomicOr(P.err, 8u);
      tg.y = 0u;
      ng.y = 0u;
      sp = 0;
      in_mesh = false;
    }
    if (tg.y != 0u) {
      // one primitive of the current leaf group
      const uint32_t b = __ffs(tg.y) - 1u;
      tg.y &= tg.y - 1u;
      const uint32_t slot = tg.x + b;
      if (in_mesh) {
        const TriRecord* tr = cur_tris + slot;
        const float4 p0 = ld4(&tr->v0), p1 = ld4(&tr->e1), p2 = ld4(&tr->e2);
        if (kCount) tris++;
        if (__float_as_uint(p1.w) == 0u) {  // zero-extent box: never hit in the reference
          Ray r;
          r.o = o;
          r.d = d;
          r.inv = inv;
          r.tm = 0.f;
          float t, u, v;
          if (tri_hit(r, V3{p0.x, p0.y, p0.z}, V3{p1.x, p1.y, p1.z}, V3{p2.x, p2.y, p2.z}, EPS,
                      tmax, t, u, v)) {
            tmax = t;
            bu = u;
            bv = v;
            best_slot = (int)slot;
          }
        }
      } else {
        const uint32_t oi = __ldg(sc.tlas_prims8 + slot);
        const DevObject& ob = sc.objects[oi];
        if (kCount) objs++;
        const Ray wr = make_ray(o, d, cf(FS_WTM));  // at the top level the ray is the world ray
        if (ob.type == 4) {
          const DevMesh& m = sc.meshes[ob.mesh];
          if (m.n_bvh8 > 0) {
            // enter the mesh tree in object space
            cu(FS_TL_NG) = ng.x;
            cu(FS_TL_NG + 1) = ng.y;
            cu(FS_TL_TG) = tg.x;
            cu(FS_TL_TG + 1) = tg.y;
            cu(FS_TL_SP) = (uint32_t)sp;
            cf(FS_TL_TMAX) = tmax;
            cu(FS_MESH_OI) = oi;
            const Ray r = to_object(ob, wr);
            o = r.o;
            d = r.d;
            inv = r.inv;
            oct4 = octant_inv4(d);
            tmax = fminf(FMAX, best * 1.0011f + cf(FS_SLACK));
            ng = make_uint2(0u, 0x80000000u);
            tg = make_uint2(0u, 0u);
            sp = 0;
            in_mesh = true;
            best_slot = -1;
            cur_nodes = m.bvh8;
            cur_n = m.n_bvh8;
            cur_tris = m.tris8;
          }
        } else {
          const Ray r = to_object(ob, wr);
          Hit h;
          auto mesh_fn = [&](const DevObject& mo, const Ray& rr, float t0, float t1, Hit& hh) {
            return mesh_hit8(sc, mo, rr, t0, t1, hh, bstk, kExtThreads, P.err);
          };
          if (object_hit_local_t(sc.cube_faces, ob, r, EPS, FMAX, h, mesh_fn)) {
            const float tw = world_t(h.p, h.n, ob, r, wr);
            if (EPS < tw && tw < best) {
              best = tw;
              tmax = best;
              cu(FS_OUT_OBJ) = oi;
              cu(FS_OUT_SLOT) = 0xffffffffu;
              cf(FS_OUT_T) = h.t;
            }
          }
        }
      }
    } else {
      // a stack pop and the node it names share one iteration
      if (ng.y <= 0x00ffffffu && sp > 0) {
        uint2* stk = in_mesh ? bstk : tstk;
        ng = stk[(--sp) * kExtThreads];
      }
      if (ng.y > 0x00ffffffu) {
        // one wide node
        const uint32_t hits = ng.y;
        const uint32_t child_bit = 31u - __clz(hits);
        ng.y &= ~(1u << child_bit);
        const uint32_t cslot = (child_bit - 24u) ^ (oct4 & 7u);
        const uint32_t node_index = ng.x + __popc((hits & 0xffu) & ~(0xffffffffu << cslot));
        if (node_index >= cur_n) {
          atomicOr(P.err, 8u);
          ng.y = 0u;
          sp = 0;
        } else {
          if (ng.y > 0x00ffffffu) {
            const int depth = in_mesh ? stack_cap(kBlasStack, sc) : stack_cap(kTlasStack, sc);
            uint2* stk = in_mesh ? bstk : tstk;
            if (sp < depth) stk[(sp++) * kExtThreads] = ng;
            else atomicOr(P.err, 1u);
          }
          float4 n0;
          uint4 n1;
          const uint32_t hm = bvh8_intersect(cur_nodes + node_index, o, inv, oct4, EPS, tmax, n0, n1);
          if (kCount) nodes++;
          ng = make_uint2(n1.x, (hm & 0xff000000u) | (__float_as_uint(n0.w) >> 24));
          tg = make_uint2(n1.y, hm & 0x00ffffffu);
        }
      } else if (in_mesh) {
        // leave the mesh tree: the candidate competes in world space
        const V3 wo{cf(FS_WO), cf(FS_WO + 1), cf(FS_WO + 2)};
        const V3 wd{cf(FS_WD), cf(FS_WD + 1), cf(FS_WD + 2)};
        float tl_tmax = cf(FS_TL_TMAX);
        if (best_slot >= 0) {
          const uint32_t oi = cu(FS_MESH_OI);
          const DevObject& ob = sc.objects[oi];
          const DevMesh& m = sc.meshes[ob.mesh];
          const uint32_t tri = __float_as_uint(__ldg(&m.tris8[best_slot].v0.w));
          Ray r;
          r.o = o;
          r.d = d;
          r.inv = inv;
          r.tm = 0.f;
          const Ray wr = make_ray(wo, wd, 0.f);
          const float tw = world_t(ray_at(r, tmax), mesh_normal(m, tri, bu, bv), ob, r, wr);
          if (EPS < tw && tw < best) {
            best = tw;
            tl_tmax = best;
            cu(FS_OUT_OBJ) = oi;
            cu(FS_OUT_SLOT) = (uint32_t)best_slot;
            cf(FS_OUT_T) = tmax;
            cf(FS_OUT_U) = bu;
            cf(FS_OUT_V) = bv;
          }
        }
        ng = make_uint2(cu(FS_TL_NG), cu(FS_TL_NG + 1));
        tg = make_uint2(cu(FS_TL_TG), cu(FS_TL_TG + 1));
        sp = (int)cu(FS_TL_SP);
        tmax = tl_tmax;
        o = wo;
        d = wd;
        inv = V3{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
        oct4 = octant_inv4(d);
        in_mesh = false;
        cur_nodes = sc.tlas8;
        cur_n = sc.n_tlas8;
      } else {
        const uint32_t p = cu(FS_PATH);
        W.hit[p] = make_uint4(cu(FS_OUT_OBJ), cu(FS_OUT_SLOT), cu(FS_OUT_U), cu(FS_OUT_V));
        W.hit_t[p] = cf(FS_OUT_T);
        if (binned) kh.add(W, sc, p, cu(FS_OUT_OBJ));
        active = false;
      }
    }
  }
  if (binned) kh.flush(W);
  if (kCount) {
    unsigned long long vals[4] = {rays, nodes, tris, objs};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      unsigned long long a = vals[k];
      for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
      if (lane == 0) atomicAdd(P.counters + k, a);
    }
  }
}

// kPerf: NR_MODE_PERF (next-event estimation + MIS); otherwise the
// reference's estimator draw for draw.
template <bool kPerf, int kMinBlocks>
__global__ void __launch_bounds__(kShadeThreads, kMinBlocks) k_wf_shade(WfParams W, int qsel,
                                                                      int identity, int sorted) {
  if (W.ctr[CTR_TAIL]) return;
  __shared__ uint2 shade_stk[kBlasStack * kShadeThreads];
  const KernelParams& P = W.kp;
  const DevScene& sc = P.scene;
  const uint32_t n = W.ctr[qsel];
  const uint32_t* queue = sorted ? W.queue_s : (qsel == 0 ? W.queue0 : W.queue1);
  uint32_t* next_queue = qsel == 0 ? W.queue1 : W.queue0;
  uint32_t* next_n = &W.ctr[qsel == 0 ? CTR_N1 : CTR_N0];
  const uint32_t N = P.W * P.H;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t wbase = wave_base(W);
  uint2* const my_stk = shade_stk + threadIdx.x;
  auto mesh_fn = [&](const DevObject& mo, const Ray& rr, float t0, float t1, Hit& hh) {
    return mesh_hit8(sc, mo, rr, t0, t1, hh, my_stk, kShadeThreads, P.err);
  };
  const bool nee_light = kPerf && light_nee_ready(sc);
  const bool nee_sky = kPerf && sky_nee_ready(sc.sky);
  const float sel = (nee_light && nee_sky) ? 0.5f : 1.0f;
  TraceStats st{0u, 0u, 0u};
  // grid-stride loop with whole warps in every iteration (for the warp-aggregated append)
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool alive = false, shadow = false;
    uint32_t p = 0;
    if (i < n) {
      p = (identity && !sorted) ? i : __ldg(queue + i);
      float4* rp = W.path + path_at(p, 0);
      float4 o, d, at, ab;
      ld8(rp + kRecO, o, d);
      ld8(rp + kRecAtten, at, ab);
      uint32_t bounce = __float_as_uint(d.w);
      PathState s;
      s.ray = make_ray(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, o.w);
      s.atten = V3{at.x, at.y, at.z};
      s.beauty = V3{ab.x, ab.y, ab.z};
      s.primary = __float_as_uint(ab.w);
      s.bounce = bounce;
      float4 aov_d = make_float4(0.f, 0.f, 0.f, 0.f), aov_n = aov_d;  // bounce 0 only
      const float pdf_prev = kPerf ? W.mis_pdf[p] : 0.0f;
      uint32_t k = p / N, pix = p - k * N;
      Rng g;
      g.init(P.seed, pix + (wbase + k) * (P.W * P.H), __float_as_uint(at.w));
      uint4 hv = W.hit[p];
      bool hit = hv.x != 0xffffffffu;
      Hit rec;
      if (hit) rebuild_hit(sc, hv.x, hv.y, W.hit_t[p], __uint_as_float(hv.z), __uint_as_float(hv.w),
                           s.ray, rec, my_stk, kShadeThreads, P.err);
      if (bounce == 0u && hit) {
        uint32_t oid = sc.objects[rec.obj].object_id;
        s.primary = (oid << 22) | (rec.prim == 0xffffffffu ? 0u : ((rec.prim + 1u) & 0x3fffffu));
      }
      if (!hit) {
        float w = 1.0f;
        if (kPerf && nee_sky && pdf_prev > 0.0f)
          w = power_heuristic(pdf_prev, sel * sky_dir_pdf(sc.sky, s.ray.d));
        s.beauty += s.atten * sky_sample(sc.sky, s.ray) * w;
      } else if (kPerf && W.nrc_bounce &&
                 !nrc_training_path(pix, wbase + k, W.nrc_train_one_in) &&
                 bounce == W.nrc_bounce) {
        // the radiance cache answers for the rest of the path
        const uint32_t qi = atomicAdd(&W.ctr[CTR_NQ], 1u);
        if (qi < W.nrc_q_cap) {
          nrc_features(sc.materials[sc.objects[rec.obj].material], rec, normalize(-s.ray.d),
                       W.nrc_q + 4 * (size_t)qi);
          W.nrc_q_beta[qi] = make_float4(s.atten.x, s.atten.y, s.atten.z, __uint_as_float(p));
        }
      } else {
        const DevMaterial& m = sc.materials[sc.objects[rec.obj].material];
        Ray r_in = s.ray;
        if (bounce == 0u) aov_n.w = rec.t;  // DEPTH layer: world distance of the first hit
        if (kPerf && W.nrc_bounce && bounce >= 1u &&
            nrc_training_path(pix, wbase + k, W.nrc_train_one_in)) {
          const uint32_t ti = atomicAdd(&W.ctr[CTR_NT], 1u);
          if (ti < W.nrc_t_cap) {
            nrc_features(m, rec, normalize(-s.ray.d), W.nrc_t + 4 * (size_t)ti);
            W.nrc_t_beta[ti] = make_float4(s.atten.x, s.atten.y, s.atten.z, __uint_as_float(p));
            W.nrc_t_before[ti] = make_float4(s.beauty.x, s.beauty.y, s.beauty.z, 0.f);
          }
        }
        {
          float w = 1.0f;
          if (kPerf && nee_light && pdf_prev > 0.0f && (int32_t)rec.obj == sc.light)
            w = power_heuristic(pdf_prev, sel * light_pdf_value(sc, r_in.o, r_in.d, st, P.err));
          s.beauty += s.atten * mat_emitted(m, rec) * w;
        }
        Scatter sr;
        bool cont = mat_scatter(m, rec, s.ray, sr, g);
        float pdf_next = 0.0f;
        if (cont) {
          if (sr.skip_pdf) {
            s.atten *= sr.atten;
            s.ray = make_ray(rec.p, sr.skip_dir, s.ray.tm);
          } else if (!kPerf) {
            cont = sample_brdf(P, m, rec, sr, r_in, s, g, st);
          } else {
            const V3 view = normalize(-r_in.d);
            // next-event estimation: one emitter sample
            if (nee_light || nee_sky) {
              bool use_light = nee_light && (!nee_sky || g.random_float() < 0.5f);
              V3 ldir, Le;
              float lpdf = 0.0f, dist = FMAX;
              bool ok;
              if (use_light) {
                ok = light_sample_nee(sc, rec.p, g, P.rtl != 0, ldir, dist, lpdf, Le, st, P.err,
                                      mesh_fn);
                dist = dist * 0.999f - 2.0f * EPS;
              } else {
                ldir = normalize(sky_sample_dir(sc.sky, g, lpdf));
                Le = sky_sample(sc.sky, make_ray(rec.p, ldir, 0.0f));
                ok = lpdf > 0.0f;
                dist = FMAX;
              }
              if (ok && dist > 0.0f) {
                const V3 f = perf_bsdf_eval(m, rec, view, ldir);
                if (f.x > 0.0f || f.y > 0.0f || f.z > 0.0f) {
                  const float pl = sel * lpdf;
                  const float wl = power_heuristic(pl, perf_bsdf_pdf(sr.pdf, ldir));
                  const V3 c = s.atten * f * Le * (wl / pl);
                  W.sh_o[p] = make_float4(rec.p.x, rec.p.y, rec.p.z, dist);
                  W.sh_d[p] = make_float4(ldir.x, ldir.y, ldir.z, 0.0f);
                  W.sh_c[p] = make_float4(c.x, c.y, c.z, 0.0f);
                  shadow = true;
                }
              }
            }
            // continue with the material's own sampler
            const V3 dir = pdf_generate(sr.pdf, g, P.rtl != 0);
            const float pb = perf_bsdf_pdf(sr.pdf, dir);
            if (pb > 0.0f) {
              s.atten *= perf_bsdf_eval(m, rec, view, dir) / pb;
              s.ray = make_ray(rec.p, dir, r_in.tm);
              pdf_next = pb;
            } else {
              cont = false;
            }
          }
        }
        if (cont) {
          if (bounce == 0u) {
            // the first-hit AOV sums start from zero (0 + x, as a running
            // sum from a cleared buffer computes it)
            aov_d = make_float4(0.f + s.atten.x, 0.f + s.atten.y, 0.f + s.atten.z, 0.f);
            aov_n = make_float4(0.f + rec.n.x, 0.f + rec.n.y, 0.f + rec.n.z, aov_n.w);
          }
          if (P.rr_enabled && bounce >= P.rr_start) {
            float survival = fmaxf(s.atten.x, fmaxf(s.atten.y, s.atten.z));
            survival = fminf(survival, P.rr_survival);
            if (g.uniform() > survival) cont = false;
            else s.atten *= v3(1.0f / survival);
          }
        }
        if (cont && bounce + 1u < P.depth) {
          alive = true;
          if (kPerf) W.mis_pdf[p] = pdf_next;
        }
      }
      if (!kPerf && W.trace_log && bounce < W.log_bounces && p < N) {
        // ray, hit (registry object id, primitive, world t), throughput and
        // beauty after this bounce, and whether the path goes on
        float* L = W.trace_log + ((size_t)p * W.log_bounces + bounce) * kTraceLogFloats;
        L[0] = o.x; L[1] = o.y; L[2] = o.z;
        L[3] = d.x; L[4] = d.y; L[5] = d.z;
        L[6] = __uint_as_float(hit ? sc.objects[rec.obj].object_id : 0xffffffffu);
        L[7] = __uint_as_float(hit ? rec.prim : 0xffffffffu);
        L[8] = hit ? rec.t : 0.0f;
        L[9] = s.atten.x; L[10] = s.atten.y; L[11] = s.atten.z;
        L[12] = s.beauty.x; L[13] = s.beauty.y; L[14] = s.beauty.z;
        L[15] = __uint_as_float(alive ? 1u : 0u);
      }
      if (bounce == 0u) {
        W.acc_d[p] = aov_d;
        W.acc_n[p] = aov_n;
      }
      const float4 b4 = make_float4(s.beauty.x, s.beauty.y, s.beauty.z, __uint_as_float(s.primary));
      if (alive) {
        st8(rp + kRecO, make_float4(s.ray.o.x, s.ray.o.y, s.ray.o.z, s.ray.tm),
            make_float4(s.ray.d.x, s.ray.d.y, s.ray.d.z, __uint_as_float(bounce + 1u)));
        st8(rp + kRecAtten, make_float4(s.atten.x, s.atten.y, s.atten.z, __uint_as_float(g.draw)), b4);
      } else {
        rp[kRecBeauty] = b4;
      }
    }
    // warp-aggregated append of the surviving paths (and, in perf mode, of
    // the shadow rays)
    uint32_t mask = __ballot_sync(0xffffffffu, alive);
    if (mask) {
      uint32_t leader = __ffs(mask) - 1u;
      uint32_t off = 0;
      if (lane == leader) off = atomicAdd(next_n, __popc(mask));
      off = __shfl_sync(0xffffffffu, off, leader);
      if (alive) next_queue[off + __popc(mask & ((1u << lane) - 1u))] = p;
    }
    if (kPerf) {
      uint32_t smask = __ballot_sync(0xffffffffu, shadow);
      if (smask) {
        uint32_t leader = __ffs(smask) - 1u;
        uint32_t off = 0;
        if (lane == leader) off = atomicAdd(&W.ctr[CTR_SH], __popc(smask));
        off = __shfl_sync(0xffffffffu, off, leader);
        if (shadow) W.sh_queue[off + __popc(smask & ((1u << lane) - 1u))] = p;
      }
    }
  }
}

// Shadow rays of one bounce (perf mode): an unoccluded ray adds its
// precomputed contribution to the path's beauty.
// Finishes every path of queue `qsel` with the per-path loop of the
// megakernel (bounce_ref: the same estimator and draws as k_wf_shade), when
// there are at most `max_paths` of them and the tail has not run yet.
__global__ void __launch_bounds__(128) k_wf_tail(WfParams W, int qsel, uint32_t max_paths) {
  if (W.ctr[CTR_TAIL]) return;
  const uint32_t n = W.ctr[qsel];
  if (n == 0u || n > max_paths) return;
  const KernelParams& P = W.kp;
  const uint32_t* queue = qsel == 0 ? W.queue0 : W.queue1;
  const uint32_t N = P.W * P.H;
  const uint32_t wbase = wave_base(W);
  TraceStats st{0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = __ldg(queue + i);
    float4 o, d, at, ab;
    ld8(W.path + path_at(p, kRecO), o, d);
    ld8(W.path + path_at(p, kRecAtten), at, ab);
    const float4 ad = W.acc_d[p], an = W.acc_n[p];
    PathState s;
    s.ray = make_ray(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, o.w);
    s.atten = V3{at.x, at.y, at.z};
    s.beauty = V3{ab.x, ab.y, ab.z};
    s.diffuse = V3{ad.x, ad.y, ad.z};
    s.normal = V3{an.x, an.y, an.z};
    s.primary = __float_as_uint(ab.w);
    s.bounce = __float_as_uint(d.w);
    const uint32_t k = p / N, pix = p - k * N;
    Rng g;
    g.init(P.seed, pix + (wbase + k) * N, __float_as_uint(at.w));
    while (bounce_ref(P, s, g, st)) {
    }
    W.path[path_at(p, kRecBeauty)] = make_float4(s.beauty.x, s.beauty.y, s.beauty.z, __uint_as_float(s.primary));
    W.acc_d[p] = make_float4(s.diffuse.x, s.diffuse.y, s.diffuse.z, 0.f);
    W.acc_n[p] = make_float4(s.normal.x, s.normal.y, s.normal.z, an.w);
  }
}

// Marks the wave finished when k_wf_tail took its queue (a separate launch,
// so that no CTA of the tail kernel can see the mark before its own work).
__global__ void k_wf_tail_mark(WfParams W, int qsel, uint32_t max_paths) {
  if (threadIdx.x != 0 || W.ctr[CTR_TAIL]) return;
  const uint32_t n = W.ctr[qsel];
  if (n > 0u && n <= max_paths) W.ctr[CTR_TAIL] = 1u;
}

__global__ void __launch_bounds__(kExtThreads) k_wf_shadow(WfParams W) {
  extern __shared__ uint2 wf_smem[];
  const KernelParams& P = W.kp;
  const uint32_t n = W.ctr[CTR_SH];
  const uint32_t lane = threadIdx.x & 31u;
  uint2* tlas_stk = wf_smem + threadIdx.x;
  uint2* blas_stk = wf_smem + kTlasStack * kExtThreads + threadIdx.x;
  TraceStats st{0u, 0u, 0u};
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&W.ctr[CTR_SHWORK], 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const uint32_t i = base + lane;
    if (i < n) {
      const uint32_t p = __ldg(W.sh_queue + i);
      const float4 o = W.sh_o[p], d = W.sh_d[p];
      const Ray r = make_ray(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, 0.0f);
      uint32_t obj, slot;
      float t, u, v;
      trace_closest<false>(P.scene, r, tlas_stk, blas_stk, kExtThreads, obj, slot, t, u, v, st,
                           P.err, o.w);
      if (obj == 0xffffffffu) {
        const float4 c = W.sh_c[p];
        float4 b = W.path[path_at(p, kRecBeauty)];
        b.x += c.x;
        b.y += c.y;
        b.z += c.z;
        W.path[path_at(p, kRecBeauty)] = b;
      }
    }
  }
}

// Clears the counters for the next bounce: the queue that was just consumed
// becomes the output of the following shade, and the extend work counter
// restarts.
__global__ void k_wf_rotate(WfParams W, int consumed) {
  if (threadIdx.x == 0) {
    W.ctr[consumed] = 0u;
    W.ctr[CTR_WORK] = 0u;
    W.ctr[CTR_SH] = 0u;
    W.ctr[CTR_SHWORK] = 0u;
  }
  if (W.sort_ctr && threadIdx.x < 2 * kSortKeys) W.sort_ctr[threadIdx.x] = 0u;
}

// Material sort, pass 2: every path of the queue to its key's segment of
// queue_s (segments in key order). A block takes 256 queue entries at a time:
// each warp ranks its lanes per key with one ballot per key, the warps'
// counts are scanned in shared memory, and one atomic per key and block
// reserves the block's run in the segment. Within a segment, blocks append
// in the order they reach their atomics and keep queue order inside a run.
constexpr int kScatterThreads = 256;
__global__ void __launch_bounds__(kScatterThreads) k_wf_bin_scatter(WfParams W, int qsel,
                                                                    int identity) {
  if (W.ctr[CTR_TAIL]) return;
  constexpr int kWarps = kScatterThreads / 32;
  __shared__ uint32_t seg[kSortKeys];
  __shared__ uint32_t run[kSortKeys];
  __shared__ uint32_t woff[kWarps][kSortKeys];
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int k = 0; k < kSortKeys; ++k) {
      seg[k] = acc;
      acc += W.sort_ctr[k];
    }
  }
  const uint32_t n = W.ctr[qsel];
  const uint32_t* queue = qsel == 0 ? W.queue0 : W.queue1;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t below = (1u << lane) - 1u;
  // the loop bound depends on the block only, so every thread reaches the
  // barriers inside it
  for (uint32_t base = blockIdx.x * kScatterThreads; base < n; base += gridDim.x * kScatterThreads) {
    const uint32_t i = base + threadIdx.x;
    uint32_t p = 0, key = kSortKeys, rank = 0;
    if (i < n) {
      p = identity ? i : __ldg(queue + i);
      key = W.skey[p];
    }
#pragma unroll
    for (uint32_t k = 0; k < (uint32_t)kSortKeys; ++k) {
      const uint32_t m = __ballot_sync(0xffffffffu, key == k);
      if (lane == 0) woff[warp][k] = (uint32_t)__popc(m);
      if (key == k) rank = (uint32_t)__popc(m & below);
    }
    __syncthreads();
    if (threadIdx.x < (unsigned)kSortKeys) {
      const uint32_t k = threadIdx.x;
      uint32_t acc = 0;
      for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = woff[w][k];
        woff[w][k] = acc;
        acc += c;
      }
      run[k] = acc ? atomicAdd(&W.sort_ctr[kSortKeys + k], acc) : 0u;
    }
    __syncthreads();
    if (key < (uint32_t)kSortKeys) W.queue_s[seg[key] + run[key] + woff[warp][key] + rank] = p;
    __syncthreads();
  }
}

__global__ void k_wf_accumulate(WfParams W) {
  const KernelParams& P = W.kp;
  const uint32_t N = P.W * P.H;
  const size_t hw = N;
  const uint32_t base = wave_base(W);
  for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < N; pix += gridDim.x * blockDim.x) {
    if (P.write_raw) {
      float4 b = W.path[path_at(pix, kRecBeauty)], d = W.acc_d[pix], n = W.acc_n[pix];
      if (P.beauty) store3(P.beauty, hw, pix, V3{b.x, b.y, b.z});
      if (P.diffuse) store3(P.diffuse, hw, pix, V3{d.x, d.y, d.z});
      if (P.normal) store3(P.normal, hw, pix, V3{n.x, n.y, n.z});
      if (P.depth_layer) P.depth_layer[pix] = n.w;
      if (P.primary) P.primary[pix] = __float_as_uint(b.w);
      continue;
    }
    V3 ab = P.beauty ? load3(P.beauty, hw, pix) : V3{0, 0, 0};
    V3 ad = P.diffuse ? load3(P.diffuse, hw, pix) : V3{0, 0, 0};
    V3 an = P.normal ? load3(P.normal, hw, pix) : V3{0, 0, 0};
    float az = P.depth_layer ? P.depth_layer[pix] : 0.0f;
    double s64[3] = {0, 0, 0};
    for (uint32_t k = 0; k < W.count; ++k) {
      uint32_t p = k * N + pix, smp = base + k;
      float4 b = W.path[path_at(p, kRecBeauty)], d = W.acc_d[p], n = W.acc_n[p];
      ab = running_mean(ab, V3{b.x, b.y, b.z}, smp);
      ad = running_mean(ad, V3{d.x, d.y, d.z}, smp);
      an = running_mean(an, V3{n.x, n.y, n.z}, smp);
      az = running_mean(V3{az, 0.f, 0.f}, V3{n.w, 0.f, 0.f}, smp).x;
      s64[0] += (double)b.x;
      s64[1] += (double)b.y;
      s64[2] += (double)b.z;
    }
    if (P.beauty) store3(P.beauty, hw, pix, ab);
    if (P.diffuse) store3(P.diffuse, hw, pix, ad);
    if (P.depth_layer) P.depth_layer[pix] = az;
    if (P.normal) store3(P.normal, hw, pix, an);
    if (W.disp8) {  // the display transform of the new running mean, in the same pass
      const V3 c = display_pixel(ab, W.disp_p);
      W.disp8[pix] = (uint8_t)quant_pre(c.x);
      W.disp8[hw + pix] = (uint8_t)quant_pre(c.y);
      W.disp8[2 * hw + pix] = (uint8_t)quant_pre(c.z);
    }
    if (P.beauty64) {
      P.beauty64[pix] += s64[0];
      P.beauty64[hw + pix] += s64[1];
      P.beauty64[2 * hw + pix] += s64[2];
    }
  }
}

__global__ void k_nrc_apply(WfParams W, const float* radiance, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 b = W.nrc_q_beta[i];
    const uint32_t p = __float_as_uint(b.w);
    float4 acc = W.path[path_at(p, kRecBeauty)];
    acc.x += b.x * radiance[3 * i];
    acc.y += b.y * radiance[3 * i + 1];
    acc.z += b.z * radiance[3 * i + 2];
    W.path[path_at(p, kRecBeauty)] = acc;
  }
}

// The radiance behind a training record: what the path gathered from this
// hit on, divided by its throughput at the hit.
__global__ void k_nrc_targets(WfParams W, float* target, float4* records, uint32_t n,
                              uint32_t groups, uint32_t per) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 b = W.nrc_t_beta[i], before = W.nrc_t_before[i];
    const float4 after = W.path[path_at(__float_as_uint(b.w), kRecBeauty)];
    const float beta[3] = {b.x, b.y, b.z};
    const float d[3] = {after.x - before.x, after.y - before.y, after.z - before.z};
    const size_t slot = (size_t)(i % groups) * per + i / groups;
    for (int c = 0; c < 3; ++c)
      target[3 * slot + c] = beta[c] > 1e-6f ? fminf(fmaxf(d[c] / beta[c], 0.0f), 1e4f) : 0.0f;
    for (int k = 0; k < 4; ++k) records[4 * slot + k] = W.nrc_t[4 * (size_t)i + k];
  }
}

__global__ void k_wf_set_base(uint32_t* ctr, uint32_t base) {
  if (threadIdx.x == 0) ctr[CTR_BASE] = base;
}

// Last launch of a wave: the next wave starts `count` sample indices later.
__global__ void k_wf_advance(WfParams W) {
  if (threadIdx.x == 0) W.ctr[CTR_BASE] += W.count;
}

// ---------------------------------------------------------------------------
// host side

static int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return sms;
}

cudaError_t wf_nrc_counts(const WfParams& W, uint32_t* n_q, uint32_t* n_t, cudaStream_t st) {
  uint32_t c[2];
  cudaError_t e = cudaMemcpyAsync(c, W.ctr + CTR_NQ, sizeof(c), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  *n_q = std::min(c[0], W.nrc_q_cap);
  *n_t = std::min(c[1], W.nrc_t_cap);
  return e;
}

cudaError_t wf_nrc_apply(const WfParams& W, const float* radiance, uint32_t n, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_nrc_apply<<<(int)std::min<uint32_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(W, radiance, n);
  return cudaGetLastError();
}

cudaError_t wf_nrc_targets(const WfParams& W, float* target, float4* records, uint32_t n,
                           uint32_t groups, cudaStream_t st) {
  if (!n) return cudaSuccess;
  groups = std::max(1u, std::min(groups, n));
  const uint32_t per = (n + groups - 1) / groups;
  k_nrc_targets<<<(int)std::min<uint32_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(
      W, target, records, n, groups, per);
  return cudaGetLastError();
}

cudaError_t wf_set_base(const WfParams& W, uint32_t first_sample, cudaStream_t st) {
  k_wf_set_base<<<1, 32, 0, st>>>(W.ctr, first_sample);
  return cudaGetLastError();
}

size_t wf_state_bytes(uint32_t n_paths, bool perf, bool sort) {
  size_t per = 6 * sizeof(float4) + sizeof(uint4) + sizeof(float) + 2 * sizeof(uint32_t);
  if (perf) per += sizeof(float) + 3 * sizeof(float4) + sizeof(uint32_t);
  if (sort) per += sizeof(uint32_t) + sizeof(uint8_t);
  return (size_t)n_paths * per;
}

cudaError_t wf_alloc(WfParams& W, uint32_t n_paths, bool perf, bool sort) {
  cudaError_t e;
#define A(ptr, T) \
  if ((e = cudaMalloc(&W.ptr, sizeof(T) * (size_t)n_paths)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&W.path, sizeof(float4) * kRecWords * (size_t)n_paths)) != cudaSuccess) return e;
  A(acc_d, float4);
  A(acc_n, float4);
  A(hit, uint4);
  A(hit_t, float);
  A(queue0, uint32_t);
  A(queue1, uint32_t);
  if (perf) {
    A(mis_pdf, float);
    A(sh_o, float4);
    A(sh_d, float4);
    A(sh_c, float4);
    A(sh_queue, uint32_t);
  }
  if (sort) {
    A(queue_s, uint32_t);
    A(skey, uint8_t);
    if ((e = cudaMalloc(&W.sort_ctr, 2 * kSortKeys * sizeof(uint32_t))) != cudaSuccess) return e;
    if ((e = cudaMemset(W.sort_ctr, 0, 2 * kSortKeys * sizeof(uint32_t))) != cudaSuccess) return e;
  }
#undef A
  if ((e = cudaMalloc(&W.ctr, 16 * sizeof(uint32_t))) != cudaSuccess) return e;
  W.capacity = n_paths;
  return cudaMemset(W.ctr, 0, 16 * sizeof(uint32_t));
}

void wf_free(WfParams& W) {
  cudaFree(W.path);
  cudaFree(W.acc_d);
  cudaFree(W.acc_n);
  cudaFree(W.hit);
  cudaFree(W.hit_t);
  cudaFree(W.queue0);
  cudaFree(W.queue1);
  cudaFree(W.mis_pdf);
  cudaFree(W.sh_o);
  cudaFree(W.sh_d);
  cudaFree(W.sh_c);
  cudaFree(W.sh_queue);
  cudaFree(W.queue_s);
  cudaFree(W.skey);
  cudaFree(W.sort_ctr);
  cudaFree(W.ctr);
  W = WfParams{};
}

using ExtendFn = void (*)(WfParams, int, int);
// Variants: 4, 5, 6, 8 = nested traversal with that many CTAs per SM;
// 14, 15, 16, 18 = flattened traversal with lane refill, 4..8 CTAs per SM.
static ExtendFn extend_fn(bool counters, int variant) {
  switch (variant) {
    case 5: return counters ? k_wf_extend<true, 5> : k_wf_extend<false, 5>;
    case 6: return counters ? k_wf_extend<true, 6> : k_wf_extend<false, 6>;
    case 8: return counters ? k_wf_extend<true, 8> : k_wf_extend<false, 8>;
    case 14: return counters ? k_wf_extend_flat<true, 4> : k_wf_extend_flat<false, 4>;
    case 15: return counters ? k_wf_extend_flat<true, 5> : k_wf_extend_flat<false, 5>;
    case 16: return counters ? k_wf_extend_flat<true, 6> : k_wf_extend_flat<false, 6>;
    case 18: return counters ? k_wf_extend_flat<true, 8> : k_wf_extend_flat<false, 8>;
    // 24 / 34 / 44: as 14 with lanes refilled once 8 / 16 / 24 of them are idle
    case 24: return counters ? k_wf_extend_flat<true, 4, 8> : k_wf_extend_flat<false, 4, 8>;
    case 34: return counters ? k_wf_extend_flat<true, 4, 16> : k_wf_extend_flat<false, 4, 16>;
    case 44: return counters ? k_wf_extend_flat<true, 4, 24> : k_wf_extend_flat<false, 4, 24>;
    // 64 / 74 / 84: as 14, each iteration running one kind of work (vote 1 / 2 / 3);
    // 65: 64 at 5 CTAs per SM; 66 / 67: 64 refilling at 8 / 16 idle lanes
    case 64: return counters ? k_wf_extend_flat<true, 4, 12, 1> : k_wf_extend_flat<false, 4, 12, 1>;
    case 65: return counters ? k_wf_extend_flat<true, 5, 12, 1> : k_wf_extend_flat<false, 5, 12, 1>;
    case 66: return counters ? k_wf_extend_flat<true, 4, 8, 1> : k_wf_extend_flat<false, 4, 8, 1>;
    case 67: return counters ? k_wf_extend_flat<true, 4, 16, 1> : k_wf_extend_flat<false, 4, 16, 1>;
    case 74: return counters ? k_wf_extend_flat<true, 4, 12, 2> : k_wf_extend_flat<false, 4, 12, 2>;
    case 84: return counters ? k_wf_extend_flat<true, 4, 12, 3> : k_wf_extend_flat<false, 4, 12, 3>;
    default: return counters ? k_wf_extend<true, 4> : k_wf_extend<false, 4>;
  }
}

static bool extend_is_flat(int variant) { return variant >= 14; }
static size_t extend_smem(int variant) {
  return extend_is_flat(variant) ? kFlatSmemBytes : kExtStackBytes;
}

static int extend_blocks(ExtendFn fn, size_t smem) {
  static ExtendFn cached_fn[32] = {nullptr};
  static int cached_blocks[32] = {0};
  for (int i = 0; i < 32; ++i) {
    if (cached_fn[i] == fn) return cached_blocks[i];
    if (!cached_fn[i]) {
      int per_sm = 0;
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kExtThreads, smem);
      cached_fn[i] = fn;
      cached_blocks[i] = sm_count() * (per_sm > 0 ? per_sm : 1);
      return cached_blocks[i];
    }
  }
  return sm_count() * 4;
}

// Launch sequence of one wave (capturable: every size is read on the device).
cudaError_t wf_launch_wave(const WfParams& W, bool counters, cudaStream_t st, WaveTimer* tm,
                           const WaveHook* hook) {
  const KernelParams& P = W.kp;
  uint32_t total = P.W * P.H * W.count;
  int gen_blocks = (int)std::min<uint32_t>((total + 255) / 256, (uint32_t)sm_count() * 16);
  k_wf_generate<<<gen_blocks, 256, 0, st>>>(W);
  if (tm) tm->mark(NR_KERNEL_GENERATE, st);
  // extend_variant v, or 100 * v0 + v: variant v0 for the camera rays of
  // bounce 0 and v for the later bounces
  const int v_rest = W.extend_variant % 100;
  const int v_first = W.extend_variant >= 100 ? W.extend_variant / 100 : v_rest;
  ExtendFn ext = extend_fn(counters, v_rest);
  ExtendFn ext0 = extend_fn(counters, v_first);
  const size_t smem = extend_smem(v_rest), smem0 = extend_smem(v_first);
  int eb = extend_blocks(ext, smem), eb0 = extend_blocks(ext0, smem0);
  int shade_blocks = (int)std::min<uint32_t>((total + kShadeThreads - 1) / kShadeThreads,
                                             (uint32_t)sm_count() * 16);
  int scatter_blocks = (int)std::min<uint32_t>((total + kScatterThreads - 1) / kScatterThreads,
                                               (uint32_t)sm_count() * 8);
  for (uint32_t b = 0; b < P.depth; ++b) {
    int q = (int)(b & 1u);
    if (b == 0) ext0<<<eb0, kExtThreads, smem0, st>>>(W, q, 1);
    else ext<<<eb, kExtThreads, smem, st>>>(W, q, 0);
    if (tm) tm->mark(NR_KERNEL_EXTEND, st);
    // the extend kernel counts the material keys and one pass sorts the
    // queue by them (the camera rays' queue is the identity)
    const int identity = b == 0 ? 1 : 0;
    const int sorted = W.queue_s ? 1 : 0;
    if (sorted) {
      k_wf_bin_scatter<<<scatter_blocks, kScatterThreads, 0, st>>>(W, q, identity);
      if (tm) tm->mark(NR_KERNEL_ROTATE, st);
    }
    if (W.mis_pdf) {
      k_wf_shade<true, 1><<<shade_blocks, kShadeThreads, 0, st>>>(W, q, identity, sorted);
      if (tm) tm->mark(NR_KERNEL_SHADE, st);
      k_wf_shadow<<<sm_count() * 4, kExtThreads, kExtStackBytes, st>>>(W);
      if (tm) tm->mark(NR_KERNEL_EXTEND, st);
    } else {
      if (W.shade_variant == 5)
        k_wf_shade<false, 5><<<shade_blocks, kShadeThreads, 0, st>>>(W, q, identity, sorted);
      else if (W.shade_variant == 6)
        k_wf_shade<false, 6><<<shade_blocks, kShadeThreads, 0, st>>>(W, q, identity, sorted);
      else
        k_wf_shade<false, 1><<<shade_blocks, kShadeThreads, 0, st>>>(W, q, identity, sorted);
      if (tm) tm->mark(NR_KERNEL_SHADE, st);
    }
    k_wf_rotate<<<1, 32, 0, st>>>(W, q);
    if (tm) tm->mark(NR_KERNEL_ROTATE, st);
    if (!W.mis_pdf && !counters && W.tail_max_paths > 0 && b >= kTailFrom && b + 1 < P.depth) {
      const int tail_blocks = (int)std::min<uint32_t>((W.tail_max_paths + 127) / 128,
                                                      (uint32_t)sm_count() * 8);
      k_wf_tail<<<tail_blocks, 128, 0, st>>>(W, 1 - q, W.tail_max_paths);
      if (tm) tm->mark(NR_KERNEL_EXTEND, st);
      k_wf_tail_mark<<<1, 32, 0, st>>>(W, 1 - q, W.tail_max_paths);
      if (tm) tm->mark(NR_KERNEL_ROTATE, st);
    }
  }
  if (hook && hook->fn) {
    cudaError_t e = hook->fn(hook->ctx, W, st);
    if (e != cudaSuccess) return e;
  }
  int acc_blocks = (int)std::min<uint32_t>((P.W * P.H + 255) / 256, (uint32_t)sm_count() * 16);
  k_wf_accumulate<<<acc_blocks, 256, 0, st>>>(W);
  if (tm) tm->mark(NR_KERNEL_ACCUMULATE, st);
  k_wf_advance<<<1, 32, 0, st>>>(W);
  if (tm) tm->mark(NR_KERNEL_ROTATE, st);
  return cudaGetLastError();
}

}  // namespace nr
