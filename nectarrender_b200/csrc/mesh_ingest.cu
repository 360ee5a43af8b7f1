// mesh_ingest.cu — OBJ vertex assembly on the GPU (see mesh_ingest.cuh). The
// result equals the host assemble_obj (host_io.cpp), which follows the
// reference loader (nectar_render/csrc/hittable/include/hittable/mesh.h:57-116),
// bit for bit:
//
// 1. Every corner's (v, vt, vn) triple is packed into one 64-bit key and
//    inserted into an open-addressing hash table (linear probing, CAS on the
//    key); each slot keeps the smallest corner index carrying its key
//    (atomicMin): the key's first use.
// 2. A corner that is its key's first use starts a vertex. An exclusive scan
//    of those flags in corner order numbers the vertices in order of first
//    use, as the host's hash map does; a corner's vertex is the number of
//    its key's first corner.
// 3. Missing normals and the tangents are per-vertex sums over the incident
//    triangles in triangle order: the corners are sorted by vertex (a stable
//    radix sort keeps ascending corner order within a vertex) and one thread
//    sums each vertex's run in that order. All arithmetic uses
//    round-to-nearest intrinsics (no FMA contraction, IEEE square root and
//    division), so every value is the host's.
#include "mesh_ingest.cuh"

#include <algorithm>

#include "bvh_build.cuh"

namespace nr {

namespace {

constexpr uint64_t kEmpty = ~0ull;

#define GRID_STRIDE(i, n) \
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

int blocks_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 ld3(const float* p, size_t i) { return F3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void st3(float* p, size_t i, F3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
__device__ __forceinline__ F3 sub(F3 a, F3 b) {
  return F3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ F3 add(F3 a, F3 b) {
  return F3{__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ F3 muls(F3 a, float t) {
  return F3{__fmul_rn(a.x, t), __fmul_rn(a.y, t), __fmul_rn(a.z, t)};
}
__device__ __forceinline__ float len(F3 v) {
  float o = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
  o = __fadd_rn(o, __fmul_rn(v.z, v.z));
  return __fsqrt_rn(o);
}
__device__ __forceinline__ F3 nrm(F3 v) { return muls(v, __fdiv_rn(1.0f, len(v))); }
__device__ __forceinline__ F3 crs(F3 u, F3 v) {
  return F3{__fsub_rn(__fmul_rn(u.y, v.z), __fmul_rn(u.z, v.y)),
            __fsub_rn(__fmul_rn(u.z, v.x), __fmul_rn(u.x, v.z)),
            __fsub_rn(__fmul_rn(u.x, v.y), __fmul_rn(u.y, v.x))};
}
__device__ __forceinline__ float dt(F3 u, F3 v) {
  return __fadd_rn(__fadd_rn(__fmul_rn(u.x, v.x), __fmul_rn(u.y, v.y)), __fmul_rn(u.z, v.z));
}

// 64-bit finaliser of MurmurHash3 (Appleby): spreads the packed keys over
// the table.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__global__ void k_insert(const int32_t* corners, uint32_t n, int bv, int bt, uint64_t* tkeys,
                         uint32_t* tfirst, uint32_t mask, uint32_t* slot, uint32_t* err) {
  GRID_STRIDE(c, n) {
    const uint64_t key = (uint64_t)(uint32_t)corners[3 * c] |
                         ((uint64_t)(uint32_t)(corners[3 * c + 1] + 1) << bv) |
                         ((uint64_t)(uint32_t)(corners[3 * c + 2] + 1) << (bv + bt));
    uint32_t h = (uint32_t)mix64(key) & mask;
    uint32_t s = 0;
    bool placed = false;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(tkeys + h),
                                      (unsigned long long)kEmpty, (unsigned long long)key);
      if (prev == kEmpty || prev == key) {
        atomicMin(tfirst + h, (uint32_t)c);
        s = h;
        placed = true;
        break;
      }
      h = (h + 1) & mask;
    }
    if (!placed) atomicOr(err, 1u);  // table full: cannot happen at load factor <= 1/2
    slot[c] = s;
  }
}

// the first corner of c's key (c itself when the table failed)
__device__ __forceinline__ uint32_t first_of(const uint32_t* slot, const uint32_t* tfirst, size_t c,
                                             uint32_t n) {
  const uint32_t f = tfirst[slot[c]];
  return f < n ? f : (uint32_t)c;
}

__global__ void k_first_flags(const uint32_t* slot, const uint32_t* tfirst, uint32_t n, uint32_t* flags) {
  GRID_STRIDE(c, n) { flags[c] = first_of(slot, tfirst, c, n) == c ? 1u : 0u; }
}

// Vertex numbers of all corners; the first corner of each key writes its
// vertex's position, normal (0 when absent) and uv (0 when absent).
__global__ void k_assign(const int32_t* corners, const uint32_t* slot, const uint32_t* tfirst,
                         const uint32_t* num, uint32_t n, const float* vpos, const float* vnor,
                         const float* vtex, float* P, float* N, float* UV, uint32_t* tri) {
  GRID_STRIDE(c, n) {
    const uint32_t f = first_of(slot, tfirst, c, n);
    const uint32_t vid = num[f];
    tri[c] = vid;
    if (f == c) {
      const int32_t v = corners[3 * c], vt = corners[3 * c + 1], vn = corners[3 * c + 2];
      st3(P, vid, ld3(vpos, (size_t)v));
      st3(N, vid, vn >= 0 ? ld3(vnor, (size_t)vn) : F3{0.f, 0.f, 0.f});
      UV[2 * vid] = vt >= 0 ? vtex[2 * (size_t)vt] : 0.0f;
      UV[2 * vid + 1] = vt >= 0 ? vtex[2 * (size_t)vt + 1] : 0.0f;
    }
  }
}

__global__ void k_face_normals(const float* P, const uint32_t* tri, uint32_t nt, float* fn) {
  GRID_STRIDE(t, nt) {
    const F3 a = ld3(P, tri[3 * t]), b = ld3(P, tri[3 * t + 1]), c = ld3(P, tri[3 * t + 2]);
    st3(fn, t, nrm(crs(sub(b, a), sub(c, a))));
  }
}

__global__ void k_face_tangents(const float* P, const float* UV, const uint32_t* tri, uint32_t nt,
                                float* tg) {
  GRID_STRIDE(t, nt) {
    const uint32_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    const F3 pa = ld3(P, a);
    const F3 e1 = sub(ld3(P, b), pa), e2 = sub(ld3(P, c), pa);
    const float du1 = __fsub_rn(UV[2 * b], UV[2 * a]), dv1 = __fsub_rn(UV[2 * b + 1], UV[2 * a + 1]);
    const float du2 = __fsub_rn(UV[2 * c], UV[2 * a]), dv2 = __fsub_rn(UV[2 * c + 1], UV[2 * a + 1]);
    const float denom = __fsub_rn(__fmul_rn(du1, dv2), __fmul_rn(du2, dv1));
    st3(tg, t, fabsf(denom) < 1e-8f ? F3{1.f, 0.f, 0.f}
                                    : muls(sub(muls(e1, dv2), muls(e2, dv1)), __fdiv_rn(1.0f, denom)));
  }
}

// One thread per vertex run of the vertex-sorted corners (vert[i] = vertex,
// corner[i] = corner index, ascending within a run): the run's face normals
// (when the file has none) and face tangents summed in triangle order, then
// finished as the host does.
__global__ void k_vertex_sums(const uint32_t* vert, const uint32_t* corner, uint32_t n,
                              const float* fn, const float* tg, bool gen_normals, float* N, float* T) {
  GRID_STRIDE(i, n) {
    const uint32_t v = vert[i];
    if (i > 0 && vert[i - 1] == v) continue;
    F3 nacc = gen_normals ? F3{0.f, 0.f, 0.f} : ld3(N, v), tacc{0.f, 0.f, 0.f};
    for (size_t j = i; j < n && vert[j] == v; ++j) {
      const uint32_t t = corner[j] / 3;
      if (gen_normals) nacc = add(nacc, ld3(fn, t));
      tacc = add(tacc, ld3(tg, t));
    }
    if (gen_normals) nacc = len(nacc) < 1e-8f ? F3{0.f, 1.f, 0.f} : nrm(nacc);
    const F3 t = sub(tacc, muls(nacc, dt(tacc, nacc)));
    st3(N, v, nacc);
    st3(T, v, len(t) < 1e-8f ? F3{1.f, 0.f, 0.f} : nrm(t));
  }
}

__global__ void k_iota(uint32_t* a, uint32_t n) {
  GRID_STRIDE(i, n) { a[i] = (uint32_t)i; }
}

int bits_for(uint64_t max_value) {
  int b = 0;
  while (b < 64 && (max_value >> b) != 0) ++b;
  return b;
}

struct DevBufs {
  std::vector<void*> p;
  ~DevBufs() {
    for (void* q : p) cudaFree(q);
  }
  template <typename T>
  cudaError_t get(T*& out, size_t count) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, std::max<size_t>(1, count) * sizeof(T));
    if (e == cudaSuccess) {
      p.push_back(v);
      out = static_cast<T*>(v);
    }
    return e;
  }
};

}  // namespace

std::string assemble_obj_device(const ObjRaw& raw, HostMesh& out, cudaStream_t st) {
  const size_t n64 = raw.corners.size() / 3;
  if (n64 == 0) {
    out = HostMesh{};
    return {};
  }
  if (n64 >= (1ull << 31)) return "device OBJ assembly: too many corners";
  const uint32_t n = (uint32_t)n64, nt = n / 3;
  const uint64_t nvr = raw.vpos.size() / 3, ntr = raw.vtex.size() / 2, nnr = raw.vnor.size() / 3;
  const int bv = bits_for(nvr ? nvr - 1 : 0), bt = bits_for(ntr), bn = bits_for(nnr);
  if (bv + bt + bn > 63)
    return "device OBJ assembly: the v/vt/vn index ranges need more than 63 key bits";
  uint32_t cap = 1;
  while (cap < 2u * n) cap <<= 1;
  DevBufs b;
  int32_t* corners;
  float *vpos, *vnor, *vtex;
  uint64_t* tkeys;
  uint32_t *tfirst, *slot, *flags, *sums, *num, *counts, *tri;
  cudaError_t e = cudaSuccess;
#define DB(ptr, cnt) \
  if ((e = b.get(ptr, cnt)) != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  DB(corners, 3 * (size_t)n);
  DB(vpos, raw.vpos.size());
  DB(vnor, raw.vnor.size());
  DB(vtex, raw.vtex.size());
  DB(tkeys, cap);
  DB(tfirst, cap);
  DB(slot, n);
  DB(flags, n);
  DB(sums, scan_scratch_words(n));
  DB(num, n);
  DB(counts, 2);
  DB(tri, n);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes && e == cudaSuccess) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  };
  up(corners, raw.corners.data(), raw.corners.size() * 4);
  up(vpos, raw.vpos.data(), raw.vpos.size() * 4);
  up(vnor, raw.vnor.data(), raw.vnor.size() * 4);
  up(vtex, raw.vtex.data(), raw.vtex.size() * 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(tkeys, 0xff, (size_t)cap * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(tfirst, 0xff, (size_t)cap * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, 8, st);
  if (e != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  k_insert<<<blocks_for(n), 256, 0, st>>>(corners, n, bv, bt, tkeys, tfirst, cap - 1, slot, counts + 1);
  k_first_flags<<<blocks_for(n), 256, 0, st>>>(slot, tfirst, n, flags);
  e = scan_exclusive(flags, num, n, sums, counts, st);
  if (e != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  uint32_t hc[2] = {0, 0};
  e = cudaMemcpyAsync(hc, counts, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  if (hc[1]) return "device OBJ assembly: hash table overflow";
  const uint32_t nv = hc[0];
  float *P, *N, *T, *UV, *fn = nullptr, *tg;
  DB(P, 3 * (size_t)nv);
  DB(N, 3 * (size_t)nv);
  DB(T, 3 * (size_t)nv);
  DB(UV, 2 * (size_t)nv);
  DB(tg, 3 * (size_t)nt);
  const bool gen_normals = raw.vnor.empty();
  if (gen_normals) DB(fn, 3 * (size_t)nt);
  k_assign<<<blocks_for(n), 256, 0, st>>>(corners, slot, tfirst, num, n, vpos, vnor, vtex, P, N, UV, tri);
  if (gen_normals) k_face_normals<<<blocks_for(nt), 256, 0, st>>>(P, tri, nt, fn);
  k_face_tangents<<<blocks_for(nt), 256, 0, st>>>(P, UV, tri, nt, tg);
  // corners grouped by vertex, ascending corner index within a vertex
  uint32_t *vk, *cv, *vk2, *cv2, *hist, *sk, *sv;
  DB(vk, n);
  DB(cv, n);
  DB(vk2, n);
  DB(cv2, n);
  DB(hist, radix_sort_hist_words(n));
#undef DB
  e = cudaMemcpyAsync(vk, tri, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  k_iota<<<blocks_for(n), 256, 0, st>>>(cv, n);
  e = radix_sort_pairs(vk, cv, vk2, cv2, n, bits_for(nv ? nv - 1 : 0), hist, st, &sk, &sv);
  if (e != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  k_vertex_sums<<<blocks_for(n), 256, 0, st>>>(sk, sv, n, fn, tg, gen_normals, N, T);
  out = HostMesh{};
  out.positions.resize(3 * (size_t)nv);
  out.normals.resize(3 * (size_t)nv);
  out.tangents.resize(3 * (size_t)nv);
  out.uvs.resize(2 * (size_t)nv);
  out.triangles.resize(n);
  auto down = [&](void* dst, const void* src, size_t bytes) {
    if (bytes && e == cudaSuccess) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
  };
  e = cudaGetLastError();
  down(out.positions.data(), P, out.positions.size() * 4);
  down(out.normals.data(), N, out.normals.size() * 4);
  down(out.tangents.data(), T, out.tangents.size() * 4);
  down(out.uvs.data(), UV, out.uvs.size() * 4);
  down(out.triangles.data(), tri, out.triangles.size() * 4);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return std::string("device OBJ assembly: ") + cudaGetErrorString(e);
  return {};
}

}  // namespace nr
