// bvh_build.cu — GPU binned-SAH BVH builder and wide-BVH collapse.
//
// Replaces the reference's single-threaded host builder BVH<T>::build
// (nectar_render/csrc/hittable/include/bvh/bvh.h:35-320): recursive top-down
// splitting with 16 centroid bins on each axis, cost A_L*N_L + A_R*N_R, a
// median split when no bin split exists, one primitive per leaf.
//
// Here:
//  1. Morton pre-sort: 30-bit Morton codes of the centroids, sorted by an LSD
//     radix sort (8-bit digits, stable per-tile ranks), so that every node's
//     primitive range is spatially coherent in memory.
//  2. Level-synchronous top-down build with 32 centroid bins per axis and the
//     reference's cost function. Nodes with more than kSmall primitives are
//     binned by many CTAs: within a warp, lanes whose primitives fall in the
//     same bin are grouped with __match_any_sync and their boxes reduced with
//     redux.sync min/max before one shared-memory atomic per group. A warp
//     per node evaluates the 32 split planes (one lane per bin, prefix and
//     suffix scans by shuffles). Primitives are partitioned stably.
//  3. Nodes with at most kSmall primitives are finished by one warp each in
//     shared memory (same binning and cost, smaller child first).
//  4. The binary tree (leaf size 1, as the reference) is laid out as 64-byte
//     two-child nodes and collapsed greedily into 8-wide nodes with quantised
//     child boxes (Ylitie et al. 2017), child slots ordered by octant.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <utility>
#include "bvh_build.cuh"

namespace nr {
namespace {

constexpr int kBins = 32;
constexpr uint32_t kSmall = 256;
constexpr int kChunk = 2048;  // primitives per CTA in the large-node passes
constexpr int kPassThreads = 256;
constexpr float kEps = 1e-4f;  // reference EPS: axes with a smaller centroid extent are skipped

__device__ __forceinline__ uint32_t f2key(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key2f(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(u);
}
__device__ __forceinline__ float3 centroid(const float4& lo, const float4& hi) {
  return make_float3((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f);
}
__device__ __forceinline__ float cget(const float3& c, int a) { return a == 0 ? c.x : (a == 1 ? c.y : c.z); }
__device__ __forceinline__ float fget(const float4& c, int a) { return a == 0 ? c.x : (a == 1 ? c.y : c.z); }
__device__ __forceinline__ int bin_of(float c, float cmin, float extent) {
  int b = (int)(kBins * (c - cmin) / extent);
  return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}
__device__ __forceinline__ float area6(float lx, float ly, float lz, float hx, float hy, float hz) {
  float dx = hx - lx, dy = hy - ly, dz = hz - lz;
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// ---------------------------------------------------------------------------
// Morton codes

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void k_bounds(const float4* lo, const float4* hi, uint32_t n, uint32_t* gk) {
  // gk: [0..2] min centroid keys, [3..5] max centroid keys, [6..8] min box, [9..11] max box
  uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
  uint32_t bmn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, bmx[3] = {0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 l = lo[i], h = hi[i];
    float3 c = centroid(l, h);
    for (int a = 0; a < 3; ++a) {
      uint32_t k = f2key(cget(c, a));
      mn[a] = min(mn[a], k);
      mx[a] = max(mx[a], k);
      bmn[a] = min(bmn[a], f2key(fget(l, a)));
      bmx[a] = max(bmx[a], f2key(fget(h, a)));
    }
  }
  for (int a = 0; a < 3; ++a) {
    uint32_t v0 = __reduce_min_sync(0xffffffffu, mn[a]);
    uint32_t v1 = __reduce_max_sync(0xffffffffu, mx[a]);
    uint32_t v2 = __reduce_min_sync(0xffffffffu, bmn[a]);
    uint32_t v3 = __reduce_max_sync(0xffffffffu, bmx[a]);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(gk + a, v0);
      atomicMax(gk + 3 + a, v1);
      atomicMin(gk + 6 + a, v2);
      atomicMax(gk + 9 + a, v3);
    }
  }
}

__global__ void k_morton(const float4* lo, const float4* hi, uint32_t n, const uint32_t* gk,
                         uint32_t* keys, uint32_t* vals) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float3 c = centroid(lo[i], hi[i]);
  uint32_t code = 0;
  for (int a = 0; a < 3; ++a) {
    float mn = key2f(gk[a]), mx = key2f(gk[3 + a]);
    float ext = mx - mn;
    float t = ext > 0.0f ? (cget(c, a) - mn) / ext : 0.0f;
    uint32_t q = (uint32_t)fminf(fmaxf(t * 1024.0f, 0.0f), 1023.0f);
    code |= expand10(q) << (2 - a);
  }
  keys[i] = code;
  vals[i] = i;
}

// ---------------------------------------------------------------------------
// LSD radix sort of (key, value) pairs, 8-bit digits, stable.

constexpr int kRsThreads = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsThreads * kRsItems;

__global__ void k_rs_hist(const uint32_t* keys, uint32_t n, int shift, uint32_t* hist,
                          uint32_t nblocks) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  uint32_t base = blockIdx.x * kRsTile;
  for (int k = 0; k < kRsItems; ++k) {
    uint32_t i = base + k * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of a uint32 array by one CTA (used for histograms and small lists).
__global__ void k_scan_single(uint32_t* a, uint32_t n, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < n; base += blockDim.x) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < n ? a[i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < blockDim.x / 32 ? warp_sums[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= (uint32_t)o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t prefix = carry + (warp > 0 ? warp_sums[warp - 1] : 0u) + x - v;
    if (i < n) a[i] = prefix;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = prefix + v;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// Multi-block exclusive scan (scan_exclusive): pass 1, the sum of each
// kScanTile-element tile.
constexpr uint32_t kScanTile = 1024;
__global__ void __launch_bounds__(kScanTile) k_scan_tile_sums(const uint32_t* a, uint32_t n,
                                                              uint32_t* sums) {
  __shared__ uint32_t w[32];
  const uint32_t i = blockIdx.x * kScanTile + threadIdx.x;
  uint32_t v = i < n ? a[i] : 0u;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31u) == 0) w[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t t = w[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = t;
  }
}

// Pass 3: the scan inside each tile plus the tile's offset (out may be in).
__global__ void __launch_bounds__(kScanTile) k_scan_tile_apply(const uint32_t* in, uint32_t n,
                                                               const uint32_t* sums,
                                                               uint32_t* out) {
  __shared__ uint32_t w[32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t i = blockIdx.x * kScanTile + threadIdx.x;
  const uint32_t v = i < n ? in[i] : 0u;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) w[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = w[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= (uint32_t)o) t += y;
    }
    w[lane] = t;
  }
  __syncthreads();
  if (i < n) out[i] = sums[blockIdx.x] + (warp ? w[warp - 1] : 0u) + x - v;
}

__global__ void k_rs_scatter(const uint32_t* kin, const uint32_t* vin, uint32_t* kout,
                             uint32_t* vout, uint32_t n, int shift, const uint32_t* hist,
                             uint32_t nblocks) {
  __shared__ uint32_t offs[256];
  __shared__ uint32_t wcnt[kRsThreads / 32][256];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  offs[threadIdx.x] = hist[threadIdx.x * nblocks + blockIdx.x];
  __syncthreads();
  uint32_t base = blockIdx.x * kRsTile;
  for (int k = 0; k < kRsItems; ++k) {
    uint32_t i = base + k * kRsThreads + threadIdx.x;
    bool valid = i < n;
    uint32_t key = valid ? kin[i] : 0u;
    uint32_t d = (key >> shift) & 0xffu;
    uint32_t tag = valid ? d : (0x100u | lane);
    uint32_t mask = __match_any_sync(0xffffffffu, tag);
    uint32_t rank = __popc(mask & ((1u << lane) - 1u));
    for (int j = lane; j < 256; j += 32) wcnt[warp][j] = 0u;
    __syncwarp();
    if (valid && rank == 0) wcnt[warp][d] = __popc(mask);
    __syncthreads();
    if (valid) {
      uint32_t pre = 0;
      for (uint32_t w = 0; w < warp; ++w) pre += wcnt[w][d];
      uint32_t pos = offs[d] + pre + rank;
      kout[pos] = key;
      vout[pos] = vin[i];
    }
    __syncthreads();
    uint32_t tot = 0;
    for (int w = 0; w < kRsThreads / 32; ++w) tot += wcnt[w][threadIdx.x];
    offs[threadIdx.x] += tot;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// build structures

struct Task {
  uint32_t node, start, count, pad;
  float cmin[3], cmax[3];
};

// Per-task bins: keys of float min/max, counts.
struct TaskBins {
  uint32_t cnt[3][kBins];
  uint32_t blo[3][kBins][3], bhi[3][kBins][3];  // primitive box bounds
  uint32_t clo[3][kBins][3], chi[3][kBins][3];  // centroid bounds
};

struct SplitInfo {
  int axis;  // -1: median split
  int bin;
  uint32_t nleft;
  uint32_t pad;
};

__global__ void k_init_bins(TaskBins* bins, uint32_t n_tasks) {
  uint32_t words = sizeof(TaskBins) / 4u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_tasks * words;
       i += gridDim.x * blockDim.x) {
    uint32_t t = i / words, w = i % words;
    uint32_t* p = reinterpret_cast<uint32_t*>(bins + t) + w;
    // layout: cnt (96 words) = 0, then [blo, bhi, clo, chi] alternating min/max init
    uint32_t v;
    if (w < 3 * kBins) v = 0u;
    else {
      uint32_t r = (w - 3 * kBins) / (3 * kBins * 3);  // 0 blo, 1 bhi, 2 clo, 3 chi
      v = (r == 0 || r == 2) ? 0xffffffffu : 0u;
    }
    *p = v;
  }
}

// Block -> task map for the large-task passes.
__global__ void k_task_blocks(const Task* tasks, uint32_t n_tasks, uint32_t* blk_start) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n_tasks) blk_start[t] = (tasks[t].count + kChunk - 1) / kChunk;
}
__global__ void k_fill_block_map(const uint32_t* blk_start, uint32_t n_tasks, uint32_t* blk_task,
                                 const Task* tasks) {
  uint32_t t = blockIdx.x;
  if (t >= n_tasks) return;
  uint32_t nb = (tasks[t].count + kChunk - 1) / kChunk;
  for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) blk_task[blk_start[t] + b] = t;
}

// Large-task binning with warp-cooperative reductions.
__global__ void __launch_bounds__(kPassThreads) k_bin_large(
    const float4* lo, const float4* hi, const uint32_t* order, const Task* tasks,
    const uint32_t* blk_task, const uint32_t* blk_start, TaskBins* gbins) {
  __shared__ TaskBins sb;
  const uint32_t t = blk_task[blockIdx.x];
  const Task T = tasks[t];
  const uint32_t chunk = blockIdx.x - blk_start[t];
  {
    uint32_t* p = reinterpret_cast<uint32_t*>(&sb);
    uint32_t words = sizeof(TaskBins) / 4u;
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
      uint32_t v;
      if (w < 3 * kBins) v = 0u;
      else {
        uint32_t r = (w - 3 * kBins) / (3 * kBins * 3);
        v = (r == 0 || r == 2) ? 0xffffffffu : 0u;
      }
      p[w] = v;
    }
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t begin = T.start + chunk * kChunk;
  uint32_t end = min(T.start + T.count, begin + kChunk);
  for (uint32_t base = begin; base < end; base += blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool valid = i < end;
    float4 l = make_float4(0, 0, 0, 0), h = make_float4(0, 0, 0, 0);
    if (valid) {
      uint32_t p = order[i];
      l = lo[p];
      h = hi[p];
    }
    float3 c = centroid(l, h);
    for (int a = 0; a < 3; ++a) {
      float ext = T.cmax[a] - T.cmin[a];
      if (ext < kEps) continue;
      int b = valid ? bin_of(cget(c, a), T.cmin[a], ext) : (kBins + (int)lane);
      uint32_t grp = __match_any_sync(0xffffffffu, b);
      bool leader = valid && ((grp & ((1u << lane) - 1u)) == 0u);
      // reductions restricted to the lanes of this bin
      uint32_t vlo[3], vhi[3], vclo[3], vchi[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        uint32_t klo = valid ? f2key(fget(l, k)) : 0xffffffffu;
        uint32_t khi = valid ? f2key(fget(h, k)) : 0u;
        uint32_t kc = valid ? f2key(cget(c, k)) : 0xffffffffu;
        uint32_t kc2 = valid ? f2key(cget(c, k)) : 0u;
        vlo[k] = __reduce_min_sync(grp, klo);
        vhi[k] = __reduce_max_sync(grp, khi);
        vclo[k] = __reduce_min_sync(grp, kc);
        vchi[k] = __reduce_max_sync(grp, kc2);
      }
      if (leader) {
        atomicAdd(&sb.cnt[a][b], (uint32_t)__popc(grp));
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          atomicMin(&sb.blo[a][b][k], vlo[k]);
          atomicMax(&sb.bhi[a][b][k], vhi[k]);
          atomicMin(&sb.clo[a][b][k], vclo[k]);
          atomicMax(&sb.chi[a][b][k], vchi[k]);
        }
      }
    }
  }
  __syncthreads();
  TaskBins* g = gbins + t;
  for (uint32_t w = threadIdx.x; w < 3 * kBins; w += blockDim.x) {
    uint32_t a = w / kBins, b = w % kBins;
    uint32_t cnt = sb.cnt[a][b];
    if (cnt == 0) continue;
    atomicAdd(&g->cnt[a][b], cnt);
    for (int k = 0; k < 3; ++k) {
      atomicMin(&g->blo[a][b][k], sb.blo[a][b][k]);
      atomicMax(&g->bhi[a][b][k], sb.bhi[a][b][k]);
      atomicMin(&g->clo[a][b][k], sb.clo[a][b][k]);
      atomicMax(&g->chi[a][b][k], sb.chi[a][b][k]);
    }
  }
}

// Warp-wide evaluation of the split planes for one set of bins. Lane b holds
// bin b of each axis. Returns the best (cost, axis, bin) and the child
// bounds on lane 0 via the out arrays.
struct SplitOut {
  float cost;
  int axis, bin;
  uint32_t nl;
  float lbox[6], rbox[6], lcb[6], rcb[6];
};

__device__ __forceinline__ void warp_eval(const uint32_t (*cnt)[kBins],
                                          const uint32_t (*blo)[kBins][3],
                                          const uint32_t (*bhi)[kBins][3],
                                          const uint32_t (*clo)[kBins][3],
                                          const uint32_t (*chi)[kBins][3],
                                          const float* cmin, const float* cmax, SplitOut& out) {
  const uint32_t lane = threadIdx.x & 31u;
  float best = 3.4e38f;
  int best_axis = -1, best_bin = -1;
  for (int a = 0; a < 3; ++a) {
    float ext = cmax[a] - cmin[a];
    if (ext < kEps) continue;
    uint32_t c = cnt[a][lane];
    uint32_t l0 = blo[a][lane][0], l1 = blo[a][lane][1], l2 = blo[a][lane][2];
    uint32_t h0 = bhi[a][lane][0], h1 = bhi[a][lane][1], h2 = bhi[a][lane][2];
    // inclusive prefix (left) and suffix (right) of counts and boxes
    uint32_t pc = c, pl0 = l0, pl1 = l1, pl2 = l2, ph0 = h0, ph1 = h1, ph2 = h2;
    uint32_t sc = c, sl0 = l0, sl1 = l1, sl2 = l2, sh0 = h0, sh1 = h1, sh2 = h2;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y;
      y = __shfl_up_sync(0xffffffffu, pc, o); if (lane >= (uint32_t)o) pc += y;
      y = __shfl_up_sync(0xffffffffu, pl0, o); if (lane >= (uint32_t)o) pl0 = min(pl0, y);
      y = __shfl_up_sync(0xffffffffu, pl1, o); if (lane >= (uint32_t)o) pl1 = min(pl1, y);
      y = __shfl_up_sync(0xffffffffu, pl2, o); if (lane >= (uint32_t)o) pl2 = min(pl2, y);
      y = __shfl_up_sync(0xffffffffu, ph0, o); if (lane >= (uint32_t)o) ph0 = max(ph0, y);
      y = __shfl_up_sync(0xffffffffu, ph1, o); if (lane >= (uint32_t)o) ph1 = max(ph1, y);
      y = __shfl_up_sync(0xffffffffu, ph2, o); if (lane >= (uint32_t)o) ph2 = max(ph2, y);
      y = __shfl_down_sync(0xffffffffu, sc, o); if (lane + o < 32) sc += y;
      y = __shfl_down_sync(0xffffffffu, sl0, o); if (lane + o < 32) sl0 = min(sl0, y);
      y = __shfl_down_sync(0xffffffffu, sl1, o); if (lane + o < 32) sl1 = min(sl1, y);
      y = __shfl_down_sync(0xffffffffu, sl2, o); if (lane + o < 32) sl2 = min(sl2, y);
      y = __shfl_down_sync(0xffffffffu, sh0, o); if (lane + o < 32) sh0 = max(sh0, y);
      y = __shfl_down_sync(0xffffffffu, sh1, o); if (lane + o < 32) sh1 = max(sh1, y);
      y = __shfl_down_sync(0xffffffffu, sh2, o); if (lane + o < 32) sh2 = max(sh2, y);
    }
    // right side of split after bin `lane` is the suffix starting at lane+1
    uint32_t rc = __shfl_down_sync(0xffffffffu, sc, 1);
    uint32_t rl0 = __shfl_down_sync(0xffffffffu, sl0, 1), rl1 = __shfl_down_sync(0xffffffffu, sl1, 1),
             rl2 = __shfl_down_sync(0xffffffffu, sl2, 1);
    uint32_t rh0 = __shfl_down_sync(0xffffffffu, sh0, 1), rh1 = __shfl_down_sync(0xffffffffu, sh1, 1),
             rh2 = __shfl_down_sync(0xffffffffu, sh2, 1);
    float cost = 3.4e38f;
    if (lane < 31 && pc > 0 && rc > 0) {
      float al = area6(key2f(pl0), key2f(pl1), key2f(pl2), key2f(ph0), key2f(ph1), key2f(ph2));
      float ar = area6(key2f(rl0), key2f(rl1), key2f(rl2), key2f(rh0), key2f(rh1), key2f(rh2));
      cost = al * (float)pc + ar * (float)rc;
    }
    // argmin over lanes, ties to the lowest bin
    float mc = cost;
    int mb = (int)lane;
    for (int o = 16; o > 0; o >>= 1) {
      float oc = __shfl_xor_sync(0xffffffffu, mc, o);
      int ob = __shfl_xor_sync(0xffffffffu, mb, o);
      if (oc < mc || (oc == mc && ob < mb)) {
        mc = oc;
        mb = ob;
      }
    }
    if (mc < best) {
      best = mc;
      best_axis = a;
      best_bin = mb;
    }
  }
  out.cost = best;
  out.axis = best_axis;
  out.bin = best_bin;
  if (best_axis < 0) return;
  // child bounds: reduce bins [0, bin] and [bin+1, 31] of the chosen axis
  int a = best_axis;
  bool left = (int)lane <= best_bin;
  uint32_t c = cnt[a][lane];
  uint32_t v[12];
  for (int k = 0; k < 3; ++k) {
    v[k] = c ? blo[a][lane][k] : 0xffffffffu;
    v[3 + k] = c ? bhi[a][lane][k] : 0u;
    v[6 + k] = c ? clo[a][lane][k] : 0xffffffffu;
    v[9 + k] = c ? chi[a][lane][k] : 0u;
  }
  uint32_t lmask = __ballot_sync(0xffffffffu, left);
  uint32_t nl = __reduce_add_sync(0xffffffffu, left ? c : 0u);
  out.nl = nl;
  for (int k = 0; k < 12; ++k) {
    bool is_min = (k < 3) || (k >= 6 && k < 9);
    uint32_t lv = left ? v[k] : (is_min ? 0xffffffffu : 0u);
    uint32_t rv = !left ? v[k] : (is_min ? 0xffffffffu : 0u);
    uint32_t L = is_min ? __reduce_min_sync(0xffffffffu, lv) : __reduce_max_sync(0xffffffffu, lv);
    uint32_t R = is_min ? __reduce_min_sync(0xffffffffu, rv) : __reduce_max_sync(0xffffffffu, rv);
    int g = k / 3, kk = k % 3;
    float* dl = g == 0 ? out.lbox : (g == 1 ? out.lbox + 3 : (g == 2 ? out.lcb : out.lcb + 3));
    float* dr = g == 0 ? out.rbox : (g == 1 ? out.rbox + 3 : (g == 2 ? out.rcb : out.rcb + 3));
    dl[kk] = key2f(L);
    dr[kk] = key2f(R);
  }
  (void)lmask;
}

__device__ __forceinline__ void write_node(BinNode* nodes, uint32_t id, const float* box,
                                           uint32_t start, uint32_t count) {
  BinNode n;
  for (int k = 0; k < 3; ++k) {
    n.lo[k] = box[k];
    n.hi[k] = box[3 + k];
  }
  n.left = -1;
  n.right = -1;
  n.start = start;
  n.count = count;
  nodes[id] = n;
}

// One warp per large task: choose the split, create the two children, queue them.
__global__ void k_split_large(const Task* tasks, uint32_t n_tasks, const TaskBins* gbins,
                              SplitInfo* splits, BinNode* nodes, uint32_t* node_counter,
                              Task* next_large, uint32_t* n_next_large, Task* small,
                              uint32_t* n_small, uint32_t* err) {
  uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (t >= n_tasks) return;
  Task T = tasks[t];
  const TaskBins& B = gbins[t];
  SplitOut so;
  warp_eval(B.cnt, B.blo, B.bhi, B.clo, B.chi, T.cmin, T.cmax, so);
  if (lane != 0) return;
  SplitInfo si;
  BinNode parent = nodes[T.node];
  float pbox[6] = {parent.lo[0], parent.lo[1], parent.lo[2], parent.hi[0], parent.hi[1], parent.hi[2]};
  Task L, R;
  if (so.axis < 0) {
    // no bin split (all centroid extents below EPS): median of the current order
    si.axis = -1;
    si.bin = -1;
    si.nleft = T.count / 2;
    for (int k = 0; k < 6; ++k) { so.lbox[k] = pbox[k]; so.rbox[k] = pbox[k]; }
    for (int k = 0; k < 3; ++k) {
      so.lcb[k] = T.cmin[k]; so.lcb[3 + k] = T.cmax[k];
      so.rcb[k] = T.cmin[k]; so.rcb[3 + k] = T.cmax[k];
    }
  } else {
    si.axis = so.axis;
    si.bin = so.bin;
    si.nleft = so.nl;
  }
  if (si.nleft == 0 || si.nleft >= T.count) {
    // cannot happen with consistent binning; guarantees progress regardless
    atomicOr(err, 16u);
    si.axis = -1;
    si.bin = -1;
    si.nleft = T.count / 2;
    for (int k = 0; k < 6; ++k) { so.lbox[k] = pbox[k]; so.rbox[k] = pbox[k]; }
    for (int k = 0; k < 3; ++k) {
      so.lcb[k] = T.cmin[k]; so.lcb[3 + k] = T.cmax[k];
      so.rcb[k] = T.cmin[k]; so.rcb[3 + k] = T.cmax[k];
    }
  }
  splits[t] = si;
  uint32_t id = atomicAdd(node_counter, 2u);
  uint32_t nl = si.nleft, nr = T.count - si.nleft;
  write_node(nodes, id, so.lbox, T.start, nl);
  write_node(nodes, id + 1, so.rbox, T.start + nl, nr);
  nodes[T.node].left = (int32_t)id;
  nodes[T.node].right = (int32_t)(id + 1);
  L.node = id; L.start = T.start; L.count = nl;
  R.node = id + 1; R.start = T.start + nl; R.count = nr;
  for (int k = 0; k < 3; ++k) {
    L.cmin[k] = so.lcb[k]; L.cmax[k] = so.lcb[3 + k];
    R.cmin[k] = so.rcb[k]; R.cmax[k] = so.rcb[3 + k];
  }
  L.pad = R.pad = 0;
  Task kids[2] = {L, R};
  for (int c = 0; c < 2; ++c) {
    if (kids[c].count > kSmall) next_large[atomicAdd(n_next_large, 1u)] = kids[c];
    else if (kids[c].count > 1) small[atomicAdd(n_small, 1u)] = kids[c];
    else if (kids[c].count == 0) atomicOr(err, 2u);
  }
}

__device__ __forceinline__ bool goes_left(const Task& T, const SplitInfo& si, uint32_t pos,
                                          const float4& l, const float4& h) {
  if (si.axis < 0) return pos < T.start + si.nleft;
  float3 c = centroid(l, h);
  float ext = T.cmax[si.axis] - T.cmin[si.axis];
  return bin_of(cget(c, si.axis), T.cmin[si.axis], ext) <= si.bin;
}

__global__ void __launch_bounds__(kPassThreads) k_part_count(
    const float4* lo, const float4* hi, const uint32_t* order, const Task* tasks,
    const SplitInfo* splits, const uint32_t* blk_task, const uint32_t* blk_start,
    uint32_t* blk_left) {
  __shared__ uint32_t s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  const uint32_t t = blk_task[blockIdx.x];
  const Task T = tasks[t];
  const SplitInfo si = splits[t];
  uint32_t chunk = blockIdx.x - blk_start[t];
  uint32_t begin = T.start + chunk * kChunk, end = min(T.start + T.count, begin + kChunk);
  uint32_t cnt = 0;
  for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    uint32_t p = order[i];
    cnt += goes_left(T, si, i, lo[p], hi[p]) ? 1u : 0u;
  }
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s, cnt);
  __syncthreads();
  if (threadIdx.x == 0) blk_left[blockIdx.x] = s;
}

// exclusive scan of the per-block left counts inside each task (one warp per task)
__global__ void k_part_scan(const Task* tasks, uint32_t n_tasks, const uint32_t* blk_start,
                            uint32_t* blk_left) {
  uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (t >= n_tasks) return;
  uint32_t nb = (tasks[t].count + kChunk - 1) / kChunk;
  uint32_t b0 = blk_start[t];
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nb; base += 32) {
    uint32_t i = base + lane;
    uint32_t v = i < nb ? blk_left[b0 + i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (i < nb) blk_left[b0 + i] = carry + x - v;
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
}

__global__ void __launch_bounds__(kPassThreads) k_part_scatter(
    const float4* lo, const float4* hi, const uint32_t* order, uint32_t* order_tmp,
    const Task* tasks, const SplitInfo* splits, const uint32_t* blk_task,
    const uint32_t* blk_start, const uint32_t* blk_left) {
  __shared__ uint32_t warp_l[kPassThreads / 32];
  __shared__ uint32_t run_l, run_r;
  const uint32_t t = blk_task[blockIdx.x];
  const Task T = tasks[t];
  const SplitInfo si = splits[t];
  uint32_t chunk = blockIdx.x - blk_start[t];
  uint32_t begin = T.start + chunk * kChunk, end = min(T.start + T.count, begin + kChunk);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t left_base = T.start + blk_left[blockIdx.x];
  uint32_t right_base = T.start + si.nleft + ((begin - T.start) - blk_left[blockIdx.x]);
  if (threadIdx.x == 0) { run_l = 0; run_r = 0; }
  __syncthreads();
  for (uint32_t base = begin; base < end; base += blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool valid = i < end;
    uint32_t p = valid ? order[i] : 0u;
    bool L = valid && goes_left(T, si, i, lo[p], hi[p]);
    uint32_t bl = __ballot_sync(0xffffffffu, L);
    uint32_t bv = __ballot_sync(0xffffffffu, valid);
    if (lane == 0) warp_l[warp] = __popc(bl);
    __syncthreads();
    uint32_t pre_l = 0, tot_l = 0;
    for (uint32_t w = 0; w < kPassThreads / 32; ++w) {
      if (w < warp) pre_l += warp_l[w];
      tot_l += warp_l[w];
    }
    uint32_t rank_l = pre_l + __popc(bl & ((1u << lane) - 1u));
    uint32_t pos_in_round = (base - begin) ;
    (void)pos_in_round;
    // rank among right elements = (index within round) - (lefts before me)
    uint32_t idx_in_round = threadIdx.x;
    uint32_t rank_r = idx_in_round - rank_l;
    if (valid) {
      if (L) order_tmp[left_base + run_l + rank_l] = p;
      else order_tmp[right_base + run_r + rank_r] = p;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t nvalid = min((uint32_t)blockDim.x, end - base);
      run_l += tot_l;
      run_r += nvalid - tot_l;
    }
    (void)bv;
    __syncthreads();
  }
}

__global__ void k_copy_ranges(const Task* tasks, const uint32_t* blk_task,
                              const uint32_t* blk_start, const uint32_t* order_tmp,
                              uint32_t* order) {
  const uint32_t t = blk_task[blockIdx.x];
  const Task T = tasks[t];
  uint32_t chunk = blockIdx.x - blk_start[t];
  uint32_t begin = T.start + chunk * kChunk, end = min(T.start + T.count, begin + kChunk);
  for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) order[i] = order_tmp[i];
}

// ---------------------------------------------------------------------------
// small tasks: one warp builds the whole subtree in shared memory

constexpr int kSmallWarps = 4;
constexpr int kSmallStack = 24;

struct SmallShared {
  float lo[kSmall][3];
  float hi[kSmall][3];
  uint32_t gidx[kSmall];   // global primitive index
  uint16_t idx[kSmall];    // current local order
  uint16_t tmp[kSmall];
  uint32_t cnt[3][kBins];
  uint32_t blo[3][kBins][3], bhi[3][kBins][3];
  uint32_t clo[3][kBins][3], chi[3][kBins][3];
  struct Entry {
    uint32_t node;
    uint16_t ls, lc;
    float cmin[3], cmax[3];
  } stack[kSmallStack];
};

__global__ void __launch_bounds__(32 * kSmallWarps) k_small(
    const float4* lo, const float4* hi, uint32_t* order, const Task* tasks, uint32_t n_tasks,
    BinNode* nodes, uint32_t* node_counter, uint32_t* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  SmallShared& S = reinterpret_cast<SmallShared*>(smem_raw)[warp];
  uint32_t t = blockIdx.x * kSmallWarps + warp;
  if (t >= n_tasks) return;
  const Task T = tasks[t];
  const uint32_t n = T.count;
  for (uint32_t i = lane; i < n; i += 32) {
    uint32_t p = order[T.start + i];
    float4 l = lo[p], h = hi[p];
    S.lo[i][0] = l.x; S.lo[i][1] = l.y; S.lo[i][2] = l.z;
    S.hi[i][0] = h.x; S.hi[i][1] = h.y; S.hi[i][2] = h.z;
    S.gidx[i] = p;
    S.idx[i] = (uint16_t)i;
  }
  int sp = 0;
  if (lane == 0) {
    S.stack[0].node = T.node;
    S.stack[0].ls = 0;
    S.stack[0].lc = (uint16_t)n;
    for (int k = 0; k < 3; ++k) { S.stack[0].cmin[k] = T.cmin[k]; S.stack[0].cmax[k] = T.cmax[k]; }
  }
  sp = 1;
  __syncwarp();
  uint32_t iterations = 0;
  while (sp > 0) {
    if (++iterations > 4u * kSmall) {  // each iteration splits a node: at most n - 1 splits
      if (lane == 0) atomicOr(err, 32u);
      break;
    }
    --sp;
    SmallShared::Entry E = S.stack[sp];
    __syncwarp();
    if (E.lc <= 1) continue;  // leaf: node already written with start/count
    // bin
    for (uint32_t w = lane; w < 3 * kBins; w += 32) {
      uint32_t a = w / kBins, b = w % kBins;
      S.cnt[a][b] = 0;
      for (int k = 0; k < 3; ++k) {
        S.blo[a][b][k] = 0xffffffffu; S.bhi[a][b][k] = 0u;
        S.clo[a][b][k] = 0xffffffffu; S.chi[a][b][k] = 0u;
      }
    }
    __syncwarp();
    for (uint32_t i = lane; i < E.lc; i += 32) {
      uint32_t q = S.idx[E.ls + i];
      float c[3];
      for (int k = 0; k < 3; ++k) c[k] = (S.lo[q][k] + S.hi[q][k]) * 0.5f;
      for (int a = 0; a < 3; ++a) {
        float ext = E.cmax[a] - E.cmin[a];
        if (ext < kEps) continue;
        int b = bin_of(c[a], E.cmin[a], ext);
        atomicAdd(&S.cnt[a][b], 1u);
        for (int k = 0; k < 3; ++k) {
          atomicMin(&S.blo[a][b][k], f2key(S.lo[q][k]));
          atomicMax(&S.bhi[a][b][k], f2key(S.hi[q][k]));
          atomicMin(&S.clo[a][b][k], f2key(c[k]));
          atomicMax(&S.chi[a][b][k], f2key(c[k]));
        }
      }
    }
    __syncwarp();
    SplitOut so;
    warp_eval(S.cnt, S.blo, S.bhi, S.clo, S.chi, E.cmin, E.cmax, so);
    uint32_t nl;
    if (so.axis >= 0 && (so.nl == 0 || so.nl >= E.lc)) {
      // cannot happen with consistent binning; guarantees progress regardless
      if (lane == 0) atomicOr(err, 16u);
      so.axis = -1;
    }
    if (so.axis < 0) {
      // median split in the current order; bounds by warp reduction
      nl = E.lc / 2;
      for (int side = 0; side < 2; ++side) {
        uint32_t b0 = side == 0 ? 0 : nl, b1 = side == 0 ? nl : E.lc;
        uint32_t v[12];
        for (int k = 0; k < 3; ++k) { v[k] = 0xffffffffu; v[3 + k] = 0u; v[6 + k] = 0xffffffffu; v[9 + k] = 0u; }
        for (uint32_t i = b0 + lane; i < b1; i += 32) {
          uint32_t q = S.idx[E.ls + i];
          for (int k = 0; k < 3; ++k) {
            float c = (S.lo[q][k] + S.hi[q][k]) * 0.5f;
            v[k] = min(v[k], f2key(S.lo[q][k]));
            v[3 + k] = max(v[3 + k], f2key(S.hi[q][k]));
            v[6 + k] = min(v[6 + k], f2key(c));
            v[9 + k] = max(v[9 + k], f2key(c));
          }
        }
        for (int k = 0; k < 12; ++k) {
          bool is_min = (k < 3) || (k >= 6 && k < 9);
          uint32_t r = is_min ? __reduce_min_sync(0xffffffffu, v[k]) : __reduce_max_sync(0xffffffffu, v[k]);
          float f = key2f(r);
          if (side == 0) { if (k < 6) so.lbox[k] = f; else so.lcb[k - 6] = f; }
          else { if (k < 6) so.rbox[k] = f; else so.rcb[k - 6] = f; }
        }
      }
    } else {
      nl = so.nl;
      // stable partition of idx[ls, ls+lc) by bin <= split bin
      float ext = E.cmax[so.axis] - E.cmin[so.axis];
      uint32_t run_l = 0, run_r = 0;
      for (uint32_t base = 0; base < E.lc; base += 32) {
        uint32_t i = base + lane;
        bool valid = i < E.lc;
        uint16_t q = valid ? S.idx[E.ls + i] : 0;
        bool L = false;
        if (valid) {
          float c = (S.lo[q][so.axis] + S.hi[q][so.axis]) * 0.5f;
          L = bin_of(c, E.cmin[so.axis], ext) <= so.bin;
        }
        uint32_t bl = __ballot_sync(0xffffffffu, L);
        uint32_t bv = __ballot_sync(0xffffffffu, valid);
        uint32_t rl = __popc(bl & ((1u << lane) - 1u));
        uint32_t rr = __popc((bv & ~bl) & ((1u << lane) - 1u));
        if (valid) {
          if (L) S.tmp[E.ls + run_l + rl] = q;
          else S.tmp[E.ls + nl + run_r + rr] = q;
        }
        run_l += __popc(bl);
        run_r += __popc(bv & ~bl);
      }
      __syncwarp();
      for (uint32_t i = lane; i < E.lc; i += 32) S.idx[E.ls + i] = S.tmp[E.ls + i];
      __syncwarp();
    }
    uint32_t id = 0;
    if (lane == 0) id = atomicAdd(node_counter, 2u);
    id = __shfl_sync(0xffffffffu, id, 0);
    uint32_t nr = E.lc - nl;
    if (lane == 0) {
      write_node(nodes, id, so.lbox, T.start + E.ls, nl);
      write_node(nodes, id + 1, so.rbox, T.start + E.ls + nl, nr);
      nodes[E.node].left = (int32_t)id;
      nodes[E.node].right = (int32_t)(id + 1);
      if (nl == 0 || nr == 0) atomicOr(err, 2u);
    }
    // push larger child first so the smaller is processed first (bounded stack)
    SmallShared::Entry Le, Re;
    Le.node = id; Le.ls = E.ls; Le.lc = (uint16_t)nl;
    Re.node = id + 1; Re.ls = (uint16_t)(E.ls + nl); Re.lc = (uint16_t)nr;
    for (int k = 0; k < 3; ++k) {
      Le.cmin[k] = so.lcb[k]; Le.cmax[k] = so.lcb[3 + k];
      Re.cmin[k] = so.rcb[k]; Re.cmax[k] = so.rcb[3 + k];
    }
    SmallShared::Entry first = nl >= nr ? Le : Re, second = nl >= nr ? Re : Le;
    if (sp + 2 > kSmallStack) {
      if (lane == 0) atomicOr(err, 4u);
      break;
    }
    if (lane == 0) {
      S.stack[sp] = first;
      S.stack[sp + 1] = second;
    }
    sp += 2;
    __syncwarp();
  }
  __syncwarp();
  for (uint32_t i = lane; i < n; i += 32) order[T.start + i] = S.gidx[S.idx[i]];
}

// ---------------------------------------------------------------------------
// SAH cost, 2-wide layout, 8-wide collapse

__global__ void k_sah(const BinNode* nodes, uint32_t n, double* out) {
  __shared__ double s[256];
  float rl[3] = {nodes[0].lo[0], nodes[0].lo[1], nodes[0].lo[2]};
  float rh[3] = {nodes[0].hi[0], nodes[0].hi[1], nodes[0].hi[2]};
  double root = (double)area6(rl[0], rl[1], rl[2], rh[0], rh[1], rh[2]);
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const BinNode& b = nodes[i];
    double a = (double)area6(b.lo[0], b.lo[1], b.lo[2], b.hi[0], b.hi[1], b.hi[2]);
    acc += (b.left < 0 ? (double)b.count : 1.0) * (root > 0 ? a / root : 0.0);
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, s[0]);
}

__global__ void k_inner_flags(const BinNode* nodes, uint32_t n, uint32_t* flags) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flags[i] = nodes[i].left >= 0 ? 1u : 0u;
}

__global__ void k_emit_bvh2(const BinNode* nodes, uint32_t n, const uint32_t* idx2,
                            Bvh2Node* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BinNode& b = nodes[i];
  if (b.left < 0) return;
  const BinNode& L = nodes[b.left];
  const BinNode& R = nodes[b.right];
  Bvh2Node o;
  o.a = make_float4(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
  o.b = make_float4(R.lo[0], R.hi[0], R.lo[1], R.hi[1]);
  o.c = make_float4(L.lo[2], L.hi[2], R.lo[2], R.hi[2]);
  int l = L.left >= 0 ? (int)idx2[b.left] : ~(int)L.start;
  int r = R.left >= 0 ? (int)idx2[b.right] : ~(int)R.start;
  o.d = make_int4(l, r, L.left >= 0 ? 0 : (int)L.count, R.left >= 0 ? 0 : (int)R.count);
  out[idx2[i]] = o;
}

// single-leaf tree: root with one leaf child and one empty child
__global__ void k_emit_bvh2_single(const BinNode* nodes, Bvh2Node* out) {
  const BinNode& L = nodes[0];
  Bvh2Node o;
  o.a = make_float4(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
  o.b = make_float4(1.0f, -1.0f, 1.0f, -1.0f);
  o.c = make_float4(L.lo[2], L.hi[2], 1.0f, -1.0f);
  o.d = make_int4(~(int)L.start, ~0, (int)L.count, 0);
  out[0] = o;
}

struct WideWork {
  uint32_t bnode;  // binary node
  uint32_t wnode;  // wide node index
};

__global__ void k_collapse(const BinNode* nodes, const uint32_t* order, const WideWork* cur,
                           uint32_t n_cur, WideWork* next, uint32_t* n_next,
                           uint32_t* wide_counter, uint32_t* prim_counter, Bvh8Node* wide,
                           uint32_t* order8, uint32_t leaf_max, uint32_t width) {
  uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_cur) return;
  WideWork item = cur[w];
  const BinNode& P = nodes[item.bnode];
  int ch[8];
  int n = 0;
  if (P.left < 0) {
    ch[n++] = (int)item.bnode;  // a leaf root: one leaf child
  } else {
    ch[n++] = P.left;
    ch[n++] = P.right;
    while (n < (int)width) {
      int best = -1;
      float best_a = -1.0f;
      for (int i = 0; i < n; ++i) {
        const BinNode& c = nodes[ch[i]];
        if (c.left < 0 || c.count <= leaf_max) continue;
        float a = area6(c.lo[0], c.lo[1], c.lo[2], c.hi[0], c.hi[1], c.hi[2]);
        if (a > best_a) { best_a = a; best = i; }
      }
      if (best < 0) break;
      int b = ch[best];
      ch[best] = nodes[b].left;
      ch[n++] = nodes[b].right;
    }
  }
  // parent box
  float plo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, phi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  for (int i = 0; i < n; ++i) {
    const BinNode& c = nodes[ch[i]];
    for (int k = 0; k < 3; ++k) {
      plo[k] = fminf(plo[k], c.lo[k]);
      phi[k] = fmaxf(phi[k], c.hi[k]);
    }
  }
  // octant slot assignment (greedy on dot(centroid - centre, slot direction))
  int slot_of[8];
  int child_in_slot[8];
  for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
  float ctr[3] = {(plo[0] + phi[0]) * 0.5f, (plo[1] + phi[1]) * 0.5f, (plo[2] + phi[2]) * 0.5f};
  bool assigned[8] = {false, false, false, false, false, false, false, false};
  for (int it = 0; it < n; ++it) {
    float best = -3.4e38f;
    int bc = -1, bs = -1;
    for (int i = 0; i < n; ++i) {
      if (assigned[i]) continue;
      const BinNode& c = nodes[ch[i]];
      float d[3];
      for (int k = 0; k < 3; ++k) d[k] = (c.lo[k] + c.hi[k]) * 0.5f - ctr[k];
      for (int s = 0; s < 8; ++s) {
        if (child_in_slot[s] >= 0) continue;
        float sc = ((s & 4) ? d[0] : -d[0]) + ((s & 2) ? d[1] : -d[1]) + ((s & 1) ? d[2] : -d[2]);
        if (sc > best) { best = sc; bc = i; bs = s; }
      }
    }
    assigned[bc] = true;
    slot_of[bc] = bs;
    child_in_slot[bs] = bc;
  }
  // quantisation frame
  uint32_t ebits[3];
  float scale[3];
  for (int k = 0; k < 3; ++k) {
    float ext = phi[k] - plo[k];
    int e = ext > 0.0f ? (int)ceilf(log2f(ext / 255.0f)) : -126;
    if (e < -126) e = -126;
    if (e > 127) e = 127;
    // guarantee 255 * 2^e >= ext
    while (ldexpf(255.0f, e) < ext && e < 127) ++e;
    ebits[k] = (uint32_t)(e + 127);
    scale[k] = ldexpf(1.0f, e);
  }
  // count inner children and leaf primitives
  uint32_t n_inner = 0, n_prims = 0;
  for (int s = 0; s < 8; ++s) {
    int i = child_in_slot[s];
    if (i < 0) continue;
    const BinNode& c = nodes[ch[i]];
    if (c.left >= 0 && c.count > leaf_max) n_inner++;
    else n_prims += c.count;
  }
  uint32_t child_base = n_inner ? atomicAdd(wide_counter, n_inner) : 0u;
  uint32_t prim_base = n_prims ? atomicAdd(prim_counter, n_prims) : 0u;
  uint8_t meta[8], qlo[3][8], qhi[3][8];
  uint32_t imask = 0;
  uint32_t inner_i = 0, prim_off = 0;
  uint32_t next_base = n_inner ? atomicAdd(n_next, n_inner) : 0u;
  for (int s = 0; s < 8; ++s) {
    int i = child_in_slot[s];
    if (i < 0) {
      meta[s] = 0;
      for (int k = 0; k < 3; ++k) { qlo[k][s] = 255; qhi[k][s] = 0; }
      continue;
    }
    const BinNode& c = nodes[ch[i]];
    for (int k = 0; k < 3; ++k) {
      float ql = floorf((c.lo[k] - plo[k]) / scale[k]);
      float qh = ceilf((c.hi[k] - plo[k]) / scale[k]);
      // conservative in float: step outwards until the decoded box contains the child
      while (ql > 0.0f && plo[k] + ql * scale[k] > c.lo[k]) ql -= 1.0f;
      while (qh < 255.0f && plo[k] + qh * scale[k] < c.hi[k]) qh += 1.0f;
      qlo[k][s] = (uint8_t)fminf(fmaxf(ql, 0.0f), 255.0f);
      qhi[k][s] = (uint8_t)fminf(fmaxf(qh, 0.0f), 255.0f);
    }
    if (c.left >= 0 && c.count > leaf_max) {
      meta[s] = (uint8_t)((1u << 5) | (24u + (uint32_t)s));
      imask |= 1u << s;
      next[next_base + inner_i] = WideWork{(uint32_t)ch[i], child_base + inner_i};
      inner_i++;
    } else {
      uint32_t k = c.count;
      uint32_t unary = k == 1 ? 1u : (k == 2 ? 3u : 7u);
      meta[s] = (uint8_t)((unary << 5) | prim_off);
      for (uint32_t j = 0; j < k; ++j) order8[prim_base + prim_off + j] = order[c.start + j];
      prim_off += k;
    }
  }
  Bvh8Node o;
  o.n0 = make_float4(plo[0], plo[1], plo[2],
                     __uint_as_float(ebits[0] | (ebits[1] << 8) | (ebits[2] << 16) | (imask << 24)));
  auto pack = [](const uint8_t* b) {
    return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
  };
  o.n1 = make_uint4(child_base, prim_base, pack(meta), pack(meta + 4));
  o.n2 = make_uint4(pack(qlo[0]), pack(qlo[0] + 4), pack(qlo[1]), pack(qlo[1] + 4));
  o.n3 = make_uint4(pack(qlo[2]), pack(qlo[2] + 4), pack(qhi[0]), pack(qhi[0] + 4));
  o.n4 = make_uint4(pack(qhi[1]), pack(qhi[1] + 4), pack(qhi[2]), pack(qhi[2] + 4));
  wide[item.wnode] = o;
}

#define NR_TRY(x)                          \
  do {                                     \
    cudaError_t e_ = (x);                  \
    if (e_ != cudaSuccess) return (int)e_; \
  } while (0)

template <typename T>
cudaError_t dalloc(T*& p, size_t n) {
  return cudaMalloc(&p, sizeof(T) * (n ? n : 1));
}

}  // namespace

void free_build(BuildResult& r) {
  cudaFree(r.d_nodes);
  cudaFree(r.d_order);
  cudaFree(r.d_bvh2);
  cudaFree(r.d_bvh8);
  cudaFree(r.d_order8);
  r = BuildResult{};
}

int build_bvh(const float4* d_lo, const float4* d_hi, uint32_t n, bool want_bvh8,
              BuildResult& out, cudaStream_t st, uint32_t leaf_max, uint32_t width) {
  if (leaf_max < 1) leaf_max = 1;
  if (leaf_max > 3) leaf_max = 3;
  if (width < 2) width = 2;
  if (width > 8) width = 8;
  out = BuildResult{};
  if (n == 0) return 0;
  cudaEvent_t ev0, ev1;
  NR_TRY(cudaEventCreate(&ev0));
  NR_TRY(cudaEventCreate(&ev1));
  NR_TRY(cudaEventRecord(ev0, st));

  // scratch
  uint32_t *gk = nullptr, *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr;
  uint32_t* hist = nullptr;
  uint32_t* counters = nullptr;  // 0 node, 1 n_next_large, 2 n_small, 3 err, 4 wide, 5 prim, 6 n_next, 7 total
  NR_TRY(dalloc(gk, 12));
  NR_TRY(dalloc(keys, n));
  NR_TRY(dalloc(vals, n));
  NR_TRY(dalloc(keys2, n));
  NR_TRY(dalloc(vals2, n));
  NR_TRY(dalloc(counters, 16));
  uint32_t rs_blocks = (n + kRsTile - 1) / kRsTile;
  NR_TRY(dalloc(hist, (size_t)radix_sort_hist_words(n)));

  // bounds and Morton codes
  {
    uint32_t init[12] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0, 0, 0,
                         0xffffffffu, 0xffffffffu, 0xffffffffu, 0, 0, 0};
    NR_TRY(cudaMemcpyAsync(gk, init, sizeof(init), cudaMemcpyHostToDevice, st));
    uint32_t blocks = std::min((n + 255) / 256, 1184u);
    k_bounds<<<blocks, 256, 0, st>>>(d_lo, d_hi, n, gk);
    k_morton<<<(n + 255) / 256, 256, 0, st>>>(d_lo, d_hi, n, gk, keys, vals);
    for (int shift = 0; shift < 32; shift += 8) {
      k_rs_hist<<<rs_blocks, kRsThreads, 0, st>>>(keys, n, shift, hist, rs_blocks);
      NR_TRY(scan_exclusive(hist, hist, 256 * rs_blocks, hist + 256 * rs_blocks, nullptr, st));
      k_rs_scatter<<<rs_blocks, kRsThreads, 0, st>>>(keys, vals, keys2, vals2, n, shift, hist, rs_blocks);
      std::swap(keys, keys2);
      std::swap(vals, vals2);
    }
    NR_TRY(cudaGetLastError());
  }
  uint32_t* order = vals;       // Morton-sorted primitive order
  uint32_t* order_tmp = vals2;  // scratch of the same size

  // nodes and tasks
  BinNode* nodes = nullptr;
  uint32_t max_nodes = 2 * n - 1;
  NR_TRY(dalloc(nodes, max_nodes));
  uint32_t max_large = n / (kSmall + 1) + 2;
  Task *large = nullptr, *large_next = nullptr, *small = nullptr;
  NR_TRY(dalloc(large, max_large));
  NR_TRY(dalloc(large_next, max_large));
  NR_TRY(dalloc(small, n / 2 + 2));
  TaskBins* bins = nullptr;
  SplitInfo* splits = nullptr;
  NR_TRY(dalloc(bins, max_large));
  NR_TRY(dalloc(splits, max_large));
  uint32_t max_blocks = (n + kChunk - 1) / kChunk + max_large + 2;
  uint32_t *blk_task = nullptr, *blk_start = nullptr, *blk_left = nullptr;
  NR_TRY(dalloc(blk_task, max_blocks));
  NR_TRY(dalloc(blk_start, max_large + 1));
  NR_TRY(dalloc(blk_left, max_blocks));

  // root node and task (host computes the root from the bounds keys)
  uint32_t hk[12];
  NR_TRY(cudaMemcpyAsync(hk, gk, sizeof(hk), cudaMemcpyDeviceToHost, st));
  NR_TRY(cudaStreamSynchronize(st));
  auto k2f = [](uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
  };
  BinNode root;
  Task rt;
  for (int a = 0; a < 3; ++a) {
    root.lo[a] = k2f(hk[6 + a]);
    root.hi[a] = k2f(hk[9 + a]);
    rt.cmin[a] = k2f(hk[a]);
    rt.cmax[a] = k2f(hk[3 + a]);
  }
  root.left = root.right = -1;
  root.start = 0;
  root.count = n;
  rt.node = 0;
  rt.start = 0;
  rt.count = n;
  rt.pad = 0;
  NR_TRY(cudaMemcpyAsync(nodes, &root, sizeof(root), cudaMemcpyHostToDevice, st));
  uint32_t hc[16] = {1u, 0u, 0u, 0u, 1u, 0u, 0u, 0u, 0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t n_large = 0, n_small = 0;
  if (n > kSmall) {
    NR_TRY(cudaMemcpyAsync(large, &rt, sizeof(rt), cudaMemcpyHostToDevice, st));
    n_large = 1;
  } else if (n > 1) {
    NR_TRY(cudaMemcpyAsync(small, &rt, sizeof(rt), cudaMemcpyHostToDevice, st));
    hc[2] = 1;
  }
  NR_TRY(cudaMemcpyAsync(counters, hc, sizeof(hc), cudaMemcpyHostToDevice, st));

  int levels = 0;
  while (n_large > 0) {
    if (++levels > 96) {
      fprintf(stderr, "nectar_b200: BVH build did not converge\n");
      return (int)cudaErrorUnknown;
    }
    k_task_blocks<<<(n_large + 255) / 256, 256, 0, st>>>(large, n_large, blk_start);
    k_scan_single<<<1, 1024, 0, st>>>(blk_start, n_large, counters + 7);
    uint32_t total_blocks = 0;
    NR_TRY(cudaMemcpyAsync(&total_blocks, counters + 7, 4, cudaMemcpyDeviceToHost, st));
    NR_TRY(cudaStreamSynchronize(st));
    k_fill_block_map<<<n_large, 128, 0, st>>>(blk_start, n_large, blk_task, large);
    k_init_bins<<<256, 256, 0, st>>>(bins, n_large);
    k_bin_large<<<total_blocks, kPassThreads, 0, st>>>(d_lo, d_hi, order, large, blk_task,
                                                       blk_start, bins);
    NR_TRY(cudaMemsetAsync(counters + 1, 0, 4, st));
    k_split_large<<<(n_large * 32 + 127) / 128, 128, 0, st>>>(
        large, n_large, bins, splits, nodes, counters + 0, large_next, counters + 1, small,
        counters + 2, counters + 3);
    k_part_count<<<total_blocks, kPassThreads, 0, st>>>(d_lo, d_hi, order, large, splits,
                                                        blk_task, blk_start, blk_left);
    k_part_scan<<<(n_large * 32 + 127) / 128, 128, 0, st>>>(large, n_large, blk_start, blk_left);
    k_part_scatter<<<total_blocks, kPassThreads, 0, st>>>(d_lo, d_hi, order, order_tmp, large,
                                                          splits, blk_task, blk_start, blk_left);
    k_copy_ranges<<<total_blocks, 256, 0, st>>>(large, blk_task, blk_start, order_tmp, order);
    NR_TRY(cudaGetLastError());
    NR_TRY(cudaMemcpyAsync(&n_large, counters + 1, 4, cudaMemcpyDeviceToHost, st));
    NR_TRY(cudaStreamSynchronize(st));
    std::swap(large, large_next);
  }
  NR_TRY(cudaMemcpyAsync(&n_small, counters + 2, 4, cudaMemcpyDeviceToHost, st));
  NR_TRY(cudaStreamSynchronize(st));
  if (n_small > 0) {
    size_t smem = sizeof(SmallShared) * kSmallWarps;
    NR_TRY(cudaFuncSetAttribute(k_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_small<<<(n_small + kSmallWarps - 1) / kSmallWarps, 32 * kSmallWarps, smem, st>>>(
        d_lo, d_hi, order, small, n_small, nodes, counters + 0, counters + 3);
    NR_TRY(cudaGetLastError());
  }
  uint32_t hcount[4];
  NR_TRY(cudaMemcpyAsync(hcount, counters, 16, cudaMemcpyDeviceToHost, st));
  NR_TRY(cudaStreamSynchronize(st));
  uint32_t n_nodes = hcount[0];
  if (hcount[3] != 0) {
    fprintf(stderr, "nectar_b200: BVH build error flags 0x%x\n", hcount[3]);
    return (int)cudaErrorUnknown;
  }

  // SAH cost of the binary tree
  double* dsah = nullptr;
  NR_TRY(dalloc(dsah, 1));
  NR_TRY(cudaMemsetAsync(dsah, 0, sizeof(double), st));
  k_sah<<<std::min((n_nodes + 255) / 256, 1184u), 256, 0, st>>>(nodes, n_nodes, dsah);
  NR_TRY(cudaMemcpyAsync(&out.sah_cost, dsah, sizeof(double), cudaMemcpyDeviceToHost, st));

  // 2-wide layout
  uint32_t* idx2 = nullptr;
  NR_TRY(dalloc(idx2, (size_t)n_nodes + scan_scratch_words(n_nodes)));
  k_inner_flags<<<(n_nodes + 255) / 256, 256, 0, st>>>(nodes, n_nodes, idx2);
  NR_TRY(scan_exclusive(idx2, idx2, n_nodes, idx2 + n_nodes, counters + 7, st));
  uint32_t n_inner = 0;
  NR_TRY(cudaMemcpyAsync(&n_inner, counters + 7, 4, cudaMemcpyDeviceToHost, st));
  NR_TRY(cudaStreamSynchronize(st));
  uint32_t n_bvh2 = n_inner > 0 ? n_inner : 1;
  NR_TRY(dalloc(out.d_bvh2, n_bvh2));
  if (n_inner > 0)
    k_emit_bvh2<<<(n_nodes + 255) / 256, 256, 0, st>>>(nodes, n_nodes, idx2, out.d_bvh2);
  else
    k_emit_bvh2_single<<<1, 1, 0, st>>>(nodes, out.d_bvh2);
  NR_TRY(cudaGetLastError());

  // 8-wide collapse
  uint32_t n_wide = 0;
  if (want_bvh8) {
    NR_TRY(dalloc(out.d_bvh8, n_nodes));  // upper bound
    NR_TRY(dalloc(out.d_order8, n));
    WideWork *wa = nullptr, *wb = nullptr;
    NR_TRY(dalloc(wa, n / 2 + 2));
    NR_TRY(dalloc(wb, n / 2 + 2));
    WideWork w0{0u, 0u};
    NR_TRY(cudaMemcpyAsync(wa, &w0, sizeof(w0), cudaMemcpyHostToDevice, st));
    uint32_t hz[3] = {1u, 0u, 0u};  // wide counter, prim counter, n_next
    NR_TRY(cudaMemcpyAsync(counters + 4, hz, sizeof(hz), cudaMemcpyHostToDevice, st));
    uint32_t n_cur = 1;
    int wide_levels = 0;
    while (n_cur > 0) {
      if (++wide_levels > 96) return (int)cudaErrorUnknown;
      NR_TRY(cudaMemsetAsync(counters + 6, 0, 4, st));
      k_collapse<<<(n_cur + 127) / 128, 128, 0, st>>>(nodes, order, wa, n_cur, wb, counters + 6,
                                                      counters + 4, counters + 5, out.d_bvh8,
                                                      out.d_order8, leaf_max, width);
      NR_TRY(cudaGetLastError());
      NR_TRY(cudaMemcpyAsync(&n_cur, counters + 6, 4, cudaMemcpyDeviceToHost, st));
      NR_TRY(cudaStreamSynchronize(st));
      std::swap(wa, wb);
    }
    NR_TRY(cudaMemcpyAsync(&n_wide, counters + 4, 4, cudaMemcpyDeviceToHost, st));
    NR_TRY(cudaStreamSynchronize(st));
    cudaFree(wa);
    cudaFree(wb);
  }

  NR_TRY(cudaEventRecord(ev1, st));
  NR_TRY(cudaEventSynchronize(ev1));
  cudaEventElapsedTime(&out.build_ms, ev0, ev1);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);

  out.d_nodes = nodes;
  out.d_order = order;
  out.n_nodes = n_nodes;
  out.n_bvh2 = n_bvh2;
  out.n_bvh8 = n_wide;

  cudaFree(gk);
  cudaFree(keys);
  cudaFree(keys2);
  cudaFree(order_tmp);
  cudaFree(hist);
  cudaFree(counters);
  cudaFree(large);
  cudaFree(large_next);
  cudaFree(small);
  cudaFree(bins);
  cudaFree(splits);
  cudaFree(blk_task);
  cudaFree(blk_start);
  cudaFree(blk_left);
  cudaFree(dsah);
  cudaFree(idx2);
  return 0;
}

uint32_t scan_scratch_words(uint32_t n) { return (n + kScanTile - 1) / kScanTile + 1u; }

cudaError_t scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* sums,
                           uint32_t* total, cudaStream_t st) {
  if (n == 0) return total ? cudaMemsetAsync(total, 0, sizeof(uint32_t), st) : cudaSuccess;
  const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
  k_scan_tile_sums<<<tiles, kScanTile, 0, st>>>(in, n, sums);
  // one CTA scans the tile sums; the last scratch word takes the total
  k_scan_single<<<1, 1024, 0, st>>>(sums, tiles, total ? total : sums + tiles);
  k_scan_tile_apply<<<tiles, kScanTile, 0, st>>>(in, n, sums, out);
  return cudaGetLastError();
}

uint32_t radix_sort_hist_words(uint32_t n) {
  const uint32_t h = 256u * ((n + kRsTile - 1) / kRsTile);
  return h + scan_scratch_words(h);
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys2, uint32_t* vals2,
                             uint32_t n, int key_bits, uint32_t* hist, cudaStream_t st,
                             uint32_t** out_keys, uint32_t** out_vals) {
  const uint32_t blocks = (n + kRsTile - 1) / kRsTile;
  for (int shift = 0; shift < key_bits && n; shift += 8) {
    k_rs_hist<<<blocks, kRsThreads, 0, st>>>(keys, n, shift, hist, blocks);
    cudaError_t e = scan_exclusive(hist, hist, 256 * blocks, hist + 256 * blocks, nullptr, st);
    if (e != cudaSuccess) return e;
    k_rs_scatter<<<blocks, kRsThreads, 0, st>>>(keys, vals, keys2, vals2, n, shift, hist, blocks);
    std::swap(keys, keys2);
    std::swap(vals, vals2);
  }
  *out_keys = keys;
  *out_vals = vals;
  return cudaGetLastError();
}

}  // namespace nr
