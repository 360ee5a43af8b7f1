// nrc.cu — neural radiance cache (see nrc.cuh).
//
// Input vector (64 BF16 channels): [0, 32) hash-grid features (16 levels x 2),
// [32, 48) real spherical harmonics of degree 0-3 of the outgoing direction,
// [48, 51) normal * 0.5 + 0.5, [51] roughness, [52, 55) diffuse albedo, zero
// padding. MLP: four hidden layers 64 -> 64 (ReLU), then 64 -> 16 (linear;
// the first three outputs are the radiance), no biases. Loss: relative squared error
// (o - t)^2 / (o^2 + 0.01) with o held constant in the denominator.
//
// The whole MLP is one fused tcgen05 kernel per call (k_mlp_infer,
// k_mlp_train): 128 queries per tile, one row per thread and one
// tensor-memory lane per row. The five weight matrices and every activation
// tile stay in shared memory (BF16, no-swizzle canonical layouts), each layer
// is 1-4 MMAs of M = 128, N = 64 (16 for the output layer), K = 16 into a
// tensor-memory accumulator, and the epilogues (ReLU, the loss gradient, the
// ReLU mask of the backward pass) run on the rows the threads load back with
// tcgen05.ld. In training the backward-data GEMM of each layer and its
// weight-gradient GEMM (dW += dZ^T X over the tile's rows, both operands read
// MN-major from the same tiles) are issued together; the weight gradients
// accumulate in tensor memory over all the CTA's tiles and are added to the
// FP32 gradient with vector atomics once at the end; the input-gradient rows
// go to global memory for the hash-grid scatter. A training step is: encode,
// k_mlp_train, grid scatter, one Adam launch for the MLP and one for the
// grid. The encoding and the scatter run one thread per (query, level).
#include "nrc.cuh"

#include <cmath>
#include <random>
#include <vector>

#include "tcgen05.cuh"

namespace nr {

namespace {

constexpr int kLevels = 16, kFeat = 2, kLog2T = 19;
constexpr uint32_t kT = 1u << kLog2T;
constexpr int kWidth = 64, kOutCh = 16;
constexpr int kHidden = 4, kLayers = kHidden + 1;
constexpr int kRows = 128;  // queries per tile = threads per CTA of k_mlp_infer
constexpr uint32_t kWaitLimit = 1u << 26;
constexpr float kNmin = 16.0f, kNmax = 2048.0f;

#define GRID_STRIDE(i, n) \
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

int blocks_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

struct GridGeo {
  float lo[3], inv_ext[3];
  float scale[kLevels];     // N_l
  uint32_t dense[kLevels];  // 1: direct index, 0: spatial hash
};

__device__ __forceinline__ uint32_t grid_index(const GridGeo& g, int l, uint32_t x, uint32_t y,
                                               uint32_t z) {
  if (g.dense[l]) {
    const uint32_t r = (uint32_t)g.scale[l] + 2u;
    return (x + r * (y + r * z)) & (kT - 1u);
  }
  return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (kT - 1u);
}

// Visits the 8 corners of level l around position u in [0,1]^3.
template <typename F>
__device__ __forceinline__ void corners(const GridGeo& g, int l, const float (&u)[3], F&& f) {
  float pos[3], fr[3];
  uint32_t base[3];
  for (int k = 0; k < 3; ++k) {
    pos[k] = u[k] * g.scale[l] + 0.5f;
    const float fl = floorf(pos[k]);
    fr[k] = pos[k] - fl;
    base[k] = (uint32_t)fl;
  }
  for (int c = 0; c < 8; ++c) {
    float w = 1.0f;
    uint32_t idx[3];
    for (int k = 0; k < 3; ++k) {
      const bool hi = (c >> k) & 1;
      w *= hi ? fr[k] : 1.0f - fr[k];
      idx[k] = base[k] + (hi ? 1u : 0u);
    }
    f(grid_index(g, l, idx[0], idx[1], idx[2]), w);
  }
}

__device__ __forceinline__ void unit_pos(const GridGeo& g, const NrcQuery& q, float (&u)[3]) {
  const float p[3] = {q.a.x, q.a.y, q.a.z};
  for (int k = 0; k < 3; ++k) u[k] = fminf(fmaxf((p[k] - g.lo[k]) * g.inv_ext[k], 0.0f), 1.0f);
}

// real spherical harmonics, degrees 0-3 (the constants are the
// normalisation factors sqrt((2l+1)/(4 pi) (l-|m|)!/(l+|m|)!) times the
// polynomial coefficients of the Cartesian forms)
__device__ __forceinline__ void sh16(float x, float y, float z, float (&s)[16]) {
  const float xx = x * x, yy = y * y, zz = z * z;
  s[0] = 0.28209479177387814f;
  s[1] = -0.48860251190291987f * y;
  s[2] = 0.48860251190291987f * z;
  s[3] = -0.48860251190291987f * x;
  s[4] = 1.0925484305920792f * x * y;
  s[5] = -1.0925484305920792f * y * z;
  s[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
  s[7] = -1.0925484305920792f * x * z;
  s[8] = 0.54627421529603959f * (xx - yy);
  s[9] = 0.59004358992664352f * y * (-3.0f * xx + yy);
  s[10] = 2.8906114426405538f * x * y * z;
  s[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
  s[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
  s[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
  s[14] = 1.4453057213202769f * z * (xx - yy);
  s[15] = 0.59004358992664352f * x * (-xx + 3.0f * yy);
}

// One thread per (query, level): the 8 corner gathers of one level, one
// spherical-harmonics coefficient and one of the remaining inputs.
__global__ void k_encode(GridGeo g, const NrcQuery* qs, const float* grid, __nv_bfloat16* x,
                         uint32_t n) {
  GRID_STRIDE(t, (size_t)n * kLevels) {
    const size_t i = t / kLevels;
    const int l = (int)(t % kLevels);
    const NrcQuery q = qs[i];
    __nv_bfloat16* row = x + i * kWidth;
    float u[3];
    unit_pos(g, q, u);
    float2 f = make_float2(0.0f, 0.0f);
    const float2* lv = reinterpret_cast<const float2*>(grid + (size_t)l * kT * kFeat);
    corners(g, l, u, [&](uint32_t idx, float w) {
      const float2 e = __ldg(lv + idx);
      f.x += w * e.x;
      f.y += w * e.y;
    });
    *reinterpret_cast<__nv_bfloat162*>(row + 2 * l) = __floats2bfloat162_rn(f.x, f.y);
    float sh[16];
    sh16(q.b.x, q.b.y, q.b.z, sh);
    row[32 + l] = __float2bfloat16(sh[l]);
    const float extra[16] = {q.c.x * 0.5f + 0.5f, q.c.y * 0.5f + 0.5f, q.c.z * 0.5f + 0.5f, q.a.w,
                             q.d.x, q.d.y, q.d.z, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    row[48 + l] = __float2bfloat16(extra[l]);
  }
}

// Hash-grid gradient, one thread per (query, level): the adjoint of the
// trilinear interpolation of that level's two feature gradients (dx: the
// BF16 gradient of the encoded input's grid features, [count][32]).
__global__ void k_encode_bwd(GridGeo g, const NrcQuery* qs, const __nv_bfloat162* dx, float* ggrid,
                             uint32_t n) {
  GRID_STRIDE(t, (size_t)n * kLevels) {
    const size_t i = t / kLevels;
    const int l = (int)(t % kLevels);
    const float2 d = __bfloat1622float2(dx[i * kLevels + l]);
    if (d.x == 0.0f && d.y == 0.0f) continue;
    float u[3];
    unit_pos(g, qs[i], u);
    static_assert(kFeat == 2, "one float2 per grid entry");
    float2* lv = reinterpret_cast<float2*>(ggrid + (size_t)l * kT * kFeat);
    corners(g, l, u, [&](uint32_t idx, float w) {
      atomicAdd(lv + idx, make_float2(w * d.x, w * d.y));  // one 8-byte vector atomic
    });
  }
}

__device__ __forceinline__ uint4 pack_bf16x8(const float (&v)[8]) {
  uint4 r;
  __nv_bfloat162 h[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  r.x = *reinterpret_cast<uint32_t*>(&h[0]);
  r.y = *reinterpret_cast<uint32_t*>(&h[1]);
  r.z = *reinterpret_cast<uint32_t*>(&h[2]);
  r.w = *reinterpret_cast<uint32_t*>(&h[3]);
  return r;
}
__device__ __forceinline__ void unpack_bf16x8(const uint4& r, float (&v)[8]) {
  const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    v[2 * i] = __low2float(h);
    v[2 * i + 1] = __high2float(h);
  }
}
__device__ __forceinline__ float round_bf16(float x) { return __bfloat162float(__float2bfloat16(x)); }

// Shared-memory layouts of the MLP kernels. An activation tile holds 128
// rows x C columns (C = 64, or 16 for the output gradient) in the K-major
// no-swizzle layout with the 8-row core matrices stacked along the rows:
// element (r, c) at r * 16 + (c / 8) * 2048 + (c % 8) * 2, i.e. LBO = 2048
// (next 8 columns) and SBO = 128 (next 8 rows) when the rows are the M
// dimension. Read as an MN-major operand over (column, row) the same bytes
// have LBO = 128 and SBO = 2048: the weight-gradient GEMMs use that view.
// Their A operand is M = 128 wide over at most 64 real columns and so reads
// up to 32 KB past the tile start (rows of the accumulator that are never
// read back), which must stay inside the CTA's shared memory.
// A weight matrix W[o][i] (nout x 64) is the K-major B operand of the forward
// GEMM (N = o, K = i): element (o, i) at o * 16 + (i / 8) * nout * 16 +
// (i % 8) * 2 (SBO = 128, LBO = nout * 16); the backward-data GEMM reads it
// MN-major over (i, o) (LBO = 128, SBO = nout * 16).
constexpr uint32_t kTileBytes = kRows * kWidth * 2;        // 16 KB
constexpr uint32_t kActLbo = kRows * 16;                   // 2048
constexpr uint32_t kWBytes = kWidth * kWidth * 2;          // 8 KB
// Inference: X, H(even), H(odd) (ping-pong), weights = 82 KB, two CTAs per SM.
constexpr uint32_t kInferSmemBytes = 3 * kTileBytes + kHidden * kWBytes + kOutCh * kWidth * 2;

__device__ __forceinline__ uint32_t act_off(uint32_t r, uint32_t c) {
  return r * 16u + (c >> 3) * kActLbo + (c & 7u) * 2u;
}

struct MlpArgs {
  const __nv_bfloat16* x0;            // [count][64] encoded inputs
  const __nv_bfloat16* w[kLayers];    // [out][in]
  uint32_t count;
  float* out;                         // inference: [count][3] radiance
  const float* target;                // training: [count][3]
  const NrcQuery* q;                  // training: queries (positions for the grid gradient)
  float* gw[kLayers];                 // training: FP32 weight gradients, accumulated
  __nv_bfloat16* dx;                  // training: [count][32] grid-feature gradients
  double* loss;                       // training: sum of the relative squared errors
  uint32_t* err;
  GridGeo geo;
};

// D (+)= A * B^T over n MMAs of K = 16, issued by the elected lane of a
// converged warp; the descriptors advance by a_inc / b_inc per MMA (added to
// the start-address field, which never carries: operands lie below 256 KB).
__device__ __forceinline__ void issue_run(uint32_t d, uint64_t da, uint64_t a_inc, uint64_t db, uint64_t b_inc,
                                          int n, uint32_t idesc, uint32_t acc0) {
  for (int kk = 0; kk < n; ++kk, da += a_inc, db += b_inc)
    if (tc::elect_one()) tc::mma_bf16(d, da, db, idesc, (acc0 || kk > 0) ? 1u : 0u);
}

// Inference: one CTA of 128 threads takes 128 queries at a time, one row per
// thread and one tensor-memory lane per row; warp 0 issues each layer's
// GEMM, the CTA waits on its commit, applies ReLU to the accumulator rows it
// loads back and writes the next layer's input tile. Two CTAs per SM overlap
// one CTA's epilogues with the other's GEMMs.
__global__ void __launch_bounds__(kRows, 2) k_mlp_infer(MlpArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  constexpr uint32_t kCols = 64u;
  constexpr uint32_t oX = 0u, oW = 3u * kTileBytes;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t base = tc::smem_u32(smem);
  if (tid == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&tmem_base, kCols);
  for (int l = 0; l < kLayers; ++l) {
    const int nout = l < kHidden ? kWidth : kOutCh;
    unsigned char* wl = smem + oW + l * kWBytes;
    for (int i = tid; i < nout * 8; i += kRows) {
      const int o = i >> 3, g = i & 7;
      *reinterpret_cast<uint4*>(wl + o * 16 + g * nout * 16) =
          *reinterpret_cast<const uint4*>(a.w[l] + (size_t)o * kWidth + g * 8);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t my_lane = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  const uint32_t tiles = (a.count + kRows - 1) / kRows;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * kRows + tid;
    const bool valid = row < a.count;
    for (int g = 0; g < 8; ++g) {
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (valid) v = *reinterpret_cast<const uint4*>(a.x0 + (size_t)row * kWidth + g * 8);
      *reinterpret_cast<uint4*>(smem + oX + act_off(tid, g * 8)) = v;
    }
    uint32_t in_off = oX;
    for (int l = 0; l < kLayers && ok; ++l) {
      const uint32_t nout = l < kHidden ? kWidth : kOutCh;
      // operands written, accumulator read: hand the tensor core the layer
      tc::fence_smem_to_async();
      tc::fence_before_sync();
      __syncthreads();
      if (warp == 0) {
        tc::fence_after_sync();
        issue_run(tmem, tc::smem_desc(base + in_off, kActLbo, 128u), (2u * kActLbo) >> 4,
                  tc::smem_desc(base + oW + (uint32_t)l * kWBytes, nout * 16u, 128u), (2u * nout * 16u) >> 4,
                  kWidth / 16, tc::idesc_bf16(128, nout, false, false), 0u);
        if (tc::elect_one()) tc::mma_commit(&bar);
        __syncwarp();
      }
      ok = __syncthreads_and(tc::mbar_wait(&bar, phase, kWaitLimit)) != 0;
      if (!ok) break;
      phase ^= 1u;
      tc::fence_after_sync();
      if (l < kHidden) {
        const uint32_t h_off = kTileBytes * (1u + (uint32_t)(l & 1));
        uint32_t r[8][8];
#pragma unroll
        for (int c = 0; c < 8; ++c) tc::tmem_ld8_nowait(my_lane + (uint32_t)(c * 8), r[c]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < kWidth / 8; ++c) {
          float v[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) v[k] = fmaxf(__uint_as_float(r[c][k]), 0.0f);
          *reinterpret_cast<uint4*>(smem + h_off + act_off(tid, c * 8)) = pack_bf16x8(v);
        }
        in_off = h_off;
      } else {
        float o[8];
        tc::tmem_ld8(my_lane, o);
        if (valid)
          for (int c = 0; c < 3; ++c) a.out[(size_t)row * 3 + c] = fmaxf(round_bf16(o[c]), 0.0f);
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicOr(a.err, 4u);
    tc::mbar_wait(&bar, phase, kWaitLimit);  // MMAs that may still be in flight
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kCols);
}

// Adam on the hash grid, lazily: only entries with a nonzero gradient move
// (the others keep their moments), and the gradient is cleared as it is
// read, so the next step needs no memset of the 64 MB gradient table.
__global__ void k_adam_grid(float* w, float* m, float* v, float4* g4, size_t n4, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  GRID_STRIDE(i, n4) {
    const float4 g = g4[i];
    if (g.x == 0.0f && g.y == 0.0f && g.z == 0.0f && g.w == 0.0f) continue;
    g4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float gs[4] = {g.x, g.y, g.z, g.w};
    for (int k = 0; k < 4; ++k) {
      if (gs[k] == 0.0f) continue;
      const size_t j = 4 * i + k;
      const float mi = b1 * m[j] + (1.0f - b1) * gs[k];
      const float vi = b2 * v[j] + (1.0f - b2) * gs[k] * gs[k];
      m[j] = mi;
      v[j] = vi;
      w[j] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
  }
}

// Adam on the MLP weights (their gradients are cleared as they are read)
// and the BF16 copies the MLP kernel reads.
struct MlpOpt {
  float *w[kLayers], *m[kLayers], *v[kLayers], *g[kLayers];
  __nv_bfloat16* wf[kLayers];
};
__global__ void k_adam_mlp(MlpOpt o, float lr, float b1, float b2, float eps, float c1, float c2) {
  constexpr size_t kHid = (size_t)kWidth * kWidth;
  GRID_STRIDE(t, kHidden * kHid + (size_t)kOutCh * kWidth) {
    const int l = (int)min(t / kHid, (size_t)kHidden);
    const size_t i = t - (size_t)l * kHid;
    const float gi = o.g[l][i];
    o.g[l][i] = 0.0f;
    const float mi = b1 * o.m[l][i] + (1.0f - b1) * gi;
    const float vi = b2 * o.v[l][i] + (1.0f - b2) * gi * gi;
    o.m[l][i] = mi;
    o.v[l][i] = vi;
    const float w = o.w[l][i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    o.w[l][i] = w;
    o.wf[l][i] = __float2bfloat16(w);
  }
}

__global__ void k_pack(const float* w, __nv_bfloat16* wf, size_t n) {
  GRID_STRIDE(i, n) { wf[i] = __float2bfloat16(w[i]); }
}

// Training with two tiles in flight. The serial chain of one tile (5
// forward and 5 backward steps, each a GEMM, a wait and a tcgen05.ld
// epilogue) leaves the tensor core idle while the epilogue runs; here two
// groups of four warps each carry their own tile through the chain and one
// more warp issues every GEMM, so that one group's epilogue overlaps the
// other group's GEMM. The issuing warp serves the groups in a fixed order
// (step k of group 0, step k of group 1, step k + 1 of group 0, ...), which
// also keeps all weight-gradient MMAs in one thread's issue order, as
// accumulation into shared tensor-memory columns needs.
//
// Per group (kGrpBytes of shared memory): G (the output gradient, 128 x 16)
// and four hidden tiles H0..H3. The encoded inputs X go to H3's tile (dead
// until layer 3 writes H3) and are copied there again for the last backward
// step; each backward step writes dZ_(j-1) over H_(j-1) in place, since the
// mask is read by the same thread just before. Tensor memory: the group's
// accumulator at 64 g, the weight gradients at 128 + 64 l.
constexpr int kGroups = 2;
constexpr int kTrainThreads = 32 * (4 * kGroups + 1);
constexpr uint32_t kGOff = 0, kHOff = kRows * kOutCh * 2;  // within a group
constexpr uint32_t kGrpBytes = kHOff + kHidden * kTileBytes;
constexpr uint32_t kOffW2 = kGroups * kGrpBytes;
constexpr uint32_t kSmemTrain = kOffW2 + kHidden * kWBytes + kOutCh * kWidth * 2;
static_assert((kGroups - 1) * kGrpBytes + kHOff + (kHidden - 1) * kTileBytes + 32768u <= kSmemTrain,
              "the padded weight-gradient reads stay inside the CTA's shared memory");
static_assert(kSmemTrain <= 227u * 1024u, "shared memory per CTA");

__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort) {
  return tc::mbar_wait_or_abort(bar, parity, abort, kWaitLimit);
}

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" :: "r"(1 + g), "r"(kRows) : "memory");
}

__global__ void __launch_bounds__(kTrainThreads, 1) k_mlp_train(MlpArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t ready[kGroups], done[kGroups], fin;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, grp_ok[kGroups];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = tc::smem_u32(smem);
  const uint32_t tiles = (a.count + kRows - 1) / kRows;
  const uint32_t stride = gridDim.x * kGroups;
  volatile int* abort_v = &abort_flag;
  if (tid == 0) {
    for (int g = 0; g < kGroups; ++g) {
      tc::mbar_init(&ready[g], 1);
      tc::mbar_init(&done[g], 1);
    }
    tc::mbar_init(&fin, 1);
    abort_flag = 0;
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, 512);
  // a group's first rows of encoded inputs are requested before the weights,
  // so that the two loads overlap
  uint4 xfirst[8];
  if (warp < 4 * kGroups) {
    const uint32_t r = (blockIdx.x * kGroups + warp / 4) * kRows + (warp % 4) * 32 + lane;
#pragma unroll
    for (int c = 0; c < 8; ++c)
      xfirst[c] = r < a.count ? *reinterpret_cast<const uint4*>(a.x0 + (size_t)r * kWidth + c * 8)
                              : make_uint4(0u, 0u, 0u, 0u);
  }
  for (int l = 0; l < kLayers; ++l) {
    const int nout = l < kHidden ? kWidth : kOutCh;
    unsigned char* wl = smem + kOffW2 + l * kWBytes;
    for (int i = tid; i < nout * 8; i += kTrainThreads) {
      const int o = i >> 3, g = i & 7;
      *reinterpret_cast<uint4*>(wl + o * 16 + g * nout * 16) =
          *reinterpret_cast<const uint4*>(a.w[l] + (size_t)o * kWidth + g * 8);
    }
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  double loss = 0.0;

  if (warp == 4 * kGroups) {
    // the issuing warp: all lanes run the loop, the elected lane issues
    uint32_t n_ready[kGroups] = {0u, 0u};
    uint32_t wg_init = 0u;  // layers whose weight gradient has been started
    bool ok = true;
    for (uint32_t r = 0; ok; ++r) {
      bool any = false;
      for (int k = 0; k < 2 * kLayers && ok; ++k) {
        for (int g = 0; g < kGroups; ++g) {
          if (blockIdx.x * kGroups + g + r * stride >= tiles) continue;
          any = true;
          int got = 0;
          if (lane == 0) got = wait_or_abort(&ready[g], n_ready[g] & 1u, abort_v) ? 1 : 0;
          ++n_ready[g];
          if (!__shfl_sync(0xffffffffu, got, 0)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t gb = base + (uint32_t)g * kGrpBytes, d = tmem + 64u * (uint32_t)g;
          // descriptors are formed before the issue loops and advance by adding
          // (byte offset >> 4) to the start-address field, which never carries
          if (k < kLayers) {  // forward layer l: D = In_l W_l^T
            const int l = k;
            const uint32_t nout = l < kHidden ? kWidth : kOutCh;
            const uint32_t in = l == 0 ? gb + kHOff + 3u * kTileBytes : gb + kHOff + (uint32_t)(l - 1) * kTileBytes;
            const uint32_t w = base + kOffW2 + (uint32_t)l * kWBytes;
            issue_run(d, tc::smem_desc(in, kActLbo, 128u), (2u * kActLbo) >> 4,
                      tc::smem_desc(w, nout * 16u, 128u), (2u * nout * 16u) >> 4, kWidth / 16,
                      tc::idesc_bf16(128, nout, false, false), 0u);
          } else {  // backward layer j: dIn = dZ_j W_j, dW_j += dZ_j^T In_j
            const int j = 2 * kLayers - 1 - k;
            const uint32_t nout = j == kHidden ? kOutCh : kWidth;
            const uint32_t dz = j == kHidden ? gb + kGOff : gb + kHOff + (uint32_t)j * kTileBytes;
            const uint32_t in = j == 0 ? gb + kHOff + 3u * kTileBytes : gb + kHOff + (uint32_t)(j - 1) * kTileBytes;
            const uint32_t w = base + kOffW2 + (uint32_t)j * kWBytes;
            issue_run(d, tc::smem_desc(dz, kActLbo, 128u), (2u * kActLbo) >> 4,
                      tc::smem_desc(w, 128u, nout * 16u), 256u >> 4, (int)nout / 16,
                      tc::idesc_bf16(128, kWidth, false, true), 0u);
            const uint32_t acc0 = (wg_init >> j) & 1u;
            wg_init |= 1u << j;
            issue_run(tmem + 128u + 64u * (uint32_t)j, tc::smem_desc(dz, 128u, kActLbo), 256u >> 4,
                      tc::smem_desc(in, 128u, kActLbo), 256u >> 4, kRows / 16,
                      tc::idesc_bf16(128, kWidth, true, true), acc0);
          }
          if (tc::elect_one()) tc::mma_commit(&done[g]);
          __syncwarp();
        }
      }
      if (!any) break;
    }
    if (tc::elect_one()) tc::mma_commit(&fin);
    __syncwarp();
  } else {
    // a group: warp gw of group g reads tensor-memory lanes 32 gw .. +31
    const int g = warp / 4, gw = warp % 4, row = gw * 32 + lane;
    unsigned char* gp = smem + (size_t)g * kGrpBytes;
    unsigned char* h3 = gp + kHOff + 3 * kTileBytes;
    const uint32_t my_lane = tmem + ((uint32_t)(gw * 32) << 16) + 64u * (uint32_t)g;
    uint32_t n_done = 0;
    // the encoded inputs of a tile's rows: fetched into registers one tile
    // ahead, and kept for the copy that the last backward step reads
    uint4 xcur[8], xnext[8];
    auto fetch_x = [&](uint32_t t, uint4 (&dst)[8]) {
      const uint32_t r = t * kRows + row;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        dst[c] = r < a.count ? *reinterpret_cast<const uint4*>(a.x0 + (size_t)r * kWidth + c * 8)
                             : make_uint4(0u, 0u, 0u, 0u);
    };
    auto store_x = [&]() {
#pragma unroll
      for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(h3 + act_off(row, c * 8)) = xcur[c];
    };
    // all 64 accumulator columns of this thread's row, one wait
    auto load_acc = [&](float (&v)[64]) {
      uint32_t r[8][8];
#pragma unroll
      for (int c = 0; c < 8; ++c) tc::tmem_ld8_nowait(my_lane + (uint32_t)(c * 8), r[c]);
      tc::tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int e = 0; e < 8; ++e) v[c * 8 + e] = __uint_as_float(r[c][e]);
    };
    // operands written: hand the next GEMM to the issuing warp
    auto hand_over = [&]() {
      tc::fence_smem_to_async();
      tc::fence_before_sync();
      group_sync(g);
      if (row == 0) tc::mbar_arrive(&ready[g]);
    };
    // the group's GEMM is done (one poller, the result shared group-wide)
    auto gemm_done = [&]() {
      if (row == 0) grp_ok[g] = wait_or_abort(&done[g], n_done & 1u, abort_v) ? 1 : 0;
      ++n_done;
      group_sync(g);
      tc::fence_after_sync();
      return grp_ok[g] != 0;
    };
    bool ok = true;
    uint32_t tile = blockIdx.x * kGroups + g;
#pragma unroll
    for (int c = 0; c < 8; ++c) xnext[c] = xfirst[c];
    for (; tile < tiles && ok; tile += stride) {
      const uint32_t grow = tile * kRows + row;
      const bool valid = grow < a.count;
#pragma unroll
      for (int c = 0; c < 8; ++c) xcur[c] = xnext[c];
      store_x();
      hand_over();
      for (int l = 0; l < kLayers && ok; ++l) {
        if (!(ok = gemm_done())) break;
        if (l < kHidden) {
          unsigned char* h = gp + kHOff + l * kTileBytes;
          float v[64];
          load_acc(v);
#pragma unroll
          for (int c = 0; c < kWidth / 8; ++c) {
            float f[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) f[e] = fmaxf(v[c * 8 + e], 0.0f);
            *reinterpret_cast<uint4*>(h + act_off(row, c * 8)) = pack_bf16x8(f);
          }
        } else {
          float o[16], gr[16];
          uint32_t r[2][8];
          tc::tmem_ld8_nowait(my_lane, r[0]);
          tc::tmem_ld8_nowait(my_lane + 8u, r[1]);
          tc::tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 16; ++c) {
            o[c] = __uint_as_float(r[c >> 3][c & 7]);
            gr[c] = 0.0f;
          }
          if (valid)
            for (int c = 0; c < 3; ++c) {
              const float oc = round_bf16(o[c]), t = a.target[(size_t)grow * 3 + c];
              const float den = oc * oc + 0.01f, dd = oc - t;
              loss += (double)(dd * dd / den);
              gr[c] = 2.0f * dd / den;
            }
          *reinterpret_cast<uint4*>(gp + kGOff + act_off(row, 0)) = pack_bf16x8(*reinterpret_cast<float(*)[8]>(gr));
          *reinterpret_cast<uint4*>(gp + kGOff + act_off(row, 8)) =
              pack_bf16x8(*reinterpret_cast<float(*)[8]>(gr + 8));
        }
        hand_over();
      }
      for (int j = kHidden; j >= 0 && ok; --j) {
        if (!(ok = gemm_done())) break;
        if (j > 0) {
          // dZ_(j-1) = BF16(dIn) where H_(j-1) > 0, over H_(j-1) in place
          unsigned char* h = gp + kHOff + (j - 1) * kTileBytes;
          float v[64];
          load_acc(v);
#pragma unroll
          for (int c = 0; c < kWidth / 8; ++c) {
            float f[8], hv[8];
            unpack_bf16x8(*reinterpret_cast<const uint4*>(h + act_off(row, c * 8)), hv);
#pragma unroll
            for (int e = 0; e < 8; ++e) f[e] = hv[e] > 0.0f ? v[c * 8 + e] : 0.0f;
            *reinterpret_cast<uint4*>(h + act_off(row, c * 8)) = pack_bf16x8(f);
          }
          if (j == 3 && tile + stride < tiles) fetch_x(tile + stride, xnext);
          if (j == 1) store_x();  // In_0 for the last step; H3's tile is free again
          hand_over();
        } else {
          // gradient of the grid features, rounded to BF16, for k_encode_bwd
          uint32_t r[4][8];
#pragma unroll
          for (int c = 0; c < 4; ++c) tc::tmem_ld8_nowait(my_lane + (uint32_t)(c * 8), r[c]);
          tc::tmem_wait_ld();
          if (valid)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              float f[8];
#pragma unroll
              for (int e = 0; e < 8; ++e) f[e] = __uint_as_float(r[c][e]);
              *reinterpret_cast<uint4*>(a.dx + (size_t)grow * 32 + c * 8) = pack_bf16x8(f);
            }
          tc::fence_before_sync();
          group_sync(g);  // every row's accumulator is read before the next tile's GEMMs
        }
      }
    }
  }

  tc::fence_before_sync();
  __syncthreads();
  bool fin_ok = false;
  if (warp < 4) {
    int got = 0;
    if (lane == 0) got = (!abort_flag && wait_or_abort(&fin, 0u, abort_v)) ? 1 : 0;
    fin_ok = __shfl_sync(0xffffffffu, got, 0) != 0;
  }
  tc::fence_after_sync();
  if (warp < 4 && fin_ok) {
    // weight gradients: accumulator row o (lane) holds dW[o][0..64)
    for (int j = 0; j < kLayers; ++j) {
      const int nout = j < kHidden ? kWidth : kOutCh;
      if (warp * 32 >= nout) continue;  // warp-uniform: tcgen05.ld is warp-wide
      for (int c = 0; c < kWidth / 8; ++c) {
        float v[8];
        tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + 128u + 64u * (uint32_t)j + (uint32_t)(c * 8), v);
        if (tid < nout) {  // two 16-byte vector atomics
          float4* dst = reinterpret_cast<float4*>(a.gw[j] + tid * kWidth + c * 8);
          atomicAdd(dst, make_float4(v[0], v[1], v[2], v[3]));
          atomicAdd(dst + 1, make_float4(v[4], v[5], v[6], v[7]));
        }
      }
    }
  }
  if (a.loss && warp < 4 * kGroups) {
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, off);
    if (lane == 0) atomicAdd(a.loss, loss);
  }
  if (abort_flag && tid == 0) {
    atomicOr(a.err, 4u);
    tc::mbar_wait(&fin, 0u, kWaitLimit);  // MMAs that may still be in flight
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

}  // namespace

struct NrcNet {
  uint32_t max_q = 0;
  GridGeo geo{};
  int nout[kLayers] = {kWidth, kWidth, kWidth, kWidth, kOutCh};
  float *w[kLayers], *mw[kLayers], *vw[kLayers], *gw[kLayers];
  __nv_bfloat16* wf[kLayers];
  float *grid, *mg, *vg, *gg;
  __nv_bfloat16 *x0, *dx;
  double* d_loss = nullptr;
  uint32_t* d_err = nullptr;
  std::vector<void*> allocs;
  int step = 0;
  uint32_t last_count = 0;
  bool gg_clear = false;  // the grid gradient table is all zero
  bool gw_clear = false;  // the MLP gradients are all zero
};

Nrc::~Nrc() {
  if (!net) return;
  for (void* p : net->allocs) cudaFree(p);
  delete net;
  net = nullptr;
}

namespace {

std::string cuda_msg(cudaError_t e, const char* what) {
  return std::string(what) + ": " + cudaGetErrorString(e);
}

template <typename T>
cudaError_t alloc(NrcNet& n, T*& p, size_t count) {
  void* v = nullptr;
  cudaError_t e = cudaMalloc(&v, count * sizeof(T));
  if (e == cudaSuccess) {
    n.allocs.push_back(v);
    p = static_cast<T*>(v);
  }
  return e;
}

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return sms;
}

cudaError_t launch_mlp_train(const MlpArgs& a, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTrain);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const uint32_t tiles = (a.count + kRows - 1) / kRows;
  const int grid = (int)std::min<uint32_t>((tiles + kGroups - 1) / kGroups, (uint32_t)sm_count());
  k_mlp_train<<<grid, kTrainThreads, kSmemTrain, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const MlpArgs& a, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmemBytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const uint32_t tiles = (a.count + kRows - 1) / kRows;
  const int grid = (int)std::min<uint32_t>(tiles, (uint32_t)sm_count() * 2u);
  k_mlp_infer<<<grid, kRows, kInferSmemBytes, st>>>(a);
  return cudaGetLastError();
}

MlpArgs mlp_args(NrcNet& n, uint32_t count) {
  MlpArgs a{};
  a.x0 = n.x0;
  for (int l = 0; l < kLayers; ++l) {
    a.w[l] = n.wf[l];
    a.gw[l] = n.gw[l];
  }
  a.count = count;
  a.dx = n.dx;
  a.err = n.d_err;
  a.geo = n.geo;
  return a;
}

std::string finish(NrcNet& n, cudaStream_t st, const char* what) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_msg(e, what);
  uint32_t err = 0;
  cudaMemcpy(&err, n.d_err, 4, cudaMemcpyDeviceToHost);
  if (err) {
    cudaMemset(n.d_err, 0, 4);
    return std::string(what) + ": a tensor-core wait timed out";
  }
  return {};
}

}  // namespace

std::string nrc_create(Nrc& c, uint32_t max_queries, const float lo[3], const float hi[3],
                       uint32_t seed) {
  if (max_queries == 0) return "nrc: max_queries must be positive";
  c.net = new NrcNet();
  NrcNet& n = *c.net;
  n.max_q = max_queries;
  for (int k = 0; k < 3; ++k) {
    n.geo.lo[k] = lo[k];
    const float ext = hi[k] - lo[k];
    n.geo.inv_ext[k] = ext > 0.0f ? 1.0f / ext : 1.0f;
  }
  const double b = std::exp((std::log((double)kNmax) - std::log((double)kNmin)) / (kLevels - 1));
  for (int l = 0; l < kLevels; ++l) {
    n.geo.scale[l] = (float)std::floor(kNmin * std::pow(b, l));
    const double r = n.geo.scale[l] + 2.0;
    n.geo.dense[l] = r * r * r <= (double)kT ? 1u : 0u;
  }
  cudaError_t e;
#define AL(p, cnt) \
  if ((e = alloc(n, p, cnt)) != cudaSuccess) return cuda_msg(e, "nrc buffers");
  std::mt19937 rng(seed);
  std::vector<float> host;
  for (int l = 0; l < kLayers; ++l) {
    const size_t k = (size_t)n.nout[l] * kWidth;
    AL(n.w[l], k);
    AL(n.mw[l], k);
    AL(n.vw[l], k);
    AL(n.gw[l], k);
    AL(n.wf[l], k);
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / kWidth));
    host.resize(k);
    for (auto& v : host) v = nd(rng);
    cudaMemcpy(n.w[l], host.data(), k * 4, cudaMemcpyHostToDevice);
    cudaMemset(n.mw[l], 0, k * 4);
    cudaMemset(n.vw[l], 0, k * 4);
    k_pack<<<blocks_for(k), 256>>>(n.w[l], n.wf[l], k);
  }
  const size_t ng = (size_t)kLevels * kT * kFeat;
  AL(n.grid, ng);
  AL(n.mg, ng);
  AL(n.vg, ng);
  AL(n.gg, ng);
  host.resize(ng);
  std::uniform_real_distribution<float> ud(-1e-4f, 1e-4f);
  for (auto& v : host) v = ud(rng);
  cudaMemcpy(n.grid, host.data(), ng * 4, cudaMemcpyHostToDevice);
  cudaMemset(n.mg, 0, ng * 4);
  cudaMemset(n.vg, 0, ng * 4);
  AL(n.x0, (size_t)max_queries * kWidth);
  AL(n.dx, (size_t)max_queries * 32);
  AL(n.d_loss, 1);
  AL(n.d_err, 1);
#undef AL
  cudaMemset(n.d_err, 0, 4);
  e = cudaDeviceSynchronize();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "nrc init");
}

std::string nrc_infer(Nrc& c, const NrcQuery* q, uint32_t count, float* out, cudaStream_t st) {
  if (!c.net) return "nrc: not created";
  NrcNet& n = *c.net;
  if (count > n.max_q) return "nrc: more queries than the cache was created for";
  if (count == 0) return {};
  k_encode<<<blocks_for((size_t)count * kLevels), 256, 0, st>>>(n.geo, q, n.grid, n.x0, count);
  MlpArgs a = mlp_args(n, count);
  a.out = out;
  cudaError_t e = launch_mlp_infer(a, st);
  return e == cudaSuccess ? std::string() : cuda_msg(e, "nrc inference");
}

std::string nrc_train(Nrc& c, const NrcQuery* q, const float* target, uint32_t count, float lr,
                      double* loss, cudaStream_t st) {
  if (!c.net) return "nrc: not created";
  NrcNet& n = *c.net;
  if (count > n.max_q) return "nrc: more queries than the cache was created for";
  if (count == 0) return {};
  if (!n.gw_clear)
    for (int l = 0; l < kLayers; ++l) cudaMemsetAsync(n.gw[l], 0, (size_t)n.nout[l] * kWidth * 4, st);
  const size_t ng = (size_t)kLevels * kT * kFeat;
  if (!n.gg_clear) cudaMemsetAsync(n.gg, 0, ng * 4, st);
  n.gw_clear = n.gg_clear = false;
  cudaMemsetAsync(n.d_loss, 0, sizeof(double), st);
  k_encode<<<blocks_for((size_t)count * kLevels), 256, 0, st>>>(n.geo, q, n.grid, n.x0, count);
  MlpArgs a = mlp_args(n, count);
  a.target = target;
  a.q = q;
  a.loss = n.d_loss;
  cudaError_t e = launch_mlp_train(a, st);
  if (e != cudaSuccess) return cuda_msg(e, "nrc training");
  k_encode_bwd<<<blocks_for((size_t)count * kLevels), 256, 0, st>>>(
      n.geo, q, reinterpret_cast<const __nv_bfloat162*>(n.dx), n.gg, count);
  n.last_count = count;
  if (lr > 0.0f) {
    n.step++;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-10f;
    const float c1 = 1.0f - std::pow(b1, (float)n.step), c2 = 1.0f - std::pow(b2, (float)n.step);
    MlpOpt o;
    for (int l = 0; l < kLayers; ++l) {
      o.w[l] = n.w[l];
      o.m[l] = n.mw[l];
      o.v[l] = n.vw[l];
      o.g[l] = n.gw[l];
      o.wf[l] = n.wf[l];
    }
    k_adam_mlp<<<blocks_for((size_t)kHidden * kWidth * kWidth + kOutCh * kWidth), 256, 0, st>>>(
        o, lr, b1, b2, eps, c1, c2);
    static_assert((kLevels * kT * kFeat) % 4 == 0, "grid table in float4 units");
    k_adam_grid<<<(int)((ng / 4 + 255) / 256), 256, 0, st>>>(n.grid, n.mg, n.vg,
                                                    reinterpret_cast<float4*>(n.gg), ng / 4, lr,
                                                    b1, b2, eps, c1, c2);
    n.gw_clear = n.gg_clear = true;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_msg(e, "nrc train");
  if (loss) {
    std::string s = finish(n, st, "nrc train");
    if (!s.empty()) return s;
    double h = 0.0;
    cudaMemcpy(&h, n.d_loss, sizeof(double), cudaMemcpyDeviceToHost);
    *loss = h / (3.0 * count);
  }
  return {};
}

uint32_t nrc_max_queries(const Nrc& c) { return c.net ? c.net->max_q : 0u; }

std::string nrc_poll_error(Nrc& c, cudaStream_t st) {
  if (!c.net) return "nrc: not created";
  uint32_t err = 0;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(&err, c.net->d_err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_msg(e, "nrc");
  if (err) {
    cudaMemset(c.net->d_err, 0, 4);
    return "nrc: a tensor-core wait timed out";
  }
  return {};
}

size_t nrc_count(const Nrc& c, int what) {
  if (!c.net) return 0;
  if (what <= 1) {
    size_t s = 0;
    for (int l = 0; l < kLayers; ++l) s += (size_t)c.net->nout[l] * kWidth;
    return s;
  }
  if (what <= 3) return (size_t)kLevels * kT * kFeat;
  return (size_t)c.net->last_count * kWidth;
}

std::string nrc_get(const Nrc& c, int what, float* host) {
  if (!c.net) return "nrc: not created";
  const NrcNet& n = *c.net;
  cudaDeviceSynchronize();
  if (what <= 1) {
    for (int l = 0; l < kLayers; ++l) {
      const size_t k = (size_t)n.nout[l] * kWidth;
      cudaMemcpy(host, what ? n.gw[l] : n.w[l], k * 4, cudaMemcpyDeviceToHost);
      host += k;
    }
  } else if (what <= 3) {
    cudaMemcpy(host, what == 2 ? n.grid : n.gg, (size_t)kLevels * kT * kFeat * 4,
               cudaMemcpyDeviceToHost);
  } else {
    std::vector<__nv_bfloat16> tmp((size_t)n.last_count * kWidth);
    cudaMemcpy(tmp.data(), n.x0, tmp.size() * 2, cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < tmp.size(); ++i) host[i] = __bfloat162float(tmp[i]);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "nrc read");
}

std::string nrc_set_weights(Nrc& c, const float* mlp, const float* grid) {
  if (!c.net) return "nrc: not created";
  NrcNet& n = *c.net;
  if (mlp)
    for (int l = 0; l < kLayers; ++l) {
      const size_t k = (size_t)n.nout[l] * kWidth;
      cudaMemcpy(n.w[l], mlp, k * 4, cudaMemcpyHostToDevice);
      k_pack<<<blocks_for(k), 256>>>(n.w[l], n.wf[l], k);
      mlp += k;
    }
  if (grid) cudaMemcpy(n.grid, grid, (size_t)kLevels * kT * kFeat * 4, cudaMemcpyHostToDevice);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "nrc write");
}

}  // namespace nr
