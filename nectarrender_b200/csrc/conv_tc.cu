// conv_tc.cu — tcgen05 implicit-GEMM 3x3 convolutions (see conv_tc.cuh).
//
// Which kernel runs (launch_conv_fwd / launch_conv_wgrad pick the first that
// fits the shape):
//  * k_conv_fwd_tma / k_conv_wgrad_tma — images whose height is a multiple
//    of 16 and width a multiple of 8, weights (forward) or two stages
//    (weight gradient) within shared memory: 8 x 16 pixel tiles copied by
//    TMA in swizzled layouts, warp-specialised issue and mbarrier
//    hand-overs (the main path; described at the kernels);
//  * k_conv_fwd_res / k_conv_fwd_halo / k_conv_wgrad_halo — the same tiles
//    copied with cp.async, for shapes whose TMA stages do not fit;
//  * k_conv_fwd / k_conv_wgrad — any image size: per-tap gathers, described
//    next.
//
// Forward / backward-data (k_conv_fwd): one CTA of 128 threads computes a
// 128-pixel x cout tile. The K loop runs over the 9 taps; per tap the 128
// shifted input rows (zero outside the image) and the tap's cout x cin
// weights are copied into shared memory with cp.async (16-byte chunks,
// zero-fill at the borders) in the K-major no-swizzle canonical layout, and
// one thread issues cin / 16 MMAs (M = 128, N = cout, K = 16) into a
// tensor-memory accumulator. Two shared-memory stages alternate: the copy of
// tap t overlaps the MMAs of tap t - 1; a stage is refilled after the
// tcgen05.commit of its previous MMAs has arrived on that stage's mbarrier.
// The epilogue loads the accumulator (tcgen05.ld, one pixel row per thread),
// adds the bias, applies ReLU and stores BF16.
//
// Backward-weights (k_conv_wgrad): CTA (g, tap) reduces chunks of 128
// pixels: D[co, ci] += dY^T[co, p] * Xshift^T[ci, p] with both operands
// MN-major in shared memory (cout rows padded to the M = 128 tile with
// zeros), then adds its FP32 partial sums to dW with atomics.
#include "conv_tc.cuh"

#include <cuda.h>  // CUtensorMap and its enums; the encoder is fetched from the driver at run time

#include <algorithm>
#include "tcgen05.cuh"

namespace nr {

namespace {

constexpr int kThreads = 128;
constexpr uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(dst), "l"(src),
               "r"(valid ? 16u : 0u) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most one committed group is still in flight
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__host__ __device__ inline uint32_t tmem_cols(int n) {
  return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : 256u));
}

__device__ __forceinline__ uint4 pack_bf16x8(const float (&v)[8]) {
  uint4 r;
  __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]);
  __nv_bfloat162 b = __floats2bfloat162_rn(v[2], v[3]);
  __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]);
  __nv_bfloat162 d = __floats2bfloat162_rn(v[6], v[7]);
  r.x = *reinterpret_cast<uint32_t*>(&a);
  r.y = *reinterpret_cast<uint32_t*>(&b);
  r.z = *reinterpret_cast<uint32_t*>(&c);
  r.w = *reinterpret_cast<uint32_t*>(&d);
  return r;
}

__global__ void __launch_bounds__(kThreads) k_conv_fwd(ConvFwdArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, cout = a.cout;
  const int P = a.B * a.H * a.W;
  const int p0 = blockIdx.x * 128;
  const uint32_t a_bytes = 128u * cin * 2u, b_bytes = (uint32_t)cout * cin * 2u;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  const uint32_t base = tc::smem_u32(smem);
  const uint32_t lbo_a = 128u * 16u, lbo_b = (uint32_t)cout * 16u;
  const uint32_t ncols = tmem_cols(cout);

  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, ncols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)cout, false, false);

  // this thread's pixel rows (fixed over the taps)
  bool ok = true;
  const int ntaps = a.taps == 1 ? 1 : 9;
  for (int t = 0; t < ntaps && ok; ++t) {
    const int s = t & 1;
    if (t >= 2) {
      // CTA-uniform: every thread polls, all agree before any of them leaves
      const bool w = tc::mbar_wait(&bar[s], (uint32_t)((t >> 1) - 1) & 1u, kWaitLimit);
      if (!__syncthreads_and(w)) {
        ok = false;
        break;
      }
    }
    const uint32_t sa = base + s * stage_bytes, sb = sa + a_bytes;
    const int dy = ntaps == 1 ? 0 : t / 3 - 1, dx = ntaps == 1 ? 0 : t % 3 - 1;
    const int kg_n = cin >> 3;
    for (int i = tid; i < 128 * kg_n; i += kThreads) {
      const int r = i & 127, kg = i >> 7;
      const int p = p0 + r;
      bool valid = p < P;
      const __nv_bfloat16* src = a.x;
      if (valid) {
        const int xw = p % a.W, rest = p / a.W;
        const int yh = rest % a.H, b = rest / a.H;
        const int sy = yh + dy, sx = xw + dx;
        valid = sy >= 0 && sy < a.H && sx >= 0 && sx < a.W;
        if (valid)
          src = a.x + ((size_t)(b * a.H + sy) * a.W + sx) * a.x_stride + a.x_off + kg * 8;
      }
      cp_async16(sa + (uint32_t)r * 16u + (uint32_t)kg * lbo_a, src, valid);
    }
    const __nv_bfloat16* wt = a.w + (size_t)t * cout * cin;
    for (int i = tid; i < cout * kg_n; i += kThreads) {
      const int n = i % cout, kg = i / cout;
      cp_async16(sb + (uint32_t)n * 16u + (uint32_t)kg * lbo_b, wt + (size_t)n * cin + kg * 8, true);
    }
    cp_async_wait_all();
    tc::fence_smem_to_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < (cin >> 4); ++kk) {
        const uint64_t da = tc::smem_desc(sa + 2u * kk * lbo_a, lbo_a, 128u);
        const uint64_t db = tc::smem_desc(sb + 2u * kk * lbo_b, lbo_b, 128u);
        tc::mma_bf16(tmem, da, db, idesc, (t > 0 || kk > 0) ? 1u : 0u);
      }
      tc::mma_commit(&bar[s]);
    }
  }
  // the last tap used stage (ntaps - 1) & 1 for the ((ntaps - 1) >> 1)-th time
  if (ok)
    ok = __syncthreads_and(tc::mbar_wait(&bar[(ntaps - 1) & 1], (uint32_t)((ntaps - 1) >> 1) & 1u,
                                         kWaitLimit));
  if (!ok && tid == 0) atomicOr(a.err, 2u);
  tc::fence_after_sync();
  __syncthreads();
  if (ok) {
    const int p = p0 + warp * 32 + lane;
    for (int c = 0; c < (cout >> 3); ++c) {
      float v[8];
      tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 8), v);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (a.bias) v[j] += a.bias[c * 8 + j];
        if (a.relu) v[j] = fmaxf(v[j], 0.0f);
      }
      if (p < P)
        *reinterpret_cast<uint4*>(a.y + (size_t)p * a.y_stride + a.y_off + c * 8) = pack_bf16x8(v);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// Halo-tile forward: the CTA's 128 output pixels are an 8 x 16 block of one
// image. Its 10 x 18 halo (zero outside the image) is copied into shared
// memory once, K-major with 8-pixel core rows: halo pixel h = hy * 10 + hx at
// byte h * 16 within each 8-channel group, groups 180 * 16 bytes apart. The
// operand of tap (dy, dx) is then the same region seen from start address
// (dy * 10 + dx) * 16 with a row-group stride (SBO) of one halo row, 160
// bytes: no per-tap gather. Only the tap's weights are streamed, through two
// stages.
constexpr int kTileW = 8, kTileH = 16;
constexpr int kHaloW = kTileW + 2, kHaloH = kTileH + 2, kHalo = kHaloW * kHaloH;

__global__ void __launch_bounds__(kThreads) k_conv_fwd_halo(ConvFwdArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, cout = a.cout;
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH, b = blockIdx.z;
  const uint32_t lbo_a = (uint32_t)kHalo * 16u, sbo_a = (uint32_t)kHaloW * 16u;
  const uint32_t a_bytes = (uint32_t)(cin >> 3) * lbo_a;
  const uint32_t b_bytes = (uint32_t)cout * cin * 2u, lbo_b = (uint32_t)cout * 16u;
  const uint32_t base = tc::smem_u32(smem);
  const uint32_t sa = base, sb0 = base + a_bytes;
  const uint32_t ncols = tmem_cols(cout);
  const int kg_n = cin >> 3;

  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, ncols);
  // halo and the weights of tap 0
  for (int i = tid; i < kHalo * kg_n; i += kThreads) {
    const int h = i % kHalo, kg = i / kHalo;
    const int yy = y0 - 1 + h / kHaloW, xx = x0 - 1 + h % kHaloW;
    const bool valid = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
    const __nv_bfloat16* src =
        valid ? a.x + ((size_t)(b * a.H + yy) * a.W + xx) * a.x_stride + a.x_off + kg * 8 : a.x;
    cp_async16(sa + (uint32_t)kg * lbo_a + (uint32_t)h * 16u, src, valid);
  }
  for (int i = tid; i < cout * kg_n; i += kThreads) {
    const int n = i % cout, kg = i / cout;
    cp_async16(sb0 + (uint32_t)n * 16u + (uint32_t)kg * lbo_b, a.w + (size_t)n * cin + kg * 8, true);
  }
  cp_async_wait_all();
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)cout, false, false);

  bool ok = true;
  for (int t = 0; t < 9; ++t) {
    const int s = t & 1;
    const uint32_t sb = sb0 + s * b_bytes;
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t tap_off = (uint32_t)((t / 3) * kHaloW + (t % 3)) * 16u;
      for (int kk = 0; kk < (cin >> 4); ++kk) {
        const uint64_t da = tc::smem_desc(sa + tap_off + 2u * kk * lbo_a, lbo_a, sbo_a);
        const uint64_t db = tc::smem_desc(sb + 2u * kk * lbo_b, lbo_b, 128u);
        tc::mma_bf16(tmem, da, db, idesc, (t > 0 || kk > 0) ? 1u : 0u);
      }
      tc::mma_commit(&bar[s]);
    }
    if (t + 1 < 9) {
      const int s1 = (t + 1) & 1;
      if (t + 1 >= 2) {
        // stage s1 last held tap t - 1: wait for its MMAs
        const bool w = tc::mbar_wait(&bar[s1], (uint32_t)((t - 1) >> 1) & 1u, kWaitLimit);
        if (!__syncthreads_and(w)) {
          ok = false;
          break;
        }
      }
      const uint32_t sbn = sb0 + s1 * b_bytes;
      const __nv_bfloat16* wt = a.w + (size_t)(t + 1) * cout * cin;
      for (int i = tid; i < cout * kg_n; i += kThreads) {
        const int n = i % cout, kg = i / cout;
        cp_async16(sbn + (uint32_t)n * 16u + (uint32_t)kg * lbo_b, wt + (size_t)n * cin + kg * 8, true);
      }
      cp_async_wait_all();
      tc::fence_smem_to_async();
      __syncthreads();
    }
  }
  if (ok) ok = __syncthreads_and(tc::mbar_wait(&bar[0], 0u, kWaitLimit));
  if (!ok && tid == 0) atomicOr(a.err, 2u);
  tc::fence_after_sync();
  __syncthreads();
  if (ok) {
    const int r = warp * 32 + lane;
    const size_t p = (size_t)(b * a.H + y0 + r / kTileW) * a.W + x0 + r % kTileW;
    for (int c = 0; c < (cout >> 3); ++c) {
      float v[8];
      tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 8), v);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (a.bias) v[j] += a.bias[c * 8 + j];
        if (a.relu) v[j] = fmaxf(v[j], 0.0f);
      }
      *reinterpret_cast<uint4*>(a.y + p * a.y_stride + a.y_off + c * 8) = pack_bf16x8(v);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// Persistent halo-tile forward with resident weights: the CTA keeps the
// weights of all nine taps for its slice of nco output channels in shared
// memory for its whole run of 8 x 16 pixel tiles, and streams only the input
// halos through three stages (two tiles ahead). Two tensor-memory
// accumulators alternate, so tile j's MMAs run while tile j - 1's epilogue
// stores and tile j + 2's halo loads. Weights of tap t: K-major over (output channel, input channel),
// element (n, k) at t * nco * cin * 2 + n * 16 + (k / 8) * nco * 16.
constexpr int kFwdStages = 3;
constexpr int kResThreads = 256;  // 8 warps: an MMA issuer, loaders, four storers
constexpr int kWgThreads = 256;   // 8 warps: an MMA issuer and seven loaders

__global__ void __launch_bounds__(kResThreads) k_conv_fwd_res(ConvFwdArgs a, int nco) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, kg_n = cin >> 3;
  const int co0 = blockIdx.y * nco;
  const int tw = a.W / kTileW, th = a.H / kTileH, n_tiles = tw * th * a.B;
  const uint32_t lbo_a = (uint32_t)kHalo * 16u, sbo_a = (uint32_t)kHaloW * 16u;
  const uint32_t h_bytes = (uint32_t)kg_n * lbo_a;
  const uint32_t w_tap = (uint32_t)nco * cin * 2u, lbo_b = (uint32_t)nco * 16u;
  const uint32_t base = tc::smem_u32(smem);
  const uint32_t sw = base, sh0 = base + 9u * w_tap;  // then kFwdStages halo stages
  const uint32_t ncols = 2u * nco <= 64u ? 64u : (2u * nco <= 128u ? 128u : 256u);

  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, ncols);
  // warp roles: warp 0 issues the MMAs, warps 1-7 load halos, warps 4-7
  // store the accumulators (one per tensor-memory subpartition), so that
  // the MMAs of one tile overlap the loads and stores of the others
  auto load_halo = [&](int t, uint32_t dst) {
    const int b = t / (tw * th), rest = t % (tw * th);
    const int y0 = (rest / tw) * kTileH, x0 = (rest % tw) * kTileW;
    if (tid < 32) return;
    for (int i = tid - 32; i < kHalo * kg_n; i += kResThreads - 32) {
      const int h = i % kHalo, kg = i / kHalo;
      const int yy = y0 - 1 + h / kHaloW, xx = x0 - 1 + h % kHaloW;
      const bool valid = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
      const __nv_bfloat16* src =
          valid ? a.x + ((size_t)(b * a.H + yy) * a.W + xx) * a.x_stride + a.x_off + kg * 8 : a.x;
      cp_async16(dst + (uint32_t)kg * lbo_a + (uint32_t)h * 16u, src, valid);
    }
  };
  // resident weights of the slice, and the first halo
  for (int i = tid; i < 9 * nco * kg_n; i += kResThreads) {
    const int n = i % nco, rest = i / nco, kg = rest % kg_n, t = rest / kg_n;
    cp_async16(sw + (uint32_t)t * w_tap + (uint32_t)n * 16u + (uint32_t)kg * lbo_b,
               a.w + ((size_t)t * a.cout + co0 + n) * cin + kg * 8, true);
  }
  const int first = blockIdx.x, step = (int)gridDim.x;
  load_halo(first, sh0);  // first < n_tiles: the grid has at most n_tiles columns
  cp_async_commit();
  if (first + step < n_tiles) load_halo(first + step, sh0 + h_bytes);
  cp_async_commit();
  cp_async_wait_1();
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)nco, false, false);

  auto epilogue = [&](int t, int s) {
    const int b = t / (tw * th), rest = t % (tw * th);
    const int y0 = (rest / tw) * kTileH, x0 = (rest % tw) * kTileW;
    // warp w (4..7) reads tensor-memory lanes 32 (w % 4) .. +31, its subpartition
    if (warp < 4) return;
    const int sub = warp & 3;
    const int r = sub * 32 + lane;
    const size_t p = (size_t)(b * a.H + y0 + r / kTileW) * a.W + x0 + r % kTileW;
    const int g0 = 0, gend = nco >> 3;
    // up to 64 columns in flight per wait
    for (int c0 = g0; c0 < gend; c0 += 8) {
      uint32_t r[8][8];
      const int nc = min(8, gend - c0);
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < nc)
          tc::tmem_ld8_nowait(tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)(s * nco + (c0 + c) * 8),
                              r[c]);
      tc::tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c >= nc) break;
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          v[q] = __uint_as_float(r[c][q]);
          if (a.bias) v[q] += a.bias[co0 + (c0 + c) * 8 + q];
          if (a.relu) v[q] = fmaxf(v[q], 0.0f);
        }
        *reinterpret_cast<uint4*>(a.y + p * a.y_stride + a.y_off + co0 + (c0 + c) * 8) = pack_bf16x8(v);
      }
    }
  };

  // One CTA barrier per tile, at its end. Warp 0 issues tile j's MMAs while
  // the other warps wait (each on the mbarrier) for tile j - 1's, load tile
  // j + 2's halo into the stage tile j - 1 used and store tile j - 1's
  // accumulator.
  bool ok = true;
  int j = 0;
  for (int t = first; t < n_tiles; t += step, ++j) {
    const int s = j & 1, hs = j % kFwdStages;
    bool fail = false;
    if (warp == 0) {
      if (lane == 0) {
        tc::fence_after_sync();
        // descriptors advance by adding (byte offset >> 4) to the start-address
        // field: every operand lies below 256 KB, so the field never carries
        const uint64_t da0 = tc::smem_desc(sh0 + (uint32_t)hs * h_bytes, lbo_a, sbo_a);
        const uint64_t db0 = tc::smem_desc(sw, lbo_b, 128u);
        const uint32_t d = tmem + (uint32_t)(s * nco);
        const int nk = cin >> 4;
        for (int tap = 0; tap < 9; ++tap) {
          const uint64_t da_t = da0 + (uint64_t)(((tap / 3) * kHaloW + (tap % 3)));  // 16-byte units
          const uint64_t db_t = db0 + (uint64_t)(((uint32_t)tap * w_tap) >> 4);
          for (int kk = 0; kk < nk; ++kk)
            tc::mma_bf16(d, da_t + (uint64_t)((2u * kk * lbo_a) >> 4),
                         db_t + (uint64_t)((2u * kk * lbo_b) >> 4), idesc, (tap > 0 || kk > 0) ? 1u : 0u);
        }
        tc::mma_commit(&bar[s]);
      }
      __syncwarp();
    } else {
      if (j >= 1) {
        // tile j - 1's MMAs: their accumulator and halo stage become free
        fail = !tc::mbar_wait(&bar[s ^ 1], (uint32_t)((j - 1) >> 1) & 1u, kWaitLimit);
        tc::fence_after_sync();
      }
      if (!fail) {
        if (t + 2 * step < n_tiles)
          load_halo(t + 2 * step, sh0 + (uint32_t)((j + 2) % kFwdStages) * h_bytes);
        cp_async_commit();
        if (j >= 1) epilogue(t - step, s ^ 1);
        cp_async_wait_1();  // tile j + 1's halo is complete
        tc::fence_smem_to_async();
      }
    }
    tc::fence_before_sync();
    if (__syncthreads_or(fail)) {
      ok = false;
      break;
    }
  }
  if (ok && j >= 1) {
    const int s = (j - 1) & 1;
    bool w = true;
    if (warp >= 4) {
      w = tc::mbar_wait(&bar[s], (uint32_t)((j - 1) >> 1) & 1u, kWaitLimit);
      tc::fence_after_sync();
      if (w) epilogue(first + (j - 1) * step, s);
    }
    ok = __syncthreads_and(w);
  }
  if (!ok) {
    if (tid == 0) atomicOr(a.err, 2u);
    tc::mbar_wait(&bar[0], 0u, kWaitLimit);  // bounded: MMAs that may still be in flight
    tc::mbar_wait(&bar[1], 0u, kWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

__global__ void __launch_bounds__(kThreads) k_conv_wgrad(ConvWgradArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, cout = a.cout;
  const int P = a.B * a.H * a.W;
  const int n_chunks = (P + 127) / 128;
  const int tap = blockIdx.y;
  const bool one = a.taps == 1;
  const int dy = one ? 0 : tap / 3 - 1, dx = one ? 0 : tap % 3 - 1;
  const int c0 = blockIdx.x * a.chunks_per_cta;
  const int c1 = min(n_chunks, c0 + a.chunks_per_cta);
  const uint32_t lbo = 128u, sbo = 2048u;  // MN-major: 8 pixels x 16 B per K group
  const uint32_t a_bytes = 16u * sbo;      // 128 (padded) output channels
  const uint32_t b_bytes = (uint32_t)(cin >> 3) * sbo;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  const uint32_t base = tc::smem_u32(smem);
  const uint32_t ncols = tmem_cols(cin);

  // zero both stages once: rows >= cout of the A tiles stay zero
  for (uint32_t i = tid * 16u; i < 2u * stage_bytes; i += kThreads * 16u)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, ncols);
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)cin, true, true);

  bool ok = true;
  int uses[2] = {0, 0};
  for (int c = c0; c < c1 && ok; ++c) {
    const int j = c - c0, s = j & 1;
    if (j >= 2) {
      const bool w = tc::mbar_wait(&bar[s], (uint32_t)(uses[s] - 1) & 1u, kWaitLimit);
      if (!__syncthreads_and(w)) {
        ok = false;
        break;
      }
    }
    const uint32_t sa = base + s * stage_bytes, sb = sa + a_bytes;
    const int pbase = c * 128;
    for (int i = tid; i < (cout >> 3) * 128; i += kThreads) {
      const int pl = i & 127, cg = i >> 7;
      const int p = pbase + pl;
      const bool valid = p < P;
      const __nv_bfloat16* src = valid ? a.dy + (size_t)p * a.dy_stride + a.dy_off + cg * 8 : a.dy;
      cp_async16(sa + (uint32_t)cg * sbo + (uint32_t)(pl >> 3) * lbo + (uint32_t)(pl & 7) * 16u,
                 src, valid);
    }
    for (int i = tid; i < (cin >> 3) * 128; i += kThreads) {
      const int pl = i & 127, cg = i >> 7;
      const int p = pbase + pl;
      bool valid = p < P;
      const __nv_bfloat16* src = a.x;
      if (valid) {
        const int xw = p % a.W, rest = p / a.W;
        const int yh = rest % a.H, b = rest / a.H;
        const int sy = yh + dy, sx = xw + dx;
        valid = sy >= 0 && sy < a.H && sx >= 0 && sx < a.W;
        if (valid)
          src = a.x + ((size_t)(b * a.H + sy) * a.W + sx) * a.x_stride + a.x_off + cg * 8;
      }
      cp_async16(sb + (uint32_t)cg * sbo + (uint32_t)(pl >> 3) * lbo + (uint32_t)(pl & 7) * 16u,
                 src, valid);
    }
    cp_async_wait_all();
    tc::fence_smem_to_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      for (int kk = 0; kk < 8; ++kk) {
        const uint64_t da = tc::smem_desc(sa + 2u * kk * lbo, lbo, sbo);
        const uint64_t db = tc::smem_desc(sb + 2u * kk * lbo, lbo, sbo);
        tc::mma_bf16(tmem, da, db, idesc, (j > 0 || kk > 0) ? 1u : 0u);
      }
      tc::mma_commit(&bar[s]);
    }
    uses[s]++;
  }
  const int n_local = c1 - c0;
  if (ok && n_local > 0) {
    const int s_last = (n_local - 1) & 1;
    ok = __syncthreads_and(tc::mbar_wait(&bar[s_last], (uint32_t)(uses[s_last] - 1) & 1u, kWaitLimit));
  }
  if (!ok && tid == 0) atomicOr(a.err, 2u);
  tc::fence_after_sync();
  __syncthreads();
  if (ok && n_local > 0) {
    const int co = warp * 32 + lane;
    for (int cg = 0; cg < (cin >> 3); ++cg) {
      float v[8];
      tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cg * 8), v);
      if (co < cout) {
        float* dst = a.dw + ((size_t)tap * cout + co) * cin + cg * 8;
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicAdd(dst + q, v[q]);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// Halo-tile weight gradient: a CTA reduces a run of 8 x 16 pixel tiles for
// one group of taps. Per tile the dY rows (MN-major over output channels,
// padded to the M = 128 tile; rows >= cout are never read back) and the
// tile's 10 x 18 input halo are copied into shared memory once; the B
// operand of tap (dy, dx) is the halo seen MN-major over input channels from
// start (dy * 10 + dx) * 16 with LBO = 160 (next tile row of 8 pixels) and
// SBO = 180 * 16 (next 8 channels), so no per-tap gather is needed. Each tap
// of the group accumulates in its own cin tensor-memory columns over all the
// CTA's tiles (two shared-memory stages: tile j loads while tile j - 1's
// MMAs run); the partial sums go to dW with vector atomics at the end.
__global__ void __launch_bounds__(kWgThreads) k_conv_wgrad_halo(ConvWgradArgs a, int tpg,
                                                               int tiles_per_cta) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, cout = a.cout, kg_n = cin >> 3;
  const int tw = a.W / kTileW, th = a.H / kTileH, n_tiles = tw * th * a.B;
  const int t0 = blockIdx.x * tiles_per_cta, t1 = min(n_tiles, t0 + tiles_per_cta);
  const int tap0 = blockIdx.y * tpg, ntap = min(tpg, 9 - tap0);
  const uint32_t a_bytes = 16u * 2048u, b_bytes = (uint32_t)kg_n * kHalo * 16u;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  const uint32_t base = tc::smem_u32(smem);
  const uint32_t ncols = (uint32_t)ntap * cin <= 256u ? 256u : 512u;

  for (uint32_t i = tid * 16u; i < 2u * stage_bytes; i += kWgThreads * 16u)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, ncols);
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)cin, true, true);

  // warp 0 issues the MMAs; warps 1-7 wait (each on the mbarrier) for the
  // stage to come free and load the next tile; one CTA barrier per tile
  bool ok = true;
  int uses[2] = {0, 0};
  for (int t = t0; t < t1; ++t) {
    const int j = t - t0, s = j & 1;
    const uint32_t sa = base + s * stage_bytes, sb = sa + a_bytes;
    bool fail = false;
    if (warp != 0) {
      if (j >= 2) fail = !tc::mbar_wait(&bar[s], (uint32_t)(uses[s] - 1) & 1u, kWaitLimit);
      if (!fail) {
        const int b = t / (tw * th), rest = t % (tw * th);
        const int y0 = (rest / tw) * kTileH, x0 = (rest % tw) * kTileW;
        for (int i = tid - 32; i < (cout >> 3) * 128; i += kWgThreads - 32) {
          const int pl = i & 127, cg = i >> 7;
          const size_t p = (size_t)(b * a.H + y0 + pl / kTileW) * a.W + x0 + pl % kTileW;
          cp_async16(sa + (uint32_t)cg * 2048u + (uint32_t)pl * 16u,
                     a.dy + p * a.dy_stride + a.dy_off + cg * 8, true);
        }
        for (int i = tid - 32; i < kHalo * kg_n; i += kWgThreads - 32) {
          const int h = i % kHalo, kg = i / kHalo;
          const int yy = y0 - 1 + h / kHaloW, xx = x0 - 1 + h % kHaloW;
          const bool valid = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
          const __nv_bfloat16* src =
              valid ? a.x + ((size_t)(b * a.H + yy) * a.W + xx) * a.x_stride + a.x_off + kg * 8 : a.x;
          cp_async16(sb + (uint32_t)kg * kHalo * 16u + (uint32_t)h * 16u, src, valid);
        }
        cp_async_wait_all();
        tc::fence_smem_to_async();
      }
    }
    if (__syncthreads_or(fail)) {
      ok = false;
      break;
    }
    if (warp == 0) {
      if (lane == 0) {
        tc::fence_after_sync();
        for (int q = 0; q < ntap; ++q) {
          const int tap = tap0 + q;
          const uint32_t tap_off = (uint32_t)((tap / 3) * kHaloW + (tap % 3)) * 16u;
          for (int kk = 0; kk < 8; ++kk) {  // K = 128 pixels = 16 tile rows, two per MMA
            const uint64_t da = tc::smem_desc(sa + 256u * kk, 128u, 2048u);
            const uint64_t db = tc::smem_desc(sb + tap_off + 2u * kk * kHaloW * 16u, kHaloW * 16u,
                                              kHalo * 16u);
            tc::mma_bf16(tmem + (uint32_t)(q * cin), da, db, idesc, (j > 0 || kk > 0) ? 1u : 0u);
          }
        }
        tc::mma_commit(&bar[s]);
      }
      __syncwarp();
    }
    uses[s]++;
  }
  const int n_local = t1 - t0;
  if (ok && n_local > 0) {
    const int s_last = (n_local - 1) & 1;
    ok = __syncthreads_and(tc::mbar_wait(&bar[s_last], (uint32_t)(uses[s_last] - 1) & 1u, kWaitLimit));
  }
  if (!ok && tid == 0) atomicOr(a.err, 2u);
  tc::fence_after_sync();
  __syncthreads();
  if (ok && n_local > 0 && warp < 4) {  // warps 0-3: one tensor-memory subpartition each
    const int co = warp * 32 + lane;
    for (int q = 0; q < ntap; ++q) {
      if (warp * 32 >= cout) break;  // warp-uniform: tcgen05.ld is warp-wide
      for (int cg = 0; cg < kg_n; ++cg) {
        float v[8];
        tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * cin + cg * 8), v);
        if (co < cout) {
          float4* dst = reinterpret_cast<float4*>(a.dw + ((size_t)(tap0 + q) * cout + co) * cin + cg * 8);
          atomicAdd(dst, make_float4(v[0], v[1], v[2], v[3]));
          atomicAdd(dst + 1, make_float4(v[4], v[5], v[6], v[7]));
        }
      }
    }
  } else if (!ok) {
    tc::mbar_wait(&bar[0], (uint32_t)(uses[0] - 1) & 1u, kWaitLimit);  // MMAs still in flight
    tc::mbar_wait(&bar[1], (uint32_t)(uses[1] - 1) & 1u, kWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// TMA-fed persistent forward. A CTA keeps the weights of all nine taps for
// its slice of nco output channels (normally all of them: the MMA's time
// hardly depends on N up to 128, so the widest slice is the fastest) and
// streams the input halos of its 8 x 16 pixel tiles in slices of sc = 16,
// 32 or 64 input channels through a ring of `ring` shared-memory slots.
// Warp 0 (one thread) copies halo slices with TMA; warp 1 (all lanes, one
// elected issuer) issues per slice the nine taps' MMAs (K = 16 each, sc / 16
// per tap) into one of `accs`
// tensor-memory accumulators and frees the slot with a commit; warps 2-5
// (one per tensor-memory subpartition) read each finished accumulator back
// and store it. Hand-overs are mbarriers: full[r] (a slice's bytes have
// landed), empty[r] (the MMAs that read slot r are done), acc_full[q] (a
// tile's MMAs are done), acc_empty[q] (its accumulator has been read). No
// CTA-wide barrier sits inside the tile loop.
//
// Shared memory, 128-byte aligned regions:
//  * weights [kg][tap][n][8] (kg: 8 input channels), copied once: B of tap t
//    and input channels 16 k .. 16 k + 15 is K-major from 2k * 9 * nco * 16 +
//    t * nco * 16 with LBO 9 * nco * 16 (next 8 input channels) and SBO 128
//    (next 8 outputs);
//  * `ring` 1024-byte aligned halo slots, each one TMA box (sc channels x
//    10 x 18 pixels, zero outside the image) of 2 sc-byte pixel rows,
//    swizzled by TMA in the mode of that row width (32, 64 or 128 bytes).
//    A of tap (dy, dx) is K-major in the same swizzle mode from
//    (dy * 10 + dx) * 2 sc (+ 32 bytes per further 16 channels) with SBO one
//    halo row, 10 * 2 sc bytes: the tensor cores apply the swizzle to the
//    absolute shared-memory address as TMA does, so a view that starts whole
//    pixel rows into the box reads the box correctly, and no per-tap gather
//    is needed.
constexpr int kTmaThreads = 192;
constexpr int kTmaMaxStages = 4, kTmaMaxAccs = 4, kTmaMaxRing = 16;
constexpr uint32_t kKgPitch = 2944;  // 180 halo pixels x 16 bytes, rounded up to 128

// Halo slot of sc channels: 180 pixel rows of 2 sc bytes, rounded up to 1 KB.
__host__ __device__ constexpr uint32_t slot_bytes(int sc) {
  return ((uint32_t)kHalo * 2u * (uint32_t)sc + 1023u) & ~1023u;
}
// Swizzle mode of the tensor-core descriptor for rows of 2 sc bytes.
__host__ __device__ constexpr uint32_t umma_swizzle(int sc) { return sc == 64 ? 2u : (sc == 32 ? 4u : 6u); }

__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort) {
  return tc::mbar_wait_or_abort(bar, parity, abort, kWaitLimit);
}

__global__ void __launch_bounds__(kTmaThreads, 1)
    k_conv_fwd_tma(const __grid_constant__ CUtensorMap tm_x, ConvFwdArgs a, int nco, int sc, int ring,
                   int accs, uint32_t ncols) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kTmaMaxRing], empty[kTmaMaxRing];
  __shared__ __align__(8) uint64_t acc_full[kTmaMaxAccs], acc_empty[kTmaMaxAccs];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, n_loaded, n_issued;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, kg_n = cin >> 3, np = cin / sc, kps = sc >> 4;  // slices per tile, K steps per slice
  const int co0 = blockIdx.y * nco;
  const int tw = a.W / kTileW, th = a.H / kTileH, n_tiles = tw * th * a.B;
  const int first = blockIdx.x, step = (int)gridDim.x;
  const uint32_t base = (tc::smem_u32(smem) + 1023u) & ~1023u;
  const uint32_t w_kg = 9u * (uint32_t)nco * 16u;  // one kg's weights
  const uint32_t sw = base, sh0 = (base + (uint32_t)kg_n * w_kg + 1023u) & ~1023u;
  const uint32_t slot = slot_bytes(sc);
  volatile int* abort_v = &abort_flag;

  if (tid == 0) {
    for (int r = 0; r < ring; ++r) {
      tc::mbar_init(&full[r], 1);
      tc::mbar_init(&empty[r], 1);
    }
    for (int q = 0; q < accs; ++q) {
      tc::mbar_init(&acc_full[q], 1);
      tc::mbar_init(&acc_empty[q], 4);  // one arrival per epilogue warp
    }
    abort_flag = 0;
    n_loaded = 0;
    n_issued = 0;
  }
  if (warp == 1) tc::tmem_alloc(&tmem_base, ncols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  if (warp >= 1) {
    // warps 1-5 copy the slice's weights, [kg][tap][n][8], while warp 0
    // already streams halos; each CTA starts at another offset so that the
    // CTAs do not all read the same lines of L2 at once
    const int total = 9 * nco * kg_n, rot = (int)((blockIdx.x * 613u + blockIdx.y * 97u) % (uint32_t)total);
    for (int i = tid - 32; i < total; i += kTmaThreads - 32) {
      int ii = i + rot;
      if (ii >= total) ii -= total;
      const int kg = ii % kg_n, rest = ii / kg_n, n = rest % nco, t = rest / nco;
      cp_async16(sw + (uint32_t)kg * w_kg + (uint32_t)(t * nco + n) * 16u,
                 a.w + ((size_t)t * a.cout + co0 + n) * cin + kg * 8, true);
    }
    cp_async_wait_all();
    tc::fence_smem_to_async();
    asm volatile("bar.sync 1, %0;" :: "r"(kTmaThreads - 32) : "memory");  // warps 1-5 only
  }

  if (warp == 0) {
    if (lane == 0) {
      tc::tma_prefetch_map(&tm_x);
      int c = 0;  // slices copied so far
      for (int t = first; t < n_tiles; t += step) {
        const int b = t / (tw * th), rest = t % (tw * th);
        const int y0 = (rest / tw) * kTileH, x0 = (rest % tw) * kTileW;
        int p = 0;
        for (; p < np; ++p, ++c) {
          const int r = c % ring, u = c / ring;
          if (u >= 1 && !wait_or_abort(&empty[r], (uint32_t)(u - 1) & 1u, abort_v)) break;
          tc::mbar_arrive_expect_tx(&full[r], (uint32_t)kHalo * 2u * (uint32_t)sc);
          tc::tma_load_5d(sh0 + (uint32_t)r * slot, &tm_x, &full[r], 0, p, x0 - 1, y0 - 1, b);
        }
        if (p < np) break;
      }
      n_loaded = c;
    }
  } else if (warp == 1) {
    // the whole warp runs the issue loop; the elected lane issues
    int j = 0, c = 0, got = 1;
    const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)nco, false, false);
    // descriptors advance by adding (byte offset >> 4) to the start-address
    // field: every operand lies below 256 KB, so the field never carries
    const uint64_t da0 =
        tc::smem_desc(sh0, 16u, (uint32_t)kHaloW * 2u * (uint32_t)sc) | ((uint64_t)umma_swizzle(sc) << 61);
    const uint64_t db0 = tc::smem_desc(sw, w_kg, 128u);
    const uint64_t b_k = (2u * w_kg) >> 4, b_tap = ((uint32_t)nco * 16u) >> 4;
    const uint32_t a_px = (2u * (uint32_t)sc) >> 4;  // one pixel row, in 16-byte units
    for (int t = first; t < n_tiles; t += step, ++j) {
      const int q = j % accs, uq = j / accs;
      if (lane == 0) got = uq < 1 || wait_or_abort(&acc_empty[q], (uint32_t)(uq - 1) & 1u, abort_v);
      if (!__shfl_sync(0xffffffffu, got, 0)) break;
      const uint32_t d = tmem + (uint32_t)(q * nco);
      int p = 0;
      for (; p < np; ++p, ++c) {
        const int r = c % ring, u = c / ring;
        if (lane == 0) got = wait_or_abort(&full[r], (uint32_t)u & 1u, abort_v);
        if (!__shfl_sync(0xffffffffu, got, 0)) break;
        tc::fence_after_sync();
        const uint64_t da = da0 + (uint64_t)(((uint32_t)r * slot) >> 4);
        for (int kk = 0; kk < kps; ++kk) {
          const uint64_t db = db0 + (uint64_t)(p * kps + kk) * b_k;
#pragma unroll
          for (int tap = 0; tap < 9; ++tap)
            if (tc::elect_one())
              tc::mma_bf16(d, da + (uint64_t)(((tap / 3) * kHaloW + (tap % 3)) * a_px + 2 * kk),
                           db + (uint64_t)tap * b_tap, idesc, (p > 0 || kk > 0 || tap > 0) ? 1u : 0u);
        }
        if (tc::elect_one()) tc::mma_commit(&empty[r]);
        __syncwarp();
      }
      if (p < np) break;
      if (tc::elect_one()) tc::mma_commit(&acc_full[q]);
      __syncwarp();
    }
    if (lane == 0) n_issued = c;
  } else {
    // warps 2-5: warp w reads tensor-memory lanes 32 (w % 4) .. +31
    const int sub = warp & 3, r = sub * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(sub * 32) << 16);
    const int gend = nco >> 3;
    int j = 0;
    for (int t = first; t < n_tiles; t += step, ++j) {
      const int q = j % accs, uq = j / accs;
      int got = 0;
      if (lane == 0) got = wait_or_abort(&acc_full[q], (uint32_t)uq & 1u, abort_v) ? 1 : 0;
      if (!__shfl_sync(0xffffffffu, got, 0)) break;
      tc::fence_after_sync();
      const int b = t / (tw * th), rest = t % (tw * th);
      const int y0 = (rest / tw) * kTileH, x0 = (rest % tw) * kTileW;
      const size_t p = (size_t)(b * a.H + y0 + r / kTileW) * a.W + x0 + r % kTileW;
      __nv_bfloat16* out = a.y + p * a.y_stride + a.y_off + co0;
      for (int c0 = 0; c0 < gend; c0 += 8) {  // up to 64 columns in flight per wait
        uint32_t v[8][8];
        const int nc = min(8, gend - c0);
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < nc) tc::tmem_ld8_nowait(lane_base + (uint32_t)(q * nco + (c0 + c) * 8), v[c]);
        tc::tmem_wait_ld();
        if (c0 + 8 >= gend) {  // the accumulator is read: hand it back before storing
          tc::fence_before_sync();
          __syncwarp();
          if (lane == 0) tc::mbar_arrive(&acc_empty[q]);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (c >= nc) break;
          float f[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            f[e] = __uint_as_float(v[c][e]);
            if (a.bias) f[e] += a.bias[co0 + (c0 + c) * 8 + e];
            if (a.relu) f[e] = fmaxf(f[e], 0.0f);
          }
          *reinterpret_cast<uint4*>(out + (c0 + c) * 8) = pack_bf16x8(f);
        }
      }
    }
  }

  tc::fence_before_sync();
  __syncthreads();
  if (abort_flag && tid == 0) {
    atomicOr(a.err, 2u);
    // bounded drain: slices copied but not consumed, and the last MMAs issued
    for (int cc = n_issued; cc < n_loaded; ++cc)
      tc::mbar_wait(&full[cc % ring], (uint32_t)(cc / ring) & 1u, kWaitLimit);
    if (n_issued > 0)
      tc::mbar_wait(&empty[(n_issued - 1) % ring], (uint32_t)((n_issued - 1) / ring) & 1u, kWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc(tmem, ncols);
}

// TMA-fed weight gradient: CTA (run of tiles, group of taps) as in
// k_conv_wgrad_halo, with the copies made by TMA and no CTA-wide barrier
// inside the tile loop. Warp 0 (one thread) copies each tile's dY rows and
// input halo into one of `stages` stages; warp 1 (all lanes, one elected
// issuer) issues the tile's ntap x 8 MMAs (K = 16 pixels each) and frees
// the stage with a commit; at the end all four warps add the accumulators to
// dW. Both operands are MN-major (channels contiguous within a pixel row)
// in the swizzle mode of their row width, one TMA box per block of so
// output or si input channels (32, 64 or 128-byte rows):
//  * A (dY^T, M = 128 output channels, K = pixels): blocks of 128 pixel rows
//    (the 8 x 16 tile) at 256 so bytes from each other (LBO); SBO 8 rows.
//    Blocks past cout are never written: they only feed accumulator rows
//    that are never read back;
//  * B (the input halo, N = cin, K = pixels): blocks of the 10 x 18 halo at
//    slot_bytes(si) (LBO); the view of tap (dy, dx) starts (dy * 10 + dx)
//    pixel rows in, and its 8-pixel K groups are one halo row apart (SBO
//    10 rows), so no per-tap gather is needed.
constexpr int kWgTmaThreads = 128;

__global__ void __launch_bounds__(kWgTmaThreads, 1)
    k_conv_wgrad_tma(const __grid_constant__ CUtensorMap tm_dy, const __grid_constant__ CUtensorMap tm_x,
                     ConvWgradArgs a, int tpg, int tiles_per_cta, int stages, int so, int si) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kTmaMaxStages], empty[kTmaMaxStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, n_loaded, n_issued;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = a.cin, cout = a.cout, kg_n = cin >> 3;
  const int ob_n = cout / so, ib_n = cin / si;  // channel blocks loaded per tile
  const int tw = a.W / kTileW, th = a.H / kTileH, n_tiles = tw * th * a.B;
  const int t0 = blockIdx.x * tiles_per_cta, t1 = min(n_tiles, t0 + tiles_per_cta);
  const int tap0 = blockIdx.y * tpg, ntap = min(tpg, 9 - tap0);
  const uint32_t a_blk = 256u * (uint32_t)so, b_blk = slot_bytes(si);
  const uint32_t a_bytes = 128u / (uint32_t)so * a_blk, stage_bytes = a_bytes + (uint32_t)ib_n * b_blk;
  const uint32_t base = (tc::smem_u32(smem) + 1023u) & ~1023u;
  const uint32_t ncols = (uint32_t)ntap * cin <= 256u ? 256u : 512u;
  volatile int* abort_v = &abort_flag;

  if (tid == 0) {
    for (int s = 0; s < stages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(&done, 1);
    abort_flag = 0;
    n_loaded = 0;
    n_issued = 0;
  }
  if (warp == 1) tc::tmem_alloc(&tmem_base, ncols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;

  if (warp == 0 && lane == 0) {
    tc::tma_prefetch_map(&tm_dy);
    tc::tma_prefetch_map(&tm_x);
    int j = 0;
    for (int t = t0; t < t1; ++t, ++j) {
      const int s = j % stages, u = j / stages;
      if (u >= 1 && !wait_or_abort(&empty[s], (uint32_t)(u - 1) & 1u, abort_v)) break;
      const int b = t / (tw * th), rest = t % (tw * th);
      const int y0 = (rest / tw) * kTileH, x0 = (rest % tw) * kTileW;
      const uint32_t sa = base + (uint32_t)s * stage_bytes, sb = sa + a_bytes;
      tc::mbar_arrive_expect_tx(&full[s], 256u * (uint32_t)cout + (uint32_t)kHalo * 2u * (uint32_t)cin);
      for (int ob = 0; ob < ob_n; ++ob)
        tc::tma_load_5d(sa + (uint32_t)ob * a_blk, &tm_dy, &full[s], 0, ob, x0, y0, b);
      for (int ib = 0; ib < ib_n; ++ib)
        tc::tma_load_5d(sb + (uint32_t)ib * b_blk, &tm_x, &full[s], 0, ib, x0 - 1, y0 - 1, b);
    }
    n_loaded = j;
  } else if (warp == 1) {
    // the whole warp runs the issue loop; the elected lane issues
    const uint32_t idesc = tc::idesc_bf16(128, (uint32_t)cin, true, true);
    const uint32_t a_row = 2u * (uint32_t)so, b_row = 2u * (uint32_t)si;
    const uint64_t a_step = (16u * a_row) >> 4, b_step = (2u * kHaloW * b_row) >> 4;  // 16 pixels
    int j = 0;
    for (int t = t0; t < t1; ++t, ++j) {
      const int s = j % stages, u = j / stages;
      int got = 0;
      if (lane == 0) got = wait_or_abort(&full[s], (uint32_t)u & 1u, abort_v) ? 1 : 0;
      if (!__shfl_sync(0xffffffffu, got, 0)) break;
      tc::fence_after_sync();
      const uint32_t sa = base + (uint32_t)s * stage_bytes, sb = sa + a_bytes;
      const uint64_t da0 = tc::smem_desc(sa, a_blk, 8u * a_row) | ((uint64_t)umma_swizzle(so) << 61);
      const uint64_t db0 = tc::smem_desc(sb, b_blk, (uint32_t)kHaloW * b_row) | ((uint64_t)umma_swizzle(si) << 61);
      for (int q = 0; q < ntap; ++q) {
        const int tap = tap0 + q;
        uint64_t da = da0, db = db0 + (uint64_t)((((tap / 3) * kHaloW + (tap % 3)) * b_row) >> 4);
        const uint32_t d = tmem + (uint32_t)(q * cin);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk, da += a_step, db += b_step)  // K = 128 pixels, 16 per MMA
          if (tc::elect_one()) tc::mma_bf16(d, da, db, idesc, (j > 0 || kk > 0) ? 1u : 0u);
      }
      if (tc::elect_one()) tc::mma_commit(&empty[s]);
      __syncwarp();
    }
    if (j > 0 && tc::elect_one()) tc::mma_commit(&done);
    if (lane == 0) n_issued = j;
  }
  __syncwarp();
  tc::fence_before_sync();
  __syncthreads();
  const int n_tiles_cta = t1 - t0;
  bool ok = !abort_flag && n_issued == n_tiles_cta;
  if (ok && n_tiles_cta > 0) {
    int got = 0;
    if (lane == 0) got = wait_or_abort(&done, 0u, abort_v) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, got, 0) != 0;
  }
  ok = __syncthreads_and(ok);
  tc::fence_after_sync();
  if (ok && n_tiles_cta > 0) {
    const int co = warp * 32 + lane;
    for (int q = 0; q < ntap; ++q) {
      if (warp * 32 >= cout) break;  // warp-uniform: tcgen05.ld is warp-wide
      for (int cg = 0; cg < kg_n; ++cg) {
        float v[8];
        tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * cin + cg * 8), v);
        if (co < cout) {
          float4* dst = reinterpret_cast<float4*>(a.dw + ((size_t)(tap0 + q) * cout + co) * cin + cg * 8);
          atomicAdd(dst, make_float4(v[0], v[1], v[2], v[3]));
          atomicAdd(dst + 1, make_float4(v[4], v[5], v[6], v[7]));
        }
      }
    }
  } else if (!ok && tid == 0) {
    atomicOr(a.err, 2u);
    // bounded drain: copies not consumed, and the last MMAs issued
    for (int jj = n_issued; jj < n_loaded; ++jj)
      tc::mbar_wait(&full[jj % stages], (uint32_t)(jj / stages) & 1u, kWaitLimit);
    if (n_issued > 0)
      tc::mbar_wait(&empty[(n_issued - 1) % stages], (uint32_t)((n_issued - 1) / stages) & 1u, kWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc(tmem, ncols);
}

// cuTensorMapEncodeTiled, looked up through the runtime so that the library
// needs no link against the driver library.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map over BF16 rows of `stride` elements, `rank` - 1 outer
// dimensions: dims[0] channels (16 to 128 bytes, always coordinate 0), then
// dims[1..] with byte strides strides[0..]; zero fill outside.
bool encode_map(CUtensorMap* m, const void* base, int rank, const cuuint64_t* dims,
                const cuuint64_t* strides, const cuuint32_t* box,
                CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn || (reinterpret_cast<uintptr_t>(base) & 15u)) return false;
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void*>(base), dims, strides,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Activations [B][H][W][stride] seen as (gc channels, channel group, x, y,
// image) with a box of one group x box_w x box_h pixels; rows of 32, 64 or
// 128 bytes are swizzled in that mode, 16-byte rows are not.
bool map_activations(CUtensorMap* m, const __nv_bfloat16* base, int groups, int W, int H, int B, int stride,
                     int box_w, int box_h, int gc = 8) {
  const cuuint64_t row = (cuuint64_t)stride * 2u;
  const cuuint64_t dims[5] = {(cuuint64_t)gc, (cuuint64_t)groups, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t strides[4] = {(cuuint64_t)gc * 2u, row, row * W, row * W * H};
  const cuuint32_t box[5] = {(cuuint32_t)gc, 1, (cuuint32_t)box_w, (cuuint32_t)box_h, 1};
  const CUtensorMapSwizzle sw = gc == 64   ? CU_TENSOR_MAP_SWIZZLE_128B
                                : gc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                : gc == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                           : CU_TENSOR_MAP_SWIZZLE_NONE;
  return encode_map(m, base, 5, dims, strides, box, sw);
}

// TMA forward launch when the shape fits: the widest slice of output
// channels whose resident weights leave room for a ring of one tile's halo
// slices and two more, with the widest halo slice (64, 32 or 16 channels)
// that divides cin and fits.
bool try_conv_fwd_tma(const ConvFwdArgs& a, cudaStream_t st, cudaError_t* err) {
  if (a.taps == 1 || a.W % kTileW != 0 || a.H % kTileH != 0) return false;
  constexpr size_t kBudget = 227u * 1024u - 1024u;  // dynamic shared memory, minus the static part
  auto w_bytes = [&](int nco) { return ((9u * (size_t)nco * a.cin * 2u) + 1023u) & ~(size_t)1023u; };
  int nco = 0, sc = 0;
  for (int n = std::min(a.cout, 256); n >= 16 && !nco; n -= 16) {
    if (a.cout % n != 0 || (n < 32 && n != a.cout)) continue;
    for (int c : {64, 32, 16}) {
      const int np = a.cin / c;
      if (a.cin % c != 0 || np + 2 > kTmaMaxRing) continue;
      if (1024u + w_bytes(n) + (size_t)(np + 2) * slot_bytes(c) <= kBudget) {
        nco = n;
        sc = c;
        break;
      }
    }
  }
  if (!nco) return false;
  const int ring = (int)std::min<size_t>(kTmaMaxRing, (kBudget - 1024u - w_bytes(nco)) / slot_bytes(sc));
  const int accs = std::min(kTmaMaxAccs, 512 / nco);
  uint32_t ncols = 32u;
  while (ncols < (uint32_t)(accs * nco)) ncols <<= 1;
  CUtensorMap mx;
  if (!map_activations(&mx, a.x + a.x_off, a.cin / sc, a.W, a.H, a.B, a.x_stride, kHaloW, kHaloH, sc))
    return false;
  const size_t smem = 1024u + w_bytes(nco) + (size_t)ring * slot_bytes(sc);
  cudaError_t e = cudaFuncSetAttribute(k_conv_fwd_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv_fwd_tma, kTmaThreads, smem);
    per_sm = std::max(1, std::min(per_sm, (int)(512u / ncols)));  // tensor memory of resident CTAs
    const int slices = a.cout / nco;
    const int n_tiles = (a.W / kTileW) * (a.H / kTileH) * a.B;
    const int workers = std::max(1, std::min(n_tiles, sms * per_sm / slices));
    k_conv_fwd_tma<<<dim3(workers, slices), kTmaThreads, smem, st>>>(mx, a, nco, sc, ring, accs, ncols);
    e = cudaGetLastError();
  }
  *err = e;
  return true;
}

// TMA weight-gradient launch when two stages fit, with the widest channel
// blocks (64, 32 or 16) that divide cout and cin.
bool try_conv_wgrad_tma(const ConvWgradArgs& a, cudaStream_t st, cudaError_t* err) {
  if (a.taps == 1 || a.W % kTileW != 0 || a.H % kTileH != 0) return false;
  auto widest = [](int c) { return c % 64 == 0 ? 64 : (c % 32 == 0 ? 32 : 16); };
  const int so = widest(a.cout), si = widest(a.cin);
  constexpr size_t kBudget = 227u * 1024u - 1024u;
  const size_t stage = (size_t)(128 / so) * 256u * so + (size_t)(a.cin / si) * slot_bytes(si);
  const int stages = (int)std::min<size_t>(kTmaMaxStages, (kBudget - 1024u) / stage);
  if (stages < 2) return false;
  CUtensorMap mdy, mx;
  if (!map_activations(&mdy, a.dy + a.dy_off, a.cout / so, a.W, a.H, a.B, a.dy_stride, kTileW, kTileH, so) ||
      !map_activations(&mx, a.x + a.x_off, a.cin / si, a.W, a.H, a.B, a.x_stride, kHaloW, kHaloH, si))
    return false;
  const size_t smem = 1024u + (size_t)stages * stage;
  cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tpg = std::min(9, 512 / a.cin);  // taps whose accumulators fit in 512 columns
    const int groups = (9 + tpg - 1) / tpg;
    const int n_tiles = (a.W / kTileW) * (a.H / kTileH) * a.B;
    const int ctas = std::max(1, std::min(n_tiles, sms / groups));  // one CTA per SM
    const int per = (n_tiles + ctas - 1) / ctas;
    dim3 grid((n_tiles + per - 1) / per, groups);
    k_conv_wgrad_tma<<<grid, kWgTmaThreads, smem, st>>>(mdy, mx, a, tpg, per, stages, so, si);
    e = cudaGetLastError();
  }
  *err = e;
  return true;
}

}  // namespace

size_t conv_fwd_smem_bytes(int cin, int cout) {
  return 2u * (128u * cin * 2u + (size_t)cout * cin * 2u);
}
size_t conv_wgrad_smem_bytes(int cin) { return 2u * (16u * 2048u + (size_t)(cin >> 3) * 2048u); }

cudaError_t launch_conv_fwd(const ConvFwdArgs& a, cudaStream_t st) {
  if (a.cin % 16 || a.cout % 16 || a.cin < 16 || a.cout < 16 || a.cin > 256 || a.cout > 256 ||
      a.x_stride % 8 || a.x_off % 8 || a.y_stride % 8 || a.y_off % 8)
    return cudaErrorInvalidValue;
  cudaError_t tma_err = cudaSuccess;
  if (try_conv_fwd_tma(a, st, &tma_err)) return tma_err;
  const bool tiles_fit = a.taps != 1 && a.W % kTileW == 0 && a.H % kTileH == 0;
  if (tiles_fit) {
    // resident weights: the widest output-channel slice whose nine taps and
    // kFwdStages halos fit
    const size_t halo = (size_t)(a.cin >> 3) * kHalo * 16u;
    int nco = a.cout;
    while (nco >= 16 && (9u * (size_t)nco * a.cin * 2u + kFwdStages * halo > 200u * 1024u ||
                         a.cout % nco != 0 || nco % 16 != 0))
      nco -= 16;
    if ((nco >= 32 || nco == a.cout) && nco >= 16 && nco <= 128) {
      const size_t smem = 9u * (size_t)nco * a.cin * 2u + kFwdStages * halo;
      cudaError_t e = cudaFuncSetAttribute(k_conv_fwd_res, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
      int dev = 0, sms = 148, per_sm = 1;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv_fwd_res, kResThreads, smem);
      const int slices = a.cout / nco;
      const int n_tiles = (a.W / kTileW) * (a.H / kTileH) * a.B;
      const int workers = std::max(1, std::min(n_tiles, sms * std::max(1, per_sm) / slices));
      k_conv_fwd_res<<<dim3(workers, slices), kResThreads, smem, st>>>(a, nco);
      return cudaGetLastError();
    }
  }
  const size_t halo_smem = (size_t)(a.cin >> 3) * kHalo * 16u + 2u * (size_t)a.cout * a.cin * 2u;
  if (tiles_fit && halo_smem <= 200u * 1024u) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_fwd_halo,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)halo_smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.W / kTileW, a.H / kTileH, a.B);
    k_conv_fwd_halo<<<grid, kThreads, halo_smem, st>>>(a);
    return cudaGetLastError();
  }
  const size_t smem = conv_fwd_smem_bytes(a.cin, a.cout);
  if (smem > 200u * 1024u) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_conv_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int P = a.B * a.H * a.W;
  k_conv_fwd<<<(P + 127) / 128, kThreads, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_conv_wgrad(const ConvWgradArgs& a, cudaStream_t st) {
  if (a.cin % 16 || a.cout % 16 || a.cin < 16 || a.cout < 16 || a.cin > 256 || a.cout > 128 ||
      a.x_stride % 8 || a.x_off % 8 || a.dy_stride % 8 || a.dy_off % 8 || a.chunks_per_cta < 1)
    return cudaErrorInvalidValue;
  cudaError_t tma_err = cudaSuccess;
  if (try_conv_wgrad_tma(a, st, &tma_err)) return tma_err;
  const size_t halo_smem = 2u * (16u * 2048u + (size_t)(a.cin >> 3) * kHalo * 16u);
  if (a.taps != 1 && a.W % kTileW == 0 && a.H % kTileH == 0 && halo_smem <= 200u * 1024u) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad_halo,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)halo_smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tpg = std::min(9, 512 / a.cin);  // taps whose accumulators fit in 512 columns
    const int groups = (9 + tpg - 1) / tpg;
    const int n_tiles = (a.W / kTileW) * (a.H / kTileH) * a.B;
    const int ctas = std::max(1, std::min(n_tiles, sms / groups));  // one CTA per SM
    const int per = (n_tiles + ctas - 1) / ctas;
    dim3 grid((n_tiles + per - 1) / per, groups);
    k_conv_wgrad_halo<<<grid, kWgThreads, halo_smem, st>>>(a, tpg, per);
    return cudaGetLastError();
  }
  const size_t smem = conv_wgrad_smem_bytes(a.cin);
  if (smem > 200u * 1024u) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int P = a.B * a.H * a.W;
  const int n_chunks = (P + 127) / 128;
  dim3 grid((n_chunks + a.chunks_per_cta - 1) / a.chunks_per_cta, a.taps == 1 ? 1 : 9);
  k_conv_wgrad<<<grid, kThreads, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace nr
