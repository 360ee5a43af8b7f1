// sky_alias.cu — HDRI importance-sampling tables built on the GPU (see
// sky_alias.cuh).
//
// Texel weight: the largest luminance in the texel's 3x3 neighbourhood (the
// bilinear lookup spreads a bright texel into its neighbours, so their
// density must not be small) times sin(theta) of the texel row (its solid
// angle). The distribution over texels factors into a marginal over rows
// and a conditional over the columns of each row; each is an alias table
// (Walker, 1977) built with Vose's method (IEEE TSE 17(9), 1991): one warp
// per row builds that row's table, one warp builds the row table, and
// texel_pdf = weight / total. A texel is drawn as row then column.
#include "sky_alias.cuh"

#include <vector>

namespace nr {

namespace {

#define GRID_STRIDE(i, n) \
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

int blocks_for(size_t n) { return (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16); }

__global__ void k_luminance(const float* chw, int W, int H, float* lum) {
  const size_t hw = (size_t)W * H;
  GRID_STRIDE(i, hw) {
    lum[i] = fmaxf(0.0f, 0.2126f * chw[i] + 0.7152f * chw[hw + i] + 0.0722f * chw[2 * hw + i]);
  }
}

__global__ void k_weights(const float* lum, int W, int H, float* w) {
  const size_t hw = (size_t)W * H;
  GRID_STRIDE(i, hw) {
    const int y = (int)(i / W), x = (int)(i % W);
    float m = 0.0f;
    for (int dy = -1; dy <= 1; ++dy) {
      const int yy = min(H - 1, max(0, y + dy));
      for (int dx = -1; dx <= 1; ++dx) m = fmaxf(m, lum[(size_t)yy * W + (x + W + dx) % W]);
    }
    w[i] = m * sinf(3.14159265358979f * ((float)y + 0.5f) / (float)H);
  }
}

// Vose's method over n weights w[0..n) (sum > 0) by one warp: q = w * n /
// sum and the small / large stacks (in index order) are built by all lanes,
// then lane 0 pairs them: each small entry takes its deficit from the large
// entry on top of the large stack. q, small and large are scratch of n
// entries.
__device__ void vose_warp(const float* w, uint32_t n, double sum, float* prob, uint32_t* alias,
                          float* q, uint32_t* small, uint32_t* large) {
  const uint32_t lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
  uint32_t ns = 0, nl = 0;  // the same in every lane
  for (uint32_t b = 0; b < n; b += 32) {
    const uint32_t i = b + lane;
    const bool valid = i < n;
    float qi = 0.0f;
    if (valid) {
      qi = (float)((double)w[i] * (double)n / sum);
      q[i] = qi;
      prob[i] = 1.0f;
      alias[i] = i;
    }
    const bool is_small = valid && qi < 1.0f, is_large = valid && !(qi < 1.0f);
    const uint32_t ms = __ballot_sync(0xffffffffu, is_small), ml = __ballot_sync(0xffffffffu, is_large);
    if (is_small) small[ns + __popc(ms & below)] = i;
    if (is_large) large[nl + __popc(ml & below)] = i;
    ns += (uint32_t)__popc(ms);
    nl += (uint32_t)__popc(ml);
  }
  __syncwarp();
  if (lane == 0) {
    while (ns > 0 && nl > 0) {
      const uint32_t l = small[--ns], g = large[nl - 1];
      prob[l] = q[l];
      alias[l] = g;
      q[g] = (q[g] + q[l]) - 1.0f;
      if (q[g] < 1.0f) {
        --nl;
        small[ns++] = g;
      }
    }
    // entries left in either stack keep prob 1 (round-off leftovers)
  }
  __syncwarp();
}

// Sum of w[0..n) in double by one warp (the same value in every lane).
__device__ double warp_sum(const float* w, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31u;
  double s = 0.0;
  for (uint32_t x = lane; x < n; x += 32) s += (double)w[x];
  for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  return s;
}

// One warp per row: the row's weight sum and its column table.
__global__ void k_row_tables(const float* w, int W, int H, double* row_sum, float* col_prob,
                             uint32_t* col_alias, float* q, uint32_t* small, uint32_t* large) {
  const int y = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (y >= H) return;  // the whole warp
  const uint32_t lane = threadIdx.x & 31u;
  const size_t o = (size_t)y * W;
  const double s = warp_sum(w + o, (uint32_t)W);
  if (lane == 0) row_sum[y] = s;
  if (s > 0.0) {
    vose_warp(w + o, (uint32_t)W, s, col_prob + o, col_alias + o, q + o, small + o, large + o);
  } else {
    for (int x = (int)lane; x < W; x += 32) {
      col_prob[o + x] = 1.0f;
      col_alias[o + x] = (uint32_t)x;
    }
  }
}

// One warp: the total, and the row table over the row sums.
__global__ void k_marginal(const double* row_sum, int H, float* row_w, double* total, float* row_prob,
                           uint32_t* row_alias, float* q, uint32_t* small, uint32_t* large) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const uint32_t lane = threadIdx.x;
  double s = 0.0;
  for (int y = (int)lane; y < H; y += 32) {
    s += row_sum[y];
    row_w[y] = (float)row_sum[y];
  }
  for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  if (lane == 0) *total = s;
  __syncwarp();
  if (s > 0.0) vose_warp(row_w, (uint32_t)H, s, row_prob, row_alias, q, small, large);
}

__global__ void k_texel_pdf(const float* w, size_t n, const double* total, float* pdf) {
  const double t = *total;
  GRID_STRIDE(i, n) { pdf[i] = t > 0.0 ? (float)((double)w[i] / t) : 0.0f; }
}

}  // namespace

void SkyTables::release() {
  cudaFree(row_prob);
  cudaFree(row_alias);
  cudaFree(col_prob);
  cudaFree(col_alias);
  cudaFree(texel_pdf);
  *this = SkyTables{};
}

cudaError_t build_sky_tables(const float* chw, int W, int H, SkyTables& t, bool& has_energy,
                             cudaStream_t st) {
  t.release();
  has_energy = false;
  const size_t hw = (size_t)W * H;
  cudaError_t e = cudaSuccess;
  auto al = [&](auto*& p, size_t n) {
    if (e == cudaSuccess) e = cudaMalloc(&p, n * sizeof(*p));
  };
  al(t.row_prob, H);
  al(t.row_alias, H);
  al(t.col_prob, hw);
  al(t.col_alias, hw);
  al(t.texel_pdf, hw);
  float *lum = nullptr, *w = nullptr, *q = nullptr, *row_w = nullptr;
  uint32_t *small = nullptr, *large = nullptr;
  double *row_sum = nullptr, *total = nullptr;
  al(lum, hw);
  al(w, hw);
  al(q, hw);
  al(small, hw);
  al(large, hw);
  al(row_sum, H);
  al(row_w, H);
  al(total, 1);
  if (e == cudaSuccess) {
    k_luminance<<<blocks_for(hw), 256, 0, st>>>(chw, W, H, lum);
    k_weights<<<blocks_for(hw), 256, 0, st>>>(lum, W, H, w);
    k_row_tables<<<(H + 3) / 4, 128, 0, st>>>(w, W, H, row_sum, t.col_prob, t.col_alias, q, small,
                                             large);
    // the row table reuses the head of the scratch arrays
    k_marginal<<<1, 32, 0, st>>>(row_sum, H, row_w, total, t.row_prob, t.row_alias, q, small, large);
    k_texel_pdf<<<blocks_for(hw), 256, 0, st>>>(w, hw, total, t.texel_pdf);
    e = cudaGetLastError();
  }
  double h_total = 0.0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_total, total, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  for (void* p : {(void*)lum, (void*)w, (void*)q, (void*)small, (void*)large, (void*)row_sum,
                  (void*)row_w, (void*)total})
    cudaFree(p);
  if (e != cudaSuccess) {
    t.release();
    return e;
  }
  has_energy = h_total > 0.0;
  t.W = W;
  t.H = H;
  return cudaSuccess;
}

}  // namespace nr
