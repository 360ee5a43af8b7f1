// nrc.cu — neural radiance cache (see nrc.cuh).
//
// Input vector (64 BF16 channels): [0, 32) hash-grid features (16 levels x 2),
// [32, 48) real spherical harmonics of degree 0-3 of the outgoing direction,
// [48, 51) normal * 0.5 + 0.5, [51] roughness, [52, 55) diffuse albedo, zero
// padding. MLP: four hidden layers 64 -> 64 (ReLU), then 64 -> 16 (linear;
// the first three outputs are the radiance), no biases. Loss: relative squared error
// (o - t)^2 / (o^2 + 0.01) with o held constant in the denominator.
#include "nrc.cuh"

#include <cmath>
#include <random>
#include <vector>

#include "conv_tc.cuh"

namespace nr {

namespace {

constexpr int kLevels = 16, kFeat = 2, kLog2T = 19;
constexpr uint32_t kT = 1u << kLog2T;
constexpr int kWidth = 64, kOutCh = 16;
constexpr int kHidden = 4, kLayers = kHidden + 1;
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

__global__ void k_encode(GridGeo g, const NrcQuery* qs, const float* grid, __nv_bfloat16* x,
                         uint32_t n) {
  GRID_STRIDE(i, n) {
    const NrcQuery q = qs[i];
    __nv_bfloat16* row = x + i * kWidth;
    float u[3];
    unit_pos(g, q, u);
    for (int l = 0; l < kLevels; ++l) {
      float f0 = 0.0f, f1 = 0.0f;
      const float* lv = grid + (size_t)l * kT * kFeat;
      corners(g, l, u, [&](uint32_t idx, float w) {
        f0 += w * lv[idx * kFeat];
        f1 += w * lv[idx * kFeat + 1];
      });
      row[2 * l] = __float2bfloat16(f0);
      row[2 * l + 1] = __float2bfloat16(f1);
    }
    float s[16];
    sh16(q.b.x, q.b.y, q.b.z, s);
    for (int k = 0; k < 16; ++k) row[32 + k] = __float2bfloat16(s[k]);
    row[48] = __float2bfloat16(q.c.x * 0.5f + 0.5f);
    row[49] = __float2bfloat16(q.c.y * 0.5f + 0.5f);
    row[50] = __float2bfloat16(q.c.z * 0.5f + 0.5f);
    row[51] = __float2bfloat16(q.a.w);
    row[52] = __float2bfloat16(q.d.x);
    row[53] = __float2bfloat16(q.d.y);
    row[54] = __float2bfloat16(q.d.z);
    for (int k = 55; k < kWidth; ++k) row[k] = __float2bfloat16(0.0f);
  }
}

// gradient of the loss with respect to the grid values: the adjoint of the
// trilinear interpolation, scattered with atomics
__global__ void k_encode_bwd(GridGeo g, const NrcQuery* qs, const __nv_bfloat16* dx, float* ggrid,
                             uint32_t n) {
  GRID_STRIDE(i, n) {
    const NrcQuery q = qs[i];
    const __nv_bfloat16* row = dx + i * kWidth;
    float u[3];
    unit_pos(g, q, u);
    for (int l = 0; l < kLevels; ++l) {
      const float d0 = __bfloat162float(row[2 * l]), d1 = __bfloat162float(row[2 * l + 1]);
      if (d0 == 0.0f && d1 == 0.0f) continue;
      float* lv = ggrid + (size_t)l * kT * kFeat;
      corners(g, l, u, [&](uint32_t idx, float w) {
        atomicAdd(lv + idx * kFeat, w * d0);
        atomicAdd(lv + idx * kFeat + 1, w * d1);
      });
    }
  }
}

__global__ void k_output(const __nv_bfloat16* o, float* out, uint32_t n) {
  GRID_STRIDE(i, n) {
    for (int c = 0; c < 3; ++c) out[i * 3 + c] = fmaxf(__bfloat162float(o[i * kOutCh + c]), 0.0f);
  }
}

__global__ void k_loss(const __nv_bfloat16* o, const float* target, __nv_bfloat16* d_o, uint32_t n,
                       double* loss) {
  double local = 0.0;
  GRID_STRIDE(i, n) {
    for (int c = 0; c < kOutCh; ++c) {
      float g = 0.0f;
      if (c < 3) {
        const float oc = __bfloat162float(o[i * kOutCh + c]);
        const float t = target[i * 3 + c];
        const float den = oc * oc + 0.01f;
        const float d = oc - t;
        local += (double)(d * d / den);
        g = 2.0f * d / den;
      }
      d_o[i * kOutCh + c] = __float2bfloat16(g);
    }
  }
  for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, local);
}

__global__ void k_mask(__nv_bfloat16* d, const __nv_bfloat16* h, size_t n) {
  GRID_STRIDE(i, n) {
    if (!(__bfloat162float(h[i]) > 0.0f)) d[i] = __float2bfloat16(0.0f);
  }
}

__global__ void k_adam(float* w, float* m, float* v, const float* g, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  GRID_STRIDE(i, n) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
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

// BF16 forward [out][in] and transposed [in][out] copies of a layer
__global__ void k_pack(const float* w, __nv_bfloat16* wf, __nv_bfloat16* wt, int nout, int nin) {
  const size_t n = (size_t)nout * nin;
  GRID_STRIDE(i, n) {
    const int in = (int)(i % nin), out = (int)(i / nin);
    const __nv_bfloat16 b = __float2bfloat16(w[i]);
    wf[i] = b;
    wt[(size_t)in * nout + out] = b;
  }
}

}  // namespace

struct NrcNet {
  uint32_t max_q = 0;
  GridGeo geo{};
  int nout[kLayers] = {kWidth, kWidth, kWidth, kWidth, kOutCh};
  float *w[kLayers], *mw[kLayers], *vw[kLayers], *gw[kLayers];
  __nv_bfloat16 *wf[kLayers], *wt[kLayers];
  float *grid, *mg, *vg, *gg;
  __nv_bfloat16 *x0, *h[kHidden], *o, *d_o, *dh, *dz;
  double* d_loss = nullptr;
  uint32_t* d_err = nullptr;
  std::vector<void*> allocs;
  int step = 0;
  uint32_t last_count = 0;
  bool gg_clear = false;  // the grid gradient table is all zero
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

// y[q, :nout] = act(W x[q, :nin]) as a one-tap tcgen05 convolution over a
// 1 x count "image"
cudaError_t gemm(NrcNet& n, const __nv_bfloat16* x, int nin, const __nv_bfloat16* w, __nv_bfloat16* y,
                 int nout, uint32_t count, bool relu, cudaStream_t st) {
  ConvFwdArgs a{x, nin, 0, w, nullptr, y, nout, 0, nin, nout, 1, 1, (int32_t)count,
                relu ? 1 : 0, n.d_err, 1};
  return launch_conv_fwd(a, st);
}

// dw[nout][nin] += dy^T x over the queries
cudaError_t gemm_wgrad(NrcNet& n, const __nv_bfloat16* dy, int nout, const __nv_bfloat16* x, int nin,
                       float* dw, uint32_t count, cudaStream_t st) {
  const int chunks = (int)((count + 127) / 128);
  const int per = std::max(1, (chunks + 295) / 296);
  ConvWgradArgs a{dy, nout, 0, x, nin, 0, dw, nin, nout, 1, 1, (int32_t)count, per, n.d_err, 1};
  return launch_conv_wgrad(a, st);
}

cudaError_t forward(NrcNet& n, const NrcQuery* q, uint32_t count, cudaStream_t st) {
  k_encode<<<blocks_for(count), 256, 0, st>>>(n.geo, q, n.grid, n.x0, count);
  cudaError_t e;
  const __nv_bfloat16* in = n.x0;
  for (int l = 0; l < kHidden; ++l) {
    if ((e = gemm(n, in, kWidth, n.wf[l], n.h[l], kWidth, count, true, st))) return e;
    in = n.h[l];
  }
  if ((e = gemm(n, in, kWidth, n.wf[kHidden], n.o, kOutCh, count, false, st))) return e;
  return cudaGetLastError();
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
    AL(n.wt[l], k);
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / kWidth));
    host.resize(k);
    for (auto& v : host) v = nd(rng);
    cudaMemcpy(n.w[l], host.data(), k * 4, cudaMemcpyHostToDevice);
    cudaMemset(n.mw[l], 0, k * 4);
    cudaMemset(n.vw[l], 0, k * 4);
    k_pack<<<blocks_for(k), 256>>>(n.w[l], n.wf[l], n.wt[l], n.nout[l], kWidth);
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
  const size_t q = max_queries;
  AL(n.x0, q * kWidth);
  for (int l = 0; l < kHidden; ++l) AL(n.h[l], q * kWidth);
  AL(n.o, q * kOutCh);
  AL(n.d_o, q * kOutCh);
  AL(n.dh, q * kWidth);
  AL(n.dz, q * kWidth);
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
  cudaError_t e = forward(n, q, count, st);
  if (e != cudaSuccess) return cuda_msg(e, "nrc forward");
  k_output<<<blocks_for(count), 256, 0, st>>>(n.o, out, count);
  e = cudaGetLastError();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "nrc output");
}

std::string nrc_train(Nrc& c, const NrcQuery* q, const float* target, uint32_t count, float lr,
                      double* loss, cudaStream_t st) {
  if (!c.net) return "nrc: not created";
  NrcNet& n = *c.net;
  if (count > n.max_q) return "nrc: more queries than the cache was created for";
  if (count == 0) return {};
  for (int l = 0; l < kLayers; ++l) cudaMemsetAsync(n.gw[l], 0, (size_t)n.nout[l] * kWidth * 4, st);
  const size_t ng = (size_t)kLevels * kT * kFeat;
  if (!n.gg_clear) cudaMemsetAsync(n.gg, 0, ng * 4, st);
  n.gg_clear = false;
  cudaMemsetAsync(n.d_loss, 0, sizeof(double), st);
  cudaError_t e = forward(n, q, count, st);
  if (e != cudaSuccess) return cuda_msg(e, "nrc forward");
  k_loss<<<blocks_for(count), 256, 0, st>>>(n.o, target, n.d_o, count, n.d_loss);
  // output layer
  if ((e = gemm_wgrad(n, n.d_o, kOutCh, n.h[kHidden - 1], kWidth, n.gw[kHidden], count, st)))
    return cuda_msg(e, "nrc");
  if ((e = gemm(n, n.d_o, kOutCh, n.wt[kHidden], n.dh, kWidth, count, false, st)))
    return cuda_msg(e, "nrc");
  // hidden layers, last to first: dz = dh * (h > 0)
  for (int l = kHidden - 1; l >= 0; --l) {
    k_mask<<<blocks_for((size_t)count * kWidth), 256, 0, st>>>(n.dh, n.h[l], (size_t)count * kWidth);
    const __nv_bfloat16* in = l > 0 ? n.h[l - 1] : n.x0;
    if ((e = gemm_wgrad(n, n.dh, kWidth, in, kWidth, n.gw[l], count, st))) return cuda_msg(e, "nrc");
    if ((e = gemm(n, n.dh, kWidth, n.wt[l], n.dz, kWidth, count, false, st))) return cuda_msg(e, "nrc");
    std::swap(n.dh, n.dz);
  }
  // n.dh now holds the gradient with respect to the encoded input
  k_encode_bwd<<<blocks_for(count), 256, 0, st>>>(n.geo, q, n.dh, n.gg, count);
  n.last_count = count;
  if (lr > 0.0f) {
    n.step++;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-10f;
    const float c1 = 1.0f - std::pow(b1, (float)n.step), c2 = 1.0f - std::pow(b2, (float)n.step);
    for (int l = 0; l < kLayers; ++l) {
      const size_t k = (size_t)n.nout[l] * kWidth;
      k_adam<<<blocks_for(k), 256, 0, st>>>(n.w[l], n.mw[l], n.vw[l], n.gw[l], k, lr, b1, b2, eps, c1, c2);
      k_pack<<<blocks_for(k), 256, 0, st>>>(n.w[l], n.wf[l], n.wt[l], n.nout[l], kWidth);
    }
    static_assert((kLevels * kT * kFeat) % 4 == 0, "grid table in float4 units");
    k_adam_grid<<<blocks_for(ng / 4), 256, 0, st>>>(n.grid, n.mg, n.vg,
                                                    reinterpret_cast<float4*>(n.gg), ng / 4, lr,
                                                    b1, b2, eps, c1, c2);
    n.gg_clear = true;
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
      k_pack<<<blocks_for(k), 256>>>(n.w[l], n.wf[l], n.wt[l], n.nout[l], kWidth);
      mlp += k;
    }
  if (grid) cudaMemcpy(n.grid, grid, (size_t)kLevels * kT * kFeat * 4, cudaMemcpyHostToDevice);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "nrc write");
}

}  // namespace nr
