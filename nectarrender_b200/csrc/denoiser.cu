// denoiser.cu — the U-Net denoiser of denoiser.cuh: activations in NHWC
// BF16, convolutions on the tcgen05 tensor cores (conv_tc.cu), everything
// else in small elementwise kernels here; FP32 master weights and Adam.
#include "denoiser.cuh"

#include <algorithm>
#include <cmath>
#include <random>

#include "conv_tc.cuh"

namespace nr {

namespace {

constexpr int kLevels = 5;
constexpr int kEnc[kLevels] = {32, 48, 64, 96, 128};
constexpr int kIn = 16;
constexpr int kOut = 16;

// A channel range of an NHWC tensor: pixel p, channel c at p * stride + off + c.
struct View {
  __nv_bfloat16* p;
  int stride, off, ch;
};

__device__ __forceinline__ float ld(const View& v, size_t pix, int c) {
  return __bfloat162float(v.p[pix * v.stride + v.off + c]);
}
__device__ __forceinline__ void st(const View& v, size_t pix, int c, float x) {
  v.p[pix * v.stride + v.off + c] = __float2bfloat16(x);
}

#define GRID_STRIDE(i, n) \
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

int blocks_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

// Network input: log(1 + beauty), diffuse, normal, log(1 + depth), zero
// padding to 16.
__global__ void k_prep(const float* beauty, const float* diffuse, const float* normal,
                       const float* depth, View out, int B, int H, int W) {
  const size_t hw = (size_t)H * W, P = (size_t)B * hw;
  GRID_STRIDE(p, P) {
    const size_t b = p / hw, i = p - b * hw;
    const size_t base = b * 3 * hw + i;
    for (int c = 0; c < 3; ++c) {
      st(out, p, c, log1pf(fmaxf(beauty[base + c * hw], 0.0f)));
      st(out, p, 3 + c, diffuse ? diffuse[base + c * hw] : 0.0f);
      st(out, p, 6 + c, normal ? normal[base + c * hw] : 0.0f);
    }
    st(out, p, 9, depth ? log1pf(fmaxf(depth[b * hw + i], 0.0f)) : 0.0f);
    for (int c = 10; c < out.ch; ++c) st(out, p, c, 0.0f);
  }
}

// The prediction is residual in log space: pred = log(1 + noisy beauty) +
// the network's first three output channels, so an untrained network (small
// output layer) starts near the identity and a clean input needs only a small
// correction. Loss (per channel, d = pred - log(1 + target)): absolute error
// |d| (kind 1, the default), gradient sign(d); or squared error 0.5 d^2
// (kind 0), gradient d. Adam is invariant to the gradient scale, so the 1/N
// of the mean is left out. The absolute error estimates the conditional
// median of the targets, the squared error their mean (the two part where
// the targets themselves still carry heavy-tailed noise).
__device__ __forceinline__ float log_beauty(const float* beauty, size_t b, size_t hw, int c,
                                            size_t i) {
  return log1pf(fmaxf(beauty[b * 3 * hw + c * hw + i], 0.0f));
}

__global__ void k_loss(View out, const float* beauty, const float* target, View dout, int B, int H,
                       int W, int kind, double* loss) {
  const size_t hw = (size_t)H * W, P = (size_t)B * hw;
  double local = 0.0;
  GRID_STRIDE(p, P) {
    const size_t b = p / hw, i = p - b * hw;
    for (int c = 0; c < 3; ++c) {
      const float t = log_beauty(target, b, hw, c, i);
      const float d = (log_beauty(beauty, b, hw, c, i) + ld(out, p, c)) - t;
      if (kind == 1) {
        local += fabs((double)d);
        st(dout, p, c, d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f));
      } else {
        local += 0.5 * (double)d * (double)d;
        st(dout, p, c, d);
      }
    }
    for (int c = 3; c < dout.ch; ++c) st(dout, p, c, 0.0f);
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, local);
}

// Output: exp(pred) - 1, planar CHW (res may be beauty: each element is read
// before it is written, by the same thread).
__global__ void k_output(View out, const float* beauty, float* res, int B, int H, int W) {
  const size_t hw = (size_t)H * W, P = (size_t)B * hw;
  GRID_STRIDE(p, P) {
    const size_t b = p / hw, i = p - b * hw;
    for (int c = 0; c < 3; ++c)
      res[b * 3 * hw + c * hw + i] =
          fmaxf(expm1f(log_beauty(beauty, b, hw, c, i) + ld(out, p, c)), 0.0f);
  }
}

// 2x2 average pooling (h, w: output size) and its adjoint.
__global__ void k_pool(View in, View out, int B, int h, int w) {
  const size_t n = (size_t)B * h * w * out.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % out.ch);
    const size_t q = i / out.ch;
    const int x = (int)(q % w), y = (int)((q / w) % h), b = (int)(q / ((size_t)w * h));
    const size_t W2 = 2 * (size_t)w, r0 = ((size_t)b * 2 * h + 2 * y) * W2 + 2 * x;
    float s = ld(in, r0, c) + ld(in, r0 + 1, c) + ld(in, r0 + W2, c) + ld(in, r0 + W2 + 1, c);
    st(out, q, c, 0.25f * s);
  }
}
__global__ void k_pool_bwd(View dout, View din, int B, int h, int w) {  // din at 2h x 2w
  const size_t n = (size_t)B * 4 * h * w * din.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % din.ch);
    const size_t q = i / din.ch;
    const int W2 = 2 * w, x = (int)(q % W2), y = (int)((q / W2) % (2 * h));
    const int b = (int)(q / ((size_t)W2 * 2 * h));
    const size_t s = ((size_t)b * h + y / 2) * w + x / 2;
    st(din, q, c, 0.25f * ld(dout, s, c));
  }
}
// nearest 2x upsampling (h, w: input size) and its adjoint
__global__ void k_up(View in, View out, int B, int h, int w) {
  const size_t n = (size_t)B * 4 * h * w * out.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % out.ch);
    const size_t q = i / out.ch;
    const int W2 = 2 * w, x = (int)(q % W2), y = (int)((q / W2) % (2 * h));
    const int b = (int)(q / ((size_t)W2 * 2 * h));
    st(out, q, c, ld(in, ((size_t)b * h + y / 2) * w + x / 2, c));
  }
}
__global__ void k_up_bwd(View dout, View din, int B, int h, int w) {  // din at h x w
  const size_t n = (size_t)B * h * w * din.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % din.ch);
    const size_t q = i / din.ch;
    const int x = (int)(q % w), y = (int)((q / w) % h), b = (int)(q / ((size_t)w * h));
    const size_t W2 = 2 * (size_t)w, r0 = ((size_t)b * 2 * h + 2 * y) * W2 + 2 * x;
    float s = ld(dout, r0, c) + ld(dout, r0 + 1, c) + ld(dout, r0 + W2, c) + ld(dout, r0 + W2 + 1, c);
    st(din, q, c, s);
  }
}
// g = dy * (y > 0): gradient through ReLU (y is the post-activation output)
__global__ void k_relu_bwd(View dy, View y, View g, size_t P) {
  const size_t n = P * g.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % g.ch);
    const size_t q = i / g.ch;
    st(g, q, c, ld(y, q, c) > 0.0f ? ld(dy, q, c) : 0.0f);
  }
}
__global__ void k_copy(View src, View dst, size_t P) {
  const size_t n = P * dst.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % dst.ch);
    const size_t q = i / dst.ch;
    st(dst, q, c, ld(src, q, c));
  }
}
__global__ void k_add(View acc, View b, size_t P) {
  const size_t n = P * acc.ch;
  GRID_STRIDE(i, n) {
    const int c = (int)(i % acc.ch);
    const size_t q = i / acc.ch;
    st(acc, q, c, ld(acc, q, c) + ld(b, q, c));
  }
}
// db[c] += sum_p g[p, c]
__global__ void k_bias_grad(View g, float* db, size_t P) {
  const int c = blockIdx.y;
  float s = 0.0f;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < P; q += (size_t)gridDim.x * blockDim.x)
    s += ld(g, q, c);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(db + c, s);
}
// Adam (Kingma & Ba 2015) on FP32 master values
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
// BF16 copies of the master weights: forward [9][co][ci] and the rotated,
// transposed backward-data layout [9][ci][co] with tap t <- 8 - t.
__global__ void k_pack(const float* w, __nv_bfloat16* wf, __nv_bfloat16* wbd, int cin, int cout) {
  const size_t n = (size_t)9 * cin * cout;
  GRID_STRIDE(i, n) {
    const int ci = (int)(i % cin), co = (int)((i / cin) % cout), t = (int)(i / ((size_t)cin * cout));
    const __nv_bfloat16 b = __float2bfloat16(w[i]);
    wf[i] = b;
    wbd[((size_t)(8 - t) * cin + ci) * cout + co] = b;
  }
}

}  // namespace

struct Layer {
  int cin, cout;
  bool relu;
  float *w, *b, *mw, *vw, *mb, *vb, *gw, *gb;  // FP32 master, Adam moments, gradients
  __nv_bfloat16 *wf, *wbd;
};

struct Tensor {
  __nv_bfloat16* p = nullptr;
  int ch = 0;
  View v(int off = 0, int n = -1) const { return View{p, ch, off, n < 0 ? ch - off : n}; }
};

struct DenoiserNet {
  uint32_t max_pixels = 0;
  std::vector<Layer> layers;
  // activations (level l has max_pixels >> 2l pixels)
  Tensor x[kLevels], ea[kLevels], eb4, cat[kLevels - 1], da[kLevels - 1], db[kLevels - 1], out;
  // gradients
  Tensor g_out, gtmp[kLevels], dcat[kLevels - 1], dea[kLevels], deb[kLevels], ddb[kLevels],
      dda[kLevels - 1], dx[kLevels];
  float* d_params = nullptr;  // one allocation for all FP32 parameter arrays
  __nv_bfloat16* d_wbf = nullptr;
  double* d_loss = nullptr;
  uint32_t* d_err = nullptr;
  std::vector<void*> allocs;
  int step = 0;
  int B = 0, H = 0, W = 0;  // shape of the last forward
  int loss_kind = 1;        // 1: absolute error, 0: squared error (log space)
};

Denoiser::~Denoiser() {
  if (!net) return;
  for (void* p : net->allocs) cudaFree(p);
  delete net;
  net = nullptr;
}

namespace {

// layer indices
enum {
  L_E0A = 0, L_E0B, L_E1A, L_E1B, L_E2A, L_E2B, L_E3A, L_E3B, L_E4A, L_E4B,
  L_D3A, L_D3B, L_D2A, L_D2B, L_D1A, L_D1B, L_D0A, L_D0B, L_OUT, L_COUNT
};

cudaError_t alloc_tensor(DenoiserNet& n, Tensor& t, size_t pixels, int ch) {
  t.ch = ch;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, pixels * ch * sizeof(__nv_bfloat16));
  if (e != cudaSuccess) return e;
  n.allocs.push_back(p);
  t.p = static_cast<__nv_bfloat16*>(p);
  return cudaSuccess;
}

std::string cuda_msg(cudaError_t e, const char* what) {
  return std::string(what) + ": " + cudaGetErrorString(e);
}

cudaError_t conv(DenoiserNet& n, const Layer& L, View x, View y, const __nv_bfloat16* w,
                 const float* bias, bool relu, int B, int h, int w_, cudaStream_t st) {
  ConvFwdArgs a{x.p, x.stride, x.off, w, bias, y.p, y.stride, y.off,
                x.ch, y.ch, B, h, w_, relu ? 1 : 0, n.d_err};
  (void)L;
  return launch_conv_fwd(a, st);
}

cudaError_t wgrad(DenoiserNet& n, Layer& L, View g, View x, int B, int h, int w, cudaStream_t st) {
  const int P = B * h * w;
  const int chunks = (P + 127) / 128;
  const int per = std::max(1, (chunks * 9 + 295) / 296);
  ConvWgradArgs a{g.p, g.stride, g.off, x.p, x.stride, x.off, L.gw, L.cin, L.cout, B, h, w, per,
                  n.d_err};
  cudaError_t e = launch_conv_wgrad(a, st);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)std::min(64, std::max(1, P / 1024)), (unsigned)L.cout);
  k_bias_grad<<<grid, 256, 0, st>>>(g, L.gb, (size_t)P);
  return cudaGetLastError();
}

}  // namespace

std::string denoiser_create(Denoiser& d, uint32_t max_pixels, uint32_t seed) {
  if (max_pixels < 256 || max_pixels % 256) return "denoiser: max_pixels must be a positive multiple of 256";
  d.net = new DenoiserNet();
  DenoiserNet& n = *d.net;
  n.max_pixels = max_pixels;
  auto add = [&](int cin, int cout, bool relu) { n.layers.push_back(Layer{cin, cout, relu}); };
  add(kIn, kEnc[0], true);
  add(kEnc[0], kEnc[0], true);
  for (int l = 1; l < kLevels; ++l) {
    add(kEnc[l - 1], kEnc[l], true);
    add(kEnc[l], kEnc[l], true);
  }
  for (int l = kLevels - 2; l >= 0; --l) {
    add(kEnc[l + 1] + kEnc[l], kEnc[l], true);
    add(kEnc[l], kEnc[l], true);
  }
  add(kEnc[0], kOut, false);
  // parameters
  size_t nw = 0, nb = 0;
  for (auto& L : n.layers) {
    nw += (size_t)9 * L.cin * L.cout;
    nb += L.cout;
  }
  const size_t total = 4 * (nw + nb) + 0;  // w,m,v,g for weights and biases
  cudaError_t e = cudaMalloc(&n.d_params, total * sizeof(float));
  if (e != cudaSuccess) return cuda_msg(e, "denoiser parameters");
  n.allocs.push_back(n.d_params);
  e = cudaMemset(n.d_params, 0, total * sizeof(float));
  if (e != cudaSuccess) return cuda_msg(e, "denoiser parameters");
  e = cudaMalloc(&n.d_wbf, 2 * nw * sizeof(__nv_bfloat16));
  if (e != cudaSuccess) return cuda_msg(e, "denoiser weights");
  n.allocs.push_back(n.d_wbf);
  float* p = n.d_params;
  __nv_bfloat16* q = n.d_wbf;
  std::mt19937 rng(seed);
  std::vector<float> host;
  for (auto& L : n.layers) {
    const size_t k = (size_t)9 * L.cin * L.cout;
    L.w = p; p += k;
    L.mw = p; p += k;
    L.vw = p; p += k;
    L.gw = p; p += k;
    L.b = p; p += L.cout;
    L.mb = p; p += L.cout;
    L.vb = p; p += L.cout;
    L.gb = p; p += L.cout;
    L.wf = q; q += k;
    L.wbd = q; q += k;
    // He initialisation for ReLU layers; small output layer
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * L.cin)) * (L.relu ? 1.0f : 0.1f));
    host.resize(k);
    for (auto& v : host) v = nd(rng);
    e = cudaMemcpy(L.w, host.data(), k * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_msg(e, "denoiser init");
    k_pack<<<blocks_for(k), 256>>>(L.w, L.wf, L.wbd, L.cin, L.cout);
  }
  // activations and gradients
  const size_t P0 = max_pixels;
  auto lv = [&](int l) { return P0 >> (2 * l); };
#define AT(t, px, ch)                                           \
  if ((e = alloc_tensor(n, t, px, ch)) != cudaSuccess) return cuda_msg(e, "denoiser buffers");
  AT(n.x[0], P0, kIn);
  for (int l = 0; l < kLevels; ++l) {
    if (l > 0) AT(n.x[l], lv(l), kEnc[l - 1]);
    AT(n.ea[l], lv(l), kEnc[l]);
    AT(n.gtmp[l], lv(l), std::max(kEnc[l], kOut));
    AT(n.dea[l], lv(l), kEnc[l]);
    AT(n.deb[l], lv(l), kEnc[l]);
    AT(n.ddb[l], lv(l), kEnc[l]);
    AT(n.dx[l], lv(l), l == 0 ? kIn : kEnc[l - 1]);
  }
  AT(n.eb4, lv(4), kEnc[4]);
  for (int l = 0; l < kLevels - 1; ++l) {
    AT(n.cat[l], lv(l), kEnc[l + 1] + kEnc[l]);
    AT(n.dcat[l], lv(l), kEnc[l + 1] + kEnc[l]);
    AT(n.da[l], lv(l), kEnc[l]);
    AT(n.db[l], lv(l), kEnc[l]);
    AT(n.dda[l], lv(l), kEnc[l]);
  }
  AT(n.out, P0, kOut);
  AT(n.g_out, P0, kOut);
#undef AT
  e = cudaMalloc(&n.d_loss, sizeof(double));
  if (e != cudaSuccess) return cuda_msg(e, "denoiser loss");
  n.allocs.push_back(n.d_loss);
  e = cudaMalloc(&n.d_err, sizeof(uint32_t));
  if (e != cudaSuccess) return cuda_msg(e, "denoiser error word");
  n.allocs.push_back(n.d_err);
  cudaMemset(n.d_err, 0, 4);
  e = cudaDeviceSynchronize();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "denoiser init");
}

namespace {

std::string check_shape(const DenoiserNet& n, int B, int H, int W) {
  if (B < 1 || H < 16 || W < 16 || H % 16 || W % 16)
    return "denoiser: H and W must be multiples of 16";
  if ((size_t)B * H * W > n.max_pixels) return "denoiser: batch exceeds the pixels it was created for";
  return {};
}

cudaError_t forward(DenoiserNet& n, const float* beauty, const float* diffuse, const float* normal,
                    const float* depth, int B, int H, int W, cudaStream_t st) {
  auto& Ls = n.layers;
  cudaError_t e;
  const size_t P0 = (size_t)B * H * W;
  k_prep<<<blocks_for(P0), 256, 0, st>>>(beauty, diffuse, normal, depth, n.x[0].v(), B, H, W);
  for (int l = 0; l < kLevels; ++l) {
    const int h = H >> l, w = W >> l;
    const Layer& A = Ls[2 * l];
    const Layer& Bl = Ls[2 * l + 1];
    if ((e = conv(n, A, n.x[l].v(), n.ea[l].v(), A.wf, A.b, true, B, h, w, st))) return e;
    View eb = l < kLevels - 1 ? n.cat[l].v(kEnc[l + 1]) : n.eb4.v();
    if ((e = conv(n, Bl, n.ea[l].v(), eb, Bl.wf, Bl.b, true, B, h, w, st))) return e;
    if (l < kLevels - 1) {
      const size_t q = (size_t)B * (h / 2) * (w / 2) * kEnc[l];
      k_pool<<<blocks_for(q), 256, 0, st>>>(eb, n.x[l + 1].v(), B, h / 2, w / 2);
    }
  }
  View below = n.eb4.v();
  for (int l = kLevels - 2; l >= 0; --l) {
    const int h = H >> l, w = W >> l;
    const size_t q = (size_t)B * h * w * kEnc[l + 1];
    k_up<<<blocks_for(q), 256, 0, st>>>(below, n.cat[l].v(0, kEnc[l + 1]), B, h / 2, w / 2);
    const int li = L_D3A + 2 * (kLevels - 2 - l);
    const Layer& A = Ls[li];
    const Layer& Bl = Ls[li + 1];
    if ((e = conv(n, A, n.cat[l].v(), n.da[l].v(), A.wf, A.b, true, B, h, w, st))) return e;
    if ((e = conv(n, Bl, n.da[l].v(), n.db[l].v(), Bl.wf, Bl.b, true, B, h, w, st))) return e;
    below = n.db[l].v();
  }
  const Layer& O = Ls[L_OUT];
  if ((e = conv(n, O, n.db[0].v(), n.out.v(), O.wf, O.b, false, B, H, W, st))) return e;
  return cudaGetLastError();
}

// Backward through one layer: y = act(conv(x)); dy given (post-activation).
// Accumulates the layer's weight and bias gradients and writes dx (unless
// dx.p is null).
cudaError_t layer_bwd(DenoiserNet& n, Layer& L, View x, View y, View dy, View dx, Tensor& tmp,
                      int B, int h, int w, cudaStream_t st) {
  const size_t P = (size_t)B * h * w;
  View g = dy;
  if (L.relu) {
    g = View{tmp.p, L.cout, 0, L.cout};
    k_relu_bwd<<<blocks_for(P * L.cout), 256, 0, st>>>(dy, y, g, P);
  }
  cudaError_t e = wgrad(n, L, g, x, B, h, w, st);
  if (e != cudaSuccess || !dx.p) return e;
  return conv(n, L, g, dx, L.wbd, nullptr, false, B, h, w, st);
}

cudaError_t backward(DenoiserNet& n, int B, int H, int W, cudaStream_t st) {
  auto& Ls = n.layers;
  cudaError_t e;
  // output layer (no activation)
  if ((e = layer_bwd(n, Ls[L_OUT], n.db[0].v(), n.out.v(), n.g_out.v(), n.ddb[0].v(), n.gtmp[0], B,
                     H, W, st)))
    return e;
  // decoder, finest level first
  for (int l = 0; l < kLevels - 1; ++l) {
    const int h = H >> l, w = W >> l;
    const size_t P = (size_t)B * h * w;
    const int li = L_D3A + 2 * (kLevels - 2 - l);
    if ((e = layer_bwd(n, Ls[li + 1], n.da[l].v(), n.db[l].v(), n.ddb[l].v(), n.dda[l].v(), n.gtmp[l],
                       B, h, w, st)))
      return e;
    if ((e = layer_bwd(n, Ls[li], n.cat[l].v(), n.da[l].v(), n.dda[l].v(), n.dcat[l].v(), n.gtmp[l],
                       B, h, w, st)))
      return e;
    // the upsampled part of the concatenation came from the level below
    View dbelow = l + 1 < kLevels - 1 ? n.ddb[l + 1].v() : n.deb[kLevels - 1].v();
    const size_t q = (size_t)B * (h / 2) * (w / 2) * kEnc[l + 1];
    k_up_bwd<<<blocks_for(q), 256, 0, st>>>(n.dcat[l].v(0, kEnc[l + 1]), dbelow, B, h / 2, w / 2);
    (void)P;
  }
  // encoder, coarsest level first
  for (int l = kLevels - 1; l >= 0; --l) {
    const int h = H >> l, w = W >> l;
    const size_t P = (size_t)B * h * w;
    View eb = l < kLevels - 1 ? n.cat[l].v(kEnc[l + 1]) : n.eb4.v();
    if (l < kLevels - 1) {
      // d(eb) = skip gradient + adjoint of the pooling into level l + 1
      const size_t q = P * kEnc[l];
      k_pool_bwd<<<blocks_for(q), 256, 0, st>>>(n.dx[l + 1].v(), n.deb[l].v(), B, h / 2, w / 2);
      k_add<<<blocks_for(q), 256, 0, st>>>(n.deb[l].v(), n.dcat[l].v(kEnc[l + 1]), P);
    }
    if ((e = layer_bwd(n, Ls[2 * l + 1], n.ea[l].v(), eb, n.deb[l].v(), n.dea[l].v(), n.gtmp[l], B,
                       h, w, st)))
      return e;
    View dxl = l > 0 ? n.dx[l].v() : View{nullptr, 0, 0, 0};
    if ((e = layer_bwd(n, Ls[2 * l], n.x[l].v(), n.ea[l].v(), n.dea[l].v(), dxl, n.gtmp[l], B, h, w,
                       st)))
      return e;
  }
  return cudaGetLastError();
}

std::string finish(DenoiserNet& n, cudaStream_t st, const char* what) {
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

std::string denoiser_forward_backward(Denoiser& d, const float* beauty, const float* diffuse,
                                      const float* normal, const float* depth, const float* target,
                                      int B, int H, int W, double* loss, cudaStream_t st) {
  if (!d.net) return "denoiser: not created";
  DenoiserNet& n = *d.net;
  std::string s = check_shape(n, B, H, W);
  if (!s.empty()) return s;
  for (auto& L : n.layers) {
    cudaMemsetAsync(L.gw, 0, sizeof(float) * 9 * L.cin * L.cout, st);
    cudaMemsetAsync(L.gb, 0, sizeof(float) * L.cout, st);
  }
  cudaMemsetAsync(n.d_loss, 0, sizeof(double), st);
  cudaError_t e = forward(n, beauty, diffuse, normal, depth, B, H, W, st);
  if (e != cudaSuccess) return cuda_msg(e, "denoiser forward");
  const size_t P0 = (size_t)B * H * W;
  k_loss<<<blocks_for(P0), 256, 0, st>>>(n.out.v(), beauty, target, n.g_out.v(), B, H, W,
                                         n.loss_kind, n.d_loss);
  e = backward(n, B, H, W, st);
  if (e != cudaSuccess) return cuda_msg(e, "denoiser backward");
  s = finish(n, st, "denoiser training step");
  if (!s.empty()) return s;
  double h = 0.0;
  cudaMemcpy(&h, n.d_loss, sizeof(double), cudaMemcpyDeviceToHost);
  if (loss) *loss = h / (3.0 * (double)P0);  // mean |d| or mean 0.5 d^2
  n.B = B;
  n.H = H;
  n.W = W;
  return {};
}

std::string denoiser_adam(Denoiser& d, float lr, cudaStream_t st) {
  if (!d.net) return "denoiser: not created";
  DenoiserNet& n = *d.net;
  n.step++;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - std::pow(b1, (float)n.step), c2 = 1.0f - std::pow(b2, (float)n.step);
  for (auto& L : n.layers) {
    const size_t k = (size_t)9 * L.cin * L.cout;
    k_adam<<<blocks_for(k), 256, 0, st>>>(L.w, L.mw, L.vw, L.gw, k, lr, b1, b2, eps, c1, c2);
    k_adam<<<blocks_for(L.cout), 256, 0, st>>>(L.b, L.mb, L.vb, L.gb, L.cout, lr, b1, b2, eps, c1, c2);
    k_pack<<<blocks_for(k), 256, 0, st>>>(L.w, L.wf, L.wbd, L.cin, L.cout);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "denoiser update");
}

std::string denoiser_infer(Denoiser& d, const float* beauty, const float* diffuse,
                           const float* normal, const float* depth, float* out, int B, int H, int W,
                           cudaStream_t st) {
  if (!d.net) return "denoiser: not created";
  DenoiserNet& n = *d.net;
  std::string s = check_shape(n, B, H, W);
  if (!s.empty()) return s;
  cudaError_t e = forward(n, beauty, diffuse, normal, depth, B, H, W, st);
  if (e != cudaSuccess) return cuda_msg(e, "denoiser forward");
  k_output<<<blocks_for((size_t)B * H * W), 256, 0, st>>>(n.out.v(), beauty, out, B, H, W);
  return finish(n, st, "denoiser inference");
}

std::string denoiser_set_loss(Denoiser& d, int kind) {
  if (!d.net) return "denoiser: not created";
  if (kind != 0 && kind != 1) return "denoiser: loss kind must be 0 (squared) or 1 (absolute)";
  d.net->loss_kind = kind;
  return {};
}

size_t denoiser_param_count(const Denoiser& d) {
  size_t c = 0;
  if (d.net)
    for (auto& L : d.net->layers) c += (size_t)9 * L.cin * L.cout + L.cout;
  return c;
}

std::string denoiser_get(const Denoiser& d, int what, float* host) {
  if (!d.net) return "denoiser: not created";
  for (auto& L : d.net->layers) {
    const size_t k = (size_t)9 * L.cin * L.cout;
    cudaError_t e = cudaMemcpy(host, what ? L.gw : L.w, k * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(host + k, what ? L.gb : L.b, L.cout * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_msg(e, "denoiser read");
    host += k + L.cout;
  }
  return {};
}

std::string denoiser_set_weights(Denoiser& d, const float* host) {
  if (!d.net) return "denoiser: not created";
  for (auto& L : d.net->layers) {
    const size_t k = (size_t)9 * L.cin * L.cout;
    cudaError_t e = cudaMemcpy(L.w, host, k * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(L.b, host + k, L.cout * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_msg(e, "denoiser write");
    k_pack<<<blocks_for(k), 256>>>(L.w, L.wf, L.wbd, L.cin, L.cout);
    host += k + L.cout;
  }
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? std::string() : cuda_msg(e, "denoiser write");
}

int denoiser_layer_count(const Denoiser& d) { return d.net ? (int)d.net->layers.size() : 0; }
void denoiser_layer_shape(const Denoiser& d, int i, int* cin, int* cout) {
  *cin = d.net->layers[i].cin;
  *cout = d.net->layers[i].cout;
}

}  // namespace nr
