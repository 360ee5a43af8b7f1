// nrc.cuh — neural radiance cache: a multiresolution hash-grid encoding of
// position (Mueller et al., "Instant Neural Graphics Primitives", 2022) and
// a 64-wide MLP predicting the radiance leaving a surface point (Mueller et
// al., "Real-time Neural Radiance Caching for Path Tracing", 2021). Every
// MLP layer (forward, backward-data, weight gradient) is a tcgen05 GEMM
// (conv_tc.cu in its one-tap mode); the encoding and its gradient are
// gather/scatter kernels here. No reference counterpart.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>
#include <string>

namespace nr {

// One query: the features the cache is keyed on, 16 floats.
//   [0..2] position, [3] roughness, [4..6] outgoing direction (unit, away
//   from the surface), [7] unused, [8..10] shading normal, [11] unused,
//   [12..14] diffuse albedo, [15] unused
struct NrcQuery {
  float4 a, b, c, d;
};

struct NrcNet;  // defined in nrc.cu

struct Nrc {
  NrcNet* net = nullptr;
  ~Nrc();
};

std::string nrc_create(Nrc& n, uint32_t max_queries, const float bounds_lo[3],
                       const float bounds_hi[3], uint32_t seed);
// radiance out[q] (float3 per query, stride 3) for q < count
std::string nrc_infer(Nrc& n, const NrcQuery* q, uint32_t count, float* out, cudaStream_t st);
// one Adam step toward target radiance (float3 per query; lazy on the hash
// grid: entries that no query touched keep their values and moments); *loss = mean
// relative squared error before the step (when loss is not null; reading
// it synchronises the stream)
std::string nrc_train(Nrc& n, const NrcQuery* q, const float* target, uint32_t count, float lr,
                      double* loss, cudaStream_t st);
// gradients only (lr = 0) and host copies for checking them
std::string nrc_get(const Nrc& n, int what, float* host);  // 0 MLP weights, 1 their gradients,
                                                            // 2 grid values, 3 grid gradients
size_t nrc_count(const Nrc& n, int what);
uint32_t nrc_max_queries(const Nrc& n);
// error flag of the tensor-core waits of the launches on st (synchronises st)
std::string nrc_poll_error(Nrc& n, cudaStream_t st);
std::string nrc_set_weights(Nrc& n, const float* mlp, const float* grid);

}  // namespace nr
