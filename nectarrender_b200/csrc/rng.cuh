// rng.cuh — counter-based random numbers and the reference's hash functions.
//
// Generator: the reference re-runs curand_init(seed, subsequence=pixel_idx +
// sample_idx*W*H, offset=draw_id) before every draw and returns
// curand_uniform (nectar_render/csrc/core/include/core/random.h:50-55). With
// Philox4x32-10 that draw is lane (draw_id % 4) of one Philox block whose
// counter is {draw_id / 4, 0, subsequence_lo, subsequence_hi} and whose key is
// {seed_lo, seed_hi}; uniform floats are x * 2^-32 + 2^-33, in (0, 1].
// Philox4x32-10 is the published counter-based generator of Salmon, Moraes,
// Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11); it is
// written here from that paper. A path therefore carries only
// (subsequence, draw_id), and the block of four words is cached so that
// consecutive draws cost one Philox evaluation per four draws.
//
// Hashes: PCG-style integer hashes of nectar_render/csrc/random/include/
// hash.h:17-191, used for the per-pixel sub-pixel shift and the medium
// free-flight distance.
#pragma once
#include "vecmath.cuh"

namespace nr {

struct Philox4 {
  uint32_t x, y, z, w;
};

NR_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
#endif
}

// Philox4x32 with 10 rounds; multipliers and Weyl key increments as published.
NR_HD Philox4 philox4x32_10(Philox4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t h0, l0, h1, l1;
    mulhilo32(0xD2511F53u, c.x, h0, l0);
    mulhilo32(0xCD9E8D57u, c.z, h1, l1);
    c = Philox4{h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

NR_HD float u32_to_uniform(uint32_t v) {
  return (float)v * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
}

// Per-path generator state: the reference Generator(seed, pixel_idx) with its
// draw counter (random.h:11-77).
struct Rng {
  uint32_t seed;
  uint32_t subseq;
  uint32_t draw;
  uint32_t cached_block;  // draw/4 of the cached block, 0xffffffff = none
  Philox4 block;

  NR_HD void init(uint32_t s, uint32_t sub, uint32_t d = 0u) {
    seed = s;
    subseq = sub;
    draw = d;
    cached_block = 0xffffffffu;
  }
  NR_HD float uniform() {
    uint32_t b = draw >> 2;
    if (b != cached_block) {
      block = philox4x32_10(Philox4{b, 0u, subseq, 0u}, seed, 0u);
      cached_block = b;
    }
    uint32_t lane = draw & 3u;
    draw += 1u;
    uint32_t v = lane == 0 ? block.x : (lane == 1 ? block.y : (lane == 2 ? block.z : block.w));
    return u32_to_uniform(v);
  }
  // random_float(min, max) = uniform()*(max-min)+min  (random.h:64-66)
  NR_HD float random_float() { return uniform() * (1.0f - 0.0f) + 0.0f; }
  NR_HD float random_float(float mn, float mx) { return uniform() * (mx - mn) + mn; }
};

// ---- hash.h ---------------------------------------------------------------
// __hash_mix multiplies by entry (stream*3 + k) of a 64-entry table of odd
// constants (hash.h:19-40). Every call on the path uses stream 0, so only the
// first three entries are reachable: the golden-ratio constant 0x9E3779B9 and
// the two MurmurHash3 finaliser multipliers 0x85EBCA6B and 0xC2B2AE35.
__device__ __forceinline__ uint32_t hash_mix(uint32_t val, uint32_t mult) {
  val ^= (val >> 16u) * mult;
  return val ^ (val >> 13u);
}

// __pcg_hash_int (hash.h:48-62)
// (stream 0 only, the only stream the path uses)
__device__ __forceinline__ uint32_t pcg_hash_int(uint32_t i, uint32_t seed) {
  uint32_t s = seed * 1759274928u;
  s = i ^ s;
  s = hash_mix(s, 0x9E3779B9u);
  s = hash_mix(s, 0x85EBCA6Bu);
  s = hash_mix(s, 0xC2B2AE35u);
  uint32_t state = s * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// (float)hash * (1/(float)0xFFFFFFFF); that scalar rounds to exactly 2^-32.
__device__ __forceinline__ float hash_to_float(uint32_t h) { return (float)h * 2.3283064365386963e-10f; }

// pcg_float(float f, seed, stream)  (hash.h:76-83)
__device__ __forceinline__ float pcg_float_f(float f, uint32_t seed) {
  return hash_to_float(pcg_hash_int(__float_as_uint(f), seed));
}

// pcg_float(const Vector3&, seed, stream)  (hash.h:98-106)
__device__ __forceinline__ float pcg_float_v3(const V3& a, uint32_t seed) {
  uint32_t s = seed * 1759274928u;
  s ^= pcg_hash_int(__float_as_uint(a.x), (seed + 0u) * 2654435761u) ^ 668265263u;
  s ^= pcg_hash_int(__float_as_uint(a.y), (seed + 1u) * 2246822519u) ^ 374761393u;
  s ^= pcg_hash_int(__float_as_uint(a.z), (seed + 2u) * 3266489917u) ^ 2654435761u;
  uint32_t state = s * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return hash_to_float((word >> 22u) ^ word);
}

// pcg_float(const Ray&) = average of the origin and direction hashes (hash.h:108-125).
__device__ __forceinline__ float pcg_float_ray(const V3& o, const V3& d) {
  float a = pcg_float_v3(o, (0u + 0u) * 2654435761u);
  float b = pcg_float_v3(d, (0u + 1u) * 3266489917u);
  return (a + b) * 0.5f;
}

// pcg_vector2(float f, seed) (hash.h:182-191); the pixel index reaches it as a float.
__device__ __forceinline__ V2 pcg_vector2(float f, uint32_t seed) {
  float x = pcg_float_f(f, seed);
  uint32_t s = seed ^ (uint32_t)(x * 4294967296.0f);
  uint32_t i = s * 747796405u + 2891336453u;
  float y = pcg_float_f((float)i, 0u);
  return V2{x, y};
}

}  // namespace nr
