// bvh_build.cuh — GPU BVH construction interface.
#pragma once
#include <vector>
#include "scene_device.cuh"

namespace nr {

// Binary node as produced by the builder (both levels). Leaves have
// left == right == -1 and reference the primitive range [start, start+count)
// of the output primitive order.
struct BinNode {
  float lo[3], hi[3];
  int32_t left, right;
  uint32_t start, count;
};

struct BuildResult {
  // device buffers owned by the caller after the build
  BinNode* d_nodes = nullptr;   // n_nodes binary nodes, root = 0
  uint32_t* d_order = nullptr;  // leaf order -> input primitive index
  Bvh2Node* d_bvh2 = nullptr;   // inner nodes, 64 B layout, root = 0
  Bvh8Node* d_bvh8 = nullptr;   // compressed 8-wide nodes, root = 0
  uint32_t* d_order8 = nullptr; // wide-leaf order -> input primitive index
  uint32_t n_nodes = 0;
  uint32_t n_bvh2 = 0;
  uint32_t n_bvh8 = 0;
  double sah_cost = 0.0;  // binary tree, leaf size 1, unit costs (node 1, prim 1)
  float build_ms = 0.0f;
};

// Builds the binary SAH tree over `n` primitive boxes given as device arrays
// lo[i] = (x, y, z, _), hi[i] = (x, y, z, _) and derives the 2-wide and
// 8-wide traversal layouts; 8-wide leaves hold at most `leaf_max` (1..3)
// primitives, and each wide node at most `width` (2..8) children (the node
// format stays 8-wide; a narrower tree leaves slots empty). Returns a
// cudaError_t value.
int build_bvh(const float4* d_lo, const float4* d_hi, uint32_t n, bool want_bvh8,
              BuildResult& out, cudaStream_t st, uint32_t leaf_max = 3, uint32_t width = 8);

void free_build(BuildResult& r);

// Exclusive prefix sum of in[0..n) into out (out == in allowed): tile sums,
// one CTA over the tile sums, tile scans plus offsets. `sums` is scratch of
// scan_scratch_words(n) words; the sum of all n values goes to *total
// (device memory) when total is not null.
uint32_t scan_scratch_words(uint32_t n);
cudaError_t scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* sums,
                           uint32_t* total, cudaStream_t st);

// Stable LSD radix sort of (key, value) pairs over the low key_bits bits
// (8 bits per pass); keys2 / vals2 are scratch of n entries, hist holds
// radix_sort_hist_words(n) words. The sorted pairs end in whichever buffers
// *out_keys / *out_vals name.
uint32_t radix_sort_hist_words(uint32_t n);
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys2, uint32_t* vals2,
                             uint32_t n, int key_bits, uint32_t* hist, cudaStream_t st,
                             uint32_t** out_keys, uint32_t** out_vals);

}  // namespace nr
