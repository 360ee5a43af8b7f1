// sky_alias.cuh — importance-sampling tables of an equirectangular HDRI for
// NR_MODE_PERF, built on the GPU: a row-marginal alias table, one alias
// table per row over its columns, and the probability of every texel.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace nr {

struct SkyTables {
  float* row_prob = nullptr;      // [H] acceptance probability of each row bucket
  uint32_t* row_alias = nullptr;  // [H] alias row
  float* col_prob = nullptr;      // [H][W] acceptance probability of each column bucket
  uint32_t* col_alias = nullptr;  // [H][W] alias column within the row
  float* texel_pdf = nullptr;     // [H][W] probability of each texel
  int W = 0, H = 0;
  void release();
};

// Builds the tables of a planar CHW float image (3 channels) on stream st;
// has_energy is false when every weight is zero (no sampling then).
cudaError_t build_sky_tables(const float* chw, int W, int H, SkyTables& t, bool& has_energy,
                             cudaStream_t st);

}  // namespace nr
