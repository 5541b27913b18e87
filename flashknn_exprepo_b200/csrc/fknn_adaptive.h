// Adaptive-neighbourhood self query (fknn_adaptive.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fknn_internal.h"

namespace fknn {

struct AdaptiveArgs {
  const int64_t* grid;   // int64 [n,3]
  const int64_t* batch;  // int64 [n] or null (one batch)
  const float* xyz;      // f32 [n,3] or null (positions = translated grid)
  int64_t n;
  int k;
  int min_factor;
  int max_factor;
  int max_shift;         // < 0: bit length of the largest translated coordinate
  float cut_r2;
  int idx_bits;
  void* idx_out;
  float* dist_out;
  int8_t* level_out;     // [n] or null
};

size_t adaptive_workspace_bytes(int64_t n);
int run_adaptive(const AdaptiveArgs& f, void* ws, size_t ws_bytes, const QueryShape& shape,
                 cudaStream_t s, int* launches);

}  // namespace fknn
