// Backward of the kNN squared distances (fknn_backward.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fknn_internal.h"

namespace fknn {

struct BackwardArgs {
  const float* q_xyz;   // f32 [m,3]
  int64_t m;
  const float* p_xyz;   // f32 [n,3]
  int64_t n;
  const int32_t* idx;   // [m,k]
  const float* dist;    // [m,k]
  const float* grad;    // [m,k]
  int k;
  float* grad_q;        // [m,3] or null
  float* grad_p;        // [n,3] or null
  int accumulate;
};

size_t backward_workspace_bytes(int64_t m, int64_t n, int k);

// Counting-sort placement of segments: from count[p] (entries per support
// point) writes start[p] (first slot), start[n] (total) and cursor[p] (one
// past the last slot, for a scatter that counts down).  tiles holds
// segment_tiles(n) words; *total receives the total.  Returns launches.
size_t segment_tiles(int64_t n);
int launch_segment_starts(const uint32_t* count, int64_t n, uint32_t* tiles, int* total,
                          uint32_t* start, uint32_t* cursor, cudaStream_t s);
int run_backward(const BackwardArgs& a, void* ws, size_t ws_bytes, cudaStream_t s, int* launches);

}  // namespace fknn
