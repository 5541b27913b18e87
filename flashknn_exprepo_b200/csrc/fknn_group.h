// Neighbour feature grouping (fknn_group.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fknn_internal.h"

namespace fknn {

struct GroupArgs {
  const float* feat;        // f32 [n,c] (forward)
  int64_t n;
  int c;
  const int32_t* idx;       // int32 [m,k]; < 0 = padding
  int64_t m;
  int k;
  const float* xyz;         // f32 [n,3] (with_xyz)
  const float* new_xyz;     // f32 [m,3] (with_xyz)
  int with_xyz;
  float* out;               // f32 [m,k,c(+3)] (forward)
  const float* grad_out;    // f32 [m,k,c(+3)] (backward)
  float* grad_feat;         // f32 [n,c] or null
  float* grad_xyz;          // f32 [n,3] or null
  int accumulate_xyz;
  float* grad_new_xyz;      // f32 [m,3] or null
  int accumulate_new_xyz;
};

size_t group_workspace_bytes(int64_t rows, int64_t n);
int run_group_forward(const GroupArgs& g, void* ws, size_t ws_bytes, cudaStream_t s,
                      int* launches);
int run_group_backward(const GroupArgs& g, void* ws, size_t ws_bytes, cudaStream_t s,
                       int* launches);

}  // namespace fknn
