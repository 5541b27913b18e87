// Voxel-first subsampling (fknn_voxel.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fknn_internal.h"

namespace fknn {

struct VoxelArgs {
  const float* xyz;      // f32 [n,3]
  const int64_t* batch;  // int64 [n] or null
  int64_t n;
  float voxel;
  int64_t* out;          // int64 [n]: representatives, ascending
  int64_t* count_out;    // int64 [1] on the device
};

size_t voxel_first_workspace_bytes(int64_t n);
int run_voxel_first(const VoxelArgs& v, void* ws, size_t ws_bytes, cudaStream_t s, int* launches);

}  // namespace fknn
