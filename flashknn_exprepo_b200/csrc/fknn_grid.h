// Fused construction + query pipelines (fknn_grid.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fknn_internal.h"

namespace fknn {

struct FusedArgs {
  int kind;                      // FKNN_QUERY_SELF / SELECTED / GENERAL
  const float* xyz;              // support f32 [n,3]
  const int64_t* grid;           // int64 [n,3] or null (then floor(xyz / voxel))
  const int64_t* batch;          // int64 [n] or null
  const int64_t* offsets;        // cumulative cloud ends or null
  int64_t n;
  int64_t n_clouds;              // batch ids must lie in [0, n_clouds)
  const int64_t* sindex;         // support point i is row sindex[i] of xyz/grid/batch, or null
  int64_t n_src;                 // rows of xyz/grid/batch when sindex is given
  int trunc_grid;                // voxelise with trunc(xyz / voxel) instead of floor
  const float* qxyz;             // general queries f32 [m,3]
  const int64_t* qoffsets;       // general queries' cloud ends
  const int64_t* qbatch;         // general queries' batch ids (instead of qoffsets), or null
  const int64_t* query_indices;  // selected queries int64 [m]
  int64_t m;
  float voxel;
  int num_down;
  int k;
  float cut_r2;
  int pad_minus_one;             // self query: pad rows with -1 instead of the own index
  int idx_bits;
  void* idx_out;
  float* dist_out;
};

size_t fused_workspace_bytes(int64_t n, int64_t m, int64_t n_clouds, int kind);
int run_fused(const FusedArgs& f, void* ws, size_t ws_bytes, const QueryShape& shape,
              cudaStream_t s, int* launches);

}  // namespace fknn
