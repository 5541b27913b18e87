// Reference table ABI on the device (fknn_tables.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fknn_internal.h"

namespace fknn {

struct TablesArgs {
  const float* xyz_sorted;     // f32 [n,3]
  int64_t n;
  const int32_t* steps;        // [p+1]
  const int32_t* neigh;        // [p,27]
  const int32_t* cnt;          // [p,28]
  int64_t p;
  const int32_t* qindex;       // selected queries [m] or null (self query)
  const int32_t* steps_query;  // [p+1] when qindex is given
  int64_t m;
  int k;
  float cut_r2;
  int32_t* idx_out;
  float* dist_out;
  const float* qxyz;           // separate query points [m,3] grouped by steps_query, or null
  const int32_t* qpad;         // with qxyz: pad index per query row, or null (pad -1)
};

struct BuildTablesArgs {
  const int64_t* grid;
  const int64_t* batch;
  int64_t n;
  int num_down;
  int64_t* order;
  int32_t* steps;
  int32_t* neigh;
  int32_t* cnt;
  int64_t* n_parents;
};

size_t tables_workspace_bytes(int64_t n, int64_t m, int64_t p);
int run_tables(const TablesArgs& t, void* ws, size_t ws_bytes, const QueryShape& shape,
               cudaStream_t s, int* launches);
size_t build_tables_workspace_bytes(int64_t n);
int run_build_tables(const BuildTablesArgs& t, void* ws, size_t ws_bytes, cudaStream_t s,
                     int* launches);
int run_morton_encode(const int64_t* grid, const int64_t* batch, int64_t n, int64_t* keys,
                      cudaStream_t s);
int run_neighbor_keys(const int64_t* gd, const int64_t* pb, int64_t p, int64_t* keys,
                      cudaStream_t s);

}  // namespace fknn
