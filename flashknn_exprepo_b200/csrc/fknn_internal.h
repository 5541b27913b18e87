// Declarations shared by the FlashKNN-B200 translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/fknn.h"

namespace fknn {

// Device-resident bookkeeping at offset 0 of every workspace.  `status` must
// stay the first member: fknn_read_status() reads the first int.
struct Meta {
  int status;       // FKNN_DEVICE_* bits
  int key_bits;     // significant bits of the support / general-query keys
  int bpa;          // bits per axis of the translated parent coordinates
  int n_cells;      // occupied support parent cells
  int n_groups;     // query groups (selected / general queries)
  int n_items;      // work items for the query kernel
  int queue_head;   // work-queue cursor of the persistent query kernel
  int qkey_bits;    // significant bits of the selected-query cell keys
  int batch_bits;   // bits of the largest batch id
  int max_extent;   // largest per-cloud parent-coordinate extent
  int reserved[6];
};
static_assert(sizeof(Meta) == 64, "Meta layout");

// One unit of query work: the queries [q_start, q_start + q_count) of the
// query-record array share the 27 candidate runs in runs[runs_row].
struct Item {
  int runs_row;
  int q_start;
  int q_count;
  int unused;
};

// Resolved launch shape of the query kernel.
struct QueryShape {
  int warps_per_cta;
  int tile_records;
  int min_candidates_per_lane;
  int ctas_per_sm;
};

QueryShape resolve_shape(const fknn_config* cfg);
bool shape_valid(const QueryShape& s);

enum PadMode : int { kPadSelf = 0, kPadArray64 = 1, kPadArray32 = 2, kPadMinusOne = 3 };

struct QueryLaunch {
  const float4* srec;  // support records (x, y, z, index bits), cell-sorted
  int n_support;
  const float4* qrec;  // query records (x, y, z, output-row bits)
  int n_qrec;
  const int2* runs;    // [rows][27] (start, count) into srec
  const int4* items;   // Item array
  Meta* meta;
  int k;
  float cut_r2;
  int idx_bits;        // 32 or 64
  void* idx_out;
  float* dist_out;
  int64_t n_rows;
  const void* pad;     // pad index per output row (pad_mode 1/2)
  int pad_mode;
  int vec_ok;          // outputs 16-byte aligned: row stores may be vectorised
};

// Launches the persistent query kernel; returns 0 or a cudaError_t.
int launch_query(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s);

// Bump allocator over a caller-provided workspace (256-byte aligned slices).
struct Arena {
  char* base;
  size_t used = 0;
  explicit Arena(void* p) : base(static_cast<char*>(p)) {}
  template <typename T>
  T* take(size_t count) {
    used = (used + 255) & ~static_cast<size_t>(255);
    T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
    used += sizeof(T) * (count ? count : 1);
    return p;
  }
};

// Library-wide bookkeeping used by the C ABI.
void note_cuda_error(cudaError_t e);
void note_launches(int n);

// Optional event brackets around the query kernel (fknn_profile_enable).
// Returns the slot to close with profile_stop, or -1 when profiling is off.
int profile_start(cudaStream_t s);
void profile_stop(int slot, cudaStream_t s);

}  // namespace fknn
