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
  int n_points_scanned;  // total of a scan over per-cell point counts (= n)
  int reserved[3];  // per-path scratch words (the adaptive octree's)
  // sum over the query groups of their 27-cell candidate totals (self and
  // general queries; read back for FlashKNN.query's traverse_info)
  unsigned long long cand_total;
};
static_assert(sizeof(Meta) == 64, "Meta layout");
static_assert(offsetof(Meta, cand_total) == 56, "Meta layout");

// Work items (int4): (q_start, q_count, g_first, g_count | flags) -- the
// queries [q_start, q_start + q_count) of the query-record array, which
// belong to the groups [g_first, g_first + g_count).  A chunked item has one
// group whose candidates exceed a tile; they are streamed tile by tile.
constexpr int kItemChunked = 1 << 30;
constexpr int kMaxGroupsPerItem = 16;

// Resolved launch shape of the query kernel.
struct QueryShape {
  int warps_per_cta;
  int tile_records;
  int min_candidates_per_lane;
  int ctas_per_sm;
  int staging_depth;  // 1: stage an item, then scan it; 2: stage the next during the scan
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
  const int32_t* group_start;  // [groups + 1] query ranges in qrec
  const int32_t* group_row;    // runs row of each group, or null (row = group)
  const int* group_count_ptr;  // device: number of groups
  const int4* items;   // work items (see above)
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

// Item construction (fknn_items.cu): per-group candidate counts, segmented
// greedy packing; *n_items_ptr receives the item count.  Returns launches.
int launch_items(const int2* runs, const int32_t* group_start, const int32_t* group_row,
                 const int* group_count_ptr, int64_t max_groups, int tile, int32_t* cands,
                 uint32_t* seg_counts, int* n_items_ptr, int4* items, cudaStream_t s,
                 int* status, int64_t n_queries, bool cands_ready);
size_t items_capacity(int64_t max_groups, int64_t n_queries);
// Bounded-wait self-test (fknn_selftest.cu): arms a barrier that never
// completes and waits at most `limit` polls; sets kStatusTimeout.
int run_selftest_wait(void* ws, size_t ws_bytes, uint32_t limit, cudaStream_t s);
// Groups per packing segment (one warp walks a segment's groups in order):
// kPackSegment for a large problem; a problem of fewer than
// kPackSegment * kPackWarps groups uses shorter segments (at least
// kPackSegmentMin groups), so its few groups still spread over about
// kPackWarps warps and no warp walks a long serial chain.
constexpr int kPackSegment = 16;
constexpr int kPackSegmentMin = 4;
constexpr int kPackWarps = 4096;
__host__ __device__ inline int pack_segment_len(int n_groups) {
  if (n_groups >= kPackSegment * kPackWarps) return kPackSegment;
  const int len = n_groups / kPackWarps;
  return len < kPackSegmentMin ? kPackSegmentMin : len;
}
// Segment counts to allocate for up to max_groups groups (every length).
inline int64_t pack_segments(int64_t max_groups) {
  return (max_groups + kPackSegmentMin - 1) / kPackSegmentMin;
}

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
