// Work items of the query kernel.
//
// A query group is a set of queries (contiguous in the query-record array)
// that share one candidate set: the 27 runs of a parent cell.  Items pack
// up to 32 consecutive queries -- possibly from several consecutive groups --
// so that every lane of a warp owns one query, as long as the candidates of
// all groups in the item fit one shared-memory tile.  Groups with more
// candidates than a tile become "chunked" items of up to 32 queries that
// stream their candidates tile by tile.
//
// Packing is a sequential greedy pass over the groups in key order; it runs
// in parallel over segments of consecutive groups (one warp each; the
// segment length follows the group count, see pack_segment_len): a
// count pass, a scan of the per-segment counts, and a write pass.  Items
// therefore keep the spatial order of the groups.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"

namespace fknn {

// cands[g] = number of candidate records of group g (sum of its 27 runs);
// a group without candidates sets kStatusNoCandidates when status is given.
__global__ void __launch_bounds__(256)
    k_group_cands(const int2* __restrict__ runs, const int32_t* __restrict__ group_row,
                  const int* group_count_ptr, int32_t* __restrict__ cands, int* status) {
  chain_wait();
  const int n_groups = *group_count_ptr;
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n_groups;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = group_row ? group_row[g] : g;
    const int2* r = runs + row * kNeighbours;
    int total = 0;
#pragma unroll
    for (int j = 0; j < kNeighbours; ++j) total += max(r[j].y, 0);
    cands[g] = total;
    if (total == 0) raise_status(status, kStatusNoCandidates);
  }
}

// One warp per segment of consecutive groups.  With items == nullptr it
// only counts (seg_counts[seg]); otherwise it writes its items at
// seg_offsets[seg].  Item = (q_start, q_count, g_first, g_count | flags).
// The segment's group ranges and candidate counts are loaded once (one
// group per lane); every lane then walks the greedy pass with the same
// values, lane 0 writes packed items and the whole warp writes a chunked
// group's items, so a group of many chunked items costs no serial stores.
// Caller tables can be malformed: a group whose query range leaves
// [0, n_queries] is reported and skipped, and no item is written at or past
// `capacity` (overlapping ranges could otherwise ask for more items than the
// buffer holds; k_scan_segments clamps the count to match).
static_assert(kPackSegment <= 32, "one group per lane");
__global__ void __launch_bounds__(256)
    k_pack(const int32_t* __restrict__ group_start, const int32_t* __restrict__ cands,
           const int* group_count_ptr, int tile, int max_q, int max_qc, int64_t n_queries,
           int64_t capacity, uint32_t* __restrict__ seg_counts,
           const uint32_t* __restrict__ seg_offsets, int4* __restrict__ items, int* status) {
  chain_wait();
  const int lane = threadIdx.x & 31;
  const int n_groups = *group_count_ptr;
  const int seg_len = pack_segment_len(n_groups);
  const int64_t n_segs = (n_groups + seg_len - 1) / seg_len;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t seg = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
       seg < n_segs; seg += warps) {
    const int64_t g_begin = seg * seg_len;
    const int64_t g_lim = g_begin + seg_len;
    const int g_end = static_cast<int>(g_lim < n_groups ? g_lim : n_groups);
    const int n_here = g_end - static_cast<int>(g_begin);
    int my_gs = 0, my_ge = 0, my_c = 0;
    if (lane < n_here) {
      my_gs = group_start[g_begin + lane];
      my_ge = group_start[g_begin + lane + 1];
      my_c = cands[g_begin + lane];
    }
    const uint32_t out = items ? seg_offsets[seg] : 0u;
    uint32_t count = 0;
    int cur_q0 = 0, cur_qn = 0, cur_g0 = 0, cur_gn = 0, cur_c = 0;
    auto put = [&](uint32_t slot, int q0, int qn, int g0, int gn, int flags) {
      if (static_cast<int64_t>(out) + slot < capacity)
        items[out + slot] = make_int4(q0, qn, g0, gn | flags);
      else
        raise_status(status, kStatusTable);
    };
    auto flush = [&]() {
      if (cur_gn > 0) {
        if (items && lane == 0) put(count, cur_q0, cur_qn, cur_g0, cur_gn, 0);
        ++count;
      }
      cur_qn = cur_gn = cur_c = 0;
    };
    for (int j = 0; j < n_here; ++j) {
      const int g = static_cast<int>(g_begin) + j;
      const int gs = __shfl_sync(kFull, my_gs, j), ge = __shfl_sync(kFull, my_ge, j);
      const int c = __shfl_sync(kFull, my_c, j);
      if (gs < 0 || ge > n_queries) {
        if (items && lane == 0) raise_status(status, kStatusTable);
        continue;
      }
      if (ge <= gs) continue;
      if (c > tile) {  // streams its candidates: items of its own
        flush();
        const int n_it = (ge - gs + max_qc - 1) / max_qc;
        if (items)
          for (int t = lane; t < n_it; t += 32) {
            const int q = gs + t * max_qc;
            put(count + t, q, min(max_qc, ge - q), g, 1, kItemChunked);
          }
        count += n_it;
        continue;
      }
      int pos = gs;
      while (pos < ge) {
        // An item spans the groups [cur_g0, g]: groups without queries inside
        // that span still count, because the kernel walks the span.
        if (cur_gn > 0 && (cur_c + c > tile || cur_qn >= max_q ||
                           g - cur_g0 + 1 > kMaxGroupsPerItem))
          flush();
        if (cur_gn == 0) {
          cur_q0 = pos;
          cur_g0 = g;
        }
        const int take = min(ge - pos, max_q - cur_qn);
        cur_qn += take;
        cur_gn = g - cur_g0 + 1;
        cur_c += c;
        pos += take;
      }
    }
    flush();
    if (!items && lane == 0) seg_counts[seg] = count;
  }
}

// Exclusive scan of the per-segment item counts over the segments that hold
// groups (the device-side group count bounds the work); the total is clamped
// to the item buffer's capacity.
__global__ void __launch_bounds__(1024)
    k_scan_segments(uint32_t* __restrict__ seg_counts, const int* group_count_ptr,
                    int64_t capacity, int* __restrict__ total_out, int* status) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int n_groups = *group_count_ptr;
  const int seg_len = pack_segment_len(n_groups);
  const int n_segs = (n_groups + seg_len - 1) / seg_len;
  uint32_t carry = 0;
  for (int t0 = 0; t0 < n_segs; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const uint32_t x = t < n_segs ? seg_counts[t] : 0u;
    const uint32_t incl = block_inclusive_scan(x, warp_sums, &s_total);
    if (t < n_segs) seg_counts[t] = carry + incl - x;
    carry += s_total;
  }
  if (threadIdx.x == 0) {
    if (static_cast<int64_t>(carry) > capacity) raise_status(status, kStatusTable);
    *total_out = static_cast<int>(static_cast<int64_t>(carry) < capacity ? carry : capacity);
  }
}

// Queries per packed item.  A large problem fills every lane (32); a small
// one -- fewer than 16 queries per resident query warp -- is cut into about
// one item per resident warp (at least 4 queries each), so its few items do
// not leave most warps idle while each one runs the whole scan.
int item_query_cap(int64_t n_queries) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
      sms = v;
    if (sms <= 0) return 32;
  }
  const int64_t warps = static_cast<int64_t>(sms) * 20;  // resident at the default shape
  if (n_queries >= warps * 16) return 32;
  const int64_t cap = ceil_div(n_queries > 0 ? n_queries : 1, warps);
  return static_cast<int>(cap < 4 ? 4 : (cap > 32 ? 32 : cap));
}

// Queries per chunked item (a group whose candidates exceed a tile: every
// query scans many of them).  An item of q queries gives each query 32 / q
// lanes.  A problem with fewer than 32 queries per resident query warp is
// cut into about two items per warp (at least 4 queries each), so a dense
// but small problem spreads every query's scan over several lanes instead
// of one lane walking all its candidates; larger ones keep full items
// (measured: the LiDAR scan at alpha 8, 118k points, is faster with full
// items; the DeLA levels of 3.7k-72k points with split ones).
int chunked_query_cap(int64_t n_queries) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    return 32;
  const int64_t warps = static_cast<int64_t>(sms) * 20;
  if (n_queries >= warps * 32) return 32;
  const int64_t cap = ceil_div(n_queries > 0 ? n_queries : 1, 2 * warps);
  return static_cast<int>(cap < 4 ? 4 : (cap > 32 ? 32 : cap));
}

int launch_items(const int2* runs, const int32_t* group_start, const int32_t* group_row,
                 const int* group_count_ptr, int64_t max_groups, int tile, int32_t* cands,
                 uint32_t* seg_counts, int* n_items_ptr, int4* items, cudaStream_t s,
                 int* status, int64_t n_queries, bool cands_ready) {
  if (max_groups <= 0) return 0;
  // grids for the host-side bound, capped: the device count drives the loops
  const int64_t gb = ceil_div(max_groups, 256);
  const int gblocks = static_cast<int>(gb < 2048 ? gb : 2048);
  const int64_t sb = ceil_div(pack_segments(max_groups), 8);  // 8 warps per block
  const int sblocks = static_cast<int>(sb < 2048 ? sb : 2048);
  if (!cands_ready)  // else the caller's run kernel wrote cands[g] already
    launch_chained(k_group_cands, gblocks, 256, 0, s, runs, group_row, group_count_ptr, cands,
        status);
  const int64_t capacity = static_cast<int64_t>(items_capacity(max_groups, n_queries));
  const int max_q = item_query_cap(n_queries);
  const int max_qc = chunked_query_cap(n_queries);
  launch_chained(k_pack, sblocks, 256, 0, s, group_start, cands, group_count_ptr, tile, max_q,
      max_qc, n_queries, capacity, seg_counts, nullptr, nullptr, status);
  launch_chained(k_scan_segments, 1, 1024, 0, s, seg_counts, group_count_ptr, capacity, n_items_ptr,
      status);
  launch_chained(k_pack, sblocks, 256, 0, s, group_start, cands, group_count_ptr, tile, max_q,
      max_qc, n_queries, capacity, nullptr, seg_counts, items, status);
  return cands_ready ? 3 : 4;
}

size_t items_capacity(int64_t max_groups, int64_t n_queries) {
  // every group yields at most ceil(q/32) + 1 items; every item holds >= 1 query
  const int64_t a = n_queries + max_groups + 32;
  return static_cast<size_t>(a);
}

}  // namespace fknn
