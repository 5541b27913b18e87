// Persistent grid-kNN query kernel for sm_100a.
//
// Semantics follow the reference production kernel
// (FlashKNN/csrc/flash_knn_query_dynamic_load.cu:469-652): every query gets
// the exact K smallest FP32 squared distances among the points of the 27
// candidate runs of its group, strict acceptance d < cut_r2, ascending output,
// (pad index, +inf) padding.  Equal distances are ordered by the lower index
// (the reference leaves their order to its network layout).
//
// Execution model (B200-first, not the reference's block-per-parent loop):
//   * persistent CTAs; each warp pulls work items from a device queue
//     (atomicAdd on Meta::queue_head);
//   * packed item: up to 32 consecutive queries from up to 32 consecutive
//     groups, one query per lane.  Each group's 27 runs are staged into the
//     warp's shared-memory tile by non-multicast cp.async.bulk copies that
//     complete on the warp's mbarrier.  Each group's candidates are then
//     counting-sorted (32 buckets of squared distance) by distance to the centroid of the
//     group's queries, so every lane fills its list with near candidates
//     first: the first KCAP candidates are sorted by a sorting network, the
//     rest go through a branch-free insertion network only when some lane
//     improves (warp vote), and a lane stops at the first bucket whose lower
//     distance bound exceeds its current K-th distance (triangle
//     inequality, with a safety margin for FP32 rounding);
//   * chunked item: one group with more candidates than a tile; G lanes per
//     query split its candidates, streamed tile by tile, and the G partial
//     lists are merged with xor-shuffle bitonic merges;
//   * lists hold packed u64 keys (distance bits << 32 | index), so ordering
//     is exact including ties; rows are written straight to the caller's
//     row / index space.
#include <algorithm>
#include <cfloat>
#include <mutex>
#include <vector>

#include "fknn_common.cuh"
#include "fknn_networks.cuh"
#include "fknn_internal.h"

namespace fknn {

constexpr uint64_t kEmpty = ~0ull;
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kBuckets = 32;
constexpr int kMaxOrderedGroup = 4096;  // queries: larger chunked groups keep record order

// Per-group scratch of the current packed item (shared memory, per warp).
struct GroupSlot {
  int seg;    // first tile slot of the group's candidates
  int len;    // number of candidates
  int a, b;   // the group's query range inside the item (query-record positions)
  float cx, cy, cz;  // centroid of those queries
  float inv_w2;      // 1 / bucket width in squared distance
  float eps;         // absolute margin of the early-exit bound
  int pad0, pad1, pad2;
};
static_assert(sizeof(GroupSlot) == 48, "GroupSlot layout");

// Staging buffers per warp (the autotuner's depth axis: 1 or 2).
constexpr int kMaxStaging = 2;

// Bytes of one warp's shared-memory region: `depth` staging buffers of T
// records (tile, group slots, flag) and one set of sort scratch.
__host__ __device__ constexpr size_t warp_smem_bytes(int T, int depth) {
  return ((static_cast<size_t>(depth) *
               (static_cast<size_t>(T) * 16 + kMaxGroupsPerItem * sizeof(GroupSlot) + 16) +
           static_cast<size_t>(T) * 4 + kMaxGroupsPerItem * (kBuckets + 1) * 2 + 32 +
           kBuckets * 4 + 127) /
          128) *
         128;
}

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

__device__ __forceinline__ uint64_t make_key(float d, float w) {
  return (static_cast<uint64_t>(__float_as_uint(d)) << 32) |
         static_cast<uint32_t>(__float_as_int(w));
}

// Insert x into the ascending list L, dropping the largest entry.  Slot j
// becomes min(L[j], max(x, L[j-1])): every slot is computed from the old
// list, so the network has no serial dependency.  x == kEmpty is a no-op.
template <int KCAP>
__device__ __forceinline__ void list_insert(uint64_t (&L)[KCAP], uint64_t x) {
#pragma unroll
  for (int j = KCAP - 1; j >= 1; --j) {
    const bool cj = x < L[j];
    const bool cm = x < L[j - 1];
    L[j] = cj ? (cm ? L[j - 1] : x) : L[j];
  }
  L[0] = x < L[0] ? x : L[0];
}

// The same network over the upper half only: valid when x does not belong
// in the lower half (x >= L[KCAP/2 - 1]), which leaves that half unchanged.
template <int KCAP>
__device__ __forceinline__ void list_insert_upper(uint64_t (&L)[KCAP], uint64_t x) {
#pragma unroll
  for (int j = KCAP - 1; j >= KCAP / 2; --j) {
    const bool cj = x < L[j];
    const bool cm = x < L[j - 1];
    L[j] = cj ? (cm ? L[j - 1] : x) : L[j];
  }
}

template <int KCAP>
__device__ __forceinline__ void cas(uint64_t (&L)[KCAP], int i, int j, bool ascending) {
  const uint64_t a = L[i], b = L[j];
  const bool sw = ascending ? (b < a) : (a < b);
  L[i] = sw ? b : a;
  L[j] = sw ? a : b;
}

// Inserts x (kEmpty = none).  Late improvements mostly belong in the upper
// half of the list: when that holds for every lane, only that half is
// updated.
template <int KCAP>
__device__ __forceinline__ void insert_one(uint64_t (&L)[KCAP], uint64_t x) {
  if constexpr (KCAP >= 8) {
    if (__all_sync(kFull, x >= L[KCAP / 2 - 1])) {
      list_insert_upper<KCAP>(L, x);
      return;
    }
  }
  list_insert<KCAP>(L, x);
}

template <int KCAP>
__device__ __forceinline__ void bitonic_clean_ascending(uint64_t (&L)[KCAP]) {
#pragma unroll
  for (int st = KCAP / 2; st > 0; st >>= 1) {
#pragma unroll
    for (int j = 0; j < KCAP; ++j)
      if ((j & st) == 0) cas<KCAP>(L, j, j + st, true);
  }
}

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int mask) {
  const uint32_t lo = __shfl_xor_sync(kFull, static_cast<uint32_t>(v), mask);
  const uint32_t hi = __shfl_xor_sync(kFull, static_cast<uint32_t>(v >> 32), mask);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Keep the KCAP smallest of this lane's list and the list of lane ^ mask.
template <int KCAP>
__device__ __forceinline__ void merge_with_lane(uint64_t (&L)[KCAP], int mask) {
  if constexpr (KCAP == 1) {
    L[0] = umin64(L[0], shfl_xor_u64(L[0], mask));
  } else {
#pragma unroll
    for (int j = 0; j < KCAP / 2; ++j) {
      const uint64_t a = L[j], b = L[KCAP - 1 - j];
      const uint64_t pa = shfl_xor_u64(b, mask);  // partner's L[KCAP-1-j]
      const uint64_t pb = shfl_xor_u64(a, mask);  // partner's L[j]
      L[j] = umin64(a, pa);
      L[KCAP - 1 - j] = umin64(b, pb);
    }
    bitonic_clean_ascending<KCAP>(L);
  }
}

// Acceptance of a candidate at squared distance d (>= +0 or NaN): d < cut_r2
// and d no larger than the current K-th.  For non-negative floats the order
// of the bit patterns is the order of the values, so d < cut_r2 is
// bits(d) <= bits(cut_r2) - 1 and both tests fold into one unsigned
// threshold min(K-th bits, cut_limit).  NaN and +inf lie above every limit.
// cut_r2 <= 0 (or NaN) accepts nothing: queries then take no candidate.
__device__ __forceinline__ bool cut_accepts_any(float cut_r2) { return cut_r2 > 0.f; }

__device__ __forceinline__ uint32_t cut_limit(float cut_r2) {
  return __float_as_uint(cut_r2) - 1u;  // valid when cut_accepts_any(cut_r2)
}

__device__ __forceinline__ uint32_t kth_limit(uint64_t last, uint32_t cut_lim) {
  return min(static_cast<uint32_t>(last >> 32), cut_lim);
}

__device__ __forceinline__ int ceil_log2(int v) { return v <= 1 ? 0 : 32 - __clz(v - 1); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(kFull, v, s);
  return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, s));
  return v;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
      : "memory");
}

// First sorted position whose bucket cannot hold a candidate closer than the
// lane's current KCAP-th distance.  Buckets are uniform in the squared
// distance to the centroid: a candidate in bucket b lies at least
// sqrt(b*w2) from the centroid, hence at least sqrt(b*w2) - rq from the
// query; buckets with b*w2 > (rq + sqrt(thr))^2 (plus margins) are skipped.
template <int KCAP>
__device__ __forceinline__ int stop_position(const uint64_t (&L)[KCAP], const GroupSlot& s,
                                             float rq, const uint16_t* bstart) {
  const uint64_t last = L[KCAP - 1];
  if (last == kEmpty) return s.len;
  // m * rsqrt(m) is within a few ulp of sqrt(m), far inside the 1e-4 margin;
  // m >= FLT_MIN keeps a K-th distance of 0 (a query on a support point) or
  // a subnormal one bounded from above, and +inf gives NaN, which skips no
  // bucket
  const float m = fmaxf(__uint_as_float(static_cast<uint32_t>(last >> 32)), FLT_MIN);
  const float reach = rq + m * rsqrtf(m) * 1.0001f + s.eps;
  const float lim = reach * reach * s.inv_w2;
  if (!(lim < static_cast<float>(kBuckets - 1))) return s.len;
  return bstart[static_cast<int>(lim) + 1];
}

template <typename IdxT, int KCAP, bool EXACT>
__device__ __forceinline__ void write_row(const QueryLaunch& a, const uint64_t (&L)[KCAP], int row,
                                          int k) {
  if (row < 0 || row >= a.n_rows) {
    raise_status(&a.meta->status, kStatusTable);
    return;
  }
  int64_t pad;
  switch (a.pad_mode) {
    case kPadArray64: pad = static_cast<const int64_t*>(a.pad)[row]; break;
    case kPadArray32: pad = static_cast<const int32_t*>(a.pad)[row]; break;
    case kPadMinusOne: pad = -1; break;
    default: pad = row; break;
  }
  IdxT* io = static_cast<IdxT*>(a.idx_out) + static_cast<int64_t>(row) * k;
  float* dout = a.dist_out + static_cast<int64_t>(row) * k;
  if (EXACT && (KCAP % 4) == 0 && a.vec_ok) {
#pragma unroll
    for (int j = 0; j < KCAP; j += 4) {
      float4 dv;
      IdxT iv[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const uint64_t e = L[j + t];
        const bool empty = e == kEmpty;
        iv[t] = empty ? static_cast<IdxT>(pad) : static_cast<IdxT>(static_cast<int32_t>(e));
        reinterpret_cast<float*>(&dv)[t] =
            empty ? __int_as_float(0x7f800000) : __uint_as_float(static_cast<uint32_t>(e >> 32));
      }
      *reinterpret_cast<float4*>(dout + j) = dv;
      if constexpr (sizeof(IdxT) == 4) {
        *reinterpret_cast<int4*>(io + j) = make_int4(iv[0], iv[1], iv[2], iv[3]);
      } else {
        *reinterpret_cast<longlong2*>(io + j) = make_longlong2(iv[0], iv[1]);
        *reinterpret_cast<longlong2*>(io + j + 2) = make_longlong2(iv[2], iv[3]);
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < KCAP; ++j) {
      if (j < k) {
        const uint64_t e = L[j];
        const bool empty = e == kEmpty;
        io[j] = empty ? static_cast<IdxT>(pad) : static_cast<IdxT>(static_cast<int32_t>(e));
        dout[j] = empty ? __int_as_float(0x7f800000) : __uint_as_float(static_cast<uint32_t>(e >> 32));
      }
    }
  }
}

__device__ __forceinline__ int2 load_run(const QueryLaunch& a, int row, int lane) {
  int2 run = make_int2(0, 0);
  if (lane < kNeighbours) run = a.runs[static_cast<int64_t>(row) * kNeighbours + lane];
  if (run.y < 0 || run.x < 0 || static_cast<int64_t>(run.x) + run.y > a.n_support) {
    raise_status(&a.meta->status, kStatusTable);
    run.y = 0;
  }
  return run;
}

// Record of query qi of a chunked item (queries q0 .. q0+qn-1 of group g0):
// the group's queries taken in octant-major order around their centroid
// (the packer cuts a chunked group into consecutive items from its first
// query, so the item covering positions [q0 - start, q0 - start + qn) of
// that order takes those queries), so every query belongs to exactly one
// item and an item's queries are close together.  A group the item holds
// whole, or one of more than kMaxOrderedGroup queries, keeps record order.
// qlist: 32 ints of scratch; hist: 8 counters.  Kept out of line so its
// registers do not add to the packed path's.
__device__ __noinline__ int ordered_query_row(const float4* __restrict__ qrec,
                                              const int32_t* __restrict__ group_start, int g0,
                                              int q0, int qn, int qi, bool active, int* qlist,
                                              uint32_t* hist) {
  const int lane = threadIdx.x & 31;
  const int gq0 = group_start[g0], gq1 = group_start[g0 + 1];
  const int nqg = gq1 - gq0;
  if (!(nqg > qn && nqg <= kMaxOrderedGroup && q0 >= gq0 && q0 + qn <= gq1))
    return q0 + qi;
  float gx = 0.f, gy = 0.f, gz = 0.f;
  for (int t = lane; t < nqg; t += 32) {
    const float4 v = qrec[gq0 + t];
    gx += v.x;
    gy += v.y;
    gz += v.z;
  }
  const float inv = 1.f / static_cast<float>(nqg);
  gx = warp_sum(gx) * inv;
  gy = warp_sum(gy) * inv;
  gz = warp_sum(gz) * inv;
  auto octant = [&](int t) {
    const float4 v = qrec[gq0 + t];
    return (v.x > gx ? 1 : 0) | (v.y > gy ? 2 : 0) | (v.z > gz ? 4 : 0);
  };
  if (lane < 8) hist[lane] = 0u;
  __syncwarp();
  for (int t = lane; t < nqg; t += 32) atomicAdd(&hist[octant(t)], 1u);
  __syncwarp();
  const uint32_t h = lane < 8 ? hist[lane] : 0u;
  const uint32_t off = static_cast<uint32_t>(warp_inclusive_scan(static_cast<int>(h))) - h;
  __syncwarp();
  if (lane < 8) hist[lane] = off;  // running position of each octant
  __syncwarp();
  const int first = q0 - gq0;
  for (int t0 = 0; t0 < nqg; t0 += 32) {
    const int t = t0 + lane;
    const int o = t < nqg ? octant(t) : 8;
    const uint32_t peers = __match_any_sync(kFull, o);
    int pos = -1;
    if (o < 8) pos = static_cast<int>(hist[o]) + __popc(peers & lanemask_lt());
    __syncwarp();
    if (o < 8 && lane == __ffs(peers) - 1) hist[o] += __popc(peers);
    if (pos >= first && pos < first + qn) qlist[pos - first] = gq0 + t;
    __syncwarp();
  }
  const int row = active ? qlist[qi] : q0 + qi;
  __syncwarp();
  return row;
}

// Register budget per list length (CTAs have at most 256 threads).  Without
// one, ptxas holds the 16-entry kernels to 64 registers and spills; 96 still
// fits the 20 resident warps per SM that the default tile's shared memory
// allows.  Lists of up to 8 entries fit in 80 without spilling.
template <int KCAP>
constexpr int query_max_regs() {
  return KCAP <= 8 ? 80 : (KCAP <= 16 ? 96 : (KCAP <= 32 ? 128 : 224));
}

// A chunked item: one group with more candidates than a tile.  Out of line,
// so its registers do not add to the packed path's.  Returns the mbarrier's
// next phase, or -1 after a bounded wait gave up (status raised; the warp
// waited once more, bounded, for its copies, and raised kStatusCopyInFlight
// if they still had not landed).
template <int KCAP, bool EXACT, typename IdxT>
__device__ __noinline__ int chunked_item(const QueryLaunch& a, int T, int min_cands_per_lane,
                                         int q0, int qn, int g0, int k, float4* tile,
                                         uint16_t* srt16, uint32_t* hist, uint64_t* bar,
                                         uint32_t phase) {
  const int lane = threadIdx.x & 31;
  // One group with more candidates than a tile, up to 32 of its queries,
  // G lanes per query.  Phase A scans the first runs (the group's own
  // cell first) until they hold 2K candidates; the G partial lists of a
  // query are then merged, so every query knows its K-th distance over
  // those candidates, an upper bound of its final K-th.  A later
  // candidate can only enter the top-K of some query q if its distance to
  // the queries' centroid c is at most |q - c| + K-th(q) <= R + D (R, D:
  // the item's largest), so phase B scans, tile by tile, only the
  // candidates inside that sphere (with a margin for FP32 rounding).
  const int row = a.group_row ? a.group_row[g0] : g0;
  const int2 run = load_run(a, row, lane);
  const int incl = warp_inclusive_scan(run.y);
  const int total = __shfl_sync(kFull, incl, 31);
  const int run_off = incl - run.y;
  int lg = 5 - ceil_log2(qn);
  while (lg > 0 && (total >> lg) < min_cands_per_lane) --lg;
  const int G = 1 << lg;
  const int qi = lane >> lg, sub = lane & (G - 1);
  const bool active = qi < qn;
  const bool takes = active && cut_accepts_any(a.cut_r2);
  // The packer cuts the group's queries into items in record order: take
  // them instead in octant-major order
  // (ordered_query_row), so an item's queries are close together and the
  // phase-B sphere below stays small.
  const int qrow = ordered_query_row(a.qrec, a.group_start, g0, q0, qn, qi, active,
                                     reinterpret_cast<int*>(tile), hist);
  float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
  if (active) q = a.qrec[qrow];
  // phase A: whole runs until 2K candidates (all of them when fewer)
  const uint32_t long_enough = __ballot_sync(kFull, lane < kNeighbours && incl >= 2 * KCAP);
  const int a_end = long_enough ? __shfl_sync(kFull, incl, __ffs(long_enough) - 1) : total;
  // centroid of the item's queries and their largest distance to it
  const bool head = active && sub == 0;
  const float inv_qn = 1.f / static_cast<float>(qn);
  const float cx = warp_sum(head ? q.x : 0.f) * inv_qn;
  const float cy = warp_sum(head ? q.y : 0.f) * inv_qn;
  const float cz = warp_sum(head ? q.z : 0.f) * inv_qn;
  const float qx = q.x - cx, qy = q.y - cy, qz = q.z - cz;
  const float rq = sqrtf(warp_max(head ? qx * qx + qy * qy + qz * qz : 0.f));
  uint64_t L[KCAP];
#pragma unroll
  for (int j = 0; j < KCAP; ++j) L[j] = kEmpty;
  const uint32_t cut_lim = cut_limit(a.cut_r2);
  uint32_t thr = cut_lim, qthr = cut_lim;
  bool timed_out = false;
  float rad2 = 0.f;
  // Stage the candidates [lo, hi) of the concatenated runs tile by tile;
  // with `filter`, keep those within sqrt(rad2) of the centroid.
  auto scan_range = [&](int lo_c, int hi_c, bool filter) {
    for (int c0 = lo_c; c0 < hi_c && !timed_out; c0 += T) {
      const int c1 = min(hi_c, c0 + T);
      __syncwarp();
      fence_proxy_async_smem();  // earlier generic reads of the tile precede the copies
      if (lane == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(c1 - c0) * 16u);
      __syncwarp();
      const int lo = max(run_off, c0), hi = min(run_off + run.y, c1);
      if (hi > lo)
        bulk_copy_g2s(tile + (lo - c0), a.srec + run.x + (lo - run_off),
                      static_cast<uint32_t>(hi - lo) * 16u, bar);
      if (!mbar_wait_bounded(bar, phase, kWaitLimit)) {
        timed_out = true;
        break;
      }
      phase ^= 1u;
      int cnt = c1 - c0;
      if (filter) {  // compact the tile to the candidates inside the sphere
        int m = 0;
        for (int t0 = 0; t0 < cnt; t0 += 32) {
          const int t = t0 + lane;
          bool keep = false;
          if (t < cnt) {
            const float4 c = tile[t];
            const float dx = c.x - cx, dy = c.y - cy, dz = c.z - cz;
            keep = dx * dx + dy * dy + dz * dz <= rad2;
          }
          const uint32_t b = __ballot_sync(kFull, keep);
          if (keep) srt16[m + __popc(b & lanemask_lt())] = static_cast<uint16_t>(t);
          m += __popc(b);
        }
        __syncwarp();
        cnt = m;
      }
      for (int i0 = 0; i0 < cnt; i0 += G) {
        const int i = i0 + sub;
        const bool ok = takes && i < cnt;
        const float4 c = ok ? tile[filter ? srt16[i] : i] : q;
        const float d = sq_dist(c.x, c.y, c.z, q.x, q.y, q.z);
        const uint32_t db = __float_as_uint(d);
        const bool acc = ok && db <= thr;
        if (__any_sync(kFull, acc)) {
          list_insert<KCAP>(L, acc ? make_key(d, c.w) : kEmpty);
          thr = min(kth_limit(L[KCAP - 1], cut_lim), qthr);
        }
      }
    }
  };
  scan_range(0, a_end, false);
  if (!timed_out && a_end < total) {
    for (int m = 1; m < G; m <<= 1) merge_with_lane<KCAP>(L, m);
    qthr = kth_limit(L[KCAP - 1], cut_lim);  // the query's bound (same in its G lanes)
    thr = qthr;
    if (sub != 0) {  // its candidates now live in lane sub == 0 only
#pragma unroll
      for (int j = 0; j < KCAP; ++j) L[j] = kEmpty;
    }
    const float d2 = warp_max(active ? __uint_as_float(qthr) : 0.f);
    const float mag = fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz))) + rq;
    const float rad = (rq + sqrtf(d2)) * 1.00001f + mag * 4e-6f + 1e-30f;
    rad2 = rad * rad * 1.00001f;
    scan_range(a_end, total, rad2 <= 3.0e38f);
  }
  if (timed_out) {  // no copy was issued after the wait that gave up
    if (lane == 0) raise_status(&a.meta->status, kStatusTimeout);
    const bool landed = mbar_wait_bounded(bar, phase, kWaitLimit);  // let them land
    if (!__all_sync(kFull, landed) && lane == 0)
      raise_status(&a.meta->status, kStatusCopyInFlight);
    return -1;
  }
  for (int m = 1; m < G; m <<= 1) merge_with_lane<KCAP>(L, m);
  if (active && sub == 0) write_row<IdxT, KCAP, EXACT>(a, L, __float_as_int(q.w), k);
  return static_cast<int>(phase);
}

// Shared memory of one staging buffer of a warp: the candidate tile, the
// item's group slots and a flag word (1 = the item's groups overflowed the
// tile, which only a malformed item can cause).
__host__ __device__ constexpr size_t buffer_bytes(int T) {
  return static_cast<size_t>(T) * 16 + kMaxGroupsPerItem * sizeof(GroupSlot) + 16;
}

// One warp's shared memory: `depth` staging buffers (at buf0 + b * stride)
// and their mbarriers, then the sort scratch shared by the buffers.
struct WarpSmem {
  unsigned char* buf0;
  size_t stride;
  int T;
  uint64_t* bars;
  uint16_t* tmp16;
  uint16_t* srt16;
  uint16_t* bstart;
  uint8_t* qgroup;
  uint32_t* hist;
  __device__ __forceinline__ float4* tile(int b) const {
    return reinterpret_cast<float4*>(buf0 + b * stride);
  }
  __device__ __forceinline__ GroupSlot* slots(int b) const {
    return reinterpret_cast<GroupSlot*>(buf0 + b * stride + static_cast<size_t>(T) * 16);
  }
  __device__ __forceinline__ int* flags(int b) const {
    return reinterpret_cast<int*>(slots(b) + kMaxGroupsPerItem);
  }
  __device__ __forceinline__ uint64_t* bar(int b) const { return bars + b; }
};

__device__ __forceinline__ WarpSmem warp_smem(unsigned char* smem_raw, int T, int depth) {
  const int warp = threadIdx.x >> 5;
  WarpSmem w;
  w.buf0 = smem_raw + 128 + static_cast<size_t>(warp) * warp_smem_bytes(T, depth);
  w.stride = buffer_bytes(T);
  w.T = T;
  w.bars = reinterpret_cast<uint64_t*>(smem_raw) + warp * kMaxStaging;
  w.tmp16 = reinterpret_cast<uint16_t*>(w.buf0 + static_cast<size_t>(depth) * buffer_bytes(T));
  w.srt16 = w.tmp16 + T;
  w.bstart = w.srt16 + T;
  w.qgroup = reinterpret_cast<uint8_t*>(w.bstart + kMaxGroupsPerItem * (kBuckets + 1));
  w.hist = reinterpret_cast<uint32_t*>(w.qgroup + 32);
  return w;
}

__device__ __forceinline__ int pop_item(Meta* meta) {
  int item = 0;
  if ((threadIdx.x & 31) == 0) item = atomicAdd(&meta->queue_head, 1);
  return __shfl_sync(kFull, item, 0);
}

// Checks item `item` and, for a packed item, issues the bulk copies of its
// groups' candidate runs into buffer b (completing on the buffer's
// mbarrier) and records the groups in the buffer's slots.  Returns 1 when
// copies were armed (the caller waits on the buffer's barrier), 0 for a
// chunked item (it streams its own tiles), -1 for a malformed item (status
// raised, nothing to do).
__device__ __forceinline__ int stage_item(const QueryLaunch& a, int item, int n_groups, int T,
                                          const WarpSmem& w, int b) {
  const int lane = threadIdx.x & 31;
  const int4 it = a.items[item];
  const int q0 = it.x, qn = it.y, g0 = it.z, gn = it.w & 0xffff;
  const bool chunked = (it.w & kItemChunked) != 0;
  if (q0 < 0 || qn < 1 || qn > 32 || static_cast<int64_t>(q0) + qn > a.n_qrec || g0 < 0 ||
      gn < 1 || gn > kMaxGroupsPerItem || g0 + gn > n_groups || (chunked && gn != 1)) {
    if (lane == 0) raise_status(&a.meta->status, kStatusTable);
    return -1;
  }
  if (chunked) return 0;
  int ga = 0, gb = 0, grow = 0;
  if (lane < gn) {
    const int g = g0 + lane;
    const int gs = a.group_start[g], ge = a.group_start[g + 1];
    ga = max(gs, q0);
    gb = max(ga, min(ge, q0 + qn));
    grow = a.group_row ? a.group_row[g] : g;
  }
  __syncwarp();
  fence_proxy_async_smem();  // earlier generic accesses of the tile precede the copies
  __syncwarp();
  float4* tile = w.tile(b);
  uint64_t* bar = w.bar(b);
  int seg = 0;
  bool overflow = false;
  for (int gi = 0; gi < gn; ++gi) {
    const int ga_ = __shfl_sync(kFull, ga, gi), gb_ = __shfl_sync(kFull, gb, gi);
    const int row = __shfl_sync(kFull, grow, gi);
    int len = 0;
    if (gb_ > ga_ && !overflow) {
      const int2 run = load_run(a, row, lane);
      const int incl = warp_inclusive_scan(run.y);
      len = __shfl_sync(kFull, incl, 31);
      if (seg + len > T) {
        overflow = true;
        len = 0;
      } else if (len > 0) {
        if (lane == 0) mbar_expect_tx(bar, static_cast<uint32_t>(len) * 16u);
        __syncwarp();
        if (run.y > 0)
          bulk_copy_g2s(tile + seg + (incl - run.y), a.srec + run.x,
                        static_cast<uint32_t>(run.y) * 16u, bar);
      }
    }
    if (lane == 0) {
      GroupSlot s{};
      s.seg = seg;
      s.len = len;
      s.a = ga_;
      s.b = overflow ? ga_ : gb_;
      w.slots(b)[gi] = s;
    }
    seg += len;
  }
  if (lane == 0) {
    *w.flags(b) = overflow ? 1 : 0;
    mbar_arrive(bar);
  }
  return 1;
}

// A packed item whose copies into buffer b have landed: up to 32 queries of
// up to 16 groups, one query per lane (see the file comment).
template <int KCAP, bool EXACT, typename IdxT>
__device__ __forceinline__ void packed_item(const QueryLaunch& a, int item, const WarpSmem& w,
                                            int b) {
  const int lane = threadIdx.x & 31;
  Meta* meta = a.meta;
  const int4 it = a.items[item];
  const int q0 = it.x, qn = it.y, gn = it.w & 0xffff;
  const float4* tile = w.tile(b);
  GroupSlot* slots = w.slots(b);
  uint16_t* tmp16 = w.tmp16;
  uint16_t* srt16 = w.srt16;
  uint16_t* bstart = w.bstart;
  uint8_t* qgroup = w.qgroup;
  uint32_t* hist = w.hist;
  const int k = a.k;
  if (*w.flags(b)) {  // the packer bounds every item by the tile; report a broken item
    if (lane == 0) raise_status(&meta->status, kStatusTable);
    return;
  }
  // query -> group map (0xff: a query no group of the item covers)
  qgroup[lane] = 0xffu;
  __syncwarp();
  if (lane < gn) {
    const GroupSlot s = slots[lane];
    for (int p = s.a; p < s.b; ++p) qgroup[p - q0] = static_cast<uint8_t>(lane);
  }
  __syncwarp();

  // Per group: centroid of its queries, distance buckets, counting sort.
  for (int gi = 0; gi < gn; ++gi) {
    const GroupSlot s = slots[gi];
    if (s.b <= s.a) continue;
    const int nq = s.b - s.a;
    float4 qv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane < nq) qv = a.qrec[s.a + lane];
    const float inv_nq = 1.f / static_cast<float>(nq);
    const float cx = warp_sum(qv.x) * inv_nq;
    const float cy = warp_sum(qv.y) * inv_nq;
    const float cz = warp_sum(qv.z) * inv_nq;
    float d2max = 0.f;
    for (int t = lane; t < s.len; t += 32) {
      const float4 c = tile[s.seg + t];
      const float dx = c.x - cx, dy = c.y - cy, dz = c.z - cz;
      d2max = fmaxf(d2max, dx * dx + dy * dy + dz * dz);
    }
    d2max = warp_max(d2max);
    const float w2 = d2max > 0.f ? d2max * (1.0f / kBuckets) * 1.0001f : 1.f;
    const float inv_w2 = 1.f / w2;
    hist[lane] = 0u;  // kBuckets == 32: one bucket per lane
    __syncwarp();
    // Bucket of every candidate and its rank inside the bucket.
    for (int t = lane; t < s.len; t += 32) {
      const float4 c = tile[s.seg + t];
      const float dx = c.x - cx, dy = c.y - cy, dz = c.z - cz;
      const int bkt = min(static_cast<int>((dx * dx + dy * dy + dz * dz) * inv_w2), kBuckets - 1);
      const uint32_t r = atomicAdd(&hist[bkt], 1u);
      tmp16[s.seg + t] = static_cast<uint16_t>((bkt << 10) | r);
    }
    __syncwarp();
    const uint32_t h = hist[lane];
    const uint32_t hi = static_cast<uint32_t>(warp_inclusive_scan(static_cast<int>(h)));
    uint16_t* bs = bstart + gi * (kBuckets + 1);
    bs[lane] = static_cast<uint16_t>(hi - h);
    if (lane == 31) bs[kBuckets] = static_cast<uint16_t>(hi);
    __syncwarp();
    hist[lane] = hi - h;
    __syncwarp();
    for (int t = lane; t < s.len; t += 32) {
      const uint16_t v = tmp16[s.seg + t];
      const int bkt = v >> 10;
      srt16[s.seg + hist[bkt] + (v & 1023)] = static_cast<uint16_t>(s.seg + t);
    }
    if (lane == 0) {
      const float mag = fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz))) + sqrtf(d2max);
      slots[gi].cx = cx;
      slots[gi].cy = cy;
      slots[gi].cz = cz;
      slots[gi].inv_w2 = inv_w2;
      slots[gi].eps = mag * 4e-6f + 1e-30f;
    }
    __syncwarp();
  }

  // One query per lane.
  const int mapped = lane < qn ? qgroup[lane] : 0;
  if (lane < qn && mapped >= gn) raise_status(&meta->status, kStatusTable);
  const bool active = lane < qn && mapped < gn;
  const int gi = active ? mapped : 0;
  const GroupSlot s = slots[gi];
  const uint16_t* bs = bstart + gi * (kBuckets + 1);
  float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
  if (active) q = a.qrec[q0 + lane];
  const float rdx = q.x - s.cx, rdy = q.y - s.cy, rdz = q.z - s.cz;
  const float rq = sqrtf(rdx * rdx + rdy * rdy + rdz * rdz);
  const int len = active && cut_accepts_any(a.cut_r2) ? s.len : 0;
  const uint32_t cut_lim = cut_limit(a.cut_r2);

  uint64_t L[KCAP];
#pragma unroll
  for (int j = 0; j < KCAP; ++j) {
    uint64_t key = kEmpty;
    if (j < len) {
      const float4 c = tile[srt16[s.seg + j]];
      const float d = sq_dist(c.x, c.y, c.z, q.x, q.y, q.z);
      if (__float_as_uint(d) <= cut_lim) key = make_key(d, c.w);
    }
    L[j] = key;
  }
  sort_network<KCAP, 0, KCAP>(L);
  uint32_t thr = kth_limit(L[KCAP - 1], cut_lim);
  int stop = len > 0 ? stop_position<KCAP>(L, s, rq, bs) : 0;
  // Candidate t of the lane's scan: accepted when it beats the K-th.
  auto test = [&](int t, uint64_t& x) {
    const float4 c = tile[srt16[s.seg + t]];
    const float d = sq_dist(c.x, c.y, c.z, q.x, q.y, q.z);
    const bool acc = __float_as_uint(d) <= thr;
    if (acc) x = make_key(d, c.w);
    return acc;
  };
  if constexpr (KCAP <= 16) {
    // Two candidates per iteration, both tested against the same K-th
    // distance: half the loop and vote overhead, and two independent loads
    // and distance chains in flight.  (With a 32- or 64-entry list the
    // extra registers cost more than this saves.)
    for (int t = KCAP;; t += 2) {
      const bool live0 = t < stop, live1 = t + 1 < stop;
      if (!__any_sync(kFull, live0)) break;
      uint64_t x0 = kEmpty, x1 = kEmpty;
      const bool acc0 = live0 && test(t, x0);
      const bool acc1 = live1 && test(t + 1, x1);
      // A lane that took only its second candidate inserts it in the first
      // step, so the second step runs only when some lane took both (the
      // list keeps the K smallest of what it is given, in any order).
      if (!acc0) {
        x0 = x1;
        x1 = kEmpty;
      }
      const bool any0 = __any_sync(kFull, acc0 || acc1);
      const bool any1 = __any_sync(kFull, acc0 && acc1);
      if (any0) insert_one<KCAP>(L, x0);
      if (any1) insert_one<KCAP>(L, x1);
      if (acc0 || acc1) {
        thr = kth_limit(L[KCAP - 1], cut_lim);
        stop = min(stop, stop_position<KCAP>(L, s, rq, bs));
      }
    }
  } else {
    for (int t = KCAP;; ++t) {
      const bool live = t < stop;
      if (!__any_sync(kFull, live)) break;
      uint64_t x = kEmpty;
      const bool acc = live && test(t, x);
      if (__any_sync(kFull, acc)) {
        insert_one<KCAP>(L, x);
        if (acc) {
          thr = kth_limit(L[KCAP - 1], cut_lim);
          stop = min(stop, stop_position<KCAP>(L, s, rq, bs));
        }
      }
    }
  }
  if (active) write_row<IdxT, KCAP, EXACT>(a, L, __float_as_int(q.w), k);
  __syncwarp();
}

// After a bounded wait gave up: waits once more (bounded) for every buffer
// that still has bulk copies in flight, so the warp does not leave while the
// copies write into its shared memory; if they still have not landed, says
// so with kStatusCopyInFlight.  The warp then stops; the other warps of its
// CTA (which keep the shared memory allocated) finish their own items.
__device__ __noinline__ void drain_after_timeout(Meta* meta, const WarpSmem& w, uint32_t phase,
                                                 uint32_t pending, int depth) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) raise_status(&meta->status, kStatusTimeout);
  bool landed = true;
  for (int b = 0; b < depth; ++b)
    if (((pending >> b) & 1u) && !mbar_wait_bounded(w.bar(b), (phase >> b) & 1u, kWaitLimit))
      landed = false;
  if (!__all_sync(kFull, landed) && lane == 0) raise_status(&meta->status, kStatusCopyInFlight);
}

// The persistent query kernel.  Each warp pulls items from the queue; with
// `depth` 2 it stages the next item's candidate runs into its second buffer
// before it scans the current one, so those copies are in flight while it
// computes.
template <int KCAP, bool EXACT, typename IdxT>
__global__ void __maxnreg__(query_max_regs<KCAP>())
    k_query(const __grid_constant__ QueryLaunch a, int T, int min_cands_per_lane, int depth) {
  chain_wait();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const WarpSmem w = warp_smem(smem_raw, T, depth);
  Meta* meta = a.meta;
  if (lane == 0) {
    for (int b = 0; b < depth; ++b) mbar_init(w.bar(b), 1);
    mbar_init_fence();
  }
  __syncwarp();
  // bit b: the parity to wait for on buffer b's barrier / copies armed there
  uint32_t phase = 0u, pending = 0u;
  const int n_items = meta->n_items;
  const int n_groups = *a.group_count_ptr;

  int buf = 0;
  int item = pop_item(meta);
  int staged = item < n_items ? stage_item(a, item, n_groups, T, w, buf) : -1;
  if (staged == 1) pending |= 1u << buf;
  while (item < n_items) {
    int next = n_items, next_staged = -1;
    if (depth > 1) {  // the next item's copies fly while this one is scanned
      next = pop_item(meta);
      if (next < n_items) next_staged = stage_item(a, next, n_groups, T, w, buf ^ 1);
      if (next_staged == 1) pending |= 1u << (buf ^ 1);
    }
    if (staged == 1) {
      if (!mbar_wait_bounded(w.bar(buf), (phase >> buf) & 1u, kWaitLimit)) {
        drain_after_timeout(meta, w, phase, pending, depth);
        return;
      }
      phase ^= 1u << buf;
      pending &= ~(1u << buf);
      packed_item<KCAP, EXACT, IdxT>(a, item, w, buf);
    } else if (staged == 0) {
      const int4 it = a.items[item];
      const int nxt = chunked_item<KCAP, EXACT, IdxT>(a, T, min_cands_per_lane, it.x, it.y, it.z,
                                                      a.k, w.tile(buf), w.srt16, w.hist,
                                                      w.bar(buf), (phase >> buf) & 1u);
      if (nxt < 0) {  // its own copies were waited for; the other buffer's may fly
        drain_after_timeout(meta, w, phase, pending, depth);
        return;
      }
      phase = (phase & ~(1u << buf)) | (static_cast<uint32_t>(nxt) << buf);
    }
    if (depth > 1) {
      buf ^= 1;
    } else {
      next = pop_item(meta);
      if (next < n_items) next_staged = stage_item(a, next, n_groups, T, w, buf);
      if (next_staged == 1) pending |= 1u << buf;
    }
    item = next;
    staged = next_staged;
  }
  __syncwarp();
}

// ------------------------------------------------------------------ host

QueryShape resolve_shape(const fknn_config* cfg) {
  QueryShape s{4, 448, 8, 0, 1};
  if (cfg) {
    if (cfg->warps_per_cta) s.warps_per_cta = cfg->warps_per_cta;
    if (cfg->tile_records) s.tile_records = cfg->tile_records;
    if (cfg->min_candidates_per_lane) s.min_candidates_per_lane = cfg->min_candidates_per_lane;
    s.ctas_per_sm = cfg->ctas_per_sm;
    if (cfg->staging_depth) s.staging_depth = cfg->staging_depth;
  }
  return s;
}

bool shape_valid(const QueryShape& s) {
  const bool warps_ok = s.warps_per_cta == 1 || s.warps_per_cta == 2 ||
                        s.warps_per_cta == 4 || s.warps_per_cta == 8;
  const bool depth_ok = s.staging_depth >= 1 && s.staging_depth <= kMaxStaging;
  return warps_ok && depth_ok && s.tile_records >= 64 && s.tile_records <= 1024 &&
         s.tile_records % 32 == 0 && s.min_candidates_per_lane >= 1 &&
         s.ctas_per_sm >= 0 && s.ctas_per_sm <= 32 &&
         128 + static_cast<size_t>(s.warps_per_cta) *
                   warp_smem_bytes(s.tile_records, s.staging_depth) <=
             227 * 1024;
}

namespace {

template <int KCAP, bool EXACT, typename IdxT>
int launch_t(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s) {
  auto kern = k_query<KCAP, EXACT, IdxT>;
  const int threads = shape.warps_per_cta * 32;
  const size_t smem = 128 + static_cast<size_t>(shape.warps_per_cta) *
                               warp_smem_bytes(shape.tile_records, shape.staging_depth);
  // Device properties and occupancy are resolved once per (device, shape) and
  // cached, so a launch inside a CUDA graph capture issues nothing but the
  // kernel itself.  The cache is shared by all host threads under a mutex,
  // and the kernel's dynamic shared-memory limit is raised once per device
  // to the device's opt-in maximum (less the kernel's static shared memory),
  // so a launch with one shape never lowers the limit under a concurrent
  // launch with a larger one.
  struct Cached {
    int dev, threads, per_sm, sms;
    size_t smem;
  };
  static std::mutex mu;
  static std::vector<Cached> cache;
  static std::vector<int> raised;  // devices whose limit is raised
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  Cached use{};
  {
    std::lock_guard<std::mutex> lock(mu);
    bool found = false;
    for (const Cached& c : cache)
      if (c.dev == dev && c.threads == threads && c.smem == smem) {
        use = c;
        found = true;
      }
    if (!found) {
      Cached c{dev, threads, 0, 0, smem};
      e = cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      if (std::find(raised.begin(), raised.end(), dev) == raised.end()) {
        int optin = 0;
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) return e;
        cudaFuncAttributes fa{};
        e = cudaFuncGetAttributes(&fa, kern);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - static_cast<int>(fa.sharedSizeBytes));
        if (e != cudaSuccess) return e;
        raised.push_back(dev);
      }
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.per_sm, kern, threads, smem);
      if (e != cudaSuccess) return e;
      if (c.per_sm < 1) c.per_sm = 1;
      cache.push_back(c);
      use = c;
    }
  }
  const int per_sm = shape.ctas_per_sm > 0 ? shape.ctas_per_sm : use.per_sm;
  const int grid = use.sms * per_sm;
  const int slot = profile_start(s);
  launch_chained(kern, grid, threads, smem, s, q, shape.tile_records, shape.min_candidates_per_lane,
      shape.staging_depth);
  e = cudaGetLastError();
  profile_stop(slot, s);
  return e;
}

template <int KCAP>
int launch_k(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s) {
  const bool exact = q.k == KCAP;
  if (q.idx_bits == 64)
    return exact ? launch_t<KCAP, true, int64_t>(q, shape, s)
                 : launch_t<KCAP, false, int64_t>(q, shape, s);
  return exact ? launch_t<KCAP, true, int32_t>(q, shape, s)
               : launch_t<KCAP, false, int32_t>(q, shape, s);
}

}  // namespace

int launch_query(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s) {
  if (q.k <= 1) return launch_k<1>(q, shape, s);
  if (q.k <= 2) return launch_k<2>(q, shape, s);
  if (q.k <= 4) return launch_k<4>(q, shape, s);
  if (q.k <= 8) return launch_k<8>(q, shape, s);
  if (q.k <= 16) return launch_k<16>(q, shape, s);
  if (q.k <= 32) return launch_k<32>(q, shape, s);
  return launch_k<64>(q, shape, s);
}

}  // namespace fknn
