// Backward of the squared distances returned by the kNN query.
//
// For d_ij = |p[idx_ij] - q_i|^2 and an upstream gradient g_ij:
//   grad_q[i] = sum_j 2 g_ij (q_i - p[idx_ij])          (one thread per query,
//                                                        j in ascending order)
//   grad_p[n] = sum_{idx_ij = n} -2 g_ij (q_i - p_n)     (segmented reduction)
// Every point's sum runs over its entries e = i*K+j in ascending e, so each
// FP32 operation happens in an order fixed by the inputs alone: the
// gradients are bitwise reproducible, and no floating-point atomics are used.
//
// The segments are built without global atomics (the bucketed path):
//   k_bwd_rows     row blocks of <= 32768 entries: grad_q, then each valid
//                  entry is placed in the block's own region of the entry
//                  array, grouped by bucket (point >> shift) through
//                  shared-memory counts, a block scan and shared-memory
//                  cursors; per (bucket, block) the run's start and length
//                  go to two small tables.  Entries are 4 bytes: the entry
//                  number within the block (15 bits) and the point within
//                  its bucket (up to 17 bits).
//   k_bwd_buckets  one CTA per bucket: gathers its runs from every block
//                  (in block order), counts entries per point, stages them
//                  grouped by point in shared memory (in passes over point
//                  ranges when a bucket holds more than the stage), orders
//                  each point's segment by e (a register sorting network, or
//                  a warp-cooperative selection when longer than 32) and sums
//                  it; a point with more entries than the whole stage is
//                  summed by a warp streaming the runs in block order.
// Sizes outside the bucketed path (K > 4096, or more buckets than a block's
// shared memory counts) take the counting-sort path below it: integer
// atomics count and place the segments, a scan, a scatter, one thread per
// point.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_networks.cuh"
#include "fknn_sort.cuh"
#include "fknn_backward.h"

#include <algorithm>
#include <mutex>
#include <vector>

namespace fknn {

namespace {

constexpr int kScanTile = 1024;
constexpr uint32_t kNoEntry = ~0u;

__device__ __forceinline__ bool entry_valid(int32_t t, int64_t n, float d) {
  return t >= 0 && t < n && !isinf(d);
}

}  // namespace

// One thread per query: grad_q over j in ascending order, and the size of
// every neighbour's segment (count[t], integer atomics).
__global__ void __launch_bounds__(256)
    k_bwd_query(const float* __restrict__ q_xyz, int64_t m, const float* __restrict__ p_xyz,
                int64_t n, const int32_t* __restrict__ idx, const float* __restrict__ dist,
                const float* __restrict__ grad, int k, float* __restrict__ grad_q, int accumulate,
                uint32_t* __restrict__ count, int vec4) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const float qx = q_xyz[3 * i], qy = q_xyz[3 * i + 1], qz = q_xyz[3 * i + 2];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  auto entry = [&](int32_t t, float d, float g) {
    if (!entry_valid(t, n, d)) return;
    if (count) atomicAdd(&count[t], 1u);
    if (!grad_q) return;
    const float g2 = 2.f * g;
    gx = __fmaf_rn(g2, __fsub_rn(qx, p_xyz[3 * static_cast<int64_t>(t)]), gx);
    gy = __fmaf_rn(g2, __fsub_rn(qy, p_xyz[3 * static_cast<int64_t>(t) + 1]), gy);
    gz = __fmaf_rn(g2, __fsub_rn(qz, p_xyz[3 * static_cast<int64_t>(t) + 2]), gz);
  };
  if (vec4) {  // k % 4 == 0 and 16-byte aligned rows: 128-bit row loads, j ascending
    const int4* i4 = reinterpret_cast<const int4*>(idx + i * k);
    const float4* d4 = reinterpret_cast<const float4*>(dist + i * k);
    const float4* g4 = reinterpret_cast<const float4*>(grad + i * k);
    for (int j = 0; j < (k >> 2); ++j) {
      const int4 t = i4[j];
      const float4 d = d4[j], g = g4[j];
      entry(t.x, d.x, g.x);
      entry(t.y, d.y, g.y);
      entry(t.z, d.z, g.z);
      entry(t.w, d.w, g.w);
    }
  } else {
    for (int j = 0; j < k; ++j) {
      const int64_t e = i * k + j;
      entry(idx[e], dist[e], grad[e]);
    }
  }
  if (grad_q) {
    if (accumulate) {
      gx = __fadd_rn(grad_q[3 * i], gx);
      gy = __fadd_rn(grad_q[3 * i + 1], gy);
      gz = __fadd_rn(grad_q[3 * i + 2], gz);
    }
    grad_q[3 * i] = gx;
    grad_q[3 * i + 1] = gy;
    grad_q[3 * i + 2] = gz;
  }
}

// Segment sizes summed per tile of kScanTile support points.
__global__ void __launch_bounds__(kScanTile)
    k_bwd_tile_sums(const uint32_t* __restrict__ count, int64_t n,
                    uint32_t* __restrict__ tile_sums) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int64_t p = static_cast<int64_t>(blockIdx.x) * kScanTile + threadIdx.x;
  block_inclusive_scan(p < n ? count[p] : 0u, warp_sums, &s_total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = s_total;
}

// start[p] = first slot of p's segment, cursor[p] = one past its last slot
// (the scatter counts it down); start[n] = number of valid entries.
__global__ void __launch_bounds__(kScanTile)
    k_bwd_starts(const uint32_t* __restrict__ count, int64_t n,
                 const uint32_t* __restrict__ tile_offsets, uint32_t* __restrict__ start,
                 uint32_t* __restrict__ cursor) {
  __shared__ uint32_t warp_sums[32];
  const int64_t p = static_cast<int64_t>(blockIdx.x) * kScanTile + threadIdx.x;
  const uint32_t c = p < n ? count[p] : 0u;
  const uint32_t incl = block_inclusive_scan(c, warp_sums, nullptr) + tile_offsets[blockIdx.x];
  if (p < n) {
    start[p] = incl - c;
    cursor[p] = incl;
    if (p == n - 1) start[n] = incl;
  }
}

// One thread per entry: scatter the entry number e into the segment of its
// neighbour (4 bytes per entry).  The slot order inside a segment depends on
// the scheduling; the reduction below orders each segment by e.
__global__ void __launch_bounds__(256)
    k_bwd_scatter(int64_t total, int64_t n, const int32_t* __restrict__ idx,
                  const float* __restrict__ dist, uint32_t* __restrict__ cursor,
                  uint32_t* __restrict__ seg, int vec4) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  auto put = [&](int64_t e, int32_t t, float d) {
    if (!entry_valid(t, n, d)) return;
    seg[atomicSub(&cursor[t], 1u) - 1u] = static_cast<uint32_t>(e);
  };
  if (vec4) {  // total % 4 == 0, 16-byte aligned: four entries (and atomics) in flight
    for (int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         w < (total >> 2); w += stride) {
      const int4 t = reinterpret_cast<const int4*>(idx)[w];
      const float4 d = reinterpret_cast<const float4*>(dist)[w];
      put(4 * w, t.x, d.x);
      put(4 * w + 1, t.y, d.y);
      put(4 * w + 2, t.z, d.z);
      put(4 * w + 3, t.w, d.w);
    }
    return;
  }
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += stride)
    put(e, idx[e], dist[e]);
}

namespace {

struct Acc {
  float x = 0.f, y = 0.f, z = 0.f;
};

// Query row i = e / K of an entry number e < 2^31 without a division
// instruction: Granlund and Montgomery's method for an invariant unsigned
// divisor ("Division by invariant integers using multiplication", PLDI
// 1994): with l = ceil(log2 K) and mul = floor(2^32 (2^l - K) / K) + 1,
// t = umulhi(mul, e) and e / K = (t + ((e - t) >> min(l, 1))) >> max(l - 1, 0).
struct DivK {
  uint32_t mul;
  int s1, s2;
};

DivK make_divk(uint32_t d) {
  int l = 0;
  while ((1ull << l) < d) ++l;
  DivK r;
  r.mul = static_cast<uint32_t>(((1ull << 32) * ((1ull << l) - d)) / d + 1);
  r.s1 = l < 1 ? l : 1;
  r.s2 = l > 1 ? l - 1 : 0;
  return r;
}

__device__ __forceinline__ uint32_t div_k(uint32_t e, const DivK& dk) {
  const uint32_t t = __umulhi(dk.mul, e);
  return (t + ((e - t) >> dk.s1)) >> dk.s2;
}

// One term of the reference-side sum, in the order the caller fixes:
// entry e = i*K+j adds -2 g_e (q_i - p).
__device__ __forceinline__ void add_entry(Acc& a, uint32_t e, const float* __restrict__ q_xyz,
                                          const float* __restrict__ grad, const DivK& k, float px,
                                          float py, float pz) {
  const int64_t i = div_k(e, k);
  const float g2 = __fmul_rn(-2.f, grad[e]);
  a.x = __fmaf_rn(g2, __fsub_rn(q_xyz[3 * i], px), a.x);
  a.y = __fmaf_rn(g2, __fsub_rn(q_xyz[3 * i + 1], py), a.y);
  a.z = __fmaf_rn(g2, __fsub_rn(q_xyz[3 * i + 2], pz), a.z);
}

// Sorts a segment of at most CAP entries in registers and sums it.
template <int CAP>
__device__ __forceinline__ void sum_short(Acc& a, const uint32_t* __restrict__ seg, uint32_t len,
                                          const float* __restrict__ q_xyz,
                                          const float* __restrict__ grad, const DivK& k, float px,
                                          float py, float pz) {
  uint32_t L[CAP];
#pragma unroll
  for (int c = 0; c < CAP; ++c) L[c] = c < static_cast<int>(len) ? seg[c] : kNoEntry;
  sort_network<CAP, 0, CAP>(L);
#pragma unroll
  for (int c = 0; c < CAP; ++c)
    if (c < static_cast<int>(len)) add_entry(a, L[c], q_xyz, grad, k, px, py, pz);
}

}  // namespace

// One thread per support point: its segment in ascending e, summed in that
// order.  Segments of more than 32 entries (hub points: many queries share
// them as a neighbour) are taken by the whole warp, one at a time: every
// round the warp selects the smallest remaining e (entries are distinct),
// so the order and the arithmetic are those of the short path.
__global__ void __maxnreg__(96)
    k_bwd_support(const float* __restrict__ q_xyz, const float* __restrict__ p_xyz, int64_t n,
                  DivK k, const uint32_t* __restrict__ start, const uint32_t* __restrict__ seg,
                  const float* __restrict__ grad, float* __restrict__ grad_p, int accumulate) {
  const int64_t p0 = static_cast<int64_t>(blockIdx.x) * blockDim.x;
  if (p0 >= n) return;  // whole warps leave together: n is the same for all
  const int64_t p = p0 + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool live = p < n;
  uint32_t s = 0, len = 0;
  float px = 0.f, py = 0.f, pz = 0.f;
  if (live) {
    s = start[p];
    len = start[p + 1] - s;
    px = p_xyz[3 * p];
    py = p_xyz[3 * p + 1];
    pz = p_xyz[3 * p + 2];
  }
  Acc a;
  const bool long_seg = len > 32;
  if (__any_sync(kFull, !long_seg && len > 16)) {
    if (!long_seg) sum_short<32>(a, seg + s, len, q_xyz, grad, k, px, py, pz);
  } else if (!long_seg && len > 0) {
    sum_short<16>(a, seg + s, len, q_xyz, grad, k, px, py, pz);
  }
  uint32_t todo = __ballot_sync(kFull, long_seg);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t ls = __shfl_sync(kFull, s, leader);
    const uint32_t ll = __shfl_sync(kFull, len, leader);
    const float lx = __shfl_sync(kFull, px, leader);
    const float ly = __shfl_sync(kFull, py, leader);
    const float lz = __shfl_sync(kFull, pz, leader);
    Acc b;
    uint32_t last = 0;
    for (uint32_t r = 0; r < ll; ++r) {
      uint32_t best = kNoEntry;
      for (uint32_t t = lane; t < ll; t += 32) {
        const uint32_t v = seg[ls + t];
        if ((r == 0 || v > last) && v < best) best = v;
      }
      best = __reduce_min_sync(kFull, best);
      add_entry(b, best, q_xyz, grad, k, lx, ly, lz);
      last = best;
    }
    if (lane == leader) a = b;
  }
  if (!live) return;
  if (accumulate) {
    a.x = __fadd_rn(grad_p[3 * p], a.x);
    a.y = __fadd_rn(grad_p[3 * p + 1], a.y);
    a.z = __fadd_rn(grad_p[3 * p + 2], a.z);
  }
  grad_p[3 * p] = a.x;
  grad_p[3 * p + 1] = a.y;
  grad_p[3 * p + 2] = a.z;
}

// --------------------------------------------------------- bucketed path

constexpr int kRowThreads = 1024;
constexpr int kEntriesPerRowBlock = 32768;  // entry numbers within a block fit 15 bits
constexpr int kLocalBits = 15;
constexpr uint32_t kLocalMask = (1u << kLocalBits) - 1u;
constexpr int kBucketThreads = 256;
constexpr int kStageCap = 12288;            // entries staged per bucket pass (48 KB)
constexpr int kMinShift = 6, kMaxShift = 12;
constexpr int kMaxRowBuckets = 16384;

struct BucketPlan {
  int64_t rows_per_block;  // rows of a row block (rows * K <= 32768)
  int64_t n_blocks;        // row blocks
  int64_t n_buckets;       // point buckets of 2^shift points
  int shift;
  int ok;                  // 0: sizes outside the bucketed path
};

BucketPlan bucket_plan(int64_t m, int64_t n, int k) {
  BucketPlan p{};
  if (k < 1 || k > 4096 || m <= 0 || n <= 0) return p;
  p.rows_per_block = kEntriesPerRowBlock / k;
  p.n_blocks = ceil_div(m, p.rows_per_block);
  // buckets holding about two thirds of the stage on average
  const double per_point = static_cast<double>(m) * k / static_cast<double>(n);
  int shift = kMinShift;
  while (shift < kMaxShift &&
         static_cast<double>(int64_t{1} << (shift + 1)) * per_point <= kStageCap * 2.0 / 3.0)
    ++shift;
  p.shift = shift;
  p.n_buckets = ceil_div(n, int64_t{1} << shift);
  p.ok = p.n_buckets <= kMaxRowBuckets ? 1 : 0;
  return p;
}

// Calls f(j, idx, dist, grad) for the entries of row i in ascending j; with
// vec4 (K % 4 == 0, 16-byte aligned rows) through 128-bit row loads.  grad
// may be null (f then gets 0).
template <typename F>
__device__ __forceinline__ void for_row_entries(const int32_t* __restrict__ idx,
                                                const float* __restrict__ dist,
                                                const float* __restrict__ grad, int64_t i, int k,
                                                int vec4, F&& f) {
  if (vec4) {
    const int4* i4 = reinterpret_cast<const int4*>(idx + i * k);
    const float4* d4 = reinterpret_cast<const float4*>(dist + i * k);
    const float4* g4 = grad ? reinterpret_cast<const float4*>(grad + i * k) : nullptr;
    for (int j = 0; j < (k >> 2); ++j) {
      const int4 t = i4[j];
      const float4 d = d4[j];
      const float4 g = g4 ? g4[j] : make_float4(0.f, 0.f, 0.f, 0.f);
      f(4 * j, t.x, d.x, g.x);
      f(4 * j + 1, t.y, d.y, g.y);
      f(4 * j + 2, t.z, d.z, g.z);
      f(4 * j + 3, t.w, d.w, g.w);
    }
  } else {
    for (int j = 0; j < k; ++j) {
      const int64_t e = i * k + j;
      f(j, idx[e], dist[e], grad ? grad[e] : 0.f);
    }
  }
}

// Row block blockIdx.x: grad_q of its rows (ascending j, as k_bwd_query),
// then the block's valid entries placed in its region of `region`, grouped
// by bucket; run_count / run_start [bucket][block] describe the runs.
__global__ void __launch_bounds__(kRowThreads)
    k_bwd_rows(const float* __restrict__ q_xyz, int64_t m, const float* __restrict__ p_xyz,
               int64_t n, const int32_t* __restrict__ idx, const float* __restrict__ dist,
               const float* __restrict__ grad, int k, float* __restrict__ grad_q,
               int accumulate, int vec4, BucketPlan plan, uint32_t* __restrict__ region,
               uint32_t* __restrict__ run_count, uint32_t* __restrict__ run_start) {
  extern __shared__ uint32_t bwd_sh[];
  __shared__ uint32_t warp_sums[32];
  const int64_t blk = blockIdx.x;
  const int64_t r0 = blk * plan.rows_per_block;
  const int64_t r1 = min(m, r0 + plan.rows_per_block);
  const int nb = static_cast<int>(plan.n_buckets);
  const int shift = plan.shift;
  uint32_t* hist = bwd_sh;
  uint32_t* cursor = bwd_sh + nb;
  const bool place = region != nullptr;
  if (place) {
    for (int b = threadIdx.x; b < nb; b += blockDim.x) hist[b] = 0u;
    __syncthreads();
  }
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    float gx = 0.f, gy = 0.f, gz = 0.f;
    float qx = 0.f, qy = 0.f, qz = 0.f;
    if (grad_q) {
      qx = q_xyz[3 * i];
      qy = q_xyz[3 * i + 1];
      qz = q_xyz[3 * i + 2];
    }
    for_row_entries(idx, dist, grad_q ? grad : nullptr, i, k, vec4,
                    [&](int j, int32_t t, float d, float g) {
      if (!entry_valid(t, n, d)) return;
      if (place) atomicAdd(&hist[t >> shift], 1u);
      if (grad_q) {
        const float g2 = 2.f * g;
        gx = __fmaf_rn(g2, __fsub_rn(qx, p_xyz[3 * static_cast<int64_t>(t)]), gx);
        gy = __fmaf_rn(g2, __fsub_rn(qy, p_xyz[3 * static_cast<int64_t>(t) + 1]), gy);
        gz = __fmaf_rn(g2, __fsub_rn(qz, p_xyz[3 * static_cast<int64_t>(t) + 2]), gz);
      }
    });
    if (grad_q) {
      if (accumulate) {
        gx = __fadd_rn(grad_q[3 * i], gx);
        gy = __fadd_rn(grad_q[3 * i + 1], gy);
        gz = __fadd_rn(grad_q[3 * i + 2], gz);
      }
      grad_q[3 * i] = gx;
      grad_q[3 * i + 1] = gy;
      grad_q[3 * i + 2] = gz;
    }
  }
  if (!place) return;  // the same for every thread of the block
  __syncthreads();
  // exclusive scan of the bucket counts: thread t takes a contiguous slice
  const int per = (nb + static_cast<int>(blockDim.x) - 1) / static_cast<int>(blockDim.x);
  const int b0 = min(nb, static_cast<int>(threadIdx.x) * per), b1 = min(nb, b0 + per);
  uint32_t sum = 0u;
  for (int b = b0; b < b1; ++b) sum += hist[b];
  uint32_t run = block_inclusive_scan(sum, warp_sums, nullptr) - sum;
  const int64_t nblk = plan.n_blocks;
  for (int b = b0; b < b1; ++b) {
    const uint32_t c = hist[b];
    cursor[b] = run;
    run_count[b * nblk + blk] = c;
    run_start[b * nblk + blk] = run;
    run += c;
  }
  __syncthreads();
  uint32_t* out = region + blk * plan.rows_per_block * k;
  const uint32_t pmask = (1u << shift) - 1u;
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const uint32_t row = static_cast<uint32_t>((i - r0) * k);
    for_row_entries(idx, dist, nullptr, i, k, vec4, [&](int j, int32_t t, float d, float) {
      if (!entry_valid(t, n, d)) return;
      const uint32_t pos = atomicAdd(&cursor[t >> shift], 1u);
      out[pos] = (row + j) | ((static_cast<uint32_t>(t) & pmask) << kLocalBits);
    });
  }
}

// Sums point p's segment seg[0, len) (full entry numbers, any order) in
// ascending e; lanes whose segment is longer than 32 are served by the
// whole warp (every round the smallest e above the last one).
__device__ __forceinline__ void sum_segment_warp(Acc& a, bool live, const uint32_t* seg,
                                                 uint32_t len, const float* __restrict__ q_xyz,
                                                 const float* __restrict__ grad, const DivK& k,
                                                 float px, float py, float pz) {
  const int lane = threadIdx.x & 31;
  const bool long_seg = live && len > 32;
  if (__any_sync(kFull, live && !long_seg && len > 16)) {
    if (live && !long_seg) sum_short<32>(a, seg, len, q_xyz, grad, k, px, py, pz);
  } else if (live && !long_seg && len > 0) {
    sum_short<16>(a, seg, len, q_xyz, grad, k, px, py, pz);
  }
  uint32_t todo = __ballot_sync(kFull, long_seg);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t* ls = reinterpret_cast<const uint32_t*>(
        __shfl_sync(kFull, reinterpret_cast<uintptr_t>(seg), leader));
    const uint32_t ll = __shfl_sync(kFull, len, leader);
    const float lx = __shfl_sync(kFull, px, leader);
    const float ly = __shfl_sync(kFull, py, leader);
    const float lz = __shfl_sync(kFull, pz, leader);
    Acc b;
    uint32_t last = 0;
    for (uint32_t r = 0; r < ll; ++r) {
      uint32_t best = kNoEntry;
      for (uint32_t t = lane; t < ll; t += 32) {
        const uint32_t v = ls[t];
        if ((r == 0 || v > last) && v < best) best = v;
      }
      best = __reduce_min_sync(kFull, best);
      add_entry(b, best, q_xyz, grad, k, lx, ly, lz);
      last = best;
    }
    if (lane == leader) a = b;
  }
}

__device__ __forceinline__ void store_grad_p(float* grad_p, int64_t p, const Acc& a,
                                             int accumulate) {
  Acc r = a;
  if (accumulate) {
    r.x = __fadd_rn(grad_p[3 * p], a.x);
    r.y = __fadd_rn(grad_p[3 * p + 1], a.y);
    r.z = __fadd_rn(grad_p[3 * p + 2], a.z);
  }
  grad_p[3 * p] = r.x;
  grad_p[3 * p + 1] = r.y;
  grad_p[3 * p + 2] = r.z;
}

// Bucket blockIdx.x: the points [b << shift, (b + 1) << shift).
__global__ void __launch_bounds__(kBucketThreads)
    k_bwd_buckets(const float* __restrict__ q_xyz, const float* __restrict__ p_xyz, int64_t n,
                  int k, DivK dk, BucketPlan plan, const uint32_t* __restrict__ region,
                  const uint32_t* __restrict__ run_count, const uint32_t* __restrict__ run_start,
                  const float* __restrict__ grad, float* __restrict__ grad_p, int accumulate) {
  extern __shared__ uint32_t bwd_sh[];
  __shared__ uint32_t warp_sums[32];
  __shared__ int range_hi;
  const int P = 1 << plan.shift;
  uint32_t* pcnt = bwd_sh;          // [P] entries per point
  uint32_t* pre = bwd_sh + P;       // [P + 1] exclusive prefix of pcnt
  uint32_t* cur = pre + P + 1;      // [P] placement cursors
  uint32_t* stage = cur + P;        // [kStageCap] entry numbers grouped by point
  const int64_t b = blockIdx.x;
  const int64_t p0 = b << plan.shift;
  const int np = static_cast<int>(min(static_cast<int64_t>(P), n - p0));
  const int64_t nblk = plan.n_blocks;
  const int64_t epb = plan.rows_per_block * k;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const uint32_t* rc = run_count + b * nblk;
  const uint32_t* rs = run_start + b * nblk;

  for (int p = threadIdx.x; p < P; p += blockDim.x) pcnt[p] = 0u;
  __syncthreads();
  for (int64_t r = warp; r < nblk; r += nwarps) {
    const uint32_t c = rc[r];
    const uint32_t* src = region + r * epb + rs[r];
    for (uint32_t t = lane; t < c; t += 32) atomicAdd(&pcnt[src[t] >> kLocalBits], 1u);
  }
  __syncthreads();
  {  // exclusive prefix over the P points (thread slices)
    const int per = (P + static_cast<int>(blockDim.x) - 1) / static_cast<int>(blockDim.x);
    const int a0 = min(P, static_cast<int>(threadIdx.x) * per), a1 = min(P, a0 + per);
    uint32_t sum = 0u;
    for (int p = a0; p < a1; ++p) sum += pcnt[p];
    uint32_t total = 0u;
    uint32_t run = block_inclusive_scan(sum, warp_sums, &total) - sum;
    for (int p = a0; p < a1; ++p) {
      pre[p] = run;
      run += pcnt[p];
    }
    if (threadIdx.x == 0) pre[P] = total;
  }
  __syncthreads();

  int lo = 0;
  while (lo < np) {
    if (threadIdx.x == 0) {  // the largest hi with pre[hi] - pre[lo] <= kStageCap
      int l = lo, h = np;
      while (l < h) {
        const int mid = (l + h + 1) >> 1;
        if (pre[mid] - pre[lo] <= static_cast<uint32_t>(kStageCap)) l = mid; else h = mid - 1;
      }
      range_hi = l;
    }
    __syncthreads();
    const int hi = range_hi;
    __syncthreads();
    if (hi == lo) {
      // one point with more entries than the stage: warp 0 streams the runs in
      // block order (ascending e), each run's entries of the point in order
      if (warp == 0) {
        const int64_t pt = p0 + lo;
        const float px = p_xyz[3 * pt], py = p_xyz[3 * pt + 1], pz = p_xyz[3 * pt + 2];
        Acc acc;
        for (int64_t r = 0; r < nblk; ++r) {
          const uint32_t c = rc[r];
          const uint32_t* src = region + r * epb + rs[r];
          const uint32_t base = static_cast<uint32_t>(r * plan.rows_per_block * k);
          uint32_t last = 0;
          bool first = true;
          for (;;) {
            uint32_t best = kNoEntry;
            for (uint32_t t = lane; t < c; t += 32) {
              const uint32_t v = src[t];
              if ((v >> kLocalBits) != static_cast<uint32_t>(lo)) continue;
              const uint32_t e = v & kLocalMask;
              if ((first || e > last) && e < best) best = e;
            }
            best = __reduce_min_sync(kFull, best);
            if (best == kNoEntry) break;
            add_entry(acc, base + best, q_xyz, grad, dk, px, py, pz);
            last = best;
            first = false;
          }
        }
        if (lane == 0) store_grad_p(grad_p, pt, acc, accumulate);
      }
      __syncthreads();
      ++lo;
      continue;
    }
    const uint32_t base_lo = pre[lo];
    for (int p = lo + static_cast<int>(threadIdx.x); p < hi; p += blockDim.x)
      cur[p] = pre[p] - base_lo;
    __syncthreads();
    for (int64_t r = warp; r < nblk; r += nwarps) {
      const uint32_t c = rc[r];
      const uint32_t* src = region + r * epb + rs[r];
      const uint32_t base = static_cast<uint32_t>(r * plan.rows_per_block * k);
      for (uint32_t t = lane; t < c; t += 32) {
        const uint32_t v = src[t];
        const int pl = static_cast<int>(v >> kLocalBits);
        if (pl >= lo && pl < hi) stage[atomicAdd(&cur[pl], 1u)] = base + (v & kLocalMask);
      }
    }
    __syncthreads();
    for (int p1 = lo; p1 < hi; p1 += blockDim.x) {  // whole warps: every thread iterates
      const int p = p1 + static_cast<int>(threadIdx.x);
      const bool live = p < hi;
      const int64_t pt = p0 + p;
      float px = 0.f, py = 0.f, pz = 0.f;
      uint32_t len = 0;
      const uint32_t* seg = stage;
      if (live) {
        px = p_xyz[3 * pt];
        py = p_xyz[3 * pt + 1];
        pz = p_xyz[3 * pt + 2];
        len = pcnt[p];
        seg = stage + (pre[p] - base_lo);
      }
      Acc acc;
      sum_segment_warp(acc, live, seg, len, q_xyz, grad, dk, px, py, pz);
      if (live) store_grad_p(grad_p, pt, acc, accumulate);
    }
    __syncthreads();
    lo = hi;
  }
}

namespace {

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

size_t bucket_smem(int shift) {
  const size_t P = size_t{1} << shift;
  return (3 * P + 1 + kStageCap) * sizeof(uint32_t);
}

struct BwdBufs {
  uint32_t* run_count;  // bucketed path: [buckets][row blocks] run lengths
  uint32_t* run_start;  // bucketed path: [buckets][row blocks] run starts
  uint32_t* count;    // [n]
  uint32_t* start;    // [n + 1]
  uint32_t* cursor;   // [n]
  uint32_t* tiles;    // [n_tiles]
  uint32_t* seg;      // [m * k] entry numbers grouped by neighbour
  int* total;         // valid entries (written by the tile scan)
};

BwdBufs bwd_layout(void* ws, int64_t m, int64_t n, int k, size_t* bytes) {
  Arena a(ws);
  BwdBufs b{};
  const BucketPlan plan = bucket_plan(m, n, k);
  b.total = a.take<int>(1);
  if (plan.ok) {  // bucketed path: entry regions and the run tables
    b.seg = a.take<uint32_t>(static_cast<size_t>(plan.n_blocks * plan.rows_per_block * k));
    b.run_count = a.take<uint32_t>(static_cast<size_t>(plan.n_buckets * plan.n_blocks));
    b.run_start = a.take<uint32_t>(static_cast<size_t>(plan.n_buckets * plan.n_blocks));
  } else {
    b.count = a.take<uint32_t>(n);
    b.start = a.take<uint32_t>(n + 1);
    b.cursor = a.take<uint32_t>(n);
    b.tiles = a.take<uint32_t>(ceil_div(n > 0 ? n : 1, kScanTile));
    b.seg = a.take<uint32_t>(m * k);
  }
  if (bytes) *bytes = a.used + 256;
  return b;
}

// Raises the dynamic shared-memory limit of the two bucketed kernels once
// per device (thread-safe).
cudaError_t bucket_kernels_ready() {
  static std::mutex mu;
  static std::vector<int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return cudaSuccess;
  e = cudaFuncSetAttribute(k_bwd_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           2 * kMaxRowBuckets * static_cast<int>(sizeof(uint32_t)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_buckets, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(bucket_smem(kMaxShift)));
  if (e == cudaSuccess) done.push_back(dev);
  return e;
}

}  // namespace

size_t segment_tiles(int64_t n) { return static_cast<size_t>(ceil_div(n > 0 ? n : 1, kScanTile)); }

int launch_segment_starts(const uint32_t* count, int64_t n, uint32_t* tiles, int* total,
                          uint32_t* start, uint32_t* cursor, cudaStream_t s) {
  const int t = blocks_for(n, kScanTile);
  k_bwd_tile_sums<<<t, kScanTile, 0, s>>>(count, n, tiles);
  k_scan_tiles<<<1, 1024, 0, s>>>(tiles, t, total);
  k_bwd_starts<<<t, kScanTile, 0, s>>>(count, n, tiles, start, cursor);
  return 3;
}

size_t backward_workspace_bytes(int64_t m, int64_t n, int k) {
  size_t bytes = 0;
  bwd_layout(nullptr, m, n, k, &bytes);
  return bytes;
}

int run_backward(const BackwardArgs& a, void* ws, size_t ws_bytes, cudaStream_t s,
                 int* launches) {
  size_t need = 0;
  BwdBufs b = bwd_layout(ws, a.m, a.n, a.k, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  const int64_t total = a.m * a.k;
  const bool want_p = a.grad_p != nullptr && a.n > 0;
  int nl = 0;
  cudaError_t e = cudaSuccess;
  const auto al16 = [](const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; };
  const bool vec4 = a.k % 4 == 0 && al16(a.idx) && al16(a.dist) && al16(a.grad);
  const BucketPlan plan = bucket_plan(a.m, a.n, a.k);
  if (plan.ok) {
    e = bucket_kernels_ready();
    if (e != cudaSuccess) {
      note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
    if (a.grad_q || want_p) {
      const size_t smem = want_p ? 2 * static_cast<size_t>(plan.n_buckets) * sizeof(uint32_t) : 0;
      k_bwd_rows<<<static_cast<int>(plan.n_blocks), kRowThreads, smem, s>>>(
          a.q_xyz, a.m, a.p_xyz, a.n, a.idx, a.dist, a.grad, a.k, a.grad_q, a.accumulate,
          vec4 ? 1 : 0, plan, want_p ? b.seg : nullptr, b.run_count, b.run_start);
      ++nl;
    }
    if (want_p) {
      k_bwd_buckets<<<static_cast<int>(plan.n_buckets), kBucketThreads, bucket_smem(plan.shift),
                      s>>>(a.q_xyz, a.p_xyz, a.n, a.k, make_divk(static_cast<uint32_t>(a.k)), plan,
                           b.seg, b.run_count, b.run_start, a.grad, a.grad_p, a.accumulate);
      ++nl;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
    if (launches) *launches = nl;
    return FKNN_OK;
  }
  if (want_p) e = cudaMemsetAsync(b.count, 0, sizeof(uint32_t) * a.n, s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (a.m > 0 && (a.grad_q || want_p)) {
    k_bwd_query<<<blocks_for(a.m, 256), 256, 0, s>>>(a.q_xyz, a.m, a.p_xyz, a.n, a.idx, a.dist,
                                                     a.grad, a.k, a.grad_q, a.accumulate,
                                                     want_p ? b.count : nullptr, vec4 ? 1 : 0);
    ++nl;
  }
  if (want_p) {
    nl += launch_segment_starts(b.count, a.n, b.tiles, b.total, b.start, b.cursor, s);
    if (total > 0) {
      const int64_t sb = ceil_div(total, 256);
      k_bwd_scatter<<<static_cast<int>(sb < 8192 ? sb : 8192), 256, 0, s>>>(
          total, a.n, a.idx, a.dist, b.cursor, b.seg, vec4 ? 1 : 0);
      ++nl;
    }
    k_bwd_support<<<blocks_for(a.n, 128), 128, 0, s>>>(a.q_xyz, a.p_xyz, a.n,
                                                       make_divk(static_cast<uint32_t>(a.k)), b.start,
                                                       b.seg, a.grad, a.grad_p, a.accumulate);
    ++nl;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (launches) *launches = nl;
  return FKNN_OK;
}

}  // namespace fknn
