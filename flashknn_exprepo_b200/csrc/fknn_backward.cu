// Backward of the squared distances returned by the kNN query.
//
// For d_ij = |p[idx_ij] - q_i|^2 and an upstream gradient g_ij:
//   grad_q[i] = sum_j 2 g_ij (q_i - p[idx_ij])          (one thread per query,
//                                                        j in ascending order)
//   grad_p[n] = sum_{idx_ij = n} -2 g_ij (q_i - p_n)     (segmented reduction)
// The reference-side sum is a segmented reduction over the entries sorted by
// neighbour index: a counting sort by idx (integer atomics count each
// segment and hand every entry its rank in it, a scan places the segments,
// an atomic-free scatter writes entry numbers e = i*K+j at segment start +
// rank), then one thread per support point orders its segment
// by e (a register sorting network; a warp-cooperative selection for
// segments longer than 32) and sums it sequentially in ascending e, reading
// g_e and q_i where it adds them.  Every FP32
// operation therefore happens in an order fixed by the inputs alone: the
// gradients are bitwise reproducible, and no floating-point atomics are used.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_networks.cuh"
#include "fknn_sort.cuh"
#include "fknn_backward.h"

namespace fknn {

namespace {

constexpr int kScanTile = 1024;
constexpr uint32_t kNoEntry = ~0u;

__device__ __forceinline__ bool entry_valid(int32_t t, int64_t n, float d) {
  return t >= 0 && t < n && !isinf(d);
}

}  // namespace

// One thread per query: grad_q over j in ascending order, the size of
// every neighbour's segment (count[t], integer atomics) and each entry's
// rank in its segment (rank[e], the atomic's old value; kNoEntry for an
// entry that carries no gradient), so the scatter needs no atomics.
__global__ void __launch_bounds__(256)
    k_bwd_query(const float* __restrict__ q_xyz, int64_t m, const float* __restrict__ p_xyz,
                int64_t n, const int32_t* __restrict__ idx, const float* __restrict__ dist,
                const float* __restrict__ grad, int k, float* __restrict__ grad_q, int accumulate,
                uint32_t* __restrict__ count, uint32_t* __restrict__ rank, int vec4) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const float qx = q_xyz[3 * i], qy = q_xyz[3 * i + 1], qz = q_xyz[3 * i + 2];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  auto entry = [&](int32_t t, float d, float g) -> uint32_t {
    if (!entry_valid(t, n, d)) return kNoEntry;
    uint32_t r = 0u;
    if (count) r = atomicAdd(&count[t], 1u);
    if (!grad_q) return r;
    const float g2 = 2.f * g;
    gx = __fmaf_rn(g2, __fsub_rn(qx, p_xyz[3 * static_cast<int64_t>(t)]), gx);
    gy = __fmaf_rn(g2, __fsub_rn(qy, p_xyz[3 * static_cast<int64_t>(t) + 1]), gy);
    gz = __fmaf_rn(g2, __fsub_rn(qz, p_xyz[3 * static_cast<int64_t>(t) + 2]), gz);
    return r;
  };
  if (vec4) {  // k % 4 == 0 and 16-byte aligned rows: 128-bit row loads, j ascending
    const int4* i4 = reinterpret_cast<const int4*>(idx + i * k);
    const float4* d4 = reinterpret_cast<const float4*>(dist + i * k);
    const float4* g4 = reinterpret_cast<const float4*>(grad + i * k);
    uint4* r4 = rank ? reinterpret_cast<uint4*>(rank + i * k) : nullptr;
    for (int j = 0; j < (k >> 2); ++j) {
      const int4 t = i4[j];
      const float4 d = d4[j], g = g4[j];
      uint4 r;
      r.x = entry(t.x, d.x, g.x);
      r.y = entry(t.y, d.y, g.y);
      r.z = entry(t.z, d.z, g.z);
      r.w = entry(t.w, d.w, g.w);
      if (r4) r4[j] = r;
    }
  } else {
    for (int j = 0; j < k; ++j) {
      const int64_t e = i * k + j;
      const uint32_t r = entry(idx[e], dist[e], grad[e]);
      if (rank) rank[e] = r;
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
  chain_wait();
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
  chain_wait();
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

// One thread per entry: the entry number e goes to slot start[t] + rank[e]
// of its neighbour's segment (4 bytes per entry, no atomics: the count pass
// handed out the ranks).  The slot order inside a segment depends on the
// count pass's scheduling; the reduction below orders each segment by e.
__global__ void __launch_bounds__(256)
    k_bwd_scatter(int64_t total, const int32_t* __restrict__ idx,
                  const uint32_t* __restrict__ rank, const uint32_t* __restrict__ start,
                  uint32_t* __restrict__ seg, int vec4) {
  chain_wait();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  auto put = [&](int64_t e, int32_t t, uint32_t r) {
    if (r == kNoEntry) return;
    seg[start[t] + r] = static_cast<uint32_t>(e);
  };
  if (vec4) {  // total % 4 == 0, 16-byte aligned: four entries per thread
    for (int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         w < (total >> 2); w += stride) {
      const int4 t = reinterpret_cast<const int4*>(idx)[w];
      const uint4 r = reinterpret_cast<const uint4*>(rank)[w];
      put(4 * w, t.x, r.x);
      put(4 * w + 1, t.y, r.y);
      put(4 * w + 2, t.z, r.z);
      put(4 * w + 3, t.w, r.w);
    }
    return;
  }
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += stride)
    put(e, idx[e], rank[e]);
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
  chain_wait();
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

namespace {

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

struct BwdBufs {
  uint32_t* count;    // [n]
  uint32_t* start;    // [n + 1]
  uint32_t* cursor;   // [n]
  uint32_t* tiles;    // [n_tiles]
  uint32_t* seg;      // [m * k] entry numbers grouped by neighbour
  uint32_t* rank;     // [m * k] each entry's rank in its segment
  int* total;         // valid entries (written by the tile scan)
};

BwdBufs bwd_layout(void* ws, int64_t m, int64_t n, int k, size_t* bytes) {
  Arena a(ws);
  BwdBufs b{};
  b.total = a.take<int>(1);
  b.count = a.take<uint32_t>(n);
  b.start = a.take<uint32_t>(n + 1);
  b.cursor = a.take<uint32_t>(n);
  b.tiles = a.take<uint32_t>(ceil_div(n > 0 ? n : 1, kScanTile));
  b.seg = a.take<uint32_t>(m * k);
  b.rank = a.take<uint32_t>(m * k);
  if (bytes) *bytes = a.used + 256;
  return b;
}

}  // namespace

size_t segment_tiles(int64_t n) { return static_cast<size_t>(ceil_div(n > 0 ? n : 1, kScanTile)); }

int launch_segment_starts(const uint32_t* count, int64_t n, uint32_t* tiles, int* total,
                          uint32_t* start, uint32_t* cursor, cudaStream_t s) {
  const int t = blocks_for(n, kScanTile);
  launch_chained(k_bwd_tile_sums, t, kScanTile, 0, s, count, n, tiles);
  launch_chained(k_scan_tiles, 1, 1024, 0, s, tiles, t, total);
  launch_chained(k_bwd_starts, t, kScanTile, 0, s, count, n, tiles, start, cursor);
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
  if (want_p) e = cudaMemsetAsync(b.count, 0, sizeof(uint32_t) * a.n, s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  const auto al16 = [](const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; };
  const bool vec4 = a.k % 4 == 0 && al16(a.idx) && al16(a.dist) && al16(a.grad);
  if (a.m > 0 && (a.grad_q || want_p)) {
    launch_chained(k_bwd_query, blocks_for(a.m, 256), 256, 0, s, a.q_xyz, a.m, a.p_xyz, a.n, a.idx,
                   a.dist, a.grad, a.k, a.grad_q, a.accumulate, want_p ? b.count : nullptr,
                   want_p ? b.rank : nullptr, vec4 ? 1 : 0);
    ++nl;
  }
  if (want_p) {
    nl += launch_segment_starts(b.count, a.n, b.tiles, b.total, b.start, b.cursor, s);
    if (total > 0) {
      const int64_t sb = ceil_div(total, 256);
      launch_chained(k_bwd_scatter, static_cast<int>(sb < 8192 ? sb : 8192), 256, 0, s, total,
                     a.idx, b.rank, b.start, b.seg, vec4 ? 1 : 0);
      ++nl;
    }
    launch_chained(k_bwd_support, blocks_for(a.n, 128), 128, 0, s, a.q_xyz, a.p_xyz, a.n,
                   make_divk(static_cast<uint32_t>(a.k)), b.start, b.seg, a.grad, a.grad_p,
                   a.accumulate);
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
