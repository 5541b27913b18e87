// Neighbour feature grouping: the gather that follows the kNN in point
// networks (Pointcept's pointops.grouping,
// Pointcept/libs/pointops/functions/grouping.py:36-60, called by
// knn_query_and_group, .../functions/utils.py:5-18).
//
// Forward: out[i, j, :] = [xyz[t] - new_xyz[i] | feat[t]] for t = idx[i, j]
// (the xyz part only with with_xyz); an index below 0 is padding and gives a
// zero row.  Threads run flat over the output words (float4 when the rows
// allow it), so every warp stores one contiguous run: a bandwidth-bound copy
// whose only re-read is the gathered feature row, served from L2 for the
// rows that neighbours share.
//
// Backward: grad_feat[t] = sum of grad_out[i, j, feat part] over the entries
// with idx[i, j] = t, grad_xyz[t] the same over the xyz part and
// grad_new_xyz[i] = -sum_j of the xyz part of row (i, j) over the valid j.
// The reference-side sums are made deterministic the same way as the
// distance backward (fknn_backward.cu): a counting sort of the entries by
// neighbour index, then one warp per support point that orders its segment
// by entry number and adds the rows in that order, so every output channel
// is summed in a fixed order -- no floating-point atomics.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"
#include "fknn_backward.h"
#include "fknn_group.h"

namespace fknn {

namespace {

constexpr uint32_t kNoEntry = 0xffffffffu;

__device__ __forceinline__ bool entry_ok(int32_t t, int64_t n, int* status) {
  if (t < 0) return false;
  if (t >= n) {
    raise_status(status, kStatusTable);
    return false;
  }
  return true;
}

}  // namespace

// ------------------------------------------------------------------ forward

// Rows of whole aligned float4s (no xyz, c % 4 == 0): a group of tpr lanes
// (a power of two, tpr >= c/4 up to 32) copies one row, so a warp writes
// 32/tpr consecutive rows as one contiguous run; the row loop is unrolled so
// several independent gathers are in flight per thread.  Otherwise flat over
// the output: thread t writes output float t.  Stores stream past L2
// (st.global.cs): the output is written once and not re-read here.
__global__ void __launch_bounds__(256)
    kg_forward(const float* __restrict__ feat, int64_t n, int c, const int32_t* __restrict__ idx,
               int64_t rows, int k, const float* __restrict__ xyz,
               const float* __restrict__ new_xyz, int with_xyz, int tpr,
               float* __restrict__ out, int* status) {
  chain_wait();
  const int off = with_xyz ? 3 : 0;
  const int cw = c + off;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  if (tpr) {  // with_xyz == 0, c % 4 == 0
    const int q4 = c >> 2;
    const int sub = threadIdx.x & (tpr - 1);
    const int64_t row_stride = stride / tpr;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 4
    for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / tpr;
         r < rows; r += row_stride) {
      const int32_t t = idx[r];
      const bool ok = entry_ok(t, n, sub == 0 ? status : nullptr);
      const float4* src = reinterpret_cast<const float4*>(feat + static_cast<int64_t>(t) * c);
      float4* dst = reinterpret_cast<float4*>(out) + r * q4;
      for (int q = sub; q < q4; q += tpr) __stcs(dst + q, ok ? __ldg(src + q) : zero);
    }
    return;
  }
  const int64_t words = rows * cw;
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < words;
       w += stride) {
    const int64_t r = w / cw;
    const int col = static_cast<int>(w - r * cw);
    const int32_t t = idx[r];
    float v = 0.f;
    if (entry_ok(t, n, col == 0 ? status : nullptr)) {
      if (col < off)
        v = __fsub_rn(xyz[3 * static_cast<int64_t>(t) + col], new_xyz[3 * (r / k) + col]);
      else
        v = __ldg(feat + static_cast<int64_t>(t) * c + (col - off));
    }
    __stcs(out + w, v);
  }
}

// ----------------------------------------------------------------- backward

// count[t] = entries naming support point t.
__global__ void __launch_bounds__(256)
    kg_count(const int32_t* __restrict__ idx, int64_t total, int64_t n,
             uint32_t* __restrict__ count, int* status) {
  chain_wait();
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t t = idx[e];
    if (entry_ok(t, n, status)) atomicAdd(&count[t], 1u);
  }
}

__global__ void __launch_bounds__(256)
    kg_scatter(const int32_t* __restrict__ idx, int64_t total, int64_t n,
               uint32_t* __restrict__ cursor, uint32_t* __restrict__ seg) {
  chain_wait();
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t t = idx[e];
    if (t < 0 || t >= n) continue;
    seg[atomicSub(&cursor[t], 1u) - 1u] = static_cast<uint32_t>(e);
  }
}

// Ascending bitonic sort of one value per lane across the warp.
__device__ __forceinline__ uint32_t warp_sort_u32(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const uint32_t o = __shfl_xor_sync(kFull, v, stride);
      const bool up = (lane & size) == 0;        // ascending block
      const bool low = (lane & stride) == 0;      // lower partner
      v = (low == up) ? min(v, o) : max(v, o);
    }
  }
  return v;
}

template <int V>
struct Vec;
template <>
struct Vec<1> {
  using T = float;
  __device__ static T zero() { return 0.f; }
  __device__ static T add(T a, T b) { return __fadd_rn(a, b); }
};
template <>
struct Vec<2> {
  using T = float2;
  __device__ static T zero() { return make_float2(0.f, 0.f); }
  __device__ static T add(T a, T b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
};

// One warp per support point: its entries in ascending order, each row of
// grad_out added channel by channel in that order.  V channels per lane (2
// when the rows are whole float2s); the rows of four entries are loaded
// before they are added, in order, so loads overlap.
template <int V>
__global__ void __launch_bounds__(256)
    kg_support(const float* __restrict__ grad_out, int c, int with_xyz,
               const uint32_t* __restrict__ start, const uint32_t* __restrict__ seg, int64_t n,
               float* __restrict__ grad_feat, float* __restrict__ grad_xyz, int accumulate_xyz) {
  chain_wait();
  using VT = typename Vec<V>::T;
  const int lane = threadIdx.x & 31;
  const int off = with_xyz ? 3 : 0;
  const int cw = c + off;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
       p < n; p += warps) {
    const uint32_t s = start[p], len = start[p + 1] - s;
    // Entries of a short segment sorted across the lanes; a long one is
    // walked by repeated selection of the next larger entry.
    uint32_t mine = kNoEntry;
    if (len <= 32) mine = warp_sort_u32(lane < static_cast<int>(len) ? seg[s + lane] : kNoEntry);
    for (int c0 = 0; c0 < cw; c0 += 32 * V) {
      const int col = c0 + lane * V;
      const bool live = col < cw;
      auto row = [&](uint32_t e) {
        return *reinterpret_cast<const VT*>(grad_out + static_cast<int64_t>(e) * cw + col);
      };
      VT acc = Vec<V>::zero();
      if (len <= 32) {
        uint32_t r = 0;
        for (; r + 4 <= len; r += 4) {
          const uint32_t e0 = __shfl_sync(kFull, mine, r), e1 = __shfl_sync(kFull, mine, r + 1);
          const uint32_t e2 = __shfl_sync(kFull, mine, r + 2), e3 = __shfl_sync(kFull, mine, r + 3);
          if (live) {
            const VT v0 = row(e0), v1 = row(e1), v2 = row(e2), v3 = row(e3);
            acc = Vec<V>::add(Vec<V>::add(Vec<V>::add(Vec<V>::add(acc, v0), v1), v2), v3);
          }
        }
        for (; r < len; ++r) {
          const uint32_t e = __shfl_sync(kFull, mine, r);
          if (live) acc = Vec<V>::add(acc, row(e));
        }
      } else {
        uint32_t last = 0;
        for (uint32_t r = 0; r < len; ++r) {
          uint32_t best = kNoEntry;
          for (uint32_t t = lane; t < len; t += 32) {
            const uint32_t v = seg[s + t];
            if ((r == 0 || v > last) && v < best) best = v;
          }
          best = __reduce_min_sync(kFull, best);
          if (live) acc = Vec<V>::add(acc, row(best));
          last = best;
        }
      }
      if (!live) continue;
      if constexpr (V == 1) {
        if (col < off) {
          if (grad_xyz) {
            float* g = grad_xyz + 3 * p + col;
            *g = accumulate_xyz ? __fadd_rn(*g, acc) : acc;
          }
        } else {
          grad_feat[p * c + (col - off)] = acc;
        }
      } else {  // no xyz part: channel col of the row is channel col of feat
        *reinterpret_cast<VT*>(grad_feat + p * c + col) = acc;
      }
    }
  }
}

// grad_new_xyz[i] = -sum_j over valid entries of the xyz part of row (i, j).
__global__ void __launch_bounds__(256)
    kg_query(const float* __restrict__ grad_out, int c, const int32_t* __restrict__ idx,
             int64_t m, int k, int64_t n, float* __restrict__ grad_new_xyz, int accumulate) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int cw = c + 3;
  float g[3] = {0.f, 0.f, 0.f};
  for (int j = 0; j < k; ++j) {
    const int32_t t = idx[i * k + j];
    if (t < 0 || t >= n) continue;
    const float* row = grad_out + (i * k + j) * cw;
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] = __fsub_rn(g[a], row[a]);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
    grad_new_xyz[3 * i + a] = accumulate ? __fadd_rn(grad_new_xyz[3 * i + a], g[a]) : g[a];
}

// --------------------------------------------------------------- host side

namespace {

struct GBufs {
  Meta* meta;
  uint32_t* count;
  uint32_t* start;
  uint32_t* cursor;
  uint32_t* tiles;
  uint32_t* seg;
};

GBufs glayout(void* ws, int64_t rows, int64_t n, size_t* bytes) {
  Arena a(ws);
  GBufs b{};
  b.meta = a.take<Meta>(1);
  b.count = a.take<uint32_t>(n);
  b.start = a.take<uint32_t>(n + 1);
  b.cursor = a.take<uint32_t>(n);
  b.tiles = a.take<uint32_t>(segment_tiles(n));
  b.seg = a.take<uint32_t>(rows);
  if (bytes) *bytes = a.used + 256;
  return b;
}

inline int capped_blocks(int64_t threads) {
  const int64_t b = ceil_div(threads > 0 ? threads : 1, 256);
  return static_cast<int>(b < 148 * 32 ? b : 148 * 32);
}

inline int capped_warp_blocks(int64_t rows) {
  const int64_t b = ceil_div(rows > 0 ? rows : 1, 8);  // 8 warps per 256-thread block
  return static_cast<int>(b < 148 * 16 ? b : 148 * 16);
}

}  // namespace

size_t group_workspace_bytes(int64_t rows, int64_t n) {
  size_t bytes = 0;
  glayout(nullptr, rows, n, &bytes);
  return bytes;
}

int run_group_forward(const GroupArgs& g, void* ws, size_t ws_bytes, cudaStream_t s,
                      int* launches) {
  size_t need = 0;
  GBufs b = glayout(ws, g.m * g.k, g.n, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  cudaError_t e = cudaMemsetAsync(b.meta, 0, sizeof(Meta), s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  const int64_t rows = g.m * g.k;
  int nl = 0;
  if (rows > 0) {
    const int cw = g.c + (g.with_xyz ? 3 : 0);
    const bool vec4 = !g.with_xyz && g.c % 4 == 0 &&
                      reinterpret_cast<uintptr_t>(g.feat) % 16 == 0 &&
                      reinterpret_cast<uintptr_t>(g.out) % 16 == 0;
    int tpr = 0;  // lanes per row of the float4 path
    if (vec4) {
      tpr = 1;
      while (tpr < 32 && tpr < g.c / 4) tpr <<= 1;
    }
    const int64_t words = vec4 ? rows * tpr : rows * cw;
    launch_chained(kg_forward, capped_blocks(words), 256, 0, s, g.feat, g.n, g.c, g.idx, rows, g.k,
                   g.xyz, g.new_xyz, g.with_xyz, tpr, g.out, &b.meta->status);
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

int run_group_backward(const GroupArgs& g, void* ws, size_t ws_bytes, cudaStream_t s,
                       int* launches) {
  size_t need = 0;
  GBufs b = glayout(ws, g.m * g.k, g.n, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  const int64_t rows = g.m * g.k;
  cudaError_t e = cudaMemsetAsync(b.meta, 0, sizeof(Meta), s);
  if (e == cudaSuccess && g.n > 0) e = cudaMemsetAsync(b.count, 0, sizeof(uint32_t) * g.n, s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  int nl = 0;
  if (g.n > 0 && g.grad_feat) {
    const int64_t eb = ceil_div(rows > 0 ? rows : 1, 256);
    const int eblocks = static_cast<int>(eb < 8192 ? eb : 8192);
    if (rows > 0) {
      launch_chained(kg_count, eblocks, 256, 0, s, g.idx, rows, g.n, b.count, &b.meta->status);
      ++nl;
    }
    nl += launch_segment_starts(b.count, g.n, b.tiles, &b.meta->n_groups, b.start, b.cursor, s);
    if (rows > 0) {
      launch_chained(kg_scatter, eblocks, 256, 0, s, g.idx, rows, g.n, b.cursor, b.seg);
      ++nl;
    }
    const bool v2 = !g.with_xyz && g.c % 2 == 0 &&
                    reinterpret_cast<uintptr_t>(g.grad_out) % 8 == 0 &&
                    reinterpret_cast<uintptr_t>(g.grad_feat) % 8 == 0;
    if (v2)
      launch_chained(kg_support<2>, capped_warp_blocks(g.n), 256, 0, s, g.grad_out, g.c, 0, b.start,
                     b.seg, g.n, g.grad_feat, nullptr, 0);
    else
      launch_chained(kg_support<1>, capped_warp_blocks(g.n), 256, 0, s, g.grad_out, g.c, g.with_xyz,
                     b.start, b.seg, g.n, g.grad_feat, g.grad_xyz, g.accumulate_xyz);
    ++nl;
  }
  if (g.with_xyz && g.grad_new_xyz && g.m > 0) {
    launch_chained(kg_query, static_cast<int>(ceil_div(g.m, 256)), 256, 0, s, g.grad_out, g.c,
                   g.idx, g.m, g.k, g.n, g.grad_new_xyz, g.accumulate_new_xyz);
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
