// Stable LSD radix sort (8-bit digits), used by the reference-table
// construction and the adaptive octree, and the block / tile scans used by
// every construction pass and the backward.
//
// Counting sort per digit, three launches per pass:
//   hist    -- per 2048-key tile, a 256-bin histogram built with
//              warp-aggregated shared-memory atomics (__match_any_sync);
//   scan    -- one CTA per digit: exclusive scan down the digit's column of
//              tile counts, offset by the totals of all smaller digits;
//   scatter -- stable ranks: each warp owns 256 consecutive keys, ranks its
//              32-key rounds with __match_any_sync, and warps are combined
//              by a per-digit prefix over the CTA.
// The number of significant key bits is read from device memory, so passes
// beyond it return immediately and the whole sort can be captured in a CUDA
// graph without knowing the data.  Pass p reads buffer p&1 and writes
// (p+1)&1; the sorted data ends in buffer (passes actually run)&1.
#pragma once

#include "fknn_common.cuh"

namespace fknn {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per CTA
constexpr int kSortMaxPasses = 8;

__host__ __device__ inline int sort_passes_for_bits(int bits) { return (bits + 7) / 8; }

template <typename KeyT>
__global__ void __launch_bounds__(kSortThreads)
    k_sort_hist(const KeyT* __restrict__ keys, int64_t n, int pass, const int* nbits,
                uint32_t* __restrict__ hist, uint32_t* __restrict__ totals, int n_tiles) {
  chain_wait();
  if (pass * 8 >= *nbits) return;
  __shared__ uint32_t sh[256];
  sh[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile;
  const int shift = pass * 8;
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const int64_t k = base + i * kSortThreads + threadIdx.x;
    const bool valid = k < n;
    const unsigned vmask = __ballot_sync(kFull, valid);
    if (valid) {
      const uint32_t d = static_cast<uint32_t>(keys[k] >> shift) & 255u;
      const unsigned peers = __match_any_sync(vmask, d);
      if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&sh[d], __popc(peers));
    }
  }
  __syncthreads();
  const uint32_t c = sh[threadIdx.x];
  hist[static_cast<int64_t>(threadIdx.x) * n_tiles + blockIdx.x] = c;
  if (c) atomicAdd(&totals[pass * 256 + threadIdx.x], c);
}

// Block-wide inclusive scan of one value per thread (blockDim.x <= 1024).
__device__ __forceinline__ uint32_t block_inclusive_scan(uint32_t v, uint32_t* warp_sums,
                                                         uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  uint32_t x = v;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, x, s);
    if (lane >= s) x += t;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < nwarps ? warp_sums[lane] : 0;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      uint32_t t = __shfl_up_sync(kFull, w, s);
      if (lane >= s) w += t;
    }
    if (lane < nwarps) warp_sums[lane] = w;
  }
  __syncthreads();
  const uint32_t result = x + (warp ? warp_sums[warp - 1] : 0);
  if (total) *total = warp_sums[nwarps - 1];
  __syncthreads();
  return result;
}

// grid = 256 CTAs (one per digit), 1024 threads.  Turns the digit-major
// histogram into global scatter offsets in place.
static __global__ void __launch_bounds__(1024)
    k_sort_scan(uint32_t* __restrict__ hist, const uint32_t* __restrict__ totals, int n_tiles,
                int pass, const int* nbits) {
  chain_wait();
  if (pass * 8 >= *nbits) return;
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int d = blockIdx.x;
  uint32_t v = threadIdx.x < static_cast<unsigned>(d) ? totals[pass * 256 + threadIdx.x] : 0u;
  block_inclusive_scan(v, warp_sums, &s_total);
  uint32_t carry = s_total;  // keys with a smaller digit
  uint32_t* col = hist + static_cast<int64_t>(d) * n_tiles;
  for (int t0 = 0; t0 < n_tiles; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const uint32_t x = t < n_tiles ? col[t] : 0u;
    const uint32_t incl = block_inclusive_scan(x, warp_sums, &s_total);
    if (t < n_tiles) col[t] = carry + incl - x;
    carry += s_total;
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(kSortThreads)
    k_sort_scatter(const KeyT* __restrict__ kin, const uint32_t* __restrict__ vin,
                   KeyT* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n, int pass,
                   const int* nbits, const uint32_t* __restrict__ offsets, int n_tiles) {
  chain_wait();
  if (pass * 8 >= *nbits) return;
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t cnt[kWarps][256];
  __shared__ uint32_t tile_off[256];
  for (int i = threadIdx.x; i < kWarps * 256; i += kSortThreads) cnt[i / 256][i % 256] = 0;
  tile_off[threadIdx.x] = offsets[static_cast<int64_t>(threadIdx.x) * n_tiles + blockIdx.x];
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int shift = pass * 8;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile + w * (32 * kSortItems);
  KeyT key[kSortItems];
  uint32_t val[kSortItems], dig[kSortItems], rank[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t k = base + r * 32 + lane;
    const bool valid = k < n;
    const unsigned vmask = __ballot_sync(kFull, valid);
    dig[r] = 256u;
    rank[r] = 0u;
    if (valid) {
      key[r] = kin[k];
      val[r] = vin[k];
      const uint32_t d = static_cast<uint32_t>(key[r] >> shift) & 255u;
      dig[r] = d;
      const unsigned peers = __match_any_sync(vmask, d);
      const uint32_t before = cnt[w][d];
      rank[r] = before + __popc(peers & lanemask_lt());
      __syncwarp(vmask);
      if (lane == 31 - __clz(peers)) cnt[w][d] = before + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  {
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) {
      const uint32_t c = cnt[ww][d];
      cnt[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    if (dig[r] < 256u) {
      const uint32_t pos = tile_off[dig[r]] + cnt[w][dig[r]] + rank[r];
      kout[pos] = key[r];
      vout[pos] = val[r];
    }
  }
}

// The two ping-pong buffers of a sort, passed by value to the kernels that
// read the sorted result (they pick the buffer from the device bit count).
template <typename KeyT>
struct SortPair {
  KeyT* keys[2];
  uint32_t* vals[2];
  // Buffer b (0 or 1) by select: indexing the arrays with a run-time value
  // would copy a by-value kernel parameter to local memory.
  __host__ __device__ KeyT* key_buf(int b) const { return b ? keys[1] : keys[0]; }
  __host__ __device__ uint32_t* val_buf(int b) const { return b ? vals[1] : vals[0]; }
};

template <typename KeyT>
struct SortBuffers {
  KeyT* keys[2];
  uint32_t* vals[2];
  uint32_t* hist;    // [256 * n_tiles]
  uint32_t* totals;  // [kSortMaxPasses * 256], zeroed by the caller
};

// Launches `max_passes` passes (the device skips the ones beyond *nbits).
// Returns the number of kernels launched.
template <typename KeyT>
inline int launch_radix_sort(const SortBuffers<KeyT>& b, int64_t n, const int* nbits,
                             int max_passes, cudaStream_t s) {
  if (n <= 0) return 0;
  const int n_tiles = static_cast<int>(ceil_div(n, kSortTile));
  int launches = 0;
  for (int p = 0; p < max_passes; ++p) {
    const int src = p & 1, dst = src ^ 1;
    launch_chained(k_sort_hist<KeyT>, n_tiles, kSortThreads, 0, s, b.keys[src], n, p, nbits, b.hist,
                   b.totals, n_tiles);
    launch_chained(k_sort_scan, 256, 1024, 0, s, b.hist, b.totals, n_tiles, p, nbits);
    launch_chained(k_sort_scatter<KeyT>, n_tiles, kSortThreads, 0, s, b.keys[src], b.vals[src],
                   b.keys[dst], b.vals[dst], n, p, nbits, b.hist, n_tiles);
    launches += 3;
  }
  return launches;
}

inline size_t sort_hist_elems(int64_t n) {
  return static_cast<size_t>(256) * static_cast<size_t>(ceil_div(n > 0 ? n : 1, kSortTile));
}

// ------------------------------------------------------------ tile scans
// A device-wide exclusive scan in three steps: a producer kernel writes one
// count per tile (tile_counts[t]); k_scan_tiles turns them into exclusive
// offsets and stores the grand total; a consumer kernel re-derives its
// per-item flags and adds its tile offset.
static __global__ void __launch_bounds__(1024)
    k_scan_tiles(uint32_t* __restrict__ tile_counts, int n_tiles, int* __restrict__ total_out) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  uint32_t carry = 0;
  for (int t0 = 0; t0 < n_tiles; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const uint32_t x = t < n_tiles ? tile_counts[t] : 0u;
    const uint32_t incl = block_inclusive_scan(x, warp_sums, &s_total);
    if (t < n_tiles) tile_counts[t] = carry + incl - x;
    carry += s_total;
  }
  if (threadIdx.x == 0) *total_out = static_cast<int>(carry);
}

}  // namespace fknn
