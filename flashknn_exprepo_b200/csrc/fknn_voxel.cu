// Voxel-first subsampling: one representative point per occupied voxel.
//
// Semantics of the reference's _voxel_first_cuda (Networks/hierarchy.py:23-35):
// voxel = floor(xyz / size) as PyTorch evaluates it on CUDA tensors (a
// product with the FP32 reciprocal of the scalar), key = the Morton key of
// the voxel's low 16 bits per axis (xyz2key, FlashKNN/functions/z_order.py;
// batch << 48 when batch ids are given), representative = the first point of
// each key in a stable sort -- the lowest index of the voxel -- and the
// representatives' indices in ascending order.
//
//   kv_keys      keys + the OR of all keys (significant bits of the sort)
//   radix sort   stable LSD sort of (key, index) over the significant bits
//   kv_heads     flag[index of every key's first sorted point] = 1
//   kv_tiles / k_scan_tiles / kv_compact
//                ordered compaction of the flags: the output comes out in
//                ascending index order without a second sort
// The count stays on the device (*count_out), so the sequence is a fixed
// launch list that can be captured in a CUDA graph.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"
#include "fknn_voxel.h"

namespace fknn {

namespace {
constexpr int kTile = 2048;  // points per 256-thread CTA (8 each)
}

// keys[i] = morton16(floor(x * inv)) | batch << 48; OR of all keys into
// bits_or[0..1] (low / high word).
__global__ void __launch_bounds__(256)
    kv_keys(const float* __restrict__ xyz, const int64_t* __restrict__ batch, int64_t n,
            float inv, Meta* meta, uint32_t* bits_or, uint64_t* __restrict__ keys,
            uint32_t* __restrict__ vals) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  uint64_t key = 0;
  if (i < n) {
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // floor conversion; saturates instead of overflowing for huge values
      const long long g = __float2ll_rd(__fmul_rn(xyz[3 * i + a], inv));
      c[a] = static_cast<uint32_t>(g) & 0xffffu;
    }
    key = morton3(c[0], c[1], c[2]);
    if (batch) {
      int64_t b = batch[i];
      if (b < 0 || b >= 32768) {
        raise_status(&meta->status, kStatusBatch);
        b = b < 0 ? 0 : 32767;
      }
      key |= static_cast<uint64_t>(b) << 48;
    }
    keys[i] = key;
    vals[i] = static_cast<uint32_t>(i);
  }
  // OR over the block first: one pair of global atomics per block, not per
  // warp (all of them hit the same two words)
  __shared__ uint32_t s_or[2][8];
  const uint32_t lo = __reduce_or_sync(kFull, static_cast<uint32_t>(key));
  const uint32_t hi = __reduce_or_sync(kFull, static_cast<uint32_t>(key >> 32));
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_or[0][warp] = lo;
    s_or[1][warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    uint32_t v = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) v |= s_or[threadIdx.x][w];
    if (v) atomicOr(bits_or + threadIdx.x, v);
  }
}

__global__ void kv_bits(const uint32_t* bits_or, Meta* meta) {
  const uint64_t v = (static_cast<uint64_t>(bits_or[1]) << 32) | bits_or[0];
  meta->key_bits = v ? 64 - __clzll(static_cast<long long>(v)) : 0;
}

// Every key's first point in the stable order is its lowest index.
__global__ void __launch_bounds__(256)
    kv_heads(int64_t n, SortPair<uint64_t> sp, const int* bits, uint8_t* __restrict__ flag) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int buf = sort_passes_for_bits(*bits) & 1;
  const uint64_t* key = sp.key_buf(buf);
  if (s == 0 || key[s] != key[s - 1]) flag[sp.val_buf(buf)[s]] = 1;
}

__global__ void __launch_bounds__(256)
    kv_tiles(int64_t n, const uint8_t* __restrict__ flag, uint32_t* __restrict__ tile_counts) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * 8;
  uint32_t c = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r)
    if (base + r < n && flag[base + r]) ++c;
  block_inclusive_scan(c, warp_sums, &s_total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = s_total;
}

__global__ void __launch_bounds__(256)
    kv_compact(int64_t n, const uint8_t* __restrict__ flag,
               const uint32_t* __restrict__ tile_offsets, const int* total,
               int64_t* __restrict__ out, int64_t* __restrict__ count_out) {
  __shared__ uint32_t warp_sums[32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * 8;
  uint32_t bits = 0, c = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r)
    if (base + r < n && flag[base + r]) {
      bits |= 1u << r;
      ++c;
    }
  const uint32_t incl = block_inclusive_scan(c, warp_sums, nullptr);
  uint32_t pos = tile_offsets[blockIdx.x] + incl - c;
#pragma unroll
  for (int r = 0; r < 8; ++r)
    if (bits & (1u << r)) out[pos++] = base + r;
  if (blockIdx.x == 0 && threadIdx.x == 0) *count_out = *total;
}

namespace {

struct VBufs {
  Meta* meta;
  uint32_t* bits_or;
  uint64_t* keys[2];
  uint32_t* vals[2];
  uint32_t* hist;
  uint32_t* totals;
  uint32_t* tile_counts;
  uint8_t* flag;
};

VBufs vlayout(void* ws, int64_t n, size_t* bytes) {
  Arena a(ws);
  VBufs b{};
  b.meta = a.take<Meta>(1);
  b.bits_or = a.take<uint32_t>(2);
  b.keys[0] = a.take<uint64_t>(n);
  b.keys[1] = a.take<uint64_t>(n);
  b.vals[0] = a.take<uint32_t>(n);
  b.vals[1] = a.take<uint32_t>(n);
  b.hist = a.take<uint32_t>(sort_hist_elems(n));
  b.totals = a.take<uint32_t>(kSortMaxPasses * 256);
  b.tile_counts = a.take<uint32_t>(static_cast<size_t>(ceil_div(n > 0 ? n : 1, kTile)));
  b.flag = a.take<uint8_t>(n);
  if (bytes) *bytes = a.used + 256;
  return b;
}

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

}  // namespace

size_t voxel_first_workspace_bytes(int64_t n) {
  size_t bytes = 0;
  vlayout(nullptr, n, &bytes);
  return bytes;
}

int run_voxel_first(const VoxelArgs& v, void* ws, size_t ws_bytes, cudaStream_t s,
                    int* launches) {
  size_t need = 0;
  VBufs b = vlayout(ws, v.n, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  cudaError_t e = cudaMemsetAsync(b.meta, 0, sizeof(Meta), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.bits_or, 0, 2 * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.totals, 0, kSortMaxPasses * 256 * sizeof(uint32_t), s);
  if (e == cudaSuccess && v.n > 0) e = cudaMemsetAsync(b.flag, 0, static_cast<size_t>(v.n), s);
  if (e == cudaSuccess && v.n == 0) e = cudaMemsetAsync(v.count_out, 0, sizeof(int64_t), s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  int nl = 0;
  if (v.n > 0) {
    const float inv = 1.0f / v.voxel;  // host FP32 division, correctly rounded
    kv_keys<<<blocks_for(v.n, 256), 256, 0, s>>>(v.xyz, v.batch, v.n, inv, b.meta, b.bits_or,
                                                 b.keys[0], b.vals[0]);
    kv_bits<<<1, 1, 0, s>>>(b.bits_or, b.meta);
    nl += 2;
    SortBuffers<uint64_t> sb{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}, b.hist, b.totals};
    nl += launch_radix_sort(sb, v.n, &b.meta->key_bits, kSortMaxPasses, s);
    const SortPair<uint64_t> sp{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}};
    const int tiles = blocks_for(v.n, kTile);
    kv_heads<<<blocks_for(v.n, 256), 256, 0, s>>>(v.n, sp, &b.meta->key_bits, b.flag);
    kv_tiles<<<tiles, 256, 0, s>>>(v.n, b.flag, b.tile_counts);
    k_scan_tiles<<<1, 1024, 0, s>>>(b.tile_counts, tiles, &b.meta->n_cells);
    kv_compact<<<tiles, 256, 0, s>>>(v.n, b.flag, b.tile_counts, &b.meta->n_cells, v.out,
                                     v.count_out);
    nl += 4;
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
