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
// No sort is needed for that: the lowest index per key comes from an
// open-addressing table of the keys (capacity >= 2n, cleared by one memset).
//   kv_insert    key, one probe per distinct key per warp, the voxel's lowest
//                index kept in the slot (atomicMax of UINT32_MAX - index, so
//                a zeroed slot is neutral), the point's slot
//   kv_flags     flag[i] = (i is the lowest index of its voxel)
//   kv_tiles / k_scan_tiles / kv_compact
//                ordered compaction of the flags: the output comes out in
//                ascending index order
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

struct __align__(16) VoxelSlot {
  uint64_t key;    // voxel key + 1; 0 = empty
  uint32_t first;  // UINT32_MAX - lowest index of the voxel (0 = none yet)
  uint32_t pad;
};

__device__ __forceinline__ uint32_t voxel_hash(uint64_t key, uint32_t mask) {
  key ^= key >> 33;
  key *= 0xff51afd7ed558ccdULL;
  key ^= key >> 33;
  key *= 0xc4ceb9fe1a85ec53ULL;
  key ^= key >> 33;
  return static_cast<uint32_t>(key) & mask;
}

// key = morton16(floor(x * inv)) | batch << 48.  Lanes with the same key
// elect their lowest lane (the lowest index among them), which probes once
// and offers that index to the slot; slot_of[i] = the point's slot.
__global__ void __launch_bounds__(256)
    kv_insert(const float* __restrict__ xyz, const int64_t* __restrict__ batch, int64_t n,
              float inv, Meta* meta, VoxelSlot* __restrict__ table, uint32_t mask,
              uint32_t* __restrict__ slot_of) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const unsigned vmask = __ballot_sync(kFull, valid);
  if (!valid) return;
  uint32_t c[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    // floor conversion; saturates instead of overflowing for huge values
    const long long g = __float2ll_rd(__fmul_rn(xyz[3 * i + a], inv));
    c[a] = static_cast<uint32_t>(g) & 0xffffu;
  }
  uint64_t key = morton3(c[0], c[1], c[2]);
  if (batch) {
    int64_t b = batch[i];
    if (b < 0 || b >= 32768) {
      raise_status(&meta->status, kStatusBatch);
      b = b < 0 ? 0 : 32767;
    }
    key |= static_cast<uint64_t>(b) << 48;
  }
  key += 1;
  const unsigned peers = __match_any_sync(vmask, key);
  const int leader = __ffs(peers) - 1;
  uint32_t slot = 0u;
  if ((threadIdx.x & 31) == leader) {
    uint32_t h = voxel_hash(key, mask);
    bool found = false;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const unsigned long long prev =
          atomicCAS(reinterpret_cast<unsigned long long*>(&table[h].key), 0ull, key);
      if (prev == 0ull || prev == key) {
        found = true;
        break;
      }
      h = (h + 1) & mask;
    }
    if (found) {
      atomicMax(&table[h].first, 0xffffffffu - static_cast<uint32_t>(i));
      slot = h;
    } else {
      raise_status(&meta->status, kStatusTable);  // cannot happen at load <= 1/2
    }
  }
  slot_of[i] = __shfl_sync(peers, slot, leader);
}

__global__ void __launch_bounds__(256)
    kv_flags(int64_t n, const VoxelSlot* __restrict__ table, const uint32_t* __restrict__ slot_of,
             uint8_t* __restrict__ flag) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = (0xffffffffu - table[slot_of[i]].first) == static_cast<uint32_t>(i) ? 1 : 0;
}

__global__ void __launch_bounds__(256)
    kv_tiles(int64_t n, const uint8_t* __restrict__ flag, uint32_t* __restrict__ tile_counts) {
  chain_wait();
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
  chain_wait();
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
  VoxelSlot* table;
  int64_t cap;
  uint32_t* slot_of;
  uint32_t* tile_counts;
  uint8_t* flag;
};

VBufs vlayout(void* ws, int64_t n, size_t* bytes) {
  Arena a(ws);
  VBufs b{};
  b.meta = a.take<Meta>(1);
  b.cap = 16;
  while (b.cap < 2 * n) b.cap <<= 1;
  b.table = a.take<VoxelSlot>(b.cap);
  b.slot_of = a.take<uint32_t>(n);
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
  if (e == cudaSuccess && v.n > 0)
    e = cudaMemsetAsync(b.table, 0, sizeof(VoxelSlot) * static_cast<size_t>(b.cap), s);
  if (e == cudaSuccess && v.n == 0) e = cudaMemsetAsync(v.count_out, 0, sizeof(int64_t), s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  int nl = 0;
  if (v.n > 0) {
    const float inv = 1.0f / v.voxel;  // host FP32 division, correctly rounded
    launch_chained(kv_insert, blocks_for(v.n, 256), 256, 0, s, v.xyz, v.batch, v.n, inv, b.meta,
                   b.table, static_cast<uint32_t>(b.cap - 1), b.slot_of);
    const int tiles = blocks_for(v.n, kTile);
    launch_chained(kv_flags, blocks_for(v.n, 256), 256, 0, s, v.n, b.table, b.slot_of, b.flag);
    launch_chained(kv_tiles, tiles, 256, 0, s, v.n, b.flag, b.tile_counts);
    launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts, tiles, &b.meta->n_cells);
    launch_chained(kv_compact, tiles, 256, 0, s, v.n, b.flag, b.tile_counts, &b.meta->n_cells,
                   v.out, v.count_out);
    nl += 5;
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
