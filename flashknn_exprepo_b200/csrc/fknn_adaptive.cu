// Adaptive-neighbourhood self query: every point picks the octree level
// whose 3x3x3 node neighbourhood holds a useful number of candidates, then
// takes its exact top-K there.  Semantics of the reference's
// AdaptiveNeighborhoodFlashKNN (FlashKNN/functions/adaptive_octree.py):
//   * grid coordinates are translated per batch to their minimum
//     (:129-147; every translated coordinate must stay below 2^16);
//   * level s groups the points by (batch, key >> 3s) (:256-274), for
//     s = 0..S, S = max_shift or the bit length of the largest translated
//     coordinate (:249-252);
//   * a node's candidate count is the number of points in the 27 nodes of
//     its level at integer offsets (0,-1,+1)^3 (:150-205, :287-302);
//   * selection (:312-351): start at S, active = count > max_f*K; for
//     s = S-1..0 an active point moves to level s when its level-s count is
//     >= min_f*K and stays active while that count is > max_f*K;
//   * the query is the exact top-K over the 27 nodes around the point's node
//     at its selected level (:369-488, :555-575), padding (own index, +inf).
//
// B200 layout.  The points are sorted once by (batch, morton(translated
// grid)); in that order every node of every level is a contiguous range, so
// no coordinates are copied per level (the reference gathers a copy of every
// referenced support node, :605-608).  Node boundaries, node sizes and the
// 27-node candidate counts do not depend on the selection, so every level is
// built at once:
//   ka_heads_all / ka_scan_all           node heads per tile and level (the
//                                        highest bit in which neighbouring
//                                        keys differ), scanned per level
//   ka_level_bases / ka_table_clear      node numbering across levels, table
//                                        capacity
//   ka_nodes_all                         node starts of every level
//   ka_insert_all                        one table for all levels: level key
//                                        -> (start, count)
//   ka_counts_all                        27-node candidate count of every node
//   ka_select_all                        per point: its level, walking the
//                                        levels from the top in registers;
//                                        group starts write their 27 runs
// A query group is a maximal run of sorted points with the same selected
// level and node; its runs address the same sorted records as its queries,
// so the packer and the top-K kernel of the fixed-level path serve it
// unchanged (fknn_items.cu, fknn_query.cu).  Every data-dependent size (the
// top level S included) stays on the device: the pipeline is a fixed launch
// sequence and can be captured in a CUDA graph.
#include <climits>

#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"
#include "fknn_adaptive.h"

namespace fknn {

namespace {

constexpr int kMaxLevel = 16;
constexpr int kBatchSlots = 32768;
constexpr int kTile = 2048;  // sorted positions per 256-thread CTA (8 each)

// Meta fields: bpa = bits per axis of the key layout, reserved[0] = S (top
// level), reserved[1] = largest batch id + 1, key_bits = 3 * bpa + batch bits.
__device__ __forceinline__ int top_level(const Meta* m) { return m->reserved[0]; }
__device__ __forceinline__ int* batch_slots_used(Meta* m) { return &m->reserved[1]; }

__device__ __forceinline__ uint32_t slot_of_key(uint64_t key, uint32_t mask) {
  key ^= key >> 33;
  key *= 0xff51afd7ed558ccdULL;
  key ^= key >> 33;
  key *= 0xc4ceb9fe1a85ec53ULL;
  key ^= key >> 33;
  return static_cast<uint32_t>(key) & mask;
}

// One 16-byte slot of the node table: level key (0 = empty) and the node's
// run (start, count).
struct __align__(16) Slot {
  uint64_t key;
  int2 run;
};

__device__ __forceinline__ const uint64_t* sorted_keys(const SortPair<uint64_t>& sp,
                                                       const int* bits) {
  return sp.key_buf(sort_passes_for_bits(*bits) & 1);
}

__device__ __forceinline__ const uint32_t* sorted_vals(const SortPair<uint64_t>& sp,
                                                       const int* bits) {
  return sp.val_buf(sort_passes_for_bits(*bits) & 1);
}

__device__ __forceinline__ bool node_head(const uint64_t* key, int64_t p, int shift) {
  return p == 0 || (key[p] >> shift) != (key[p - 1] >> shift);
}

}  // namespace

// ------------------------------------------------------------ boxes, keys

__global__ void ka_init(Meta* meta, long long* box, uint32_t* totals, int n_totals) {
  chain_wait();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  if (t < static_cast<int64_t>(sizeof(Meta) / sizeof(int))) reinterpret_cast<int*>(meta)[t] = 0;
  for (int64_t i = t; i < static_cast<int64_t>(kBatchSlots) * 6; i += stride)
    box[i] = (i % 6) < 3 ? LLONG_MAX : LLONG_MIN;
  for (int64_t i = t; i < n_totals; i += stride) totals[i] = 0u;
}

__device__ __forceinline__ int batch_of(const int64_t* batch, int64_t i, int* status) {
  if (!batch) return 0;
  int64_t b = batch[i];
  if (b < 0 || b >= kBatchSlots) {
    raise_status(status, kStatusBatch);
    b = b < 0 ? 0 : kBatchSlots - 1;
  }
  return static_cast<int>(b);
}

// Per-batch bounding boxes of the grid coordinates.  2048 points per CTA;
// the batches of the tile's first and last point are reduced in shared
// memory (offset batching puts one or two batches in most tiles), any other
// batch goes straight to global atomics.
__global__ void __launch_bounds__(256)
    ka_box(const int64_t* __restrict__ grid, const int64_t* __restrict__ batch, int64_t n,
           long long* __restrict__ box, Meta* meta) {
  chain_wait();
  __shared__ long long sh[2][6];
  int* status = &meta->status;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile;
  const int64_t last = min(base + kTile - 1, n - 1);
  const int b_lo = batch_of(batch, base, status);
  const int b_hi = batch_of(batch, last, status);
  if (threadIdx.x < 12) sh[threadIdx.x / 6][threadIdx.x % 6] = (threadIdx.x % 6) < 3 ? LLONG_MAX
                                                                                       : LLONG_MIN;
  __syncthreads();
  long long lo[2][6];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int a = 0; a < 6; ++a) lo[h][a] = a < 3 ? LLONG_MAX : LLONG_MIN;
  int b_max = -1;
  for (int r = 0; r < 8; ++r) {
    const int64_t i = base + r * 256 + threadIdx.x;
    if (i >= n) break;
    const int b = batch_of(batch, i, status);
    b_max = max(b_max, b);
    const long long g[3] = {grid[3 * i], grid[3 * i + 1], grid[3 * i + 2]};
    if (b == b_lo || b == b_hi) {
      const int h = b == b_lo ? 0 : 1;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lo[h][a] = min(lo[h][a], g[a]);
        lo[h][a + 3] = max(lo[h][a + 3], g[a]);
      }
    } else {
      long long* dst = box + 6 * static_cast<int64_t>(b);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        atomicMin(dst + a, g[a]);
        atomicMax(dst + a + 3, g[a]);
      }
    }
  }
  b_max = __reduce_max_sync(kFull, b_max);
  if ((threadIdx.x & 31) == 0 && b_max >= 0) atomicMax(batch_slots_used(meta), b_max + 1);
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      long long v = lo[h][a];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const long long w = __shfl_xor_sync(kFull, v, o);
        v = a < 3 ? min(v, w) : max(v, w);
      }
      if ((threadIdx.x & 31) == 0) {
        if (a < 3) atomicMin(&sh[h][a], v); else atomicMax(&sh[h][a], v);
      }
    }
  __syncthreads();
  if (threadIdx.x < 12) {
    const int h = threadIdx.x / 6, a = threadIdx.x % 6;
    const int b = h == 0 ? b_lo : b_hi;
    if (h == 1 && b_hi == b_lo) return;
    const long long v = sh[h][a];
    long long* dst = box + 6 * static_cast<int64_t>(b) + a;
    if (a < 3) {
      if (v != LLONG_MAX) atomicMin(dst, v);
    } else if (v != LLONG_MIN) {
      atomicMax(dst, v);
    }
  }
}

// One CTA: top level S, key layout (bits per axis, batch bits), span check.
__global__ void __launch_bounds__(1024)
    ka_meta(const long long* __restrict__ box, int max_shift, Meta* meta) {
  chain_wait();
  __shared__ long long s_span[32];
  __shared__ int s_b[32];
  long long span = 0;
  int maxb = 0;
  const int used = min(*batch_slots_used(meta), kBatchSlots);  // boxes above are empty
  for (int b = threadIdx.x; b < used; b += blockDim.x) {
    const long long* bx = box + 6 * static_cast<int64_t>(b);
    if (bx[0] <= bx[3]) {
      span = max(span, max(bx[3] - bx[0], max(bx[4] - bx[1], bx[5] - bx[2])));
      maxb = max(maxb, b);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    span = max(span, __shfl_xor_sync(kFull, span, o));
    maxb = max(maxb, __shfl_xor_sync(kFull, maxb, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s_span[threadIdx.x >> 5] = span;
    s_b[threadIdx.x >> 5] = maxb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) {
      span = max(span, s_span[w]);
      maxb = max(maxb, s_b[w]);
    }
    if (span >= 65536) {
      raise_status(&meta->status, kStatusRange);
      span = 65535;
    }
    const int auto_s = span > 0 ? 64 - __clzll(span) : 0;
    const int top = max_shift >= 0 ? max_shift : auto_s;
    const int bpa = max(auto_s, top);
    const int bb = maxb > 0 ? 32 - __clz(maxb) : 0;
    meta->bpa = bpa;
    meta->batch_bits = bb;
    meta->max_extent = static_cast<int>(span);
    meta->key_bits = 3 * bpa + bb;
    meta->reserved[0] = top;
  }
}

__device__ __forceinline__ void translated(const int64_t* grid, const long long* box, int b,
                                           int64_t i, uint32_t* c) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    long long v = grid[3 * i + a] - box[6 * static_cast<int64_t>(b) + a];
    v = v < 0 ? 0 : (v > 65535 ? 65535 : v);  // out of range: status already raised
    c[a] = static_cast<uint32_t>(v);
  }
}

__global__ void __launch_bounds__(256)
    ka_keys(const int64_t* __restrict__ grid, const int64_t* __restrict__ batch, int64_t n,
            const long long* __restrict__ box, Meta* meta, uint64_t* __restrict__ keys,
            uint32_t* __restrict__ vals) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = batch_of(batch, i, &meta->status);
  uint32_t c[3];
  translated(grid, box, b, i, c);
  keys[i] = (static_cast<uint64_t>(b) << (3 * meta->bpa)) | morton3(c[0], c[1], c[2]);
  vals[i] = static_cast<uint32_t>(i);
}

// Sorted records (position, input index); positions are xyz, or the
// translated grid coordinates when xyz is null.
__global__ void __launch_bounds__(256)
    ka_records(const float* __restrict__ xyz, const int64_t* __restrict__ grid,
               const int64_t* __restrict__ batch, int64_t n, const long long* __restrict__ box,
               SortPair<uint64_t> sp, const int* bits, Meta* meta, float4* __restrict__ rec) {
  chain_wait();
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int64_t id = sorted_vals(sp, bits)[s];
  float4 r;
  if (xyz) {
    r = make_float4(xyz[3 * id], xyz[3 * id + 1], xyz[3 * id + 2], 0.f);
  } else {
    uint32_t c[3];
    translated(grid, box, batch_of(batch, id, &meta->status), id, c);
    r = make_float4(static_cast<float>(c[0]), static_cast<float>(c[1]), static_cast<float>(c[2]),
                    0.f);
  }
  r.w = __int_as_float(static_cast<int>(id));
  rec[s] = r;
}

// ------------------------------------------------------------------ levels

struct LevelArgs {
  SortPair<uint64_t> sp;
  const int* bits;
  const Meta* meta;
  int64_t n;
  int s;
};

// Node heads of every level in one pass.  Position p heads a level-s node
// when key[p] >> 3s differs from key[p-1] >> 3s, i.e. when the highest bit in
// which the two keys differ is at least 3s: so p heads the nodes of levels
// 0..hb/3.  tile_counts[s * n_tiles + tile] = heads of level s in the tile.
__global__ void __launch_bounds__(256)
    ka_heads_all(LevelArgs a, int n_tiles, uint32_t* __restrict__ tile_counts) {
  chain_wait();
  __shared__ uint32_t hist[kMaxLevel + 1];
  if (threadIdx.x <= kMaxLevel) hist[threadIdx.x] = 0u;
  __syncthreads();
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * 8;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t p = base + r;
    if (p >= a.n) break;
    int lvl = kMaxLevel;
    if (p > 0) {
      const uint64_t x = key[p] ^ key[p - 1];
      if (x == 0) continue;  // same leaf key: heads no node
      lvl = min((63 - __clzll(static_cast<long long>(x))) / 3, kMaxLevel);
    }
    atomicAdd(&hist[lvl], 1u);
  }
  __syncthreads();
  if (threadIdx.x <= kMaxLevel) {  // heads of level s = points whose lvl >= s
    uint32_t c = 0;
    for (int l = threadIdx.x; l <= kMaxLevel; ++l) c += hist[l];
    tile_counts[static_cast<int64_t>(threadIdx.x) * n_tiles + blockIdx.x] = c;
  }
}

// One CTA per level: exclusive scan of that level's tile counts in place,
// level_nodes[s] = the level's node count.
__global__ void __launch_bounds__(1024)
    ka_scan_all(uint32_t* __restrict__ tile_counts, int n_tiles, int* __restrict__ level_nodes) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  uint32_t* col = tile_counts + static_cast<int64_t>(blockIdx.x) * n_tiles;
  uint32_t carry = 0;
  for (int t0 = 0; t0 < n_tiles; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const uint32_t x = t < n_tiles ? col[t] : 0u;
    const uint32_t incl = block_inclusive_scan(x, warp_sums, &s_total);
    if (t < n_tiles) col[t] = carry + incl - x;
    carry += s_total;
  }
  if (threadIdx.x == 0) level_nodes[blockIdx.x] = static_cast<int>(carry);
}

// ---- all levels at once.  Node boundaries, node tables and 27-node counts
// do not depend on the selection, so they are built for every level in one
// pass each; only the selection walks the levels, per point, in registers.
//
// One open-addressing table holds the nodes of every level under the key
// level_key(key, s) = (key >> 3s) | 2^(63 - 3s): keys have at most 63 bits,
// so a level-s node key has at most 63 - 3s bits and the marker bit keeps the
// levels' key ranges disjoint (and every key non-zero: 0 marks an empty slot).
// A slot holds the node's run (start, count); cand_slot[slot] its 27-node
// candidate count.  Global node g of level s is node g - base[s] of that
// level; base[s + 1] = base[s] + nodes(s) + 1 (one sentinel per level), so
// node_start[g + 1] - node_start[g] is always the node's size.

__device__ __forceinline__ uint64_t level_key(uint64_t key, int s) {
  return (key >> (3 * s)) | (1ull << (63 - 3 * s));
}

struct LTable {
  Slot* slots;
  const int* mask_word;  // capacity - 1, set on the device
};

// Run of the node with level key v: one 16-byte load per probe; (0, 0)
// when absent.
__device__ __forceinline__ int2 level_find(const Slot* slots, uint32_t mask, uint64_t v) {
  uint32_t h = slot_of_key(v, mask);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const ulonglong2 e = __ldcg(reinterpret_cast<const ulonglong2*>(slots + h));
    if (e.x == v)
      return make_int2(static_cast<int>(static_cast<uint32_t>(e.y)),
                       static_cast<int>(static_cast<uint32_t>(e.y >> 32)));
    if (e.x == 0ull) break;
    h = (h + 1) & mask;
  }
  return make_int2(0, 0);
}

// Run of neighbour j of the level-s node with node key nk, or (0, 0) when
// the neighbour is outside the grid or empty.
__device__ __forceinline__ int2 level_neighbour_run(const Slot* slots, uint32_t mask, uint64_t nk,
                                                    int s, int bpa, int j) {
  const int sb = 3 * (bpa - s);  // spatial bits of a level-s node key
  const uint64_t batch = nk >> sb;
  const uint64_t m = sb ? (nk & ((1ull << sb) - 1)) : 0ull;
  const int lim = 1 << (bpa - s);
  const int x = static_cast<int>(compact3(m >> 2)) + (j / 9 == 0 ? 0 : (j / 9 == 1 ? -1 : 1));
  const int jy = (j / 3) % 3, jz = j % 3;
  const int y = static_cast<int>(compact3(m >> 1)) + (jy == 0 ? 0 : (jy == 1 ? -1 : 1));
  const int z = static_cast<int>(compact3(m)) + (jz == 0 ? 0 : (jz == 1 ? -1 : 1));
  if (x < 0 || y < 0 || z < 0 || x >= lim || y >= lim || z >= lim) return make_int2(0, 0);
  const uint64_t key = (batch << sb) | morton3(static_cast<uint32_t>(x), static_cast<uint32_t>(y),
                                               static_cast<uint32_t>(z));
  return level_find(slots, mask, key | (1ull << (63 - 3 * s)));
}

// Level of global node g (base[] has top + 2 entries).
__device__ __forceinline__ int level_of_node(const int* base, int top, int64_t g) {
  int s = 0;
  while (s < top && g >= base[s + 1]) ++s;
  return s;
}

// Meta words of the all-levels pipeline.
__device__ __forceinline__ int* level_mask_word(Meta* m) { return &m->reserved[2]; }

// One warp: base[s] for s = 0..top+1 and the table mask: capacity = next
// power of two >= 4 x all nodes (most neighbour lookups miss, and misses end
// at the first empty slot), at most the allocated capacity, which holds
// twice the largest possible node count.
__global__ void ka_level_bases(const int* __restrict__ level_nodes, Meta* meta,
                               int* __restrict__ base, int64_t max_cap) {
  chain_wait();
  if (threadIdx.x != 0) return;
  const int top = top_level(meta);
  int b = 0;
  for (int s = 0; s <= top; ++s) {
    base[s] = b;
    b += level_nodes[s] + 1;
  }
  base[top + 1] = b;
  int64_t cap = 16;
  while (cap < 4 * static_cast<int64_t>(b)) cap <<= 1;
  if (cap > max_cap) cap = max_cap;
  *level_mask_word(meta) = static_cast<int>(cap - 1);
}

__global__ void __launch_bounds__(256)
    ka_table_clear(Slot* __restrict__ slots, const Meta* meta) {
  chain_wait();
  const int64_t cap = static_cast<int64_t>(static_cast<uint32_t>(meta->reserved[2])) + 1;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < cap;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    slots[i].key = 0ull;
}

// Head level of sorted position p: p heads the nodes of levels 0..hl, or
// hl = -1 when its key equals its predecessor's.
__device__ __forceinline__ int head_level(const uint64_t* key, int64_t p) {
  if (p == 0) return kMaxLevel;
  const uint64_t x = key[p] ^ key[p - 1];
  if (x == 0) return -1;
  return min((63 - __clzll(static_cast<long long>(x))) / 3, kMaxLevel);
}

// Node starts of every level, and node_of[s * n + p] = the global node of
// sorted position p at level s: tile of 2048 positions, 8 per thread, one
// block scan per level over the precomputed per-level tile offsets.
__global__ void __launch_bounds__(256)
    ka_nodes_all(LevelArgs a, int n_tiles, const uint32_t* __restrict__ tile_offsets,
                 const int* __restrict__ level_nodes, const int* __restrict__ base,
                 int32_t* __restrict__ node_start, int32_t* __restrict__ node_of) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  const int top = top_level(a.meta);
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int64_t p0 = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * 8;
  int hl[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) hl[r] = p0 + r < a.n ? head_level(key, p0 + r) : -1;
  for (int s = 0; s <= top; ++s) {
    uint32_t heads = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r) heads += hl[r] >= s ? 1u : 0u;
    const uint32_t incl = block_inclusive_scan(heads, warp_sums, nullptr);
    int64_t g = base[s] + static_cast<int64_t>(tile_offsets[static_cast<int64_t>(s) * n_tiles +
                                                            blockIdx.x]) + incl - heads - 1;
    int32_t* nof = node_of + static_cast<int64_t>(s) * a.n;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      if (p0 + r >= a.n) break;
      if (hl[r] >= s) node_start[++g] = static_cast<int32_t>(p0 + r);
      nof[p0 + r] = static_cast<int32_t>(g);
    }
    if (p0 <= a.n - 1 && a.n - 1 < p0 + 8)  // the sentinel after the level's last node
      node_start[base[s] + level_nodes[s]] = static_cast<int32_t>(a.n);
  }
}

// Every node of every level into the table: (start, count) under its level
// key.  One thread per global node.
__global__ void __launch_bounds__(256)
    ka_insert_all(LevelArgs a, const int* __restrict__ base, const int32_t* __restrict__ node_start,
                  Slot* __restrict__ slots) {
  chain_wait();
  const int top = top_level(a.meta);
  const uint32_t mask = static_cast<uint32_t>(a.meta->reserved[2]);
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int64_t total = base[top + 1];
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int s = level_of_node(base, top, g);
    if (g == base[s + 1] - 1) continue;  // the level's sentinel
    const int32_t st = node_start[g];
    const uint64_t v = level_key(key[st], s);
    uint32_t h = slot_of_key(v, mask);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const unsigned long long prev =
          atomicCAS(reinterpret_cast<unsigned long long*>(&slots[h].key), 0ull, v);
      if (prev == 0ull) {
        slots[h].run = make_int2(st, node_start[g + 1] - st);
        break;
      }
      h = (h + 1) & mask;
    }
  }
}

// cand[g] = points in the 27 same-level nodes around global node g.  One
// warp per node, one lookup per lane.
__global__ void __launch_bounds__(256)
    ka_counts_all(LevelArgs a, const int* __restrict__ base,
                  const int32_t* __restrict__ node_start, const Slot* __restrict__ slots,
                  int32_t* __restrict__ cand) {
  chain_wait();
  const int top = top_level(a.meta);
  const uint32_t mask = static_cast<uint32_t>(a.meta->reserved[2]);
  const int bpa = a.meta->bpa;
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int64_t total = base[top + 1];
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; g < total;
       g += warps) {
    const int s = level_of_node(base, top, g);
    if (g == base[s + 1] - 1) continue;  // sentinel (warp-uniform)
    const uint64_t nk = key[node_start[g]] >> (3 * s);
    const int len = lane < kNeighbours ? level_neighbour_run(slots, mask, nk, s, bpa, lane).y : 0;
    const int t = __reduce_add_sync(kFull, len);
    if (lane == 0) cand[g] = t;
  }
}

// Selected level of sorted position q: from the top level down, an active
// point moves to level s when its level-s count is >= min_count and stays
// active while it is > max_count (adaptive_octree.py:312-351).  The counts
// of all levels are loaded first (independent loads), then walked.
__device__ __forceinline__ int select_level(int64_t q, int64_t n, int top,
                                            const int32_t* __restrict__ node_of,
                                            const int32_t* __restrict__ cand, int min_count,
                                            int max_count) {
  int cnt[kMaxLevel + 1];
#pragma unroll
  for (int s = 0; s <= kMaxLevel; ++s)
    cnt[s] = s <= top ? __ldcg(cand + __ldcg(node_of + static_cast<int64_t>(s) * n + q)) : 0;
  int sel = top;
  bool act = false;
#pragma unroll
  for (int s = kMaxLevel; s >= 0; --s) {
    if (s > top) continue;
    if (s == top) {
      act = cnt[s] > max_count;
    } else if (act) {
      const bool use = cnt[s] >= min_count;
      if (use) sel = s;
      act = use && cnt[s] > max_count;
    }
  }
  return sel;
}

// Level selection of every point, then the query groups: a group is a
// maximal run of sorted positions with the same selected level L and the
// same level-L node; its start writes group_flag and the 27 runs (row p).
// One warp per 32 positions; lane 0 recomputes its predecessor's level.
__global__ void __launch_bounds__(256)
    ka_select_all(LevelArgs a, const Slot* __restrict__ slots, const int32_t* __restrict__ node_of,
                  const int32_t* __restrict__ cand, int min_count, int max_count,
                  uint8_t* __restrict__ sel_out, uint8_t* __restrict__ group_flag,
                  int2* __restrict__ runs) {
  chain_wait();
  const int top = top_level(a.meta);
  const uint32_t mask = static_cast<uint32_t>(a.meta->reserved[2]);
  const int bpa = a.meta->bpa;
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t base = ((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * 32;
       base < a.n; base += warps * 32) {
    const int64_t p = base + lane;
    int L = -1;
    if (p < a.n) {
      L = select_level(p, a.n, top, node_of, cand, min_count, max_count);
      sel_out[p] = static_cast<uint8_t>(L);
    }
    int prev = __shfl_up_sync(kFull, L, 1);
    if (lane == 0 && p > 0 && p < a.n)
      prev = select_level(p - 1, a.n, top, node_of, cand, min_count, max_count);
    bool start = false;
    if (p < a.n) {
      start = p == 0 || prev != L || node_head(key, p, 3 * L);
      group_flag[p] = start ? 1 : 0;
    }
    uint32_t starts = __ballot_sync(kFull, start);
    while (starts) {
      const int src = __ffs(starts) - 1;
      starts &= starts - 1;
      const int64_t ps = base + src;
      const int Ls = __shfl_sync(kFull, L, src);
      if (lane < kNeighbours)
        runs[ps * kNeighbours + lane] =
            level_neighbour_run(slots, mask, key[ps] >> (3 * Ls), Ls, bpa, lane);
    }
  }
}

// ------------------------------------------------------------------ groups

__global__ void __launch_bounds__(256)
    ka_group_tiles(int64_t n, const uint8_t* __restrict__ flag, uint32_t* __restrict__ tile_counts) {
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
    ka_groups(int64_t n, const uint8_t* __restrict__ flag, const uint32_t* __restrict__ tile_offsets,
              const int* count_ptr, int32_t* __restrict__ group_start,
              int32_t* __restrict__ group_row) {
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
  int g = static_cast<int>(tile_offsets[blockIdx.x] + incl - c);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t p = base + r;
    if (p >= n) break;
    if (bits & (1u << r)) {
      group_start[g] = static_cast<int32_t>(p);
      group_row[g] = static_cast<int32_t>(p);
      ++g;
    }
    if (p == n - 1) group_start[*count_ptr] = static_cast<int32_t>(n);
  }
}

__global__ void __launch_bounds__(256)
    ka_levels_out(int64_t n, const float4* __restrict__ rec, const uint8_t* __restrict__ sel,
                  int8_t* __restrict__ out) {
  chain_wait();
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= n) return;
  out[__float_as_int(rec[p].w)] = static_cast<int8_t>(sel[p]);
}

// --------------------------------------------------------------- host side

namespace {

struct ABufs {
  Meta* meta;
  long long* box;
  uint64_t* keys[2];
  uint32_t* vals[2];
  uint32_t* hist;
  uint32_t* totals;
  uint32_t* tile_counts;
  float4* rec;
  int* level_nodes;        // [kMaxLevel + 1]
  int* level_base;         // [kMaxLevel + 2]
  int32_t* node_start;     // nodes of every level, one sentinel per level
  int32_t* node_of;        // [kMaxLevel + 1][n] global node of each sorted position
  Slot* slots;             // node table of every level
  int32_t* cand;           // 27-node count per global node
  int64_t cap;             // table allocation: twice the largest possible node count
  uint8_t* sel;
  uint8_t* group_flag;
  int2* runs;
  int32_t* group_start;
  int32_t* group_row;
  int4* items;
  int32_t* cands;
  uint32_t* seg_counts;
};

ABufs alayout(void* ws, int64_t n, size_t* bytes) {
  Arena a(ws);
  ABufs b{};
  b.meta = a.take<Meta>(1);
  b.box = a.take<long long>(6 * static_cast<size_t>(kBatchSlots));
  b.keys[0] = a.take<uint64_t>(n);
  b.keys[1] = a.take<uint64_t>(n);
  b.vals[0] = a.take<uint32_t>(n);
  b.vals[1] = a.take<uint32_t>(n);
  b.hist = a.take<uint32_t>(sort_hist_elems(n));
  b.totals = a.take<uint32_t>(kSortMaxPasses * 256);
  b.tile_counts = a.take<uint32_t>(static_cast<size_t>(kMaxLevel + 1) *
                                   static_cast<size_t>(ceil_div(n > 0 ? n : 1, kTile)));
  b.rec = a.take<float4>(n);
  b.level_nodes = a.take<int>(kMaxLevel + 1);
  b.level_base = a.take<int>(kMaxLevel + 2);
  // at most n nodes (+ a sentinel) on each of the kMaxLevel + 1 levels
  const int64_t max_nodes = static_cast<int64_t>(kMaxLevel + 1) * (n + 1);
  b.node_start = a.take<int32_t>(max_nodes);
  b.node_of = a.take<int32_t>(static_cast<size_t>(kMaxLevel + 1) * static_cast<size_t>(n));
  b.cap = 16;
  while (b.cap < 2 * max_nodes) b.cap <<= 1;
  b.slots = a.take<Slot>(b.cap);
  b.cand = a.take<int32_t>(max_nodes);
  b.sel = a.take<uint8_t>(n);
  b.group_flag = a.take<uint8_t>(n);
  b.runs = a.take<int2>(static_cast<size_t>(n) * kNeighbours);
  b.group_start = a.take<int32_t>(n + 1);
  b.group_row = a.take<int32_t>(n);
  b.items = a.take<int4>(items_capacity(n, n));
  b.cands = a.take<int32_t>(n);
  b.seg_counts = a.take<uint32_t>(pack_segments(n));
  if (bytes) *bytes = a.used + 256;
  return b;
}

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

inline int capped_blocks(int64_t threads) {
  const int64_t b = ceil_div(threads > 0 ? threads : 1, 256);
  return static_cast<int>(b < 2048 ? b : 2048);
}

}  // namespace

size_t adaptive_workspace_bytes(int64_t n) {
  size_t bytes = 0;
  alayout(nullptr, n, &bytes);
  return bytes;
}

int run_adaptive(const AdaptiveArgs& f, void* ws, size_t ws_bytes, const QueryShape& shape,
                 cudaStream_t s, int* launches) {
  const int64_t n = f.n;
  size_t need = 0;
  ABufs b = alayout(ws, n, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  if (n <= 0) {
    if (launches) *launches = 0;
    return FKNN_OK;
  }
  int nl = 0;
  cudaError_t e;
  launch_chained(ka_init, 64, 256, 0, s, b.meta, b.box, b.totals, kSortMaxPasses * 256);
  launch_chained(ka_box, blocks_for(n, kTile), 256, 0, s, f.grid, f.batch, n, b.box, b.meta);
  launch_chained(ka_meta, 1, 1024, 0, s, b.box, f.max_shift, b.meta);
  launch_chained(ka_keys, blocks_for(n, 256), 256, 0, s, f.grid, f.batch, n, b.box, b.meta,
                 b.keys[0], b.vals[0]);
  nl += 4;
  const int* key_bits = &b.meta->key_bits;
  SortBuffers<uint64_t> sb{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}, b.hist, b.totals};
  nl += launch_radix_sort(sb, n, key_bits, sort_passes_for_bits(3 * kMaxLevel + 15), s);
  const SortPair<uint64_t> sp{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}};
  launch_chained(ka_records, blocks_for(n, 256), 256, 0, s, f.xyz, f.grid, f.batch, n, b.box, sp,
                 key_bits, b.meta, b.rec);
  ++nl;

  const int tiles = blocks_for(n, kTile);
  const int min_count = f.min_factor * f.k, max_count = f.max_factor * f.k;
  const int top_host = f.max_shift >= 0 ? f.max_shift : kMaxLevel;
  const LevelArgs la{sp, key_bits, b.meta, n, 0};
  const int64_t node_bound = static_cast<int64_t>(top_host + 1) * (n + 1);
  launch_chained(ka_heads_all, tiles, 256, 0, s, la, tiles, b.tile_counts);
  launch_chained(ka_scan_all, kMaxLevel + 1, 1024, 0, s, b.tile_counts, tiles, b.level_nodes);
  launch_chained(ka_level_bases, 1, 32, 0, s, b.level_nodes, b.meta, b.level_base, b.cap);
  launch_chained(ka_table_clear, capped_blocks(b.cap), 256, 0, s, b.slots, b.meta);
  launch_chained(ka_nodes_all, tiles, 256, 0, s, la, tiles, b.tile_counts, b.level_nodes,
                 b.level_base, b.node_start, b.node_of);
  launch_chained(ka_insert_all, capped_blocks(node_bound), 256, 0, s, la, b.level_base,
                 b.node_start, b.slots);
  launch_chained(ka_counts_all, capped_blocks(node_bound * 32), 256, 0, s, la, b.level_base,
                 b.node_start, b.slots, b.cand);
  launch_chained(ka_select_all, capped_blocks(n), 256, 0, s, la, b.slots, b.node_of, b.cand,
                 min_count, max_count, b.sel, b.group_flag, b.runs);
  launch_chained(ka_group_tiles, tiles, 256, 0, s, n, b.group_flag, b.tile_counts);
  launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts, tiles, &b.meta->n_groups);
  launch_chained(ka_groups, tiles, 256, 0, s, n, b.group_flag, b.tile_counts, &b.meta->n_groups,
                 b.group_start, b.group_row);
  nl += 11;
  if (f.level_out) {
    launch_chained(ka_levels_out, blocks_for(n, 256), 256, 0, s, n, b.rec, b.sel, f.level_out);
    ++nl;
  }
  nl += launch_items(b.runs, b.group_start, b.group_row, &b.meta->n_groups, n, shape.tile_records,
                     b.cands, b.seg_counts, &b.meta->n_items, b.items, s, &b.meta->status, n,
                     false);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  QueryLaunch q{};
  q.srec = b.rec;
  q.n_support = static_cast<int>(n);
  q.qrec = b.rec;
  q.n_qrec = static_cast<int>(n);
  q.runs = b.runs;
  q.group_start = b.group_start;
  q.group_row = b.group_row;
  q.group_count_ptr = &b.meta->n_groups;
  q.items = b.items;
  q.meta = b.meta;
  q.k = f.k;
  q.cut_r2 = f.cut_r2;
  q.idx_bits = f.idx_bits;
  q.idx_out = f.idx_out;
  q.dist_out = f.dist_out;
  q.n_rows = n;
  q.pad = nullptr;
  q.pad_mode = kPadSelf;
  q.vec_ok = (reinterpret_cast<uintptr_t>(f.idx_out) % 16 == 0) &&
             (reinterpret_cast<uintptr_t>(f.dist_out) % 16 == 0);
  const int rc = launch_query(q, shape, s);
  if (rc != 0) {
    note_cuda_error(static_cast<cudaError_t>(rc));
    return FKNN_ERR_CUDA;
  }
  ++nl;
  if (launches) *launches = nl;
  return FKNN_OK;
}

}  // namespace fknn
