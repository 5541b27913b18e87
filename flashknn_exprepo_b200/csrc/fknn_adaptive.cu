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
// referenced support node, :605-608).  Once for all levels:
//   ka_heads_all / ka_scan_all           node heads per tile and level (the
//                                        highest bit in which neighbouring
//                                        keys differ), scanned per level
// then per level, from the coarsest down (four launches):
//   ka_nodes                             node starts; empties the table
//                                        last used two levels up
//   ka_insert                            open-addressing table: node key ->
//                                        (start, count); two tables alternate
//                                        between consecutive levels
//   ka_counts                            27-node candidate count per node
//   ka_select                            per-point level selection step;
//                                        points that stopped one level up
//                                        open query groups there and write
//                                        their 27 (start, count) runs
// and ka_finalize opens the groups of the points that reach level 0.
// A query group is a maximal run of sorted points with the same selected
// level and node; its runs address the same sorted records as its queries,
// so the packer and the top-K kernel of the fixed-level path serve it
// unchanged (fknn_items.cu, fknn_query.cu).  Every data-dependent size stays
// on the device: the pipeline is a fixed launch sequence (levels above the
// device-side S return at once) and can be captured in a CUDA graph.
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
constexpr uint64_t kEmptyKey = ~0ull;

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

// One 16-byte slot: node key and its run, so a probe is a single load.
struct __align__(16) Slot {
  uint64_t key;
  int2 run;
};

struct Table {
  Slot* slots;
  uint32_t mask;
};

__device__ __forceinline__ int2 table_find(const Table& t, uint64_t key) {
  uint32_t h = slot_of_key(key, t.mask);
  for (uint32_t probe = 0; probe <= t.mask; ++probe) {
    const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(t.slots + h));
    if (v.x == key) {
      int2 r;
      r.x = static_cast<int>(static_cast<uint32_t>(v.y));
      r.y = static_cast<int>(static_cast<uint32_t>(v.y >> 32));
      return r;
    }
    if (v.x == kEmptyKey) break;
    h = (h + 1) & t.mask;
  }
  return make_int2(0, 0);
}

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

// Neighbour j of the node with key nk at level s: runs of the 27 offsets in
// the reference's order (centre first, (0,-1,+1)^3 ij), or (0,0).
__device__ __forceinline__ int2 neighbour_run(const Table& t, uint64_t nk, int s, int bpa,
                                              int j) {
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
  return table_find(t, key);
}

}  // namespace

// ------------------------------------------------------------ boxes, keys

__global__ void ka_init(Meta* meta, long long* box, uint32_t* totals, int n_totals) {
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

// ---- per-level passes (device functions over an explicit tile, thread or
// warp range; the kernels below launch them, four per level).  Arrays that a
// pass rewrites on every level (node starts, node of, counts, selection,
// slots) are read with ld.global.cg, straight from L2.

// Positions of tile `tile` (kTile of them, 8 per thread of a 256-thread CTA):
// node_of[p] = node of sorted position p at level s; node_start[c] = first
// position of node c, node_start[nodes] = n.  Called by every thread of the
// CTA (block-wide scan).
__device__ __forceinline__ void nodes_tile(const LevelArgs& a, int tile,
                                           const uint32_t* __restrict__ tile_offsets, int nodes,
                                           int32_t* __restrict__ node_of,
                                           int32_t* __restrict__ node_start, uint32_t* warp_sums) {
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int64_t base = static_cast<int64_t>(tile) * kTile + threadIdx.x * 8;
  uint32_t flags = 0, heads = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t p = base + r;
    if (p < a.n && node_head(key, p, 3 * a.s)) {
      flags |= 1u << r;
      ++heads;
    }
  }
  const uint32_t incl = block_inclusive_scan(heads, warp_sums, nullptr);
  int c = static_cast<int>(tile_offsets[tile] + incl - heads) - 1;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t p = base + r;
    if (p >= a.n) break;
    if (flags & (1u << r)) {
      ++c;
      node_start[c] = static_cast<int32_t>(p);
    }
    node_of[p] = c;
    if (p == a.n - 1) node_start[nodes] = static_cast<int32_t>(a.n);
  }
}

// Empties the `stale` slots listed in slot_of (the nodes a table held two
// levels up), so the table can take this level's nodes.
__device__ __forceinline__ void erase_nodes(int64_t t, int64_t stride, int stale,
                                            const int32_t* __restrict__ slot_of,
                                            Slot* __restrict__ table) {
  for (int64_t c = t; c < stale; c += stride) table[__ldcg(slot_of + c)].key = kEmptyKey;
}

// Node key -> (start, count) into the table of this level; the slot is kept
// for the erase.  One thread per node.
__device__ __forceinline__ void insert_nodes(const LevelArgs& a, int64_t t, int64_t stride,
                                             int nodes, const int32_t* __restrict__ node_start,
                                             const Table& tab, int32_t* __restrict__ slot_of) {
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  for (int64_t c = t; c < nodes; c += stride) {
    const int32_t st = __ldcg(node_start + c);
    const uint64_t nk = key[st] >> (3 * a.s);
    uint32_t h = slot_of_key(nk, tab.mask);
    for (uint32_t probe = 0; probe <= tab.mask; ++probe) {
      const unsigned long long prev =
          atomicCAS(reinterpret_cast<unsigned long long*>(&tab.slots[h].key), kEmptyKey, nk);
      if (prev == kEmptyKey) {
        tab.slots[h].run = make_int2(st, __ldcg(node_start + c + 1) - st);
        slot_of[c] = static_cast<int32_t>(h);
        break;
      }
      h = (h + 1) & tab.mask;
    }
  }
}

// cand[c] = points in the 27 nodes around node c.  One warp per node, one
// lookup per lane, so the 27 probes are in flight together.  Below the top
// level only points still active read their count, so a node of at most
// kScanActive points none of which is active (act_in, the previous level's
// flags) is skipped.
constexpr int kScanActive = 128;

__device__ __forceinline__ void count_nodes(const LevelArgs& a, int top, int64_t w,
                                            int64_t wstride, int nodes,
                                            const int32_t* __restrict__ node_start,
                                            const Table& tab, const uint8_t* __restrict__ act_in,
                                            int32_t* __restrict__ cand) {
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int bpa = a.meta->bpa;
  const int lane = threadIdx.x & 31;
  for (int64_t c = w; c < nodes; c += wstride) {
    const int32_t st = __ldcg(node_start + c);
    if (a.s < top) {
      const int32_t len = __ldcg(node_start + c + 1) - st;
      if (len <= kScanActive) {
        bool any = false;
#pragma unroll
        for (int i = 0; i < kScanActive / 32; ++i) {
          const int j = lane + 32 * i;
          any |= j < len && __ldcg(act_in + st + j) != 0;
        }
        if (!__any_sync(kFull, any)) continue;
      }
    }
    const uint64_t nk = key[st] >> (3 * a.s);
    const int len = lane < kNeighbours ? neighbour_run(tab, nk, a.s, bpa, lane).y : 0;
    const int total = __reduce_add_sync(kFull, len);
    if (lane == 0) cand[c] = total;
  }
}

// New (level, active) of sorted position q after the step at level s; only
// points still active read their node's count.
__device__ __forceinline__ void select_step(int64_t q, int s, int top,
                                            const int32_t* __restrict__ node_of,
                                            const int32_t* __restrict__ cand,
                                            const uint8_t* __restrict__ sel_in,
                                            const uint8_t* __restrict__ act_in, int min_count,
                                            int max_count, uint8_t* sel_new, uint8_t* act_new) {
  if (s == top) {
    *sel_new = static_cast<uint8_t>(top);
    *act_new = __ldcg(cand + __ldcg(node_of + q)) > max_count;
  } else if (__ldcg(act_in + q)) {
    const int cnt = __ldcg(cand + __ldcg(node_of + q));
    const bool use = cnt >= min_count;
    *sel_new = use ? static_cast<uint8_t>(s) : __ldcg(sel_in + q);
    *act_new = use && cnt > max_count;
  } else {
    *sel_new = __ldcg(sel_in + q);
    *act_new = 0;
  }
}

struct SelectArgs {
  const int32_t* node_of;
  const int32_t* cand;
  int min_count, max_count;
  const uint8_t* sel_in;
  const uint8_t* act_in;
  uint8_t* sel_out;
  uint8_t* act_out;
  Table t_up;  // table of level s + 1
  uint8_t* group_flag;
  int2* runs;
};

// One step of the coarse-to-fine level selection, fused with the
// finalisation of level s+1: points whose selection stays at s+1 open their
// query groups there (a group is a maximal run of sorted positions with the
// same level and level-(s+1) node) and write the group's 27 runs (row p).
// The new selection goes to sel_out / act_out, the previous one is read from
// sel_in / act_in, so a warp can recompute its left neighbour's new level
// without racing the warp that writes it.  One warp per 32 positions.
__device__ __forceinline__ void select_positions(const LevelArgs& a, int top, int64_t w,
                                                 int64_t wstride, const SelectArgs& g) {
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int bpa = a.meta->bpa;
  const int L = a.s + 1;  // level finalised here (when <= top)
  const int lane = threadIdx.x & 31;
  for (int64_t base = w * 32; base < a.n; base += wstride * 32) {
    const int64_t p = base + lane;
    uint8_t ns = 0xff, na = 0;
    if (p < a.n) {
      select_step(p, a.s, top, g.node_of, g.cand, g.sel_in, g.act_in, g.min_count, g.max_count,
                  &ns, &na);
      g.sel_out[p] = ns;
      g.act_out[p] = na;
    }
    if (L > top) continue;
    uint8_t prev = static_cast<uint8_t>(__shfl_up_sync(kFull, ns, 1));
    if (lane == 0 && p > 0 && p < a.n) {  // the previous warp's last position
      uint8_t pa;
      select_step(p - 1, a.s, top, g.node_of, g.cand, g.sel_in, g.act_in, g.min_count,
                  g.max_count, &prev, &pa);
    }
    bool start = false;
    if (p < a.n && ns == L) {
      start = p == 0 || prev != L || node_head(key, p, 3 * L);
      g.group_flag[p] = start ? 1 : 0;
    }
    uint32_t starts = __ballot_sync(kFull, start);
    while (starts) {
      const int src = __ffs(starts) - 1;
      starts &= starts - 1;
      const int64_t ps = base + src;
      if (lane < kNeighbours)
        g.runs[ps * kNeighbours + lane] = neighbour_run(g.t_up, key[ps] >> (3 * L), L, bpa, lane);
    }
  }
}

// ---- per-level kernels

// Also empties the table this level is about to reuse: it still holds the
// nodes of level s+2 (erase_count of them, at erase_slot), whose last reader
// was the finalisation of level s+2 in the previous step.
__global__ void __launch_bounds__(256)
    ka_nodes(LevelArgs a, const uint32_t* __restrict__ tile_offsets, const int* count_ptr,
             int32_t* __restrict__ node_of, int32_t* __restrict__ node_start,
             const int* erase_count, const int32_t* __restrict__ erase_slot,
             Slot* __restrict__ table) {
  __shared__ uint32_t warp_sums[32];
  const int top = top_level(a.meta);
  if (a.s > top) return;
  if (a.s + 2 <= top)
    erase_nodes(static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x,
                static_cast<int64_t>(gridDim.x) * blockDim.x, *erase_count, erase_slot, table);
  nodes_tile(a, blockIdx.x, tile_offsets, *count_ptr, node_of, node_start, warp_sums);
}

__global__ void __launch_bounds__(256)
    ka_insert(LevelArgs a, const int* count_ptr, const int32_t* __restrict__ node_start, Table t,
              int32_t* __restrict__ slot_of) {
  if (a.s > top_level(a.meta)) return;
  insert_nodes(a, static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x,
               static_cast<int64_t>(gridDim.x) * blockDim.x, *count_ptr, node_start, t, slot_of);
}

__global__ void __launch_bounds__(256)
    ka_counts(LevelArgs a, const int* count_ptr, const int32_t* __restrict__ node_start, Table t,
              const uint8_t* __restrict__ act_in, int32_t* __restrict__ cand) {
  const int top = top_level(a.meta);
  if (a.s > top) return;
  count_nodes(a, top, (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5,
              (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5, *count_ptr, node_start, t,
              act_in, cand);
}

__global__ void __launch_bounds__(256) ka_select(LevelArgs a, SelectArgs g) {
  const int top = top_level(a.meta);
  if (a.s > top) return;
  select_positions(a, top, (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5,
                   (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5, g);
}

// Points whose selection stopped at level L open their query groups: a
// group is a maximal run of sorted positions with level L and the same
// level-L node.  group_flag[p] and the group's 27 runs (row p).  One warp per
// 32 consecutive points: every lane decides for its point, then the warp
// looks up the 27 runs of each group start together, one run per lane.
__global__ void __launch_bounds__(256)
    ka_finalize(LevelArgs a, int L, Table t, const uint8_t* __restrict__ sel,
                uint8_t* __restrict__ group_flag, int2* __restrict__ runs) {
  if (L > top_level(a.meta)) return;
  const uint64_t* key = sorted_keys(a.sp, a.bits);
  const int bpa = a.meta->bpa;
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32;
       base < a.n; base += warps * 32) {
    const int64_t p = base + lane;
    bool start = false;
    if (p < a.n && sel[p] == L) {
      start = p == 0 || sel[p - 1] != L || node_head(key, p, 3 * L);
      group_flag[p] = start ? 1 : 0;
    }
    uint32_t starts = __ballot_sync(kFull, start);
    while (starts) {
      const int src = __ffs(starts) - 1;
      starts &= starts - 1;
      const int64_t ps = base + src;
      if (lane < kNeighbours)
        runs[ps * kNeighbours + lane] = neighbour_run(t, key[ps] >> (3 * L), L, bpa, lane);
    }
  }
}

// ------------------------------------------------------------------ groups

__global__ void __launch_bounds__(256)
    ka_group_tiles(int64_t n, const uint8_t* __restrict__ flag, uint32_t* __restrict__ tile_counts) {
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
  int32_t* node_of;
  int32_t* node_start;
  int32_t* cand;
  int32_t* slot_of[2];
  int* level_nodes;  // [kMaxLevel + 1]
  uint8_t* sel[2];     // selection of the previous / current level (ping-pong by level parity)
  uint8_t* active[2];
  uint8_t* group_flag;
  Slot* tslots[2];
  int64_t cap;
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
  b.node_of = a.take<int32_t>(n);
  b.node_start = a.take<int32_t>(n + 1);
  b.cand = a.take<int32_t>(n);
  b.slot_of[0] = a.take<int32_t>(n);
  b.slot_of[1] = a.take<int32_t>(n);
  b.level_nodes = a.take<int>(kMaxLevel + 1);
  for (int h = 0; h < 2; ++h) {
    b.sel[h] = a.take<uint8_t>(n);
    b.active[h] = a.take<uint8_t>(n);
  }
  b.group_flag = a.take<uint8_t>(n);
  b.cap = 16;
  while (b.cap < 2 * n) b.cap <<= 1;
  for (int h = 0; h < 2; ++h) {
    b.tslots[h] = a.take<Slot>(b.cap);
  }
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
  cudaError_t e = cudaMemsetAsync(b.tslots[0], 0xff, sizeof(Slot) * b.cap, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.tslots[1], 0xff, sizeof(Slot) * b.cap, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.group_flag, 0, static_cast<size_t>(n), s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  ka_init<<<64, 256, 0, s>>>(b.meta, b.box, b.totals, kSortMaxPasses * 256);
  ka_box<<<blocks_for(n, kTile), 256, 0, s>>>(f.grid, f.batch, n, b.box, b.meta);
  ka_meta<<<1, 1024, 0, s>>>(b.box, f.max_shift, b.meta);
  ka_keys<<<blocks_for(n, 256), 256, 0, s>>>(f.grid, f.batch, n, b.box, b.meta, b.keys[0],
                                              b.vals[0]);
  nl += 4;
  const int* key_bits = &b.meta->key_bits;
  SortBuffers<uint64_t> sb{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}, b.hist, b.totals};
  nl += launch_radix_sort(sb, n, key_bits, sort_passes_for_bits(3 * kMaxLevel + 15), s);
  const SortPair<uint64_t> sp{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}};
  ka_records<<<blocks_for(n, 256), 256, 0, s>>>(f.xyz, f.grid, f.batch, n, b.box, sp, key_bits,
                                                b.meta, b.rec);
  ++nl;

  const int tiles = blocks_for(n, kTile);
  const int min_count = f.min_factor * f.k, max_count = f.max_factor * f.k;
  const int top_host = f.max_shift >= 0 ? f.max_shift : kMaxLevel;
  const Table tab[2] = {{b.tslots[0], static_cast<uint32_t>(b.cap - 1)},
                        {b.tslots[1], static_cast<uint32_t>(b.cap - 1)}};
  {
    const LevelArgs la{sp, key_bits, b.meta, n, 0};
    ka_heads_all<<<tiles, 256, 0, s>>>(la, tiles, b.tile_counts);
    ka_scan_all<<<kMaxLevel + 1, 1024, 0, s>>>(b.tile_counts, tiles, b.level_nodes);
    nl += 2;
  }
  for (int lv = top_host; lv >= 0; --lv) {
    const LevelArgs la{sp, key_bits, b.meta, n, lv};
    int* nodes = b.level_nodes + lv;
    const int* stale = b.level_nodes + (lv + 2 <= kMaxLevel ? lv + 2 : kMaxLevel);
    const int h = lv & 1, up = (lv + 1) & 1;
    ka_nodes<<<tiles, 256, 0, s>>>(la, b.tile_counts + static_cast<int64_t>(lv) * tiles, nodes,
                                   b.node_of, b.node_start, stale, b.slot_of[h], b.tslots[h]);
    ka_insert<<<capped_blocks(n), 256, 0, s>>>(la, nodes, b.node_start, tab[h], b.slot_of[h]);
    ka_counts<<<capped_blocks(n * 32), 256, 0, s>>>(la, nodes, b.node_start, tab[h],
                                                     b.active[up], b.cand);
    const SelectArgs sa{b.node_of, b.cand, min_count, max_count, b.sel[up], b.active[up],
                        b.sel[h], b.active[h], tab[up], b.group_flag, b.runs};
    ka_select<<<capped_blocks(n), 256, 0, s>>>(la, sa);
    nl += 4;
  }
  {
    const LevelArgs la{sp, key_bits, b.meta, n, 0};
    ka_finalize<<<capped_blocks(n), 256, 0, s>>>(la, 0, tab[0], b.sel[0], b.group_flag, b.runs);
    ka_group_tiles<<<tiles, 256, 0, s>>>(n, b.group_flag, b.tile_counts);
    k_scan_tiles<<<1, 1024, 0, s>>>(b.tile_counts, tiles, &b.meta->n_groups);
    ka_groups<<<tiles, 256, 0, s>>>(n, b.group_flag, b.tile_counts, &b.meta->n_groups,
                                    b.group_start, b.group_row);
    nl += 4;
    if (f.level_out) {
      ka_levels_out<<<blocks_for(n, 256), 256, 0, s>>>(n, b.rec, b.sel[0], f.level_out);
      ++nl;
    }
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
