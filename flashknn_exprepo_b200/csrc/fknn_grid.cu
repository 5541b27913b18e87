// Grid construction and the fused query pipelines (self / selected / general).
//
// The reference builds its tables with ~15 ATen calls and host syncs
// (FlashKNN/functions/FlashKnnWrapper.py:220-337).  Here the whole pipeline
// is a fixed sequence of launches with every data-dependent size kept on the
// device, so it is CUDA-graph capturable:
//
//   k_init          zero the Meta block, empty the per-cloud boxes
//   k_bbox          parent cell (grid >> num_down) and cloud of each point,
//                   range checks, per-cloud bounding boxes (block-aggregated
//                   atomics)
//   k_meta          bits per axis of the translated parent coordinates
//   support cells   counting sort by cell through an open-addressing table
//                   keyed by cloud << 3*bpa | morton(parent - cloud min):
//     k_cell_insert   per point its cell's slot and its rank in the cell
//                     (warp-aggregated count atomics), cell ids in order of
//                     creation
//     k_cell_tiles / k_scan_tiles / k_cell_starts
//                     cell starts in id order, written into the table
//     k_scatter       float4 records (x, y, z, point id) at start + rank
//   query groups    general queries: query cells by the same counting sort
//                   through a second table; selected queries: support cells
//                   holding queries, by a counting sort over the dense cell
//                   ids (k_sel_count / k_sel_tiles / k_sel_starts /
//                   k_sel_scatter)
//   k_runs          27 (start, count) candidate runs per cell / query group,
//                   centre first, (0,-1,+1)^3 in ij order like the reference
//                   neighbour table (flash_knn_construction.cu:42-63)
//   items           work items for the query kernel: up to 32 consecutive
//                   queries of consecutive groups whose candidates fit one
//                   shared-memory tile (fknn_items.cu)
//
// Parent cells and their 3x3x3 adjacency are those of the reference: for grid
// coordinates inside [-2^15, 2^15) the reference's key >> 3*num_down groups
// exactly the points with equal grid >> num_down, and its neighbour lookup
// finds exactly the integer-adjacent parent cells.  The per-cloud translation
// only shortens the keys; it changes neither the cells nor their adjacency.
#include <climits>

#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"
#include "fknn_grid.h"

namespace fknn {

// ---------------------------------------------------------------- sources

struct PointSrc {
  const float* xyz;        // f32 [n_src,3]
  const int64_t* grid;     // int64 [n_src,3] or null: floor(xyz / voxel)
  const int64_t* batch;    // int64 [n_src] or null
  const int64_t* offsets;  // cumulative cloud ends or null
  int64_t n_clouds;        // clouds addressable by this source
  int64_t n;               // points of this source
  float inv_voxel;         // FP32 reciprocal of the voxel edge
  int num_down;
  const int64_t* index;    // point i is row index[i] of xyz / grid / batch, or null
  int64_t n_src;           // rows of xyz / grid / batch when index is given
  int trunc;               // voxelise with trunc(xyz / voxel) instead of floor
};

// Row of point i in the source arrays; an index outside the rows is
// reported (kStatusTable) and read as row 0.
__device__ __forceinline__ int64_t row_of(const PointSrc& p, int64_t i, int* status) {
  if (!p.index) return i;
  const int64_t r = p.index[i];
  if (r < 0 || r >= p.n_src) {
    raise_status(status, kStatusTable);
    return 0;
  }
  return r;
}

__device__ __forceinline__ int grid_axis(const PointSrc& p, int64_t i, int a, int* status) {
  int64_t g;
  const int64_t row = row_of(p, i, status);
  if (p.grid) {
    g = p.grid[3 * row + a];
  } else {
    // x * (1 / voxel): the rounding of PyTorch's CUDA tensor / scalar
    // division, which the reference's callers voxelise with
    // (Query/benchmark_s3dis.py:159, Networks/hierarchy.py:30)
    const float q = __fmul_rn(p.xyz[3 * row + a], p.inv_voxel);
    const float f = p.trunc ? truncf(q) : floorf(q);
    if (!(f >= -32768.f && f <= 32767.f)) {
      raise_status(status, kStatusRange);
      return 0;
    }
    g = static_cast<int64_t>(f);
  }
  if (g < -32768 || g > 32767) {
    raise_status(status, kStatusRange);
    g = g < 0 ? -32768 : 32767;
  }
  return static_cast<int>(g);
}

__device__ __forceinline__ int cloud_of(const PointSrc& p, int64_t i, int* status) {
  int64_t b = 0;
  if (p.batch) {
    b = p.batch[row_of(p, i, status)];
  } else if (p.offsets) {
    int64_t lo = 0, hi = p.n_clouds;  // first cloud whose end exceeds i
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (p.offsets[mid] > i) hi = mid; else lo = mid + 1;
    }
    b = lo;
  }
  if (b < 0 || b >= p.n_clouds) {
    raise_status(status, kStatusBatch);
    b = b < 0 ? 0 : p.n_clouds - 1;
  }
  return static_cast<int>(b);
}

// ------------------------------------------------------------------ init

__global__ void k_init(Meta* meta, int* bbox, int64_t n_clouds) {
  chain_wait();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  if (t < static_cast<int64_t>(sizeof(Meta) / sizeof(int))) reinterpret_cast<int*>(meta)[t] = 0;
  for (int64_t i = t; i < n_clouds * 6; i += stride) bbox[i] = (i % 6) < 3 ? INT_MAX : INT_MIN;
}

// ------------------------------------------------------------------ bbox

struct Box6 {
  int v[6];  // min x, y, z, max x, y, z
  __device__ void reset() {
    v[0] = v[1] = v[2] = INT_MAX;
    v[3] = v[4] = v[5] = INT_MIN;
  }
  __device__ void add(int x, int y, int z) {
    v[0] = min(v[0], x); v[1] = min(v[1], y); v[2] = min(v[2], z);
    v[3] = max(v[3], x); v[4] = max(v[4], y); v[5] = max(v[5], z);
  }
};

__device__ __forceinline__ void box_atomic(int* bbox, int b, const Box6& box) {
  if (box.v[0] > box.v[3]) return;  // empty
  int* dst = bbox + 6 * b;
  atomicMin(dst + 0, box.v[0]); atomicMin(dst + 1, box.v[1]); atomicMin(dst + 2, box.v[2]);
  atomicMax(dst + 3, box.v[3]); atomicMax(dst + 4, box.v[4]); atomicMax(dst + 5, box.v[5]);
}

// Block-wide reduction of a box; result valid in thread 0.
__device__ __forceinline__ Box6 box_reduce(Box6 box, int (*sh)[6]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    box.v[a] = __reduce_min_sync(kFull, box.v[a]);
    box.v[a + 3] = __reduce_max_sync(kFull, box.v[a + 3]);
  }
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < 6; ++a) sh[warp][a] = box.v[a];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int w = 1; w < nw; ++w) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        box.v[a] = min(box.v[a], sh[w][a]);
        box.v[a + 3] = max(box.v[a + 3], sh[w][a + 3]);
      }
    }
  }
  __syncthreads();
  return box;
}

// 256 threads x ppt points (1, 2, 4 or 8).  Writes the parent cell and cloud
// of every point and grows the per-cloud boxes.  Most tiles hold one or two clouds (offset
// batching): those are reduced in the block, other clouds go straight to
// global atomics.
__global__ void __launch_bounds__(256) k_bbox(PointSrc p, int4* __restrict__ pc,
                                              int* __restrict__ bbox, Meta* meta, int ppt) {
  chain_wait();
  __shared__ int sh[8][6];
  int* status = &meta->status;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 256 * ppt;
  const int64_t last = min(base + 256 * ppt - 1, p.n - 1);
  const int b_lo = cloud_of(p, base, status);
  const int b_hi = cloud_of(p, last, status);
  // offset batching: a point of this tile below the end of b_lo is in b_lo,
  // one below the end of b_lo + 1 = b_hi in b_hi; only others search
  const bool by_offsets = p.offsets && !p.batch;
  const int64_t end_lo = by_offsets ? p.offsets[b_lo] : 0;
  const int64_t end_hi = by_offsets && b_hi == b_lo + 1 ? p.offsets[b_hi] : 0;
  Box6 lo, hi;
  lo.reset();
  hi.reset();
#pragma unroll 2
  for (int r = 0; r < ppt; ++r) {
    const int64_t i = base + r * 256 + threadIdx.x;
    if (i >= p.n) break;
    const int gx = grid_axis(p, i, 0, status) >> p.num_down;
    const int gy = grid_axis(p, i, 1, status) >> p.num_down;
    const int gz = grid_axis(p, i, 2, status) >> p.num_down;
    const int b = !by_offsets ? cloud_of(p, i, status)
                  : i < end_lo  ? b_lo
                  : i < end_hi  ? b_hi
                                : cloud_of(p, i, status);
    pc[i] = make_int4(gx, gy, gz, b);
    if (b == b_lo) {
      lo.add(gx, gy, gz);
    } else if (b == b_hi) {
      hi.add(gx, gy, gz);
    } else {
      Box6 one;
      one.reset();
      one.add(gx, gy, gz);
      box_atomic(bbox, b, one);
    }
  }
  lo = box_reduce(lo, sh);
  hi = box_reduce(hi, sh);
  if (threadIdx.x == 0) {
    box_atomic(bbox, b_lo, lo);
    if (b_hi != b_lo) box_atomic(bbox, b_hi, hi);
  }
}

// One CTA: bits per axis of the largest per-cloud extent, batch bits.
__global__ void __launch_bounds__(1024) k_meta(const int* __restrict__ bbox, int64_t n_clouds,
                                               Meta* meta) {
  chain_wait();
  __shared__ int s_ext[32], s_b[32];
  int ext = 0, maxb = 0;
  for (int64_t c = threadIdx.x; c < n_clouds; c += blockDim.x) {
    const int* bx = bbox + 6 * c;
    if (bx[0] <= bx[3]) {
      ext = max(ext, max(bx[3] - bx[0], max(bx[4] - bx[1], bx[5] - bx[2])));
      maxb = max(maxb, static_cast<int>(c));
    }
  }
  ext = __reduce_max_sync(kFull, ext);
  maxb = __reduce_max_sync(kFull, maxb);
  if ((threadIdx.x & 31) == 0) {
    s_ext[threadIdx.x >> 5] = ext;
    s_b[threadIdx.x >> 5] = maxb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) {
      ext = max(ext, s_ext[w]);
      maxb = max(maxb, s_b[w]);
    }
    const int bpa = ext > 0 ? 32 - __clz(ext) : 0;
    const int bb = maxb > 0 ? 32 - __clz(maxb) : 0;
    meta->bpa = bpa;
    meta->batch_bits = bb;
    meta->max_extent = ext;
    meta->key_bits = 3 * bpa + bb;
  }
}

__device__ __forceinline__ uint64_t cell_key_of(int4 c, const int* bbox, int bpa) {
  const int* bx = bbox + 6 * c.w;
  const uint32_t x = static_cast<uint32_t>(c.x - bx[0]);
  const uint32_t y = static_cast<uint32_t>(c.y - bx[1]);
  const uint32_t z = static_cast<uint32_t>(c.z - bx[2]);
  return (static_cast<uint64_t>(c.w) << (3 * bpa)) | morton3(x, y, z);
}

// ------------------------------------------------------------- neighbours

__device__ __forceinline__ int axis_offset(int position) {
  return position == 0 ? 0 : (position == 1 ? -1 : 1);
}

// ------------------------------------------------------- cell hash table
// Open addressing over the support cells (linear probing, capacity >= 2n, so
// the load stays <= 1/2 whatever the cell count).  A slot holds key + 1 (0 =
// empty, so the whole table clears with one memset) and the cell's run
// (start, count): a neighbour lookup is one 16-byte load.
//
// The table also builds the cells, as a counting sort by cell instead of a
// sort by key.  k_cell_insert counts the points of every cell in its slot
// and gives each point its rank inside the cell; new cells take ids in
// creation order (one global atomic per CTA); k_cell_tiles / k_scan_tiles /
// k_cell_starts lay the cells out in id order; k_scatter writes each point's
// record at start + rank.  Cell and in-cell order are therefore not
// deterministic, but nothing downstream depends on them: every query's
// candidates are the same 27 cells and its top-K is exact under the
// (distance, index) order.

// One 16-byte slot: key + 1 and the cell's run.
struct __align__(16) HashSlot {
  uint64_t key;  // cell key + 1; 0 = empty
  int2 run;      // (start, count)
};

__device__ __forceinline__ uint32_t hash_slot(uint64_t key, uint32_t mask) {
  key ^= key >> 33;
  key *= 0xff51afd7ed558ccdULL;
  key ^= key >> 33;
  key *= 0xc4ceb9fe1a85ec53ULL;
  key ^= key >> 33;
  return static_cast<uint32_t>(key) & mask;
}

// Warp-cooperative insertion of 256 x ppt points per CTA (ppt <= 8).  Lanes with
// the same cell key elect one leader, which probes once and adds the group's
// size to the cell count; slot_of[i] / rank_of[i] = the point's slot and its
// rank in the cell.  cell_slot[id] = slot of cell id; *cell_count = cells.
__global__ void __launch_bounds__(256)
    k_cell_insert(const int4* __restrict__ pc, int64_t n, const int* __restrict__ bbox,
                  Meta* meta, HashSlot* __restrict__ table, uint32_t mask,
                  uint32_t* __restrict__ slot_of, uint32_t* __restrict__ rank_of,
                  uint32_t* __restrict__ cell_slot, int* cell_count, int ppt) {
  chain_wait();
  __shared__ uint32_t s_new;
  __shared__ uint32_t s_base;
  __shared__ uint32_t s_list[2048];
  if (threadIdx.x == 0) s_new = 0u;
  __syncthreads();
  const int bpa = meta->bpa;
  const int lane = threadIdx.x & 31;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 256 * ppt;
#pragma unroll 2
  for (int r = 0; r < ppt; ++r) {
    const int64_t i = base + r * 256 + threadIdx.x;
    const bool valid = i < n;
    const unsigned vmask = __ballot_sync(kFull, valid);
    if (!valid) continue;
    const uint64_t key = cell_key_of(pc[i], bbox, bpa) + 1;
    const unsigned peers = __match_any_sync(vmask, key);
    const int leader = __ffs(peers) - 1;
    uint32_t slot = 0u, before = 0u;
    if (lane == leader) {
      uint32_t h = hash_slot(key, mask);
      bool found = false;
      for (uint32_t probe = 0; probe <= mask; ++probe) {
        const unsigned long long prev =
            atomicCAS(reinterpret_cast<unsigned long long*>(&table[h].key), 0ull, key);
        if (prev == 0ull) {
          s_list[atomicAdd(&s_new, 1u)] = h;
          found = true;
          break;
        }
        if (prev == key) {
          found = true;
          break;
        }
        h = (h + 1) & mask;
      }
      if (found) {
        slot = h;
        before = static_cast<uint32_t>(atomicAdd(&table[h].run.y, __popc(peers)));
      } else {
        raise_status(&meta->status, kStatusTable);  // cannot happen at load <= 1/2
      }
    }
    slot = __shfl_sync(peers, slot, leader);
    before = __shfl_sync(peers, before, leader);
    slot_of[i] = slot;
    rank_of[i] = before + __popc(peers & lanemask_lt());
  }
  __syncthreads();
  if (threadIdx.x == 0)
    s_base = s_new ? atomicAdd(reinterpret_cast<unsigned*>(cell_count), s_new) : 0u;
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < s_new; j += blockDim.x) cell_slot[s_base + j] = s_list[j];
}

// Points per 256 x ppt cell ids (ppt per thread): tile_counts[tile].
__global__ void __launch_bounds__(256)
    k_cell_tiles(const int* cell_count_ptr, const uint32_t* __restrict__ cell_slot,
                 const HashSlot* __restrict__ table, uint32_t* __restrict__ tile_counts, int ppt) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int cells = *cell_count_ptr;
  const int64_t base = (static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x) * ppt;
  uint32_t c = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r)
    if (r < ppt && base + r < cells)
      c += static_cast<uint32_t>(table[cell_slot[base + r]].run.y);
  block_inclusive_scan(c, warp_sums, &s_total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = s_total;
}

// Cell starts in id order from the scanned tile counts: the slot's run,
// cell_key[id], cell_start[id] (cell_start[cells] = n) and, when asked,
// slot_cell[slot] = id and zero_per_cell[id] = 0.
__global__ void __launch_bounds__(256)
    k_cell_starts(const int* cell_count_ptr, const uint32_t* __restrict__ cell_slot,
                  HashSlot* __restrict__ table, const uint32_t* __restrict__ tile_offsets,
                  int64_t n, uint64_t* __restrict__ cell_key, int32_t* __restrict__ cell_start,
                  uint32_t* __restrict__ slot_cell, uint32_t* __restrict__ zero_per_cell, int ppt) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  const int cells = *cell_count_ptr;
  const int64_t base = (static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x) * ppt;
  uint32_t cnt[8], slot[8], sum = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    cnt[r] = 0u;
    slot[r] = 0u;
    if (r < ppt && base + r < cells) {
      slot[r] = cell_slot[base + r];
      cnt[r] = static_cast<uint32_t>(table[slot[r]].run.y);
    }
    sum += cnt[r];
  }
  const uint32_t incl = block_inclusive_scan(sum, warp_sums, nullptr);
  uint32_t start = tile_offsets[blockIdx.x] + incl - sum;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t c = base + r;
    if (r >= ppt || c >= cells) break;
    HashSlot& hs = table[slot[r]];
    hs.run.x = static_cast<int>(start);
    cell_key[c] = hs.key - 1;
    cell_start[c] = static_cast<int32_t>(start);
    if (slot_cell) slot_cell[slot[r]] = static_cast<uint32_t>(c);
    if (zero_per_cell) zero_per_cell[c] = 0u;
    start += cnt[r];
    if (c == cells - 1) cell_start[cells] = static_cast<int32_t>(n);
  }
}

// rec[pos] = (xyz of point i, i) at pos = cell start + rank; optional
// pos_of[i] = pos and cell_of[pos] = cell id.
__global__ void __launch_bounds__(256)
    k_scatter(const float* __restrict__ xyz, const int64_t* __restrict__ index, int64_t n_src,
              int64_t n, const uint32_t* __restrict__ slot_of, const uint32_t* __restrict__ rank_of,
              const HashSlot* __restrict__ table, const uint32_t* __restrict__ slot_cell,
              float4* __restrict__ rec, int32_t* __restrict__ pos_of,
              int32_t* __restrict__ cell_of, int* status) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t slot = slot_of[i];
  const int64_t pos = static_cast<int64_t>(table[slot].run.x) + rank_of[i];
  if (pos < 0 || pos >= n) {
    raise_status(status, kStatusTable);
    return;
  }
  int64_t row = i;
  if (index) {
    row = index[i];
    if (row < 0 || row >= n_src) row = 0;  // reported by k_bbox
  }
  rec[pos] = make_float4(xyz[3 * row], xyz[3 * row + 1], xyz[3 * row + 2],
                         __int_as_float(static_cast<int>(i)));
  if (pos_of) pos_of[i] = static_cast<int32_t>(pos);
  if (cell_of) cell_of[pos] = static_cast<int32_t>(slot_cell[slot]);
}

__device__ __forceinline__ int2 hash_find(const HashSlot* table, uint32_t mask, uint64_t key) {
  const uint64_t stored = key + 1;
  uint32_t h = hash_slot(stored, mask);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(table + h));
    if (v.x == stored)
      return make_int2(static_cast<int>(static_cast<uint32_t>(v.y)),
                       static_cast<int>(static_cast<uint32_t>(v.y >> 32)));
    if (v.x == 0ull) break;
    h = (h + 1) & mask;
  }
  return make_int2(0, 0);  // no such cell: an empty run
}

// One warp per group, one lane per neighbour position.  group_key[g] is a
// key in the support key space; runs[g*27 + j] = (start, count) of the
// support cell at offset j, or (0, 0) when that cell is empty.  With cands,
// cands[g] = the group's candidate total (the work-item packer's input; a
// group without candidates sets kStatusNoCandidates in *status) and
// meta->cand_total receives the sum of the totals (one atomic per block).
__global__ void __launch_bounds__(256)
    k_runs(const uint64_t* __restrict__ group_key, const int* group_count_ptr,
           const HashSlot* __restrict__ table, uint32_t hmask, const int* cell_count_ptr,
           Meta* meta, int2* __restrict__ runs, int32_t* __restrict__ cands,
           int* status) {
  chain_wait();
  __shared__ unsigned long long block_total;
  if (threadIdx.x == 0) block_total = 0ull;
  __syncthreads();
  unsigned long long my_total = 0ull;
  const int groups = *group_count_ptr;
  const int bpa = meta->bpa;
  const int cells = *cell_count_ptr;
  const uint64_t mask = bpa ? ((1ull << (3 * bpa)) - 1) : 0ull;
  const int lim = 1 << bpa;
  const int j = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
       g < groups; g += warps) {
    int2 run = make_int2(0, 0);
    if (j < kNeighbours) {
      const uint64_t key = group_key[g];
      const uint64_t cloud = key >> (3 * bpa);
      const uint64_t m = key & mask;
      const int x = static_cast<int>(compact3(m >> 2)) + axis_offset(j / 9);
      const int y = static_cast<int>(compact3(m >> 1)) + axis_offset((j / 3) % 3);
      const int z = static_cast<int>(compact3(m)) + axis_offset(j % 3);
      if (cells > 0 && x >= 0 && y >= 0 && z >= 0 && x < lim && y < lim && z < lim) {
        const uint64_t nk = (cloud << (3 * bpa)) |
                            morton3(static_cast<uint32_t>(x), static_cast<uint32_t>(y),
                                    static_cast<uint32_t>(z));
        run = hash_find(table, hmask, nk);
      }
      runs[g * kNeighbours + j] = run;
    }
    if (cands) {
      const int total = __reduce_add_sync(kFull, run.y);
      if (j == 0) {
        cands[g] = total;
        my_total += static_cast<unsigned long long>(total);
        if (total == 0) raise_status(status, kStatusNoCandidates);
      }
    }
  }
  if (cands) {
    if (my_total) atomicAdd(&block_total, my_total);
    __syncthreads();
    if (threadIdx.x == 0 && block_total) atomicAdd(&meta->cand_total, block_total);
  }
}

// ------------------------------------------------------ selected queries
// Groups = support cells holding at least one selected query, in cell id
// order; group_row[g] = that cell (its runs row).  A counting sort over the
// dense cell ids: k_sel_count (warp-aggregated counts and ranks), two tile
// scans (non-empty cells, queries), k_sel_starts, k_sel_scatter.

// Per query r: the cell of its support point and its rank among that
// cell's queries (qcount is zeroed by k_cell_starts).
__global__ void __launch_bounds__(256)
    k_sel_count(const int64_t* __restrict__ query_indices, int64_t m, int64_t n,
                const int32_t* __restrict__ pos_of, const int32_t* __restrict__ cell_of,
                Meta* meta, uint32_t* __restrict__ qcount, uint32_t* __restrict__ cell_r,
                uint32_t* __restrict__ rank_r) {
  chain_wait();
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool valid = r < m;
  const unsigned vmask = __ballot_sync(kFull, valid);
  if (!valid) return;
  int64_t qi = query_indices[r];
  if (qi < 0 || qi >= n) {
    raise_status(&meta->status, kStatusTable);
    qi = 0;
  }
  const uint32_t c = static_cast<uint32_t>(cell_of[pos_of[qi]]);
  const unsigned peers = __match_any_sync(vmask, c);
  const int leader = __ffs(peers) - 1;
  uint32_t before = 0u;
  if ((threadIdx.x & 31) == leader)
    before = atomicAdd(&qcount[c], static_cast<uint32_t>(__popc(peers)));
  before = __shfl_sync(peers, before, leader);
  cell_r[r] = c;
  rank_r[r] = before + __popc(peers & lanemask_lt());
}

// Per 2048 cells (8 per thread): non-empty cells and their queries.
__global__ void __launch_bounds__(256)
    k_sel_tiles(const int* cell_count_ptr, const uint32_t* __restrict__ qcount,
                uint32_t* __restrict__ tile_groups, uint32_t* __restrict__ tile_queries) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int cells = *cell_count_ptr;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 2048 + threadIdx.x * 8;
  uint32_t g = 0, q = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const uint32_t c = base + r < cells ? qcount[base + r] : 0u;
    g += c ? 1u : 0u;
    q += c;
  }
  block_inclusive_scan(g, warp_sums, &s_total);
  if (threadIdx.x == 0) tile_groups[blockIdx.x] = s_total;
  block_inclusive_scan(q, warp_sums, &s_total);
  if (threadIdx.x == 0) tile_queries[blockIdx.x] = s_total;
}

// Group ids of the non-empty cells from the scanned tile counts:
// group_start[g] = first query record, group_row[g] = cell, qstart[cell] =
// first record of the cell's queries; group_start[groups] = m.
__global__ void __launch_bounds__(256)
    k_sel_starts(const int* cell_count_ptr, const uint32_t* __restrict__ qcount,
                 const uint32_t* __restrict__ tile_goff, const uint32_t* __restrict__ tile_qoff,
                 int64_t m, const int* group_count_ptr, int32_t* __restrict__ group_start,
                 int32_t* __restrict__ group_row, uint32_t* __restrict__ qstart) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  const int cells = *cell_count_ptr;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 2048 + threadIdx.x * 8;
  uint32_t cnt[8], g = 0, q = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    cnt[r] = base + r < cells ? qcount[base + r] : 0u;
    g += cnt[r] ? 1u : 0u;
    q += cnt[r];
  }
  const uint32_t gi = block_inclusive_scan(g, warp_sums, nullptr);
  const uint32_t qi = block_inclusive_scan(q, warp_sums, nullptr);
  uint32_t gid = tile_goff[blockIdx.x] + gi - g;
  uint32_t qs = tile_qoff[blockIdx.x] + qi - q;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t c = base + r;
    if (c >= cells) break;
    if (cnt[r]) {
      group_start[gid] = static_cast<int32_t>(qs);
      group_row[gid] = static_cast<int32_t>(c);
      qstart[c] = qs;
      ++gid;
      qs += cnt[r];
    }
    if (c == cells - 1) group_start[*group_count_ptr] = static_cast<int32_t>(m);
  }
}

// qrec[qstart[cell] + rank] = (support xyz of query r, output row r).
__global__ void __launch_bounds__(256)
    k_sel_scatter(int64_t m, int64_t n, const int64_t* __restrict__ query_indices,
                  const int32_t* __restrict__ pos_of, const float4* __restrict__ srec,
                  const uint32_t* __restrict__ cell_r, const uint32_t* __restrict__ rank_r,
                  const uint32_t* __restrict__ qstart, float4* __restrict__ qrec, int* status) {
  chain_wait();
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t qi = query_indices[r];
  if (qi < 0 || qi >= n) qi = 0;  // reported by k_sel_count
  const int64_t pos = static_cast<int64_t>(qstart[cell_r[r]]) + rank_r[r];
  if (pos < 0 || pos >= m) {
    raise_status(status, kStatusTable);
    return;
  }
  float4 v = srec[pos_of[qi]];
  v.w = __int_as_float(static_cast<int>(r));
  qrec[pos] = v;
}

// ------------------------------------------------------------ host side

namespace {

struct Bufs {
  Meta* meta;
  int* bbox;
  int4* pc_s;
  int4* pc_q;
  uint32_t* slot_of;    // per point: cell slot (support, then general queries)
  uint32_t* rank_of;    // per point: rank inside its cell
  uint32_t* cell_slot;  // per cell / query group id: its slot
  uint32_t* tile_counts;
  uint32_t* tile_counts2;
  float4* srec;
  float4* qrec;
  int32_t* pos_of;
  int32_t* cell_of;
  uint64_t* cell_key;
  int32_t* cell_start;
  int2* runs;
  uint64_t* group_key;
  int32_t* group_start;
  int32_t* group_row;
  int4* items;
  int32_t* cands;
  uint32_t* seg_counts;
  HashSlot* hslots;
  int64_t hash_cap;
  uint32_t* slot_cell;  // cell id of each occupied slot (selected queries)
  uint32_t* qcount;     // selected queries per support cell
  uint32_t* qstart;     // first query record of each support cell
  HashSlot* qslots;     // query-cell table (general queries)
  int64_t qhash_cap;
};

Bufs layout(void* ws, int64_t n, int64_t m, int64_t n_clouds, int kind, size_t* bytes) {
  Arena a(ws);
  Bufs b{};
  const int64_t nm = n > m ? n : m;
  b.meta = a.take<Meta>(1);
  // Sized for every valid batch id (< 2^15) so one size serves all callers.
  b.bbox = a.take<int>(6 * static_cast<size_t>(n_clouds > 32768 ? n_clouds : 32768));
  b.pc_s = a.take<int4>(n);
  b.pc_q = kind == FKNN_QUERY_GENERAL ? a.take<int4>(m) : nullptr;
  b.slot_of = a.take<uint32_t>(nm);
  b.rank_of = a.take<uint32_t>(nm);
  b.cell_slot = a.take<uint32_t>(nm);
  b.tile_counts = a.take<uint32_t>(static_cast<size_t>(ceil_div(nm > 0 ? nm : 1, 256)));
  b.tile_counts2 = a.take<uint32_t>(static_cast<size_t>(ceil_div(nm > 0 ? nm : 1, 2048)));
  b.srec = a.take<float4>(n);
  b.cell_key = a.take<uint64_t>(n);
  b.cell_start = a.take<int32_t>(n + 1);
  b.hash_cap = 16;
  while (b.hash_cap < 2 * n) b.hash_cap <<= 1;
  b.hslots = a.take<HashSlot>(b.hash_cap);
  if (kind == FKNN_QUERY_SELECTED) {
    b.pos_of = a.take<int32_t>(n);
    b.cell_of = a.take<int32_t>(n);
    b.slot_cell = a.take<uint32_t>(b.hash_cap);
    b.qcount = a.take<uint32_t>(n);
    b.qstart = a.take<uint32_t>(n);
  }
  if (kind == FKNN_QUERY_GENERAL) {
    b.runs = a.take<int2>(static_cast<size_t>(m) * kNeighbours);
    b.group_key = a.take<uint64_t>(m);
    b.qhash_cap = 16;
    while (b.qhash_cap < 2 * m) b.qhash_cap <<= 1;
    b.qslots = a.take<HashSlot>(b.qhash_cap);
  } else {
    b.runs = a.take<int2>(static_cast<size_t>(n) * kNeighbours);
  }
  if (kind != FKNN_QUERY_SELF) {
    b.qrec = a.take<float4>(m);
    b.group_start = a.take<int32_t>(m + 1);
    b.group_row = kind == FKNN_QUERY_SELECTED ? a.take<int32_t>(m) : nullptr;
  }
  const int64_t q = kind == FKNN_QUERY_SELF ? n : m;
  const int64_t max_groups = kind == FKNN_QUERY_SELF ? n : m;
  b.items = a.take<int4>(items_capacity(max_groups, q));
  b.cands = a.take<int32_t>(max_groups);
  b.seg_counts = a.take<uint32_t>(pack_segments(max_groups));
  if (bytes) *bytes = a.used + 256;
  return b;
}

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

// Points (or cells) per thread of the construction kernels: 8 once the
// problem gives at least two 2048-point CTAs per SM, fewer for smaller
// problems so that their CTAs still spread over the SMs instead of a few
// threads walking eight points each.
int points_per_thread(int64_t n) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
      sms = v;
    else
      return 8;
  }
  int ppt = 8;
  while (ppt > 1 && ceil_div(n > 0 ? n : 1, 256 * ppt) < 2 * sms) ppt >>= 1;
  return ppt;
}

// Grid for kernels whose real extent is only known on the device: enough
// blocks to fill the GPU, a grid-stride loop covers the rest.
inline int capped_blocks(int64_t upper_threads) {
  return static_cast<int>(ceil_div(upper_threads > 0 ? upper_threads : 1, 256) < 2048
                              ? ceil_div(upper_threads > 0 ? upper_threads : 1, 256)
                              : 2048);
}

}  // namespace

size_t fused_workspace_bytes(int64_t n, int64_t m, int64_t n_clouds, int kind) {
  size_t bytes = 0;
  layout(nullptr, n, m, n_clouds, kind, &bytes);
  return bytes;
}

int run_fused(const FusedArgs& f, void* ws, size_t ws_bytes, const QueryShape& shape,
              cudaStream_t s, int* launches) {
  const int64_t n = f.n;
  const int kind = f.kind;
  const int64_t m = kind == FKNN_QUERY_SELF ? n : f.m;
  const int64_t n_clouds = f.n_clouds;
  size_t need = 0;
  Bufs b = layout(ws, n, m, n_clouds, kind, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  int nl = 0;
  cudaError_t e;
  const uint32_t hmask = static_cast<uint32_t>(b.hash_cap - 1);

  launch_chained(k_init, 64, 256, 0, s, b.meta, b.bbox, n_clouds);
  ++nl;

  const float inv_voxel = 1.0f / f.voxel;  // host FP32 division, correctly rounded
  PointSrc ps{f.xyz, f.grid, f.batch, f.offsets, n_clouds, n, inv_voxel, f.num_down,
              f.sindex, f.n_src, f.trunc_grid};
  const int ppt_s = points_per_thread(n);
  if (n > 0) {
    launch_chained(k_bbox, blocks_for(n, 256 * ppt_s), 256, 0, s, ps, b.pc_s, b.bbox, b.meta,
                   ppt_s);
    ++nl;
  }
  PointSrc pq{f.qxyz, nullptr, f.qbatch, f.qbatch ? nullptr : f.qoffsets, n_clouds, m, inv_voxel,
              f.num_down, nullptr, m, f.trunc_grid};
  const int ppt_q = points_per_thread(m);
  if (kind == FKNN_QUERY_GENERAL && m > 0) {
    launch_chained(k_bbox, blocks_for(m, 256 * ppt_q), 256, 0, s, pq, b.pc_q, b.bbox, b.meta,
                   ppt_q);
    ++nl;
  }
  launch_chained(k_meta, 1, 1024, 0, s, b.bbox, n_clouds, b.meta);
  ++nl;

  // --- support cells
  if (n > 0) {
    // Counting sort by cell through the hash table.
    e = cudaMemsetAsync(b.hslots, 0, sizeof(HashSlot) * static_cast<size_t>(b.hash_cap), s);
    if (e != cudaSuccess) {
      note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
    const int tiles = blocks_for(n, 256 * ppt_s);
    launch_chained(k_cell_insert, tiles, 256, 0, s, b.pc_s, n, b.bbox, b.meta, b.hslots, hmask,
                   b.slot_of, b.rank_of, b.cell_slot, &b.meta->n_cells, ppt_s);
    launch_chained(k_cell_tiles, tiles, 256, 0, s,
        &b.meta->n_cells, b.cell_slot, b.hslots, b.tile_counts, ppt_s);
    launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts, tiles, &b.meta->n_points_scanned);
    launch_chained(k_cell_starts, tiles, 256, 0, s, &b.meta->n_cells, b.cell_slot, b.hslots,
                   b.tile_counts, n, b.cell_key, b.cell_start, b.slot_cell, b.qcount, ppt_s);
    launch_chained(k_scatter, blocks_for(n, 256), 256, 0, s, f.xyz, f.sindex, f.n_src, n, b.slot_of,
        b.rank_of, b.hslots, b.slot_cell, b.srec, b.pos_of, b.cell_of, &b.meta->status);
    nl += 5;
  }

  const float4* qrec = b.srec;
  int n_qrec = static_cast<int>(n);
  const int2* runs = b.runs;
  int pad_mode = f.pad_minus_one ? kPadMinusOne : kPadSelf;
  const void* pad = nullptr;
  const int32_t* group_start = b.cell_start;
  const int32_t* group_row = nullptr;
  const int* group_count_ptr = &b.meta->n_cells;

  if (kind == FKNN_QUERY_SELF) {
    if (n > 0) {
      launch_chained(k_runs, capped_blocks(n * 32), 256, 0, s, b.cell_key, &b.meta->n_cells,
                     b.hslots, hmask, &b.meta->n_cells, b.meta, b.runs, b.cands,
                     &b.meta->status);
      ++nl;
      nl += launch_items(b.runs, b.cell_start, nullptr, &b.meta->n_cells, n, shape.tile_records,
                         b.cands, b.seg_counts, &b.meta->n_items, b.items, s, &b.meta->status, n,
                         true);
    }
  } else if (kind == FKNN_QUERY_SELECTED) {
    pad_mode = kPadArray64;
    pad = f.query_indices;
    qrec = b.qrec;
    n_qrec = static_cast<int>(m);
    group_start = b.group_start;
    group_row = b.group_row;
    group_count_ptr = &b.meta->n_groups;
    if (n > 0) {
      launch_chained(k_runs, capped_blocks(n * 32), 256, 0, s, b.cell_key,
          &b.meta->n_cells, b.hslots, hmask, &b.meta->n_cells, b.meta, b.runs, nullptr, nullptr);
      ++nl;
    }
    if (m > 0 && n > 0) {
      // per-query cell and rank in slot_of / rank_of (free again once the
      // support records are written)
      const int ctiles = blocks_for(n, 2048);
      launch_chained(k_sel_count, blocks_for(m, 256), 256, 0, s, f.query_indices, m, n, b.pos_of,
          b.cell_of, b.meta, b.qcount, b.slot_of, b.rank_of);
      launch_chained(k_sel_tiles, ctiles, 256, 0, s,
          &b.meta->n_cells, b.qcount, b.tile_counts, b.tile_counts2);
      launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts, ctiles, &b.meta->n_groups);
      launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts2, ctiles,
                     &b.meta->n_points_scanned);
      launch_chained(k_sel_starts, ctiles, 256, 0, s, &b.meta->n_cells, b.qcount, b.tile_counts,
                     b.tile_counts2, m, &b.meta->n_groups, b.group_start, b.group_row,
                     b.qstart);
      launch_chained(k_sel_scatter, blocks_for(m, 256), 256, 0, s, m, n, f.query_indices, b.pos_of,
          b.srec, b.slot_of, b.rank_of, b.qstart, b.qrec, &b.meta->status);
      nl += 6;
      nl += launch_items(b.runs, b.group_start, b.group_row, &b.meta->n_groups, m,
                         shape.tile_records, b.cands, b.seg_counts, &b.meta->n_items, b.items, s,
                         &b.meta->status, m, false);
    }
  } else {  // general queries
    pad_mode = kPadMinusOne;
    qrec = b.qrec;
    n_qrec = static_cast<int>(m);
    runs = b.runs;
    group_start = b.group_start;
    group_count_ptr = &b.meta->n_groups;
    if (m > 0) {
      // query groups = query cells, by the same counting sort through a
      // second table (slot_of / rank_of / cell_slot are free again once the
      // support records are written)
      e = cudaMemsetAsync(b.qslots, 0, sizeof(HashSlot) * static_cast<size_t>(b.qhash_cap), s);
      if (e != cudaSuccess) {
        note_cuda_error(e);
        return FKNN_ERR_CUDA;
      }
      const uint32_t qmask = static_cast<uint32_t>(b.qhash_cap - 1);
      const int tiles = blocks_for(m, 256 * ppt_q);
      launch_chained(k_cell_insert, tiles, 256, 0, s, b.pc_q, m, b.bbox, b.meta, b.qslots, qmask,
          b.slot_of, b.rank_of, b.cell_slot, &b.meta->n_groups, ppt_q);
      launch_chained(k_cell_tiles, tiles, 256, 0, s,
          &b.meta->n_groups, b.cell_slot, b.qslots, b.tile_counts, ppt_q);
      launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts, tiles, &b.meta->n_points_scanned);
      launch_chained(k_cell_starts, tiles, 256, 0, s, &b.meta->n_groups, b.cell_slot, b.qslots,
                     b.tile_counts, m, b.group_key, b.group_start, nullptr, nullptr, ppt_q);
      launch_chained(k_scatter, blocks_for(m, 256), 256, 0, s, f.qxyz, nullptr, m, m, b.slot_of,
          b.rank_of, b.qslots, nullptr, b.qrec, nullptr, nullptr, &b.meta->status);
      nl += 5;
      launch_chained(k_runs, capped_blocks(m * 32), 256, 0, s, b.group_key, &b.meta->n_groups,
                     b.hslots, hmask, &b.meta->n_cells, b.meta, b.runs, b.cands,
                     &b.meta->status);
      ++nl;
      nl += launch_items(b.runs, b.group_start, nullptr, &b.meta->n_groups, m, shape.tile_records,
                         b.cands, b.seg_counts, &b.meta->n_items, b.items, s, &b.meta->status, m,
                         true);
    }
  }

  e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (m > 0) {
    QueryLaunch q{};
    q.srec = b.srec;
    q.n_support = static_cast<int>(n);
    q.qrec = qrec;
    q.n_qrec = n_qrec;
    q.runs = runs;
    q.group_start = group_start;
    q.group_row = group_row;
    q.group_count_ptr = group_count_ptr;
    q.items = b.items;
    q.meta = b.meta;
    q.k = f.k;
    q.cut_r2 = f.cut_r2;
    q.idx_bits = f.idx_bits;
    q.idx_out = f.idx_out;
    q.dist_out = f.dist_out;
    q.n_rows = m;
    q.pad = pad;
    q.pad_mode = pad_mode;
    q.vec_ok = (reinterpret_cast<uintptr_t>(f.idx_out) % 16 == 0) &&
               (reinterpret_cast<uintptr_t>(f.dist_out) % 16 == 0);
    const int rc = launch_query(q, shape, s);
    if (rc != 0) {
      note_cuda_error(static_cast<cudaError_t>(rc));
      return FKNN_ERR_CUDA;
    }
    ++nl;
  }
  if (launches) *launches = nl;
  return FKNN_OK;
}

}  // namespace fknn
