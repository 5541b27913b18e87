// The reference's table ABI on the device:
//   * morton encode / neighbour keys (FlashKNN/csrc/flash_knn_construction.cu),
//   * the reference table construction (FlashKNN/functions/FlashKnnWrapper.py
//     :220-337: stable key sort, parent grouping by key >> 3*num_down, steps,
//     sorted-key neighbour lookup, candidate prefix table),
//   * queries over caller-provided tables (FlashKNN_Query_Dynamic_Load and
//     FlashKNN_Selected_Query_DL), run by the same persistent query kernel as
//     the fused path after two small preparation kernels.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"
#include "fknn_tables.h"

namespace fknn {

// Reference key: low 16 bits of each coordinate interleaved, batch << 48.
__device__ __forceinline__ uint64_t ref_key(int64_t x, int64_t y, int64_t z, int64_t b) {
  return morton3(static_cast<uint32_t>(x) & 0xffffu, static_cast<uint32_t>(y) & 0xffffu,
                 static_cast<uint32_t>(z) & 0xffffu) |
         (static_cast<uint64_t>(b) << 48);
}

__device__ __forceinline__ int ref_axis_offset(int position) {
  return position == 0 ? 0 : (position == 1 ? -1 : 1);
}

__global__ void k_morton_encode(const int64_t* __restrict__ grid, const int64_t* __restrict__ batch,
                                int64_t n, int64_t* __restrict__ keys) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = static_cast<int64_t>(
      ref_key(grid[3 * i], grid[3 * i + 1], grid[3 * i + 2], batch ? batch[i] : 0));
}

__global__ void k_neighbor_keys(const int64_t* __restrict__ gd, const int64_t* __restrict__ pb,
                                int64_t p, int64_t* __restrict__ keys) {
  chain_wait();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= p * 27) return;
  const int64_t q = t / 27;
  const int j = static_cast<int>(t - q * 27);
  keys[t] = static_cast<int64_t>(ref_key(gd[3 * q] + ref_axis_offset(j / 9),
                                         gd[3 * q + 1] + ref_axis_offset((j / 3) % 3),
                                         gd[3 * q + 2] + ref_axis_offset(j % 3),
                                         pb ? pb[q] : 0));
}

// ------------------------------------------------- queries over tables

__global__ void k_tab_records(const float* __restrict__ xyz, int64_t n, float4* __restrict__ rec) {
  chain_wait();
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n) return;
  rec[s] = make_float4(xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2],
                       __int_as_float(static_cast<int>(s)));
}

// runs[p*27+j] = (steps[neigh], cnt[j+1] - cnt[j]): the candidates the
// reference loader enumerates for neighbour position j
// (flash_knn_query_dynamic_load.cu:87-155).
__global__ void k_tab_runs(const int32_t* __restrict__ steps, const int32_t* __restrict__ neigh,
                           const int32_t* __restrict__ cnt, int64_t p, Meta* meta,
                           int2* __restrict__ runs) {
  chain_wait();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t == 0) meta->n_groups = static_cast<int>(p);
  if (t >= p * 27) return;
  const int64_t q = t / 27;
  const int j = static_cast<int>(t - q * 27);
  const int32_t c = cnt[q * 28 + j + 1] - cnt[q * 28 + j];
  int2 run = make_int2(0, 0);
  if (c > 0) {
    const int32_t nb = neigh[t];
    if (nb < 0 || nb >= p) {
      raise_status(&meta->status, kStatusTable);
    } else {
      run = make_int2(steps[nb], c);
    }
  } else if (c < 0) {
    raise_status(&meta->status, kStatusTable);
  }
  runs[t] = run;
}

__global__ void k_tab_qrec(const float* __restrict__ xyz, int64_t n, const int32_t* __restrict__ qindex,
                           int64_t m, Meta* meta, float4* __restrict__ qrec) {
  chain_wait();
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t s = qindex[r];
  if (s < 0 || s >= n) {
    raise_status(&meta->status, kStatusTable);
    s = 0;
  }
  qrec[r] = make_float4(xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2],
                        __int_as_float(static_cast<int>(r)));
}

// Separate query points (FlashKNN_Query_GM, the back-query kernels): row r
// is qxyz[r], already grouped by the caller's steps_query.
__global__ void k_tab_qxyz(const float* __restrict__ qxyz, int64_t m, float4* __restrict__ qrec) {
  chain_wait();
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= m) return;
  qrec[r] = make_float4(qxyz[3 * r], qxyz[3 * r + 1], qxyz[3 * r + 2],
                        __int_as_float(static_cast<int>(r)));
}

namespace {

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

struct TabBufs {
  Meta* meta;
  float4* srec;
  float4* qrec;
  int2* runs;
  int4* items;
  int32_t* cands;
  uint32_t* seg_counts;
};

TabBufs tab_layout(void* ws, int64_t n, int64_t m, int64_t p, size_t* bytes) {
  Arena a(ws);
  TabBufs b{};
  b.meta = a.take<Meta>(1);
  b.srec = a.take<float4>(n);
  b.qrec = a.take<float4>(m);
  b.runs = a.take<int2>(static_cast<size_t>(p) * 27);
  b.items = a.take<int4>(items_capacity(p, m));
  b.cands = a.take<int32_t>(p);
  b.seg_counts = a.take<uint32_t>(pack_segments(p));
  if (bytes) *bytes = a.used + 256;
  return b;
}

}  // namespace

size_t tables_workspace_bytes(int64_t n, int64_t m, int64_t p) {
  size_t bytes = 0;
  tab_layout(nullptr, n, m, p, &bytes);
  return bytes;
}

int run_tables(const TablesArgs& t, void* ws, size_t ws_bytes, const QueryShape& shape,
               cudaStream_t s, int* launches) {
  const bool general = t.qxyz != nullptr;
  const bool selected = t.qindex != nullptr || general;
  const int64_t m = selected ? t.m : t.n;
  size_t need = 0;
  TabBufs b = tab_layout(ws, t.n, m, t.p, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  int nl = 0;
  cudaError_t e = cudaMemsetAsync(b.meta, 0, sizeof(Meta), s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (t.n > 0) {
    launch_chained(k_tab_records, blocks_for(t.n, 256), 256, 0, s, t.xyz_sorted, t.n, b.srec);
    ++nl;
  }
  launch_chained(k_tab_runs, blocks_for(t.p * 27, 256), 256, 0, s, t.steps, t.neigh, t.cnt, t.p,
                 b.meta, b.runs);
  ++nl;
  if (general && m > 0) {
    launch_chained(k_tab_qxyz, blocks_for(m, 256), 256, 0, s, t.qxyz, m, b.qrec);
    ++nl;
  } else if (selected && m > 0) {
    launch_chained(k_tab_qrec, blocks_for(m, 256), 256, 0, s, t.xyz_sorted, t.n, t.qindex, m,
                   b.meta, b.qrec);
    ++nl;
  }
  if (t.p > 0)
    nl += launch_items(b.runs, selected ? t.steps_query : t.steps, nullptr, &b.meta->n_groups, t.p,
                       shape.tile_records, b.cands, b.seg_counts, &b.meta->n_items, b.items, s,
                       &b.meta->status, selected ? m : t.n, false);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (m > 0 && t.p > 0) {
    QueryLaunch q{};
    q.srec = b.srec;
    q.n_support = static_cast<int>(t.n);
    q.qrec = selected ? b.qrec : b.srec;
    q.n_qrec = static_cast<int>(m);
    q.runs = b.runs;
    q.group_start = selected ? t.steps_query : t.steps;
    q.group_row = nullptr;
    q.group_count_ptr = &b.meta->n_groups;
    q.items = b.items;
    q.meta = b.meta;
    q.k = t.k;
    q.cut_r2 = t.cut_r2;
    q.idx_bits = 32;
    q.idx_out = t.idx_out;
    q.dist_out = t.dist_out;
    q.n_rows = m;
    if (general) {
      q.pad = t.qpad;
      q.pad_mode = t.qpad ? kPadArray32 : kPadMinusOne;
    } else {
      q.pad = selected ? static_cast<const void*>(t.qindex) : nullptr;
      q.pad_mode = selected ? kPadArray32 : kPadSelf;
    }
    q.vec_ok = (reinterpret_cast<uintptr_t>(t.idx_out) % 16 == 0) &&
               (reinterpret_cast<uintptr_t>(t.dist_out) % 16 == 0);
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

// ------------------------------------------- reference table construction

__global__ void k_ref_keys(const int64_t* __restrict__ grid, const int64_t* __restrict__ batch,
                           int64_t n, Meta* meta, unsigned long long* max_key,
                           uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  chain_wait();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  uint64_t key = 0;
  if (i < n) {
    const int64_t b = batch ? batch[i] : 0;
    if (b < 0 || b >= 32768) raise_status(&meta->status, kStatusBatch);
    key = ref_key(grid[3 * i], grid[3 * i + 1], grid[3 * i + 2], b);
    keys[i] = key;
    vals[i] = static_cast<uint32_t>(i);
  }
  // One atomic per warp for the largest key.
  unsigned long long wmax = key;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const unsigned long long o = __shfl_xor_sync(kFull, wmax, s);
    wmax = o > wmax ? o : wmax;
  }
  if ((threadIdx.x & 31) == 0 && wmax) atomicMax(max_key, wmax);
}

__global__ void k_ref_bits(const unsigned long long* max_key, Meta* meta) {
  chain_wait();
  const unsigned long long k = *max_key;
  meta->key_bits = k ? 64 - __clzll(static_cast<long long>(k)) : 0;
}

// order[s] = sorted point id; parent heads (key >> 3*num_down changes).
__global__ void __launch_bounds__(256)
    k_ref_order(int64_t n, SortPair<uint64_t> sp, const int* bits_ptr, int num_down,
                int64_t* __restrict__ order, uint32_t* __restrict__ tile_counts) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_total;
  const int buf = sort_passes_for_bits(*bits_ptr) & 1;
  const uint64_t* keys = sp.key_buf(buf);
  const uint32_t* vals = sp.val_buf(buf);
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 2048 + threadIdx.x * 8;
  uint32_t heads = 0;
  const int sh = 3 * num_down;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t s = base + r;
    if (s >= n) break;
    order[s] = vals[s];
    heads += (s == 0 || (keys[s] >> sh) != (keys[s - 1] >> sh)) ? 1u : 0u;
  }
  block_inclusive_scan(heads, warp_sums, &s_total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = s_total;
}

// steps[p] = first sorted position of parent p; parent grid (>> num_down),
// batch and reference key of its first point (FlashKnnWrapper.py:250-263).
__global__ void __launch_bounds__(256)
    k_ref_parents(int64_t n, SortPair<uint64_t> sp, const int* bits_ptr, int num_down,
                  const uint32_t* __restrict__ tile_offsets, const int* count_ptr,
                  const int64_t* __restrict__ grid, const int64_t* __restrict__ batch,
                  const int64_t* __restrict__ order, int32_t* __restrict__ steps,
                  int64_t* __restrict__ gd, int64_t* __restrict__ pb,
                  uint64_t* __restrict__ pkey, int64_t* __restrict__ n_parents) {
  chain_wait();
  __shared__ uint32_t warp_sums[32];
  const uint64_t* keys = sp.key_buf(sort_passes_for_bits(*bits_ptr) & 1);
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 2048 + threadIdx.x * 8;
  const int sh = 3 * num_down;
  uint32_t flags = 0, heads = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t s = base + r;
    if (s < n && (s == 0 || (keys[s] >> sh) != (keys[s - 1] >> sh))) {
      flags |= 1u << r;
      ++heads;
    }
  }
  const uint32_t incl = block_inclusive_scan(heads, warp_sums, nullptr);
  int c = static_cast<int>(tile_offsets[blockIdx.x] + incl - heads);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t s = base + r;
    if (s >= n) break;
    if (flags & (1u << r)) {
      const int64_t src = order[s];
      steps[c] = static_cast<int32_t>(s);
      const int64_t x = grid[3 * src] >> num_down, y = grid[3 * src + 1] >> num_down,
                    z = grid[3 * src + 2] >> num_down;
      const int64_t b = batch ? batch[src] : 0;
      gd[3 * c] = x;
      gd[3 * c + 1] = y;
      gd[3 * c + 2] = z;
      pb[c] = b;
      pkey[c] = ref_key(x, y, z, b);
      ++c;
    }
    if (s == n - 1) {
      steps[*count_ptr] = static_cast<int32_t>(n);
      *n_parents = *count_ptr;
    }
  }
}

// neigh[p*27+j] = index of the parent whose reference key equals the j-th
// neighbour key, else -1 (the searchsorted lookup, FlashKnnWrapper.py:279-287).
__global__ void k_ref_neigh(const int64_t* __restrict__ gd, const int64_t* __restrict__ pb,
                            const uint64_t* __restrict__ pkey, const int* count_ptr,
                            int32_t* __restrict__ neigh) {
  chain_wait();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int p = *count_ptr;
  if (t >= static_cast<int64_t>(p) * 27) return;
  const int64_t q = t / 27;
  const int j = static_cast<int>(t - q * 27);
  const uint64_t key = ref_key(gd[3 * q] + ref_axis_offset(j / 9),
                               gd[3 * q + 1] + ref_axis_offset((j / 3) % 3),
                               gd[3 * q + 2] + ref_axis_offset(j % 3), pb[q]);
  int lo = 0, hi = p;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (pkey[mid] < key) lo = mid + 1; else hi = mid;
  }
  neigh[t] = (lo < p && pkey[lo] == key) ? lo : -1;
}

// cnt[p*28 + j] = exclusive prefix of the neighbour counts (FlashKnnWrapper.py:337).
__global__ void k_ref_cnt(const int32_t* __restrict__ steps, const int32_t* __restrict__ neigh,
                          const int* count_ptr, int32_t* __restrict__ cnt) {
  chain_wait();
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= *count_ptr) return;
  int32_t acc = 0;
  cnt[q * 28] = 0;
  for (int j = 0; j < 27; ++j) {
    const int32_t nb = neigh[q * 27 + j];
    acc += nb >= 0 ? steps[nb + 1] - steps[nb] : 0;
    cnt[q * 28 + j + 1] = acc;
  }
}

namespace {

struct RefBufs {
  Meta* meta;
  unsigned long long* max_key;
  uint64_t* keys[2];
  uint32_t* vals[2];
  uint32_t* hist;
  uint32_t* totals;
  uint32_t* tile_counts;
  int64_t* gd;
  int64_t* pb;
  uint64_t* pkey;
};

RefBufs ref_layout(void* ws, int64_t n, size_t* bytes) {
  Arena a(ws);
  RefBufs b{};
  b.meta = a.take<Meta>(1);
  b.max_key = a.take<unsigned long long>(1);
  b.keys[0] = a.take<uint64_t>(n);
  b.keys[1] = a.take<uint64_t>(n);
  b.vals[0] = a.take<uint32_t>(n);
  b.vals[1] = a.take<uint32_t>(n);
  b.hist = a.take<uint32_t>(sort_hist_elems(n));
  b.totals = a.take<uint32_t>(kSortMaxPasses * 256);
  b.tile_counts = a.take<uint32_t>(static_cast<size_t>(ceil_div(n > 0 ? n : 1, 2048)));
  b.gd = a.take<int64_t>(3 * static_cast<size_t>(n));
  b.pb = a.take<int64_t>(n);
  b.pkey = a.take<uint64_t>(n);
  if (bytes) *bytes = a.used + 256;
  return b;
}

}  // namespace

size_t build_tables_workspace_bytes(int64_t n) {
  size_t bytes = 0;
  ref_layout(nullptr, n, &bytes);
  return bytes;
}

int run_build_tables(const BuildTablesArgs& t, void* ws, size_t ws_bytes, cudaStream_t s,
                     int* launches) {
  size_t need = 0;
  RefBufs b = ref_layout(ws, t.n, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  cudaError_t e = cudaMemsetAsync(b.meta, 0, 512, s);  // Meta + max_key
  if (e == cudaSuccess) e = cudaMemsetAsync(b.totals, 0, kSortMaxPasses * 256 * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t.n_parents, 0, sizeof(int64_t), s);
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  int nl = 0;
  if (t.n > 0) {
    const int tiles = blocks_for(t.n, 2048);
    launch_chained(k_ref_keys, blocks_for(t.n, 256), 256, 0, s, t.grid, t.batch, t.n, b.meta,
                   b.max_key, b.keys[0], b.vals[0]);
    launch_chained(k_ref_bits, 1, 1, 0, s, b.max_key, b.meta);
    nl += 2;
    SortBuffers<uint64_t> sb{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}, b.hist, b.totals};
    nl += launch_radix_sort(sb, t.n, &b.meta->key_bits, kSortMaxPasses, s);
    const SortPair<uint64_t> sp{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}};
    launch_chained(k_ref_order, tiles, 256, 0, s, t.n, sp, &b.meta->key_bits, t.num_down, t.order,
                   b.tile_counts);
    launch_chained(k_scan_tiles, 1, 1024, 0, s, b.tile_counts, tiles, &b.meta->n_cells);
    launch_chained(k_ref_parents, tiles, 256, 0, s, t.n, sp, &b.meta->key_bits, t.num_down,
                   b.tile_counts, &b.meta->n_cells, t.grid, t.batch, t.order, t.steps, b.gd, b.pb,
                   b.pkey, t.n_parents);
    launch_chained(k_ref_neigh, blocks_for(t.n * 27, 256), 256, 0, s, b.gd, b.pb, b.pkey,
                   &b.meta->n_cells, t.neigh);
    launch_chained(k_ref_cnt, blocks_for(t.n, 256), 256, 0, s, t.steps, t.neigh, &b.meta->n_cells,
                   t.cnt);
    nl += 5;
  } else {
    e = cudaMemsetAsync(t.steps, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) {
      note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (launches) *launches = nl;
  return FKNN_OK;
}

int run_morton_encode(const int64_t* grid, const int64_t* batch, int64_t n, int64_t* keys,
                      cudaStream_t s) {
  if (n <= 0) return FKNN_OK;
  launch_chained(k_morton_encode, blocks_for(n, 256), 256, 0, s, grid, batch, n, keys);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  return FKNN_OK;
}

int run_neighbor_keys(const int64_t* gd, const int64_t* pb, int64_t p, int64_t* keys,
                      cudaStream_t s) {
  if (p <= 0) return FKNN_OK;
  launch_chained(k_neighbor_keys, blocks_for(p * 27, 256), 256, 0, s, gd, pb, p, keys);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  return FKNN_OK;
}

}  // namespace fknn
