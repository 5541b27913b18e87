/*
 * CPU restatement of FlashKNN's grid kNN -- TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the product library links or calls this file.  It is the
 * checker for the CUDA path: the parity tests, the smoke check and the CPU
 * baseline leg of the benchmark call it through ctypes (oracle/oracle.py).
 *
 * What it restates (paths are relative to the reference project root):
 *   - morton key: FlashKNN/csrc/flash_knn_construction.cu:13-27
 *     (low 16 bits per axis, x at bit 3b+2, y at 3b+1, z at 3b, batch << 48);
 *   - 27 neighbour keys, offsets (0,-1,+1) per axis in ij order, centre first:
 *     FlashKNN/csrc/flash_knn_construction.cu:42-63;
 *   - table construction (sort, parent grouping by key >> 3*num_down, steps,
 *     searchsorted neighbour lookup, candidate prefix table):
 *     FlashKNN/functions/FlashKnnWrapper.py:220-337;
 *   - the SMPS query semantics: FlashKNN/csrc/flash_knn_query_dynamic_load.cu
 *     :469-652 (candidate enumeration through CumCntInNeigh :87-155, initial
 *     fill (self index, +inf) :562, strict acceptance d < K-th and d < cut_r2
 *     :587-616, ascending output :640-647).  The reference kernel is an exact
 *     top-K over the candidate set; this restatement computes that top-K
 *     directly and breaks equal distances by the lower index;
 *   - the selected-query variant: flash_knn_query_dynamic_load.cu:1211-1370;
 *   - the output remap order[idx[inverse_order]]: FlashKnnWrapper.py:427-429.
 *
 * Distances are FP32.  The contraction order of the reference's expression
 * dx*dx + dy*dy + dz*dz is not specified by the source; `variant` selects one
 * of the candidate evaluation orders so the tests can find the one that
 * reproduces the reference kernel's output bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ keys */

static uint64_t morton16(uint32_t ux, uint32_t uy, uint32_t uz) {
  uint64_t key = 0;
  for (int bit = 0; bit < 16; ++bit) {
    key |= (uint64_t)((ux >> bit) & 1u) << (3 * bit + 2);
    key |= (uint64_t)((uy >> bit) & 1u) << (3 * bit + 1);
    key |= (uint64_t)((uz >> bit) & 1u) << (3 * bit);
  }
  return key;
}

int64_t orc_morton_key(int64_t x, int64_t y, int64_t z, int64_t batch) {
  uint64_t key = morton16((uint32_t)x & 0xffffu, (uint32_t)y & 0xffffu,
                          (uint32_t)z & 0xffffu);
  key |= (uint64_t)batch << 48;
  return (int64_t)key;
}

void orc_morton_encode(const int64_t* grid, const int64_t* batch, int64_t n,
                       int64_t* keys) {
  for (int64_t i = 0; i < n; ++i)
    keys[i] = orc_morton_key(grid[3 * i], grid[3 * i + 1], grid[3 * i + 2],
                             batch ? batch[i] : 0);
}

static int axis_offset(int position) {
  return position == 0 ? 0 : (position == 1 ? -1 : 1);
}

void orc_neighbor_keys(const int64_t* grid_down, const int64_t* parent_batch,
                       int64_t p, int64_t* out) {
  for (int64_t q = 0; q < p; ++q)
    for (int j = 0; j < 27; ++j) {
      const int64_t* g = grid_down + 3 * q;
      out[q * 27 + j] = orc_morton_key(g[0] + axis_offset(j / 9),
                                       g[1] + axis_offset((j / 3) % 3),
                                       g[2] + axis_offset(j % 3),
                                       parent_batch ? parent_batch[q] : 0);
    }
}

/* ------------------------------------------------------- stable argsort */

typedef struct {
  int64_t key;
  int64_t index;
} KeyIndex;

static int cmp_key_index(const void* a, const void* b) {
  const KeyIndex* x = (const KeyIndex*)a;
  const KeyIndex* y = (const KeyIndex*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->index < y->index ? -1 : (x->index > y->index);
}

/* Stable argsort of signed 64-bit keys (ties keep input order). */
void orc_argsort_i64(const int64_t* keys, int64_t n, int64_t* order) {
  KeyIndex* tmp = (KeyIndex*)malloc(sizeof(KeyIndex) * (size_t)(n ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    tmp[i].key = keys[i];
    tmp[i].index = i;
  }
  qsort(tmp, (size_t)n, sizeof(KeyIndex), cmp_key_index);
  for (int64_t i = 0; i < n; ++i) order[i] = tmp[i].index;
  free(tmp);
}

static int64_t search_sorted(const int64_t* keys, int64_t n, int64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = lo + (hi - lo) / 2;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < n && keys[lo] == key) ? lo : -1;
}

/*
 * Reference table construction (FlashKnnWrapper.py:220-337, fused branch).
 * Outputs: order[n] (stable argsort of the keys), steps[P+1], neigh[P*27],
 * cnt[P*28] (exclusive prefix of neighbour counts), and grid_down[P*3] /
 * parent_batch[P] when non-NULL.  Every output buffer must hold the n-point
 * worst case (P <= n).  Returns P.
 */
int64_t orc_build_tables(const int64_t* grid, const int64_t* batch, int64_t n,
                         int num_down, int64_t* order, int32_t* steps,
                         int32_t* neigh, int32_t* cnt, int64_t* grid_down_out,
                         int64_t* parent_batch_out) {
  int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  orc_morton_encode(grid, batch, n, keys);
  orc_argsort_i64(keys, n, order);
  int64_t p = 0;
  int64_t prev = 0;
  for (int64_t s = 0; s < n; ++s) {
    int64_t kd = keys[order[s]] >> (3 * num_down);
    if (s == 0 || kd != prev) steps[p++] = (int32_t)s;
    prev = kd;
  }
  steps[p] = (int32_t)n;
  int64_t* gd = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)(p ? p : 1));
  int64_t* pb = (int64_t*)malloc(sizeof(int64_t) * (size_t)(p ? p : 1));
  for (int64_t q = 0; q < p; ++q) {
    int64_t src = order[steps[q]];
    for (int a = 0; a < 3; ++a) gd[3 * q + a] = grid[3 * src + a] >> num_down;
    pb[q] = batch ? batch[src] : 0;
  }
  int64_t* nk = (int64_t*)malloc(sizeof(int64_t) * 27 * (size_t)(p ? p : 1));
  orc_neighbor_keys(gd, pb, p, nk);
  int64_t* parent_keys = (int64_t*)malloc(sizeof(int64_t) * (size_t)(p ? p : 1));
  for (int64_t q = 0; q < p; ++q) parent_keys[q] = nk[27 * q];
  for (int64_t q = 0; q < p; ++q) {
    cnt[28 * q] = 0;
    for (int j = 0; j < 27; ++j) {
      int64_t hit = search_sorted(parent_keys, p, nk[27 * q + j]);
      neigh[27 * q + j] = (int32_t)hit;
      int32_t c = hit >= 0 ? steps[hit + 1] - steps[hit] : 0;
      cnt[28 * q + j + 1] = cnt[28 * q + j] + c;
    }
  }
  if (grid_down_out) memcpy(grid_down_out, gd, sizeof(int64_t) * 3 * (size_t)p);
  if (parent_batch_out) memcpy(parent_batch_out, pb, sizeof(int64_t) * (size_t)p);
  free(parent_keys);
  free(nk);
  free(pb);
  free(gd);
  free(keys);
  return p;
}

/* ------------------------------------------------------------ distances */

/*
 * FP32 squared distance between candidate c and query q, dx = c - q.
 * variant 0: fma(dz,dz, fma(dy,dy, dx*dx))
 * variant 1: fma(dz,dz, fma(dx,dx, dy*dy))
 * variant 2: ((dx*dx + dy*dy) + dz*dz), every operation rounded
 */
static inline float sqdist(const float* c, const float* q, int variant) {
  float dx = c[0] - q[0];
  float dy = c[1] - q[1];
  float dz = c[2] - q[2];
  switch (variant) {
    case 0: return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    case 1: return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
    default: {
      volatile float xx = dx * dx;
      volatile float yy = dy * dy;
      volatile float zz = dz * dz;
      volatile float s = xx + yy;
      return s + zz;
    }
  }
}

/* Sorted (distance, index) list of length k; insertion keeps the k smallest
 * under the lexicographic order (d, index). */
static inline void topk_insert(float d, int64_t id, float* dl, int64_t* il,
                               int k) {
  if (d > dl[k - 1] || (d == dl[k - 1] && id >= il[k - 1])) return;
  int j = k - 1;
  while (j > 0 && (d < dl[j - 1] || (d == dl[j - 1] && id < il[j - 1]))) {
    dl[j] = dl[j - 1];
    il[j] = il[j - 1];
    --j;
  }
  dl[j] = d;
  il[j] = id;
}

#define ORC_MAXK 1024

/*
 * Query over the reference table ABI (FlashKNN_Query_Dynamic_Load).
 * xyz_sorted[n*3], steps[p+1], neigh[p*27], cnt[p*28].  Output rows are in
 * sorted-point space; reported indices are idx_map[t] when idx_map is given,
 * else the sorted position t.  Ties break by the reported index.
 * Returns 0, or -1 for K out of range, -2 for a table that names an empty
 * neighbour with a non-zero count.
 */
int orc_query_tables(const float* xyz_sorted, const int32_t* steps,
                     const int32_t* neigh, const int32_t* cnt, int64_t p,
                     int k, float cut_r2, int variant, const int64_t* idx_map,
                     int64_t* idx_out, float* dist_out, int nthreads) {
  if (k < 1 || k > ORC_MAXK) return -1;
  int bad = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad)
#endif
  for (int64_t q = 0; q < p; ++q) {
    float dl[ORC_MAXK];
    int64_t il[ORC_MAXK];
    for (int32_t s = steps[q]; s < steps[q + 1]; ++s) {
      int64_t self = idx_map ? idx_map[s] : s;
      for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
      for (int j = 0; j < 27; ++j) {
        int32_t c = cnt[28 * q + j + 1] - cnt[28 * q + j];
        if (c <= 0) continue;
        int32_t nb = neigh[27 * q + j];
        if (nb < 0) { bad = 1; continue; }
        for (int32_t t = steps[nb]; t < steps[nb] + c; ++t) {
          float d = sqdist(xyz_sorted + 3 * (int64_t)t, xyz_sorted + 3 * (int64_t)s, variant);
          if (!(d < cut_r2)) continue;
          topk_insert(d, idx_map ? idx_map[t] : t, dl, il, k);
        }
      }
      for (int j = 0; j < k; ++j) {
        idx_out[(int64_t)s * k + j] = (il[j] == INT64_MAX) ? self : il[j];
        dist_out[(int64_t)s * k + j] = dl[j];
      }
    }
  }
  return bad ? -2 : 0;
}

/*
 * Selected query over the reference table ABI (FlashKNN_Selected_Query_DL).
 * qindex[m] holds the sorted support index of each query, grouped by parent
 * through steps_query[p+1].  Output row r belongs to query qindex[r]; the pad
 * index is the query's own support index (flash_knn_query_dynamic_load.cu:1289).
 */
int orc_selected_query_tables(const float* xyz_sorted, const int32_t* qindex,
                              const int32_t* steps, const int32_t* steps_query,
                              const int32_t* neigh, const int32_t* cnt,
                              int64_t p, int k, float cut_r2, int variant,
                              const int64_t* idx_map, int64_t* idx_out,
                              float* dist_out, int nthreads) {
  if (k < 1 || k > ORC_MAXK) return -1;
  int bad = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad)
#endif
  for (int64_t q = 0; q < p; ++q) {
    float dl[ORC_MAXK];
    int64_t il[ORC_MAXK];
    for (int32_t r = steps_query[q]; r < steps_query[q + 1]; ++r) {
      int32_t s = qindex[r];
      int64_t self = idx_map ? idx_map[s] : s;
      for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
      for (int j = 0; j < 27; ++j) {
        int32_t c = cnt[28 * q + j + 1] - cnt[28 * q + j];
        if (c <= 0) continue;
        int32_t nb = neigh[27 * q + j];
        if (nb < 0) { bad = 1; continue; }
        for (int32_t t = steps[nb]; t < steps[nb] + c; ++t) {
          float d = sqdist(xyz_sorted + 3 * (int64_t)t, xyz_sorted + 3 * (int64_t)s, variant);
          if (!(d < cut_r2)) continue;
          topk_insert(d, idx_map ? idx_map[t] : t, dl, il, k);
        }
      }
      for (int j = 0; j < k; ++j) {
        idx_out[(int64_t)r * k + j] = (il[j] == INT64_MAX) ? self : il[j];
        dist_out[(int64_t)r * k + j] = dl[j];
      }
    }
  }
  return bad ? -2 : 0;
}

/* ------------------------------------------------------- general queries */

/*
 * Grid kNN in original-index space, for queries that need not be support
 * points.  A query's candidates are the support points whose parent cell
 * (grid >> num_down, same batch) lies in the 3x3x3 block of parent cells
 * around the query's own parent cell -- for a query that is a support point
 * this is exactly the reference's candidate set.  Ties break by the lower
 * support index.  Rows with fewer than K candidates are padded with
 * (pad[r], +inf); pad == NULL pads with -1.
 * sgrid/sbatch: support grid coords [n*3] and batch [n]; qgrid/qbatch: query.
 */
int orc_knn_general(const float* sxyz, const int64_t* sgrid,
                    const int64_t* sbatch, int64_t n, const float* qxyz,
                    const int64_t* qgrid, const int64_t* qbatch, int64_t m,
                    int num_down, int k, float cut_r2, int variant,
                    const int64_t* pad, int32_t* idx_out, float* dist_out,
                    int nthreads) {
  if (k < 1 || k > ORC_MAXK) return -1;
  /* Parent-cell keys.  For grid coordinates inside [-2^15, 2^15) the 16-bit
   * truncation of the morton key is injective on parent cells and a +-1
   * neighbour key never aliases an occupied cell, so the key lookup below is
   * integer adjacency of parent cells. */
  int64_t* pk = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  for (int64_t i = 0; i < n; ++i)
    pk[i] = orc_morton_key(sgrid[3 * i] >> num_down, sgrid[3 * i + 1] >> num_down,
                           sgrid[3 * i + 2] >> num_down, sbatch ? sbatch[i] : 0);
  orc_argsort_i64(pk, n, order);
  int64_t* cell_key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  int64_t* cell_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t p = 0;
  for (int64_t s = 0; s < n; ++s) {
    int64_t key = pk[order[s]];
    if (s == 0 || key != cell_key[p - 1]) { cell_key[p] = key; cell_start[p] = s; ++p; }
  }
  cell_start[p] = n;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t r = 0; r < m; ++r) {
    float dl[ORC_MAXK];
    int64_t il[ORC_MAXK];
    for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
    int64_t gx = qgrid[3 * r] >> num_down, gy = qgrid[3 * r + 1] >> num_down,
            gz = qgrid[3 * r + 2] >> num_down;
    int64_t b = qbatch ? qbatch[r] : 0;
    for (int j = 0; j < 27; ++j) {
      int64_t key = orc_morton_key(gx + axis_offset(j / 9), gy + axis_offset((j / 3) % 3),
                                   gz + axis_offset(j % 3), b);
      int64_t c = search_sorted(cell_key, p, key);
      if (c < 0) continue;
      for (int64_t s = cell_start[c]; s < cell_start[c + 1]; ++s) {
        int64_t t = order[s];
        float d = sqdist(sxyz + 3 * t, qxyz + 3 * r, variant);
        if (!(d < cut_r2)) continue;
        topk_insert(d, t, dl, il, k);
      }
    }
    int64_t padv = pad ? pad[r] : -1;
    for (int j = 0; j < k; ++j) {
      idx_out[r * k + j] = (int32_t)((il[j] == INT64_MAX) ? padv : il[j]);
      dist_out[r * k + j] = dl[j];
    }
  }
  free(cell_start);
  free(cell_key);
  free(order);
  free(pk);
  return 0;
}

/*
 * Pointcept-style offset batching on top of orc_knn_general: offsets are
 * cumulative cloud ends, grid = floor(xyz * (1 / voxel)) in FP32, batch =
 * cloud id.  The reference's callers voxelise with torch.floor(coord /
 * voxel_size) on CUDA tensors (Query/benchmark_s3dis.py:159,
 * Networks/hierarchy.py:30): PyTorch evaluates a CUDA tensor divided by a
 * Python scalar as a product with the scalar's FP32 reciprocal, so that is
 * the rounding restated here.
 * qxyz == NULL means a self query (pad = own index); otherwise pad = -1.
 */
int orc_knn_offsets(const float* xyz, const int64_t* offsets, int64_t b,
                    const float* qxyz, const int64_t* qoffsets, float voxel,
                    int num_down, int k, float cut_r2, int variant,
                    int32_t* idx_out, float* dist_out, int nthreads) {
  int64_t n = b ? offsets[b - 1] : 0;
  const float inv = 1.0f / voxel;
  int self = qxyz == NULL;
  if (self) { qxyz = xyz; qoffsets = offsets; }
  int64_t m = b ? qoffsets[b - 1] : 0;
  int64_t* sg = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)(n ? n : 1));
  int64_t* sb = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  int64_t* qg = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)(m ? m : 1));
  int64_t* qb = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
  int64_t* pad = self ? (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1)) : NULL;
  int64_t c = 0;
  for (int64_t i = 0; i < n; ++i) {
    while (c < b && i >= offsets[c]) ++c;
    sb[i] = c;
    for (int a = 0; a < 3; ++a) sg[3 * i + a] = (int64_t)floorf(xyz[3 * i + a] * inv);
  }
  c = 0;
  for (int64_t i = 0; i < m; ++i) {
    while (c < b && i >= qoffsets[c]) ++c;
    qb[i] = c;
    for (int a = 0; a < 3; ++a) qg[3 * i + a] = (int64_t)floorf(qxyz[3 * i + a] * inv);
    if (pad) pad[i] = i;
  }
  int rc = orc_knn_general(xyz, sg, sb, n, qxyz, qg, qb, m, num_down, k, cut_r2,
                           variant, pad, idx_out, dist_out, nthreads);
  free(pad);
  free(qb);
  free(qg);
  free(sb);
  free(sg);
  return rc;
}

/* --------------------------------------------------------- brute force */

/*
 * Exact FP64 k nearest neighbours inside each cloud (offset batching), the
 * recall reference.  Ties break by the lower index.  Rows with fewer than K
 * points in their cloud are padded with (-1, +inf).
 */
int orc_brute_knn_f64(const float* xyz, const int64_t* offsets, int64_t b,
                      const float* qxyz, const int64_t* qoffsets, int k,
                      int32_t* idx_out, double* dist_out, int nthreads) {
  if (k < 1 || k > ORC_MAXK) return -1;
  if (qxyz == NULL) { qxyz = xyz; qoffsets = offsets; }
  int64_t m = b ? qoffsets[b - 1] : 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t r = 0; r < m; ++r) {
    double dl[ORC_MAXK];
    int64_t il[ORC_MAXK];
    int64_t c = 0;
    while (c < b && r >= qoffsets[c]) ++c;
    int64_t s0 = c ? offsets[c - 1] : 0, s1 = offsets[c];
    for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
    double qx = qxyz[3 * r], qy = qxyz[3 * r + 1], qz = qxyz[3 * r + 2];
    for (int64_t t = s0; t < s1; ++t) {
      double dx = (double)xyz[3 * t] - qx, dy = (double)xyz[3 * t + 1] - qy,
             dz = (double)xyz[3 * t + 2] - qz;
      double d = dx * dx + dy * dy + dz * dz;
      if (d > dl[k - 1] || (d == dl[k - 1] && t >= il[k - 1])) continue;
      int j = k - 1;
      while (j > 0 && (d < dl[j - 1] || (d == dl[j - 1] && t < il[j - 1]))) {
        dl[j] = dl[j - 1];
        il[j] = il[j - 1];
        --j;
      }
      dl[j] = d;
      il[j] = t;
    }
    for (int j = 0; j < k; ++j) {
      idx_out[r * k + j] = (int32_t)(il[j] == INT64_MAX ? -1 : il[j]);
      dist_out[r * k + j] = dl[j];
    }
  }
  return 0;
}

/* ------------------------------------------------------------ backward */

/*
 * FP64 gradient of L = sum_ij g_ij * d_ij with d_ij = |p_idx_ij - q_i|^2 and
 * the indices held fixed: grad_q[i] = sum_j 2 g_ij (q_i - p_idx_ij),
 * grad_p[n] = sum_{idx_ij = n} -2 g_ij (q_i - p_n).  Entries whose distance
 * is +inf (padding) carry no gradient.
 */
void orc_backward_f64(const float* qxyz, int64_t m, const float* pxyz,
                      int64_t n, const int32_t* idx, const float* dist,
                      const double* g, int k, double* grad_q, double* grad_p) {
  memset(grad_q, 0, sizeof(double) * 3 * (size_t)m);
  memset(grad_p, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t i = 0; i < m; ++i)
    for (int j = 0; j < k; ++j) {
      int64_t e = i * k + j;
      if (isinf(dist[e]) || idx[e] < 0) continue;
      int64_t t = idx[e];
      for (int a = 0; a < 3; ++a) {
        double diff = (double)qxyz[3 * i + a] - (double)pxyz[3 * t + a];
        grad_q[3 * i + a] += 2.0 * g[e] * diff;
        grad_p[3 * t + a] -= 2.0 * g[e] * diff;
      }
    }
}

/* ------------------------------------------------- adaptive neighbourhood */

/* Morton interleave of non-negative coordinates below 2^21. */
static uint64_t morton21(uint64_t x, uint64_t y, uint64_t z) {
  uint64_t key = 0;
  for (int bit = 0; bit < 21; ++bit) {
    key |= ((x >> bit) & 1u) << (3 * bit + 2);
    key |= ((y >> bit) & 1u) << (3 * bit + 1);
    key |= ((z >> bit) & 1u) << (3 * bit);
  }
  return key;
}

/*
 * Adaptive-neighbourhood self query
 * (FlashKNN/functions/adaptive_octree.py:211-351 and :531-575):
 *   - grid coordinates are translated per batch to their minimum
 *     (:129-147); every translated coordinate must be below 2^16;
 *   - the octree levels s = 0..S group the points by (batch, spatial key
 *     >> 3s) (:256-274), S = max_shift, or the bit length of the largest
 *     translated coordinate when max_shift < 0 (:249-252);
 *   - a node's candidate count is the number of points in the 27 nodes of
 *     its level at integer offsets (0,-1,+1)^3 (:150-205, :287-302); offsets
 *     that leave [0, 2^(16-s)) name no node;
 *   - level selection (:312-351): start at S, active = count > max_f*K; for
 *     s = S-1..0 a still-active point moves to level s when its level-s
 *     count is >= min_f*K, and stays active while that count is > max_f*K;
 *   - the query is the exact top-K over the points of the 27 nodes around
 *     the point's node at its selected level (the compatible-table kernel
 *     launch, :369-488 and :555-575), FP32 distances, d < cut_r2, padding
 *     (own index, +inf), ties by the lower original index.
 * Positions are xyz, or the translated grid coordinates when xyz is NULL
 * (:545-549).  Outputs in input order: level_out[n] (may be NULL),
 * idx_out[n*k], dist_out[n*k].
 * Returns 0; -1 bad K or n < K or n == 0; -2 batch outside [0, 32768);
 * -3 a batch spans 2^16 or more; -4 max_shift > 16.
 */
int orc_adaptive_query(const int64_t* grid, const int64_t* batch, int64_t n,
                       const float* xyz, int k, int min_f, int max_f,
                       int max_shift, float cut_r2, int variant,
                       int32_t* level_out, int64_t* idx_out, float* dist_out,
                       int nthreads) {
  if (k < 1 || k > ORC_MAXK || n <= 0 || n < k) return -1;
  enum { NB = 32768 };
  int64_t* bmin = (int64_t*)malloc(sizeof(int64_t) * 3 * NB);
  for (int64_t i = 0; i < 3 * NB; ++i) bmin[i] = INT64_MAX;
  for (int64_t i = 0; i < n; ++i) {
    if (batch[i] < 0 || batch[i] >= NB) { free(bmin); return -2; }
    for (int a = 0; a < 3; ++a)
      if (grid[3 * i + a] < bmin[3 * batch[i] + a]) bmin[3 * batch[i] + a] = grid[3 * i + a];
  }
  int64_t* norm = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)n);
  int64_t maxc = 0;
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      int64_t v = grid[3 * i + a] - bmin[3 * batch[i] + a];
      if (v >= 65536) { free(norm); free(bmin); return -3; }
      norm[3 * i + a] = v;
      if (v > maxc) maxc = v;
    }
  free(bmin);
  int auto_s = 0;
  while ((1ll << auto_s) <= maxc) ++auto_s;  /* bit length of maxc */
  int S = max_shift >= 0 ? max_shift : auto_s;
  if (S > 16) { free(norm); return -4; }
  int L = S + 1;

  int64_t* key = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  for (int64_t i = 0; i < n; ++i)
    key[i] = (int64_t)(((uint64_t)batch[i] << 48) |
                       morton21((uint64_t)norm[3 * i], (uint64_t)norm[3 * i + 1],
                                (uint64_t)norm[3 * i + 2]));
  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  orc_argsort_i64(key, n, order);

  /* per level: node of every sorted position, node keys / starts, counts */
  int64_t* node_of = (int64_t*)malloc(sizeof(int64_t) * (size_t)n * L);
  int64_t** nkey = (int64_t**)malloc(sizeof(int64_t*) * L);
  int64_t** nstart = (int64_t**)malloc(sizeof(int64_t*) * L);
  int64_t** ncand = (int64_t**)malloc(sizeof(int64_t*) * L);
  int64_t* ncount = (int64_t*)malloc(sizeof(int64_t) * L);
  const uint64_t spatial_mask = (1ull << 48) - 1;
  for (int s = 0; s < L; ++s) {
    nkey[s] = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    nstart[s] = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t p = 0;
    for (int64_t q = 0; q < n; ++q) {
      uint64_t kk = (uint64_t)key[order[q]];
      int64_t nk = (int64_t)(((kk >> 48) << 48) | ((kk & spatial_mask) >> (3 * s)));
      if (q == 0 || nk != nkey[s][p - 1]) { nkey[s][p] = nk; nstart[s][p] = q; ++p; }
      node_of[(size_t)s * n + q] = p - 1;
    }
    nstart[s][p] = n;
    ncount[s] = p;
    ncand[s] = (int64_t*)malloc(sizeof(int64_t) * (size_t)(p ? p : 1));
    const int64_t lim = 1ll << (16 - s);
    for (int64_t c = 0; c < p; ++c) {
      int64_t f = order[nstart[s][c]];
      int64_t cx = norm[3 * f] >> s, cy = norm[3 * f + 1] >> s, cz = norm[3 * f + 2] >> s;
      int64_t b = batch[f], total = 0;
      for (int j = 0; j < 27; ++j) {
        int64_t x = cx + axis_offset(j / 9), y = cy + axis_offset((j / 3) % 3),
                z = cz + axis_offset(j % 3);
        if (x < 0 || y < 0 || z < 0 || x >= lim || y >= lim || z >= lim) continue;
        int64_t nk = (int64_t)(((uint64_t)b << 48) | morton21((uint64_t)x, (uint64_t)y, (uint64_t)z));
        int64_t hit = search_sorted(nkey[s], p, nk);
        if (hit >= 0) total += nstart[s][hit + 1] - nstart[s][hit];
      }
      ncand[s][c] = total;
    }
  }

  /* level selection, sorted order */
  int* sel = (int*)malloc(sizeof(int) * (size_t)n);
  for (int64_t q = 0; q < n; ++q) {
    int level = S;
    int active = ncand[S][node_of[(size_t)S * n + q]] > (int64_t)max_f * k;
    for (int s = S - 1; s >= 0; --s) {
      int64_t child = ncand[s][node_of[(size_t)s * n + q]];
      int use = active && child >= (int64_t)min_f * k;
      if (use) level = s;
      active = use && child > (int64_t)max_f * k;
    }
    sel[q] = level;
  }

#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t q = 0; q < n; ++q) {
    float dl[ORC_MAXK];
    int64_t il[ORC_MAXK];
    for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
    const int64_t i = order[q];
    const int s = sel[q];
    const int64_t lim = 1ll << (16 - s);
    float qp[3], cp[3];
    for (int a = 0; a < 3; ++a) qp[a] = xyz ? xyz[3 * i + a] : (float)norm[3 * i + a];
    int64_t cx = norm[3 * i] >> s, cy = norm[3 * i + 1] >> s, cz = norm[3 * i + 2] >> s;
    for (int j = 0; j < 27; ++j) {
      int64_t x = cx + axis_offset(j / 9), y = cy + axis_offset((j / 3) % 3),
              z = cz + axis_offset(j % 3);
      if (x < 0 || y < 0 || z < 0 || x >= lim || y >= lim || z >= lim) continue;
      int64_t nk = (int64_t)(((uint64_t)batch[i] << 48) | morton21((uint64_t)x, (uint64_t)y, (uint64_t)z));
      int64_t hit = search_sorted(nkey[s], ncount[s], nk);
      if (hit < 0) continue;
      for (int64_t r = nstart[s][hit]; r < nstart[s][hit + 1]; ++r) {
        int64_t t = order[r];
        for (int a = 0; a < 3; ++a) cp[a] = xyz ? xyz[3 * t + a] : (float)norm[3 * t + a];
        float d = sqdist(cp, qp, variant);
        if (!(d < cut_r2)) continue;
        topk_insert(d, t, dl, il, k);
      }
    }
    for (int j = 0; j < k; ++j) {
      idx_out[i * k + j] = il[j] == INT64_MAX ? i : il[j];
      dist_out[i * k + j] = dl[j];
    }
    if (level_out) level_out[i] = s;
  }

  free(sel);
  for (int s = 0; s < L; ++s) { free(nkey[s]); free(nstart[s]); free(ncand[s]); }
  free(ncount); free(ncand); free(nstart); free(nkey); free(node_of);
  free(order); free(key); free(norm);
  return 0;
}

/* ------------------------------------------------------------ back query */

/*
 * FlashKNN_Back_Query_DL / FlashKNN_Nearest_Back_Query_DL over the tables
 * FlashKNN.back_query builds (FlashKnnWrapper.py:459-585; kernels
 * flash_knn_query_dynamic_load.cu:949-1208): xyz_h [*,3] every point in key
 * order, xyz_l [*,3] the subset in key order, steps_h / steps_l [p+1] the
 * cell ranges of both, neigh [p*27] (-1 = no cell).  For each point of cell
 * c, the k nearest subset points of the 27 cells around c.  Rows follow
 * xyz_h; indices are subset positions (rows of xyz_l); rows ascending by
 * (distance, position), padding (-1, +inf).  The reference keeps the k best
 * under strict '<' and writes them in heap order (k > 1) or keeps the first
 * nearest met (k == 1); the neighbour set is the same up to equal distances.
 */
int orc_back_query_tables(const float* xyz_h, const float* xyz_l,
                          const int32_t* steps_h, const int32_t* steps_l,
                          const int32_t* neigh, int64_t p, int k, int variant,
                          int64_t* idx_out, float* dist_out, int nthreads) {
  if (k < 1 || k > ORC_MAXK) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
  for (int64_t c = 0; c < p; ++c) {
    for (int64_t q = steps_h[c]; q < steps_h[c + 1]; ++q) {
      float dl[ORC_MAXK];
      int64_t il[ORC_MAXK];
      for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
      for (int j = 0; j < 27; ++j) {
        int32_t nb = neigh[c * 27 + j];
        if (nb < 0) continue;
        for (int64_t t = steps_l[nb]; t < steps_l[nb + 1]; ++t)
          topk_insert(sqdist(xyz_l + 3 * t, xyz_h + 3 * q, variant), t, dl, il, k);
      }
      for (int j = 0; j < k; ++j) {
        idx_out[q * k + j] = il[j] == INT64_MAX ? -1 : il[j];
        dist_out[q * k + j] = dl[j];
      }
    }
  }
  return 0;
}

/*
 * FlashKNN.back_query end to end (FlashKnnWrapper.py:459-644) from its
 * inputs: cells = trunc(xyz * (1 / size)) in FP32 (the wrapper's
 * (xyz / size).long() on CUDA tensors, where PyTorch multiplies by the FP32
 * reciprocal of the Python scalar),
 * keyed like FlashKNN_Morton_Encode (16 bits per axis, batch << 48); for
 * every point i the k nearest subset points sel[j] among the subset points
 * whose cell is one of the 27 cells around i's cell; reported index = j,
 * the position in sel (the wrapper's order_l remap).  Ties by the lower j;
 * padding (-1, +inf); empty_out[i] = 1 when i has no candidate (the wrapper
 * asserts that none has).  batch may be NULL.
 */
int orc_back_query(const float* xyz, int64_t n, const int64_t* sel, int64_t m,
                   const int64_t* batch, float size, int k, int variant,
                   int64_t* idx_out, float* dist_out, int32_t* empty_out, int nthreads) {
  if (k < 1 || k > ORC_MAXK) return -1;
  int64_t* g = (int64_t*)malloc(sizeof(int64_t) * 3 * (size_t)(n ? n : 1));
  const float inv = 1.0f / size;
  for (int64_t i = 0; i < 3 * n; ++i) g[i] = (int64_t)(xyz[i] * inv);
  int64_t* skey = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
  int64_t* sorder = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
  for (int64_t j = 0; j < m; ++j) {
    int64_t r = sel[j];
    skey[j] = orc_morton_key(g[3 * r], g[3 * r + 1], g[3 * r + 2], batch ? batch[r] : 0);
  }
  orc_argsort_i64(skey, m, sorder);
  int64_t* cell_key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
  int64_t* cell_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
  int64_t p = 0;
  for (int64_t s = 0; s < m; ++s) {
    int64_t key = skey[sorder[s]];
    if (s == 0 || key != cell_key[p - 1]) { cell_key[p] = key; cell_start[p] = s; ++p; }
  }
  cell_start[p] = m;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t i = 0; i < n; ++i) {
    float dl[ORC_MAXK];
    int64_t il[ORC_MAXK];
    for (int j = 0; j < k; ++j) { dl[j] = INFINITY; il[j] = INT64_MAX; }
    int64_t b = batch ? batch[i] : 0;
    int any = 0;
    for (int j = 0; j < 27; ++j) {
      int64_t key = orc_morton_key(g[3 * i] + axis_offset(j / 9),
                                   g[3 * i + 1] + axis_offset((j / 3) % 3),
                                   g[3 * i + 2] + axis_offset(j % 3), b);
      int64_t c = search_sorted(cell_key, p, key);
      if (c < 0) continue;
      for (int64_t s = cell_start[c]; s < cell_start[c + 1]; ++s) {
        int64_t t = sorder[s];
        any = 1;
        topk_insert(sqdist(xyz + 3 * sel[t], xyz + 3 * i, variant), t, dl, il, k);
      }
    }
    for (int j = 0; j < k; ++j) {
      idx_out[i * k + j] = il[j] == INT64_MAX ? -1 : il[j];
      dist_out[i * k + j] = dl[j];
    }
    if (empty_out) empty_out[i] = any ? 0 : 1;
  }
  free(cell_start); free(cell_key); free(sorder); free(skey); free(g);
  return 0;
}

/* -------------------------------------------------- voxel-first subsampling */

/*
 * Voxel-first subsampling (Networks/hierarchy.py:23-35, _voxel_first_cuda):
 * voxel = floor(xyz * (1 / size)) in FP32 (torch.floor(xyz / size) on CUDA
 * tensors multiplies by the FP32 reciprocal), key = the 16-bit-per-axis
 * Morton key of the voxel (xyz2key, no batch unless batch != NULL: then
 * batch << 48), one representative per key -- the first point of the key in
 * a stable sort, i.e. the lowest index -- and the representatives' indices
 * ascending.  out[n] receives them; returns their count.
 */
int64_t orc_voxel_first(const float* xyz, int64_t n, const int64_t* batch, float size,
                        int64_t* out) {
  const float inv = 1.0f / size;
  int64_t* key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  unsigned char* keep = (unsigned char*)calloc((size_t)(n ? n : 1), 1);
  for (int64_t i = 0; i < n; ++i)
    key[i] = orc_morton_key((int64_t)floorf(xyz[3 * i] * inv), (int64_t)floorf(xyz[3 * i + 1] * inv),
                            (int64_t)floorf(xyz[3 * i + 2] * inv), batch ? batch[i] : 0);
  orc_argsort_i64(key, n, order);
  for (int64_t s = 0; s < n; ++s)
    if (s == 0 || key[order[s]] != key[order[s - 1]]) keep[order[s]] = 1;
  int64_t c = 0;
  for (int64_t i = 0; i < n; ++i)
    if (keep[i]) out[c++] = i;
  free(keep); free(order); free(key);
  return c;
}
