// extern "C" entry points of libfknn.so (declared in include/fknn.h).
// Host-side checks only: argument errors return before any launch.
#include <atomic>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/fknn.h"
#include "fknn_backward.h"
#include "fknn_adaptive.h"
#include "fknn_grid.h"
#include "fknn_group.h"
#include "fknn_internal.h"
#include "fknn_tables.h"
#include "fknn_voxel.h"

namespace fknn {

static std::atomic<int> g_last_cuda_error{0};
static std::atomic<int> g_last_launches{0};

void note_cuda_error(cudaError_t e) { g_last_cuda_error.store(static_cast<int>(e)); }
void note_launches(int n) { g_last_launches.store(n); }

namespace {

struct Profiler {
  std::mutex mu;
  std::vector<cudaEvent_t> start, stop;
  std::vector<int> used;  // slot order of the recorded brackets
  int next = 0;
  long long recorded = 0;
};

Profiler& profiler() {
  static Profiler p;
  return p;
}

cudaError_t record(cudaEvent_t ev, cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &st);
  // Inside a capture an external record becomes a timing node of the graph.
  return st == cudaStreamCaptureStatusActive
             ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal)
             : cudaEventRecord(ev, s);
}

}  // namespace

int profile_start(cudaStream_t s) {
  Profiler& p = profiler();
  std::lock_guard<std::mutex> lock(p.mu);
  if (p.start.empty()) return -1;
  const int slot = p.next;
  p.next = (p.next + 1) % static_cast<int>(p.start.size());
  if (record(p.start[slot], s) != cudaSuccess) return -1;
  return slot;
}

void profile_stop(int slot, cudaStream_t s) {
  if (slot < 0) return;
  Profiler& p = profiler();
  std::lock_guard<std::mutex> lock(p.mu);
  if (slot >= static_cast<int>(p.stop.size())) return;
  if (record(p.stop[slot], s) == cudaSuccess) {
    p.used.push_back(slot);
    if (p.used.size() > p.stop.size()) p.used.erase(p.used.begin());
    ++p.recorded;
  }
}

}  // namespace fknn

using fknn::QueryShape;

namespace {

constexpr int64_t kMaxPoints = (1ll << 31) - 1;

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

inline int check_k(int32_t k) { return (k >= 1 && k <= 64) ? FKNN_OK : FKNN_ERR_K; }

inline int finish(int rc, int launches) {
  if (rc == FKNN_OK) fknn::note_launches(launches);
  return rc;
}

inline int shape_from(const fknn_config* cfg, QueryShape* out) {
  *out = fknn::resolve_shape(cfg);
  return fknn::shape_valid(*out) ? FKNN_OK : FKNN_ERR_ARG;
}

}  // namespace

extern "C" {

const char* fknn_version(void) { return "flashknn-b200 0.1 (sm_100a)"; }

const char* fknn_error_string(int code) {
  switch (code) {
    case FKNN_OK: return "ok";
    case FKNN_ERR_ARG: return "invalid argument (null pointer, negative size or misaligned buffer)";
    case FKNN_ERR_K: return "K must lie in [1, 64]";
    case FKNN_ERR_WORKSPACE: return "workspace too small";
    case FKNN_ERR_CUDA: return "CUDA launch failed";
    case FKNN_ERR_SIZE: return "too many points for 32-bit indexing";
    case FKNN_ERR_NUM_DOWN: return "num_down must lie in [0, 8]";
    case FKNN_ERR_SCRATCH_LIMIT:
      return "problem exceeds the built-in scratch of fknn_query_tables_noalloc "
             "(at most 32768 points and 32768 parent cells)";
    default: return "unknown error";
  }
}

int fknn_last_cuda_error(void) { return fknn::g_last_cuda_error.load(); }

int fknn_last_launch_count(void) { return fknn::g_last_launches.load(); }

int fknn_profile_enable(int slots) {
  if (slots < 0 || slots > 4096) return FKNN_ERR_ARG;
  fknn::Profiler& p = fknn::profiler();
  std::lock_guard<std::mutex> lock(p.mu);
  for (auto ev : p.start) cudaEventDestroy(ev);
  for (auto ev : p.stop) cudaEventDestroy(ev);
  p.start.clear();
  p.stop.clear();
  p.used.clear();
  p.next = 0;
  for (int i = 0; i < slots; ++i) {
    cudaEvent_t a, b;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e != cudaSuccess) {
      fknn::note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
    p.start.push_back(a);
    p.stop.push_back(b);
  }
  return FKNN_OK;
}

int fknn_profile_read(float* ms_out, int max) {
  if (!ms_out || max < 0) return FKNN_ERR_ARG;
  fknn::Profiler& p = fknn::profiler();
  std::lock_guard<std::mutex> lock(p.mu);
  const int have = static_cast<int>(p.used.size());
  const int count = have < max ? have : max;
  for (int i = 0; i < count; ++i) {
    const int slot = p.used[have - count + i];
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(p.stop[slot]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p.start[slot], p.stop[slot]);
    if (e != cudaSuccess) {
      fknn::note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
    ms_out[i] = ms;
  }
  return count;
}

int fknn_selftest_bounded_wait(void* workspace, size_t workspace_bytes, uint32_t limit,
                               void* stream) {
  if (!workspace || limit < 1 || limit > (1u << 20)) return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  return fknn::run_selftest_wait(workspace, workspace_bytes, limit, as_stream(stream));
}

int fknn_read_status(const void* workspace, int* status, void* stream) {
  if (!workspace || !status) return FKNN_ERR_ARG;
  cudaError_t e = cudaMemcpyAsync(status, workspace, sizeof(int), cudaMemcpyDeviceToHost,
                                  as_stream(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
  if (e != cudaSuccess) {
    fknn::note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  return FKNN_OK;
}

int fknn_read_candidate_stats(const void* workspace, int64_t* total, int64_t* groups,
                              void* stream) {
  if (!workspace || !total || !groups) return FKNN_ERR_ARG;
  fknn::Meta meta{};
  cudaError_t e = cudaMemcpyAsync(&meta, workspace, sizeof(meta), cudaMemcpyDeviceToHost,
                                  as_stream(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
  if (e != cudaSuccess) {
    fknn::note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  *total = static_cast<int64_t>(meta.cand_total);
  // self queries group by support cell (n_groups stays 0), general queries
  // by query cell
  *groups = meta.n_groups > 0 ? meta.n_groups : meta.n_cells;
  return FKNN_OK;
}

size_t fknn_workspace_bytes(int64_t n_support, int64_t n_query, int64_t n_clouds,
                            int32_t query_kind) {
  if (n_support < 0 || n_query < 0 || n_clouds < 1 || query_kind < 0 || query_kind > 2) return 0;
  return fknn::fused_workspace_bytes(n_support, n_query, n_clouds, query_kind);
}

}  // extern "C"

namespace {

// Offset-batched grid query shared by fknn_knn_offsets and fknn_ball_query.
int offsets_query(const float* xyz, int64_t n, const int64_t* offsets, int64_t n_clouds,
                  const float* new_xyz, int64_t m, const int64_t* new_offsets, int32_t k,
                  float voxel, int32_t num_down, float cut_r2, bool pad_minus_one,
                  int32_t* idx_out, float* dist_out, void* workspace, size_t workspace_bytes,
                  const fknn_config* config, void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  const bool general = new_xyz != nullptr;
  if (n < 0 || n_clouds < 1 || n_clouds > 32768 || (general && m < 0)) return FKNN_ERR_ARG;
  if (n > kMaxPoints || (general && m > kMaxPoints)) return FKNN_ERR_SIZE;
  if (num_down < 0 || num_down > 8) return FKNN_ERR_NUM_DOWN;
  if (!(voxel > 0.f)) return FKNN_ERR_ARG;
  const int64_t rows = general ? m : n;
  if (!offsets || !workspace || (n > 0 && !xyz) || (general && m > 0 && !new_offsets) ||
      (rows > 0 && (!idx_out || !dist_out)))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  fknn::FusedArgs f{};
  f.kind = general ? FKNN_QUERY_GENERAL : FKNN_QUERY_SELF;
  f.xyz = xyz;
  f.offsets = offsets;
  f.n = n;
  f.n_clouds = n_clouds;
  f.qxyz = new_xyz;
  f.qoffsets = new_offsets;
  f.m = rows;
  f.voxel = voxel;
  f.num_down = num_down;
  f.k = k;
  f.cut_r2 = cut_r2;
  f.pad_minus_one = pad_minus_one ? 1 : 0;
  f.idx_bits = 32;
  f.idx_out = idx_out;
  f.dist_out = dist_out;
  int launches = 0;
  rc = fknn::run_fused(f, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

}  // namespace

extern "C" {

int fknn_knn_offsets(const float* xyz, int64_t n, const int64_t* offsets, int64_t n_clouds,
                     const float* new_xyz, int64_t m, const int64_t* new_offsets, int32_t k,
                     float voxel, int32_t num_down, float cut_r2, int32_t* idx_out,
                     float* dist_out, void* workspace, size_t workspace_bytes,
                     const fknn_config* config, void* stream) {
  return offsets_query(xyz, n, offsets, n_clouds, new_xyz, m, new_offsets, k, voxel, num_down,
                       cut_r2, false, idx_out, dist_out, workspace, workspace_bytes, config,
                       stream);
}

int fknn_ball_query(const float* xyz, int64_t n, const int64_t* offsets, int64_t n_clouds,
                    const float* new_xyz, int64_t m, const int64_t* new_offsets, int32_t nsample,
                    float voxel, int32_t num_down, float max_radius, int32_t* idx_out,
                    float* dist_out, void* workspace, size_t workspace_bytes,
                    const fknn_config* config, void* stream) {
  if (!(max_radius > 0.f)) return FKNN_ERR_ARG;
  const float r2 = max_radius * max_radius;  // FP32, as the ball-query kernels square it
  return offsets_query(xyz, n, offsets, n_clouds, new_xyz, m, new_offsets, nsample, voxel,
                       num_down, r2, true, idx_out, dist_out, workspace, workspace_bytes, config,
                       stream);
}

int fknn_knn_grid(const float* xyz, const int64_t* grid_coord, const int64_t* batch_idx,
                  int64_t n, const int64_t* query_indices, int64_t m, int32_t k,
                  int32_t num_down, float cut_r2, int32_t idx_bits, void* idx_out,
                  float* dist_out, void* workspace, size_t workspace_bytes,
                  const fknn_config* config, void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  const bool selected = query_indices != nullptr;
  if (n < 0 || (selected && m < 0)) return FKNN_ERR_ARG;
  if (n > kMaxPoints || (selected && m > kMaxPoints)) return FKNN_ERR_SIZE;
  if (num_down < 0 || num_down > 8) return FKNN_ERR_NUM_DOWN;
  if (idx_bits != 32 && idx_bits != 64) return FKNN_ERR_ARG;
  const int64_t rows = selected ? m : n;
  if (!workspace || (n > 0 && (!xyz || !grid_coord)) || (rows > 0 && (!idx_out || !dist_out)))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  fknn::FusedArgs f{};
  f.kind = selected ? FKNN_QUERY_SELECTED : FKNN_QUERY_SELF;
  f.xyz = xyz;
  f.grid = grid_coord;
  f.batch = batch_idx;
  f.n = n;
  // Batch ids below 2^15 are valid (the reference keeps them in key bits 48-62).
  f.n_clouds = batch_idx ? 32768 : 1;
  f.query_indices = query_indices;
  f.m = rows;
  f.voxel = 1.f;
  f.num_down = num_down;
  f.k = k;
  f.cut_r2 = cut_r2;
  f.idx_bits = idx_bits;
  f.idx_out = idx_out;
  f.dist_out = dist_out;
  int launches = 0;
  rc = fknn::run_fused(f, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

int fknn_general_query_tables(const float* xyz_support, int64_t n, const float* xyz_query,
                              int64_t m, const int32_t* pad_index, const int32_t* steps,
                              const int32_t* steps_query, const int32_t* neigh,
                              const int32_t* cnt, int64_t p, int32_t k, float cut_r2,
                              int32_t* idx_out, float* dist_out, void* workspace,
                              size_t workspace_bytes, const fknn_config* config, void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  if (n < 0 || m < 0 || p < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints || m > kMaxPoints || p > kMaxPoints / 28) return FKNN_ERR_SIZE;
  if (!workspace || (n > 0 && !xyz_support) || (m > 0 && (!xyz_query || !idx_out || !dist_out)) ||
      (p > 0 && (!steps || !steps_query || !neigh || !cnt)))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  fknn::TablesArgs t{xyz_support, n, steps, neigh, cnt, p, nullptr, steps_query, m, k, cut_r2,
                     idx_out, dist_out, xyz_query, pad_index};
  int launches = 0;
  rc = fknn::run_tables(t, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

size_t fknn_tables_workspace_bytes(int64_t n, int64_t m, int64_t p) {
  if (n < 0 || m < 0 || p < 0) return 0;
  return fknn::tables_workspace_bytes(n, m, p);
}

int fknn_query_tables(const float* xyz_sorted, int64_t n, const int32_t* steps,
                      const int32_t* neigh, const int32_t* cnt, int64_t p, int32_t k,
                      float cut_r2, int32_t* idx_out, float* dist_out, void* workspace,
                      size_t workspace_bytes, const fknn_config* config, void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  if (n < 0 || p < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints || p > kMaxPoints / 28) return FKNN_ERR_SIZE;
  if (!workspace || (n > 0 && (!xyz_sorted || !idx_out || !dist_out)) ||
      (p > 0 && (!steps || !neigh || !cnt)))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  fknn::TablesArgs t{xyz_sorted, n, steps, neigh, cnt, p, nullptr, nullptr, n, k, cut_r2,
                     idx_out, dist_out};
  int launches = 0;
  rc = fknn::run_tables(t, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

int fknn_selected_query_tables(const float* xyz_sorted, int64_t n, const int32_t* qindex,
                               int64_t m, const int32_t* steps, const int32_t* steps_query,
                               const int32_t* neigh, const int32_t* cnt, int64_t p, int32_t k,
                               float cut_r2, int32_t* idx_out, float* dist_out,
                               void* workspace, size_t workspace_bytes,
                               const fknn_config* config, void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  if (n < 0 || m < 0 || p < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints || m > kMaxPoints || p > kMaxPoints / 28) return FKNN_ERR_SIZE;
  if (!workspace || (n > 0 && !xyz_sorted) || (m > 0 && (!qindex || !idx_out || !dist_out)) ||
      (p > 0 && (!steps || !steps_query || !neigh || !cnt)))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  fknn::TablesArgs t{xyz_sorted, n, steps, neigh, cnt, p, qindex, steps_query, m, k, cut_r2,
                     idx_out, dist_out};
  int launches = 0;
  rc = fknn::run_tables(t, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

int fknn_morton_encode(const int64_t* grid_coord, const int64_t* batch_idx, int64_t n,
                       int64_t* keys, void* stream) {
  if (n < 0 || (n > 0 && (!grid_coord || !keys))) return FKNN_ERR_ARG;
  return fknn::run_morton_encode(grid_coord, batch_idx, n, keys, as_stream(stream));
}

int fknn_morton_neighbor_keys(const int64_t* grid_down, const int64_t* parent_batch,
                              int64_t p, int64_t* keys, void* stream) {
  if (p < 0 || (p > 0 && (!grid_down || !keys))) return FKNN_ERR_ARG;
  if (p > INT64_MAX / 27) return FKNN_ERR_SIZE;
  return fknn::run_neighbor_keys(grid_down, parent_batch, p, keys, as_stream(stream));
}

size_t fknn_build_tables_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  return fknn::build_tables_workspace_bytes(n);
}

int fknn_build_tables(const int64_t* grid_coord, const int64_t* batch_idx, int64_t n,
                      int32_t num_down, int64_t* order, int32_t* steps, int32_t* neigh,
                      int32_t* cnt, int64_t* n_parents, void* workspace,
                      size_t workspace_bytes, void* stream) {
  if (n < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints / 28) return FKNN_ERR_SIZE;
  if (num_down < 0 || num_down > 8) return FKNN_ERR_NUM_DOWN;
  if (!workspace || !steps || !n_parents ||
      (n > 0 && (!grid_coord || !order || !neigh || !cnt)))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  fknn::BuildTablesArgs t{grid_coord, batch_idx, n, num_down, order, steps, neigh, cnt, n_parents};
  int launches = 0;
  const int rc = fknn::run_build_tables(t, workspace, workspace_bytes, as_stream(stream), &launches);
  return finish(rc, launches);
}

size_t fknn_back_query_workspace_bytes(int64_t n, int64_t m) {
  if (n < 0 || m < 0) return 0;
  return fknn::fused_workspace_bytes(m, n, 32768, FKNN_QUERY_GENERAL);
}

int fknn_back_query(const float* xyz, int64_t n, const int64_t* sel_indices, int64_t m,
                    const int64_t* batch_idx, float query_grid_size, int32_t k,
                    int32_t idx_bits, void* idx_out, float* dist_out, void* workspace,
                    size_t workspace_bytes, const fknn_config* config, void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  if (n < 0 || m < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints || m > kMaxPoints) return FKNN_ERR_SIZE;
  if (!(query_grid_size > 0.f) || (idx_bits != 32 && idx_bits != 64)) return FKNN_ERR_ARG;
  if (!workspace || (n > 0 && (!xyz || !idx_out || !dist_out)) || (m > 0 && !sel_indices))
    return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  fknn::FusedArgs f{};
  f.kind = FKNN_QUERY_GENERAL;
  f.xyz = xyz;                 // support = the rows sel_indices of xyz
  f.sindex = sel_indices;
  f.n = m;
  f.n_src = n;
  f.batch = batch_idx;
  f.n_clouds = batch_idx ? 32768 : 1;
  f.qxyz = xyz;                // queries = every point
  f.qbatch = batch_idx;
  f.m = n;
  f.voxel = query_grid_size;
  f.num_down = 0;
  f.trunc_grid = 1;            // the reference voxelises with (xyz / size).long()
  f.k = k;
  f.cut_r2 = INFINITY;
  f.idx_bits = idx_bits;
  f.idx_out = idx_out;
  f.dist_out = dist_out;
  int launches = 0;
  rc = fknn::run_fused(f, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

size_t fknn_voxel_first_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  return fknn::voxel_first_workspace_bytes(n);
}

int fknn_voxel_first(const float* xyz, int64_t n, const int64_t* batch_idx, float voxel,
                     int64_t* out, int64_t* count_out, void* workspace, size_t workspace_bytes,
                     void* stream) {
  if (n < 0 || !(voxel > 0.f)) return FKNN_ERR_ARG;
  if (n > kMaxPoints) return FKNN_ERR_SIZE;
  if (!workspace || !count_out || (n > 0 && (!xyz || !out))) return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  const fknn::VoxelArgs v{xyz, batch_idx, n, voxel, out, count_out};
  int launches = 0;
  const int rc = fknn::run_voxel_first(v, workspace, workspace_bytes, as_stream(stream), &launches);
  return finish(rc, launches);
}

size_t fknn_group_workspace_bytes(int64_t m, int32_t k, int64_t n) {
  if (m < 0 || k < 1 || n < 0) return 0;
  return fknn::group_workspace_bytes(m * k, n);
}

namespace {
int group_args_check(int64_t n, int32_t c, const int32_t* idx, int64_t m, int32_t k,
                     void* workspace) {
  if (n < 0 || m < 0 || c < 1 || k < 1) return FKNN_ERR_ARG;
  if (n > kMaxPoints || m * static_cast<int64_t>(k) > kMaxPoints) return FKNN_ERR_SIZE;
  if (!workspace || (m > 0 && !idx)) return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  return FKNN_OK;
}
}  // namespace

int fknn_group_features(const float* feat, int64_t n, int32_t c, const int32_t* idx,
                        int64_t m, int32_t k, const float* xyz, const float* new_xyz,
                        int32_t with_xyz, float* out, void* workspace, size_t workspace_bytes,
                        void* stream) {
  int rc = group_args_check(n, c, idx, m, k, workspace);
  if (rc) return rc;
  if (m > 0 && (!out || (n > 0 && !feat) || (with_xyz && (!new_xyz || (n > 0 && !xyz)))))
    return FKNN_ERR_ARG;
  fknn::GroupArgs g{};
  g.feat = feat;
  g.n = n;
  g.c = c;
  g.idx = idx;
  g.m = m;
  g.k = k;
  g.xyz = xyz;
  g.new_xyz = new_xyz;
  g.with_xyz = with_xyz ? 1 : 0;
  g.out = out;
  int launches = 0;
  rc = fknn::run_group_forward(g, workspace, workspace_bytes, as_stream(stream), &launches);
  return finish(rc, launches);
}

int fknn_group_backward(const float* grad_out, int64_t n, int32_t c, const int32_t* idx,
                        int64_t m, int32_t k, int32_t with_xyz, float* grad_feat,
                        float* grad_xyz, int32_t accumulate_xyz, float* grad_new_xyz,
                        int32_t accumulate_new_xyz, void* workspace, size_t workspace_bytes,
                        void* stream) {
  int rc = group_args_check(n, c, idx, m, k, workspace);
  if (rc) return rc;
  if (m > 0 && !grad_out) return FKNN_ERR_ARG;
  if (!with_xyz && (grad_xyz || grad_new_xyz)) return FKNN_ERR_ARG;
  if (grad_xyz && !grad_feat) return FKNN_ERR_ARG;  // both come from the segment pass
  fknn::GroupArgs g{};
  g.n = n;
  g.c = c;
  g.idx = idx;
  g.m = m;
  g.k = k;
  g.with_xyz = with_xyz ? 1 : 0;
  g.grad_out = grad_out;
  g.grad_feat = grad_feat;
  g.grad_xyz = grad_xyz;
  g.accumulate_xyz = accumulate_xyz ? 1 : 0;
  g.grad_new_xyz = grad_new_xyz;
  g.accumulate_new_xyz = accumulate_new_xyz ? 1 : 0;
  int launches = 0;
  rc = fknn::run_group_backward(g, workspace, workspace_bytes, as_stream(stream), &launches);
  return finish(rc, launches);
}

size_t fknn_adaptive_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  return fknn::adaptive_workspace_bytes(n);
}

int fknn_adaptive_query(const int64_t* grid_coord, const int64_t* batch_idx, int64_t n,
                        const float* xyz, int32_t k, int32_t min_candidates_factor,
                        int32_t max_candidates_factor, int32_t max_shift, float cut_r2,
                        int32_t idx_bits, void* idx_out, float* dist_out, int8_t* level_out,
                        void* workspace, size_t workspace_bytes, const fknn_config* config,
                        void* stream) {
  int rc = check_k(k);
  if (rc) return rc;
  if (n < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints) return FKNN_ERR_SIZE;
  if (n > 0 && n < k) return FKNN_ERR_ARG;
  if (min_candidates_factor < 1 || max_candidates_factor < min_candidates_factor ||
      static_cast<int64_t>(max_candidates_factor) * k > (1ll << 30))
    return FKNN_ERR_ARG;
  if (max_shift > 16) return FKNN_ERR_ARG;
  if (idx_bits != 32 && idx_bits != 64) return FKNN_ERR_ARG;
  if (!workspace || (n > 0 && (!grid_coord || !idx_out || !dist_out))) return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  QueryShape shape;
  if ((rc = shape_from(config, &shape))) return rc;
  const fknn::AdaptiveArgs a{grid_coord, batch_idx, xyz, n, k, min_candidates_factor,
                             max_candidates_factor, max_shift < 0 ? -1 : max_shift, cut_r2,
                             idx_bits, idx_out, dist_out, level_out};
  int launches = 0;
  rc = fknn::run_adaptive(a, workspace, workspace_bytes, shape, as_stream(stream), &launches);
  return finish(rc, launches);
}

size_t fknn_backward_workspace_bytes(int64_t m, int64_t n, int32_t k) {
  if (m < 0 || n < 0 || k < 1) return 0;
  return fknn::backward_workspace_bytes(m, n, k);
}

int fknn_backward(const float* q_xyz, int64_t m, const float* p_xyz, int64_t n,
                  const int32_t* idx, const float* dist, const float* grad_dist, int32_t k,
                  float* grad_q, float* grad_p, int32_t accumulate, void* workspace,
                  size_t workspace_bytes, void* stream) {
  if (k < 1 || m < 0 || n < 0) return FKNN_ERR_ARG;
  if (m * static_cast<int64_t>(k) > kMaxPoints || n > kMaxPoints - 1) return FKNN_ERR_SIZE;
  if (!workspace || (m > 0 && (!q_xyz || !idx || !dist || !grad_dist)) ||
      (n > 0 && grad_p && !p_xyz) || (m > 0 && !p_xyz))
    return FKNN_ERR_ARG;
  if (grad_q && grad_p && grad_q == grad_p && !accumulate) return FKNN_ERR_ARG;
  if (!aligned(workspace, 256)) return FKNN_ERR_ARG;
  fknn::BackwardArgs a{q_xyz, m, p_xyz, n, idx, dist, grad_dist, k, grad_q, grad_p, accumulate};
  int launches = 0;
  const int rc = fknn::run_backward(a, workspace, workspace_bytes, as_stream(stream), &launches);
  return finish(rc, launches);
}

}  // extern "C"
