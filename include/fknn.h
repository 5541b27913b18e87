/*
 * FlashKNN-B200: C ABI of the grid k-nearest-neighbour path on sm_100a.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*), launches asynchronously on that stream, never
 * synchronises the device, never allocates, and never throws.  Host-side
 * argument errors are returned as a negative FKNN_ERR_* code before anything
 * is launched.  Problems that only the device can see (coordinates outside
 * the Morton range, inconsistent tables, a bounded wait that gave up) are
 * OR-ed into a status word inside the caller's workspace; read it with
 * fknn_read_status().
 *
 * Index and distance conventions (same as the reference kernel):
 *   - squared FP32 distances, ascending per row, ties broken by lower index;
 *   - a row with fewer than K candidates is padded with (pad index, +inf),
 *     where the pad index is the query's own index for self / selected
 *     queries (flash_knn_query_dynamic_load.cu:562,1289) and -1 for general
 *     queries (Pointcept libs/pointops/functions/query.py:12);
 *   - K in [1, 64] (flash_knn_query_dynamic_load.cu:694-777 rejects K > 64).
 *
 * Reference paths below are relative to the FlashKNN_ExpRepo project root.
 */
#ifndef FKNN_H_
#define FKNN_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FKNN_API __attribute__((visibility("default")))
#else
#define FKNN_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------- return codes */
#define FKNN_OK 0
#define FKNN_ERR_ARG (-1)       /* null pointer, negative size, misaligned buffer */
#define FKNN_ERR_K (-2)         /* K outside [1, 64] */
#define FKNN_ERR_WORKSPACE (-3) /* workspace smaller than the *_workspace_bytes() size */
#define FKNN_ERR_CUDA (-4)      /* a launch failed: see fknn_last_cuda_error() */
#define FKNN_ERR_SIZE (-5)      /* more points than 32-bit indexing allows */
#define FKNN_ERR_NUM_DOWN (-6)  /* num_down outside [0, 8] */
#define FKNN_ERR_SCRATCH_LIMIT (-7) /* larger than the built-in scratch of fknn_query_tables_noalloc */

/* --------------------------------------------------- device status bits */
#define FKNN_DEVICE_COORD_RANGE 1 /* grid coordinate outside [-2^15, 2^15) */
#define FKNN_DEVICE_BAD_TABLE 2   /* a table names rows outside the point array */
#define FKNN_DEVICE_TIMEOUT 4     /* a bounded wait on a bulk copy gave up */
#define FKNN_DEVICE_BATCH_RANGE 8 /* batch id outside [0, 2^15) */
#define FKNN_DEVICE_NO_CANDIDATES 16 /* informational: a query saw no candidate
                                        (general / back queries pad it with -1) */
#define FKNN_DEVICE_COPY_IN_FLIGHT 32 /* after FKNN_DEVICE_TIMEOUT, a second bounded
                                         wait also gave up: a warp stopped while bulk
                                         copies into its CTA's shared memory may still
                                         have been in flight */

/* Optional launch shape of the query kernel; NULL selects the defaults.
 * warps_per_cta in {1,2,4,8}; tile_records (candidate records staged per
 * warp) a multiple of 32 in [64, 1024] whose shared memory fits a CTA;
 * min_candidates_per_lane >= 1 caps how many lanes share one query;
 * ctas_per_sm 0 = occupancy maximum; staging_depth 1 (stage a work item's
 * candidates, then scan them) or 2 (two tiles per warp: the next item's
 * bulk copies are in flight while the current one is scanned).  Zero
 * fields take the defaults.  flashknn_exprepo_b200/autotune.py picks these
 * per K and point density by timing them. */
typedef struct fknn_config {
  int32_t warps_per_cta;
  int32_t tile_records;
  int32_t min_candidates_per_lane;
  int32_t ctas_per_sm;
  int32_t staging_depth;
} fknn_config;

/* ----------------------------------------------------------- utilities */
FKNN_API const char* fknn_version(void);
FKNN_API const char* fknn_error_string(int code);
/* cudaError_t value of the last launch failure seen by this library. */
FKNN_API int fknn_last_cuda_error(void);
/* Copies the workspace's device status word to *status (synchronises
 * `stream`).  0 means no device-side problem was seen. */
FKNN_API int fknn_read_status(const void* workspace, int* status, void* stream);
/* Candidate statistics of the last fused self or general query that used
 * `workspace` (fknn_knn_grid / fknn_knn_offsets / fknn_ball_query):
 * *total = the sum over query groups (parent cells) of the number of points
 * in their 27-cell neighbourhoods, *groups = the number of groups.  The
 * reference's FlashKNN.query reports total / groups as traverse_info[0]
 * (FlashKNN/functions/FlashKnnWrapper.py:351-352).  Synchronises `stream`. */
FKNN_API int fknn_read_candidate_stats(const void* workspace, int64_t* total, int64_t* groups,
                                       void* stream);
/* Number of kernels the last successful fused call launched. */
FKNN_API int fknn_last_launch_count(void);
/* Kernel timing for benchmarks (no reference counterpart).  With slots > 0
 * every query-kernel launch is bracketed by a pair of CUDA events on its
 * stream, taken round-robin from `slots` pairs (inside a CUDA graph capture
 * the pair becomes event-record nodes of the graph); slots == 0 disables it.
 * fknn_profile_read waits for the most recent min(max, recorded) pairs and
 * writes their durations in milliseconds, newest last; returns the count. */
FKNN_API int fknn_profile_enable(int slots);
FKNN_API int fknn_profile_read(float* ms_out, int max);

/* No reference counterpart.  Failure-path self-test: launches one CTA that
 * waits, with the query kernel's bounded wait, on a shared-memory barrier
 * that nothing completes, and gives up after `limit` polls (1..2^20),
 * setting FKNN_DEVICE_TIMEOUT in the workspace's status word (read it with
 * fknn_read_status).  Nothing faults and nothing is left in flight; the
 * call lets a test check that a stalled wait ends and is reported. */
FKNN_API int fknn_selftest_bounded_wait(void* workspace, size_t workspace_bytes, uint32_t limit,
                               void* stream);

/* --------------------------------------------- fused queries (a1..a9)
 * Grid construction + candidate gather + top-K + remap in one stream of
 * launches.  Output rows follow the caller's query order; indices are in
 * the caller's point numbering.
 */
#define FKNN_QUERY_SELF 0     /* queries = support points, pad = own index */
#define FKNN_QUERY_SELECTED 1 /* queries = a subset of the support points */
#define FKNN_QUERY_GENERAL 2  /* queries = separate points, pad = -1 */

FKNN_API size_t fknn_workspace_bytes(int64_t n_support, int64_t n_query, int64_t n_clouds,
                            int32_t query_kind);

/* Pointcept-style offset batching (Pointcept libs/pointops/functions/query.py
 * :7-24 knn_query(nsample, xyz, offset, new_xyz, new_offset)): offsets are
 * cumulative cloud ends, grid = floor(xyz / voxel) (FP32 division), parent
 * cell = grid >> num_down.  new_xyz == NULL selects the self query (m and
 * new_offsets ignored).  idx_out int32 [m, k], dist_out f32 [m, k]. */
FKNN_API int fknn_knn_offsets(const float* xyz, int64_t n, const int64_t* offsets, int64_t n_clouds,
                     const float* new_xyz, int64_t m, const int64_t* new_offsets, int32_t k,
                     float voxel, int32_t num_down, float cut_r2, int32_t* idx_out,
                     float* dist_out, void* workspace, size_t workspace_bytes,
                     const fknn_config* config, void* stream);

/* Radius-limited grid query, the cut-radius variant of the reference query
 * (FlashKnnWrapper.py:172,370: a candidate counts only when d < cut_r^2)
 * with the calling convention of Pointcept's ball query
 * (Pointcept/libs/pointops/functions/query.py:73-108): the nsample nearest
 * points with squared distance < max_radius^2 among the 27 parent cells,
 * ascending; rows with fewer are padded with (-1, +inf), also for the self
 * query.  When voxel * 2^num_down >= max_radius the 27 cells hold the whole
 * ball and the rows are exact.  (Pointcept's brute-force kernel returns a
 * strided subset when the ball holds more than nsample points; this returns
 * the nearest ones.)  Arguments as fknn_knn_offsets; workspace from
 * fknn_workspace_bytes with the same kind. */
FKNN_API int fknn_ball_query(const float* xyz, int64_t n, const int64_t* offsets, int64_t n_clouds,
                    const float* new_xyz, int64_t m, const int64_t* new_offsets, int32_t nsample,
                    float voxel, int32_t num_down, float max_radius, int32_t* idx_out,
                    float* dist_out, void* workspace, size_t workspace_bytes,
                    const fknn_config* config, void* stream);

/* FlashKNN.query (FlashKNN/functions/FlashKnnWrapper.py:165-449) when
 * query_indices == NULL, FlashKNN.selected_query (:646-849) otherwise.
 * grid_coord int64 [n,3], batch_idx int64 [n] (NULL = one cloud), xyz f32
 * [n,3].  idx_bits 64 writes int64 indices (the reference's return type),
 * 32 writes int32.  idx_out [m,k] with m = n for the self query. */
FKNN_API int fknn_knn_grid(const float* xyz, const int64_t* grid_coord, const int64_t* batch_idx,
                  int64_t n, const int64_t* query_indices, int64_t m, int32_t k,
                  int32_t num_down, float cut_r2, int32_t idx_bits, void* idx_out,
                  float* dist_out, void* workspace, size_t workspace_bytes,
                  const fknn_config* config, void* stream);

/* FlashKNN.back_query (FlashKNN/functions/FlashKnnWrapper.py:459-644, kernels
 * FlashKNN_Nearest_Back_Query_DL / FlashKNN_Back_Query_DL,
 * flash_knn_query_dynamic_load.cu:949-1208): for every point of xyz [n,3]
 * the k nearest points of the subset sel_indices [m] (rows of xyz) among the
 * subset points in the 27 cells around the point's cell, cells =
 * trunc(xyz / query_grid_size) per batch (batch_idx int64 [n] or NULL).
 * idx_out [n,k] (idx_bits 64: int64, 32: int32) holds positions in
 * sel_indices (0..m-1), ascending by (distance, position); dist_out f32
 * [n,k].  A point with no subset point around it gets (-1, +inf) and sets
 * FKNN_DEVICE_NO_CANDIDATES (the reference asserts that this never
 * happens). */
FKNN_API size_t fknn_back_query_workspace_bytes(int64_t n, int64_t m);
FKNN_API int fknn_back_query(const float* xyz, int64_t n, const int64_t* sel_indices, int64_t m,
                    const int64_t* batch_idx, float query_grid_size, int32_t k,
                    int32_t idx_bits, void* idx_out, float* dist_out, void* workspace,
                    size_t workspace_bytes, const fknn_config* config, void* stream);

/* Voxel-first subsampling, _voxel_first_cuda (Networks/hierarchy.py:23-35):
 * one representative per occupied voxel -- voxel = floor(xyz * (1/voxel))
 * in FP32 (PyTorch's evaluation of torch.floor(xyz / voxel) on CUDA), keyed
 * by its 16-bit-per-axis Morton key (batch << 48 when batch_idx is given,
 * ids in [0, 32768)) -- the lowest index of each voxel.  out [n] int64
 * receives the representatives in ascending order, *count_out (int64, device
 * memory) their number. */
FKNN_API size_t fknn_voxel_first_workspace_bytes(int64_t n);
FKNN_API int fknn_voxel_first(const float* xyz, int64_t n, const int64_t* batch_idx, float voxel,
                     int64_t* out, int64_t* count_out, void* workspace, size_t workspace_bytes,
                     void* stream);

/* Neighbour feature grouping, Pointcept's pointops.grouping
 * (Pointcept/libs/pointops/functions/grouping.py:36-60) as used by
 * knn_query_and_group (.../functions/utils.py:5-18): out [m,k,c'] with
 * out[i,j] = [xyz[t] - new_xyz[i] | feat[t]] for t = idx[i,j] (the xyz part,
 * 3 channels, only when with_xyz != 0; c' = c or c + 3); an index below 0 is
 * padding and gives a zero row.  feat f32 [n,c], idx int32 [m,k], xyz f32
 * [n,3] and new_xyz f32 [m,3] (with_xyz only).  Requires m*k < 2^31. */
FKNN_API size_t fknn_group_workspace_bytes(int64_t m, int32_t k, int64_t n);
FKNN_API int fknn_group_features(const float* feat, int64_t n, int32_t c, const int32_t* idx,
                        int64_t m, int32_t k, const float* xyz, const float* new_xyz,
                        int32_t with_xyz, float* out, void* workspace, size_t workspace_bytes,
                        void* stream);
/* Gradients of fknn_group_features for grad_out f32 [m,k,c']: grad_feat
 * [n,c] (overwritten), grad_xyz [n,3] (with_xyz; added to when
 * accumulate_xyz != 0) and grad_new_xyz [m,3] (with_xyz; added to when
 * accumulate_new_xyz != 0; written after grad_xyz, so one buffer may serve
 * both for a self query).  Every point's sum runs over its entries in
 * ascending i*k+j order: the result is bitwise reproducible (the reference
 * op accumulates with atomics).  Any output may be NULL. */
FKNN_API int fknn_group_backward(const float* grad_out, int64_t n, int32_t c, const int32_t* idx,
                        int64_t m, int32_t k, int32_t with_xyz, float* grad_feat,
                        float* grad_xyz, int32_t accumulate_xyz, float* grad_new_xyz,
                        int32_t accumulate_new_xyz, void* workspace, size_t workspace_bytes,
                        void* stream);

/* AdaptiveNeighborhoodFlashKNN.query (FlashKNN/functions/adaptive_octree.py
 * :505-612): every point takes its exact top-K over the 27 same-level nodes
 * of the octree level picked by coarse-to-fine candidate counting (descend
 * while the count exceeds max_candidates_factor*K, provided the finer count
 * is at least min_candidates_factor*K).  grid_coord int64 [n,3], batch_idx
 * int64 [n] in [0, 32768) (NULL = one batch), xyz f32 [n,3] or NULL (then
 * the positions are the grid coordinates translated to each batch's
 * minimum, as in the reference).  max_shift < 0 builds levels up to the bit
 * length of the largest translated coordinate; otherwise 0..max_shift (<=
 * 16).  Requires n >= k.  idx_out [n,k] (idx_bits 64: int64, 32: int32) in
 * input index space, dist_out f32 [n,k], padding (own index, +inf);
 * level_out int8 [n] (NULL = not wanted) receives the selected level.
 * Device status: FKNN_DEVICE_BATCH_RANGE for a batch id outside the range,
 * FKNN_DEVICE_COORD_RANGE for a batch spanning 2^16 grid cells or more. */
FKNN_API size_t fknn_adaptive_workspace_bytes(int64_t n);
FKNN_API int fknn_adaptive_query(const int64_t* grid_coord, const int64_t* batch_idx, int64_t n,
                        const float* xyz, int32_t k, int32_t min_candidates_factor,
                        int32_t max_candidates_factor, int32_t max_shift, float cut_r2,
                        int32_t idx_bits, void* idx_out, float* dist_out, int8_t* level_out,
                        void* workspace, size_t workspace_bytes, const fknn_config* config,
                        void* stream);

/* ------------------------------------------ reference table ABI (a8, a10)
 * Replaces FlashKNN_Query_Dynamic_Load (FlashKNN/csrc/flash_knn_query.h:144-154):
 * xyz_sorted f32 [n,3], steps int32 [p+1], neigh int32 [p,27] (-1 = empty),
 * cnt int32 [p,28]; idx_out int32 [n,k] in sorted-point space, dist_out f32
 * [n,k].  batch_for_prune is not an argument: the reference accepts and
 * ignores it (flash_knn_query_dynamic_load.cu:622-624). */
FKNN_API size_t fknn_tables_workspace_bytes(int64_t n, int64_t m, int64_t p);
FKNN_API int fknn_query_tables(const float* xyz_sorted, int64_t n, const int32_t* steps,
                      const int32_t* neigh, const int32_t* cnt, int64_t p, int32_t k,
                      float cut_r2, int32_t* idx_out, float* dist_out, void* workspace,
                      size_t workspace_bytes, const fknn_config* config, void* stream);

/* No counterpart in the reference.  Same inputs, outputs and results as
 * fknn_query_tables, for callers that cannot give the library device memory
 * (a plugin whose host framework owns all device allocations, a real-time
 * loop that must not allocate after start-up, a binding that only forwards
 * tensors): the scratch is a fixed array inside the library (about 10 MiB on
 * every GPU that loads it, kept until exit), so n and p are limited to 32768
 * each; larger problems return FKNN_ERR_SCRATCH_LIMIT.  All calls on a device
 * share that array: calls that overlap on the GPU race, so order them on one
 * stream.  The first call on a device looks up the array's address with that
 * device current; make it before any stream capture.  The address is kept
 * until exit: calls after a device reset are not supported.  Device-side
 * problems are reported by fknn_query_tables_noalloc_read_status. */
FKNN_API int fknn_query_tables_noalloc(const float* xyz_sorted, int64_t n, const int32_t* steps,
                                       const int32_t* neigh, const int32_t* cnt, int64_t p,
                                       int32_t k, float cut_r2, int32_t* idx_out,
                                       float* dist_out, void* stream);
/* No counterpart in the reference.  The device status word of the last
 * fknn_query_tables_noalloc call on the current device (the FKNN_DEVICE_*
 * bits that fknn_read_status reports for a workspace; each call clears it
 * first), copied to *status after `stream` is synchronised.  Order it after
 * that call on the same stream.  Allocates nothing. */
FKNN_API int fknn_query_tables_noalloc_read_status(int* status, void* stream);

/* Replaces FlashKNN_Selected_Query_DL (FlashKNN/csrc/flash_knn_query.h:206-218):
 * qindex int32 [m] (sorted support index of each query, grouped by parent
 * through steps_query int32 [p+1]); idx_out int32 [m,k], dist_out f32 [m,k]. */
FKNN_API int fknn_selected_query_tables(const float* xyz_sorted, int64_t n, const int32_t* qindex,
                               int64_t m, const int32_t* steps, const int32_t* steps_query,
                               const int32_t* neigh, const int32_t* cnt, int64_t p, int32_t k,
                               float cut_r2, int32_t* idx_out, float* dist_out,
                               void* workspace, size_t workspace_bytes,
                               const fknn_config* config, void* stream);

/* Queries that are separate points over caller tables.  Replaces
 * FlashKNN_Query_GM (FlashKNN/csrc/flash_knn_query.h:220-233) and the
 * back-query table kernels FlashKNN_Nearest_Back_Query_DL /
 * FlashKNN_Back_Query_DL (flash_knn_query.h:183-204): xyz_query f32 [m,3]
 * grouped by parent through steps_query int32 [p+1]; candidates are the
 * points of xyz_support f32 [n,3] in the 27 runs of the query's parent
 * (steps int32 [p+1] support starts, neigh int32 [p,27], cnt int32 [p,28]
 * over the support counts).  idx_out int32 [m,k] (rows of xyz_support) and
 * dist_out f32 [m,k], ascending by (distance, index); a row with fewer than k
 * candidates is padded with (pad_index[r], +inf), or (-1, +inf) when
 * pad_index is NULL.  (The reference's back-query kernels leave K > 1 rows in
 * heap order and its nearest kernel pads with (0, -1).)  Workspace:
 * fknn_tables_workspace_bytes(n, m, p). */
FKNN_API int fknn_general_query_tables(const float* xyz_support, int64_t n,
                                       const float* xyz_query, int64_t m,
                                       const int32_t* pad_index, const int32_t* steps,
                                       const int32_t* steps_query, const int32_t* neigh,
                                       const int32_t* cnt, int64_t p, int32_t k, float cut_r2,
                                       int32_t* idx_out, float* dist_out, void* workspace,
                                       size_t workspace_bytes, const fknn_config* config,
                                       void* stream);

/* ------------------------------------------------- construction (a1..a6)
 * Replaces FlashKNN_Morton_Encode (FlashKNN/csrc/flash_knn_construction.h:7-9,
 * kernel flash_knn_construction.cu:29-40): keys int64 [n]; batch NULL = 0. */
FKNN_API int fknn_morton_encode(const int64_t* grid_coord, const int64_t* batch_idx, int64_t n,
                       int64_t* keys, void* stream);

/* Replaces FlashKNN_Morton_Neighbor_Keys (flash_knn_construction.h:11-13,
 * kernel flash_knn_construction.cu:46-63): keys int64 [p*27], centre first. */
FKNN_API int fknn_morton_neighbor_keys(const int64_t* grid_down, const int64_t* parent_batch,
                              int64_t p, int64_t* keys, void* stream);

/* The reference's table construction (FlashKnnWrapper.py:220-337) on the
 * device: order int64 [n] (stable sort by morton key), steps int32 [n+1],
 * neigh int32 [n*27], cnt int32 [n*28] (sized for the worst case p = n),
 * n_parents int64 [1] receives p.  Nothing is read back to the host. */
FKNN_API size_t fknn_build_tables_workspace_bytes(int64_t n);
FKNN_API int fknn_build_tables(const int64_t* grid_coord, const int64_t* batch_idx, int64_t n,
                      int32_t num_down, int64_t* order, int32_t* steps, int32_t* neigh,
                      int32_t* cnt, int64_t* n_parents, void* workspace,
                      size_t workspace_bytes, void* stream);

/* ----------------------------------------------------------- backward
 * No reference counterpart (the reference query is @torch.no_grad,
 * FlashKnnWrapper.py:165).  For d_ij = |p[idx_ij] - q_i|^2:
 *   grad_q[i] (+)= sum_j 2 g_ij (q_i - p[idx_ij])
 *   grad_p[n] (+)= sum_{idx_ij = n} -2 g_ij (q_i - p_n)
 * summed in a fixed order (grad_p: a counting sort of the entries by
 * neighbour index, each segment summed in ascending entry order i*K+j), so
 * results are bitwise reproducible.  Requires m*k < 2^31.
 * Entries with dist == +inf or idx < 0 (padding) carry no gradient.
 * accumulate != 0 adds into grad_q / grad_p instead of overwriting them
 * (grad_q may alias grad_p for a self query only with accumulate != 0). */
FKNN_API size_t fknn_backward_workspace_bytes(int64_t m, int64_t n, int32_t k);
FKNN_API int fknn_backward(const float* q_xyz, int64_t m, const float* p_xyz, int64_t n,
                  const int32_t* idx, const float* dist, const float* grad_dist, int32_t k,
                  float* grad_q, float* grad_p, int32_t accumulate, void* workspace,
                  size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FKNN_H_ */
