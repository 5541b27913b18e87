// Backward of the squared distances returned by the kNN query.
//
// For d_ij = |p[idx_ij] - q_i|^2 and an upstream gradient g_ij:
//   grad_q[i] = sum_j 2 g_ij (q_i - p[idx_ij])          (one thread per query,
//                                                        j in ascending order)
//   grad_p[n] = sum_{idx_ij = n} -2 g_ij (q_i - p_n)     (segmented reduction)
// The reference-side sum runs over the (i, j) entries grouped by neighbour
// index with a stable radix sort of (idx, i*K+j); each segment is summed in
// ascending i*K+j order, so the result does not depend on scheduling and is
// bitwise reproducible.  No floating-point atomics are used.
#include "fknn_common.cuh"
#include "fknn_internal.h"
#include "fknn_sort.cuh"
#include "fknn_backward.h"

namespace fknn {

// One thread per query: grad_q, and the (neighbour index, entry) pairs.
// Padding entries (dist == +inf or idx outside [0, n)) get the key n, which
// sorts after every real index and is never summed.
__global__ void __launch_bounds__(256)
    k_bwd_query(const float* __restrict__ q_xyz, int64_t m, const float* __restrict__ p_xyz,
                int64_t n, const int32_t* __restrict__ idx, const float* __restrict__ dist,
                const float* __restrict__ grad, int k, float* __restrict__ grad_q, int accumulate,
                uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const float qx = q_xyz[3 * i], qy = q_xyz[3 * i + 1], qz = q_xyz[3 * i + 2];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  for (int j = 0; j < k; ++j) {
    const int64_t e = i * k + j;
    const int32_t t = idx[e];
    const bool valid = t >= 0 && t < n && !isinf(dist[e]);
    if (keys) {
      keys[e] = valid ? static_cast<uint32_t>(t) : static_cast<uint32_t>(n);
      vals[e] = static_cast<uint32_t>(e);
    }
    if (!valid) continue;
    const float g2 = 2.f * grad[e];
    gx = __fmaf_rn(g2, __fsub_rn(qx, p_xyz[3 * static_cast<int64_t>(t)]), gx);
    gy = __fmaf_rn(g2, __fsub_rn(qy, p_xyz[3 * static_cast<int64_t>(t) + 1]), gy);
    gz = __fmaf_rn(g2, __fsub_rn(qz, p_xyz[3 * static_cast<int64_t>(t) + 2]), gz);
  }
  if (grad_q) {
    if (accumulate) {
      gx = __fadd_rn(grad_q[3 * i], gx);
      gy = __fadd_rn(grad_q[3 * i + 1], gy);
      gz = __fadd_rn(grad_q[3 * i + 2], gz);
    }
    grad_q[3 * i] = gx;
    grad_q[3 * i + 1] = gy;
    grad_q[3 * i + 2] = gz;
  }
}

// Segment bounds in the sorted pairs: first[key] / last[key] (exclusive);
// both arrays are zeroed beforehand, so indices without entries stay empty.
__global__ void k_bwd_bounds(int64_t total, SortPair<uint32_t> sp, const int* bits_ptr,
                             uint32_t n, uint32_t* __restrict__ first, uint32_t* __restrict__ last) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const uint32_t* keys = sp.keys[sort_passes_for_bits(*bits_ptr) & 1];
  const uint32_t key = keys[t];
  if (key >= n) return;
  if (t == 0 || keys[t - 1] != key) first[key] = static_cast<uint32_t>(t);
  if (t == total - 1 || keys[t + 1] != key) last[key] = static_cast<uint32_t>(t + 1);
}

// One thread per support point: ordered sum over its segment.
__global__ void __launch_bounds__(256)
    k_bwd_support(const float* __restrict__ q_xyz, const float* __restrict__ p_xyz, int64_t n,
                  const float* __restrict__ grad, int k, SortPair<uint32_t> sp,
                  const int* bits_ptr, const uint32_t* __restrict__ first,
                  const uint32_t* __restrict__ last, float* __restrict__ grad_p, int accumulate) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t* vals = sp.vals[sort_passes_for_bits(*bits_ptr) & 1];
  const float px = p_xyz[3 * p], py = p_xyz[3 * p + 1], pz = p_xyz[3 * p + 2];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  for (uint32_t t = first[p]; t < last[p]; ++t) {
    const uint32_t e = vals[t];
    const int64_t i = e / static_cast<uint32_t>(k);
    const float g2 = -2.f * grad[e];
    gx = __fmaf_rn(g2, __fsub_rn(q_xyz[3 * i], px), gx);
    gy = __fmaf_rn(g2, __fsub_rn(q_xyz[3 * i + 1], py), gy);
    gz = __fmaf_rn(g2, __fsub_rn(q_xyz[3 * i + 2], pz), gz);
  }
  if (accumulate) {
    gx = __fadd_rn(grad_p[3 * p], gx);
    gy = __fadd_rn(grad_p[3 * p + 1], gy);
    gz = __fadd_rn(grad_p[3 * p + 2], gz);
  }
  grad_p[3 * p] = gx;
  grad_p[3 * p + 1] = gy;
  grad_p[3 * p + 2] = gz;
}

__global__ void k_bwd_bits(Meta* meta, int bits) { meta->key_bits = bits; }

namespace {

inline int blocks_for(int64_t n, int per_block) {
  return static_cast<int>(ceil_div(n > 0 ? n : 1, per_block));
}

struct BwdBufs {
  Meta* meta;
  uint32_t* keys[2];
  uint32_t* vals[2];
  uint32_t* hist;
  uint32_t* totals;
  uint32_t* first;
  uint32_t* last;
};

BwdBufs bwd_layout(void* ws, int64_t m, int64_t n, int k, size_t* bytes) {
  Arena a(ws);
  BwdBufs b{};
  const int64_t total = m * k;
  b.meta = a.take<Meta>(1);
  b.keys[0] = a.take<uint32_t>(total);
  b.keys[1] = a.take<uint32_t>(total);
  b.vals[0] = a.take<uint32_t>(total);
  b.vals[1] = a.take<uint32_t>(total);
  b.hist = a.take<uint32_t>(sort_hist_elems(total));
  b.totals = a.take<uint32_t>(kSortMaxPasses * 256);
  b.first = a.take<uint32_t>(n);
  b.last = a.take<uint32_t>(n);
  if (bytes) *bytes = a.used + 256;
  return b;
}

int bits_for(int64_t count) {
  int b = 0;
  while ((1ll << b) < count) ++b;
  return b;
}

}  // namespace

size_t backward_workspace_bytes(int64_t m, int64_t n, int k) {
  size_t bytes = 0;
  bwd_layout(nullptr, m, n, k, &bytes);
  return bytes;
}

int run_backward(const BackwardArgs& a, void* ws, size_t ws_bytes, cudaStream_t s,
                 int* launches) {
  size_t need = 0;
  BwdBufs b = bwd_layout(ws, a.m, a.n, a.k, &need);
  if (ws_bytes < need) return FKNN_ERR_WORKSPACE;
  const int64_t total = a.m * a.k;
  const bool want_p = a.grad_p != nullptr && a.n > 0;
  cudaError_t e = cudaMemsetAsync(b.meta, 0, sizeof(Meta), s);
  if (e == cudaSuccess && want_p) {
    e = cudaMemsetAsync(b.totals, 0, kSortMaxPasses * 256 * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.first, 0, sizeof(uint32_t) * a.n, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.last, 0, sizeof(uint32_t) * a.n, s);
  }
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  int nl = 0;
  if (a.m > 0) {
    k_bwd_query<<<blocks_for(a.m, 256), 256, 0, s>>>(
        a.q_xyz, a.m, a.p_xyz, a.n, a.idx, a.dist, a.grad, a.k, a.grad_q, a.accumulate,
        want_p ? b.keys[0] : nullptr, want_p ? b.vals[0] : nullptr);
    ++nl;
  }
  if (want_p) {
    const int bits = bits_for(a.n + 1);
    if (total > 0) {
      k_bwd_bits<<<1, 1, 0, s>>>(b.meta, bits);
      SortBuffers<uint32_t> sb{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}, b.hist, b.totals};
      nl += 1 + launch_radix_sort(sb, total, &b.meta->key_bits, sort_passes_for_bits(bits), s);
      const SortPair<uint32_t> sp{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}};
      k_bwd_bounds<<<blocks_for(total, 256), 256, 0, s>>>(total, sp, &b.meta->key_bits,
                                                         static_cast<uint32_t>(a.n), b.first,
                                                         b.last);
      ++nl;
    }
    const SortPair<uint32_t> sp{{b.keys[0], b.keys[1]}, {b.vals[0], b.vals[1]}};
    k_bwd_support<<<blocks_for(a.n, 256), 256, 0, s>>>(a.q_xyz, a.p_xyz, a.n, a.grad, a.k, sp,
                                                       &b.meta->key_bits, b.first, b.last,
                                                       a.grad_p, a.accumulate);
    ++nl;
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
