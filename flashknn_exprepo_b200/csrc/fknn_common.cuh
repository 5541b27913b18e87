// Shared device helpers for the FlashKNN-B200 kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/fknn.h"

namespace fknn {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kNeighbours = 27;
constexpr int kMaxK = 64;
// Device-side status bits, OR-ed into the status word of a workspace.
constexpr int kStatusRange = FKNN_DEVICE_COORD_RANGE;
constexpr int kStatusTable = FKNN_DEVICE_BAD_TABLE;
constexpr int kStatusTimeout = FKNN_DEVICE_TIMEOUT;
constexpr int kStatusBatch = FKNN_DEVICE_BATCH_RANGE;
constexpr int kStatusNoCandidates = FKNN_DEVICE_NO_CANDIDATES;
constexpr int kStatusCopyInFlight = FKNN_DEVICE_COPY_IN_FLIGHT;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

__device__ __forceinline__ void raise_status(int* status, int bit) {
  if (status) atomicOr(status, bit);
}

// ------------------------------------------- programmatic dependent launch
// A kernel launched with launch_chained() may be scheduled while the kernel
// before it in the stream is still finishing (its launch overlaps that
// kernel's tail); it calls chain_wait() before it touches global memory,
// which returns once the previous kernel has completed and its writes are
// visible.  Launched the ordinary way, chain_wait() returns at once.
__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                  cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// ------------------------------------------------------------ morton codes
// Interleave the low 16 bits of x, y, z: x bit b -> 3b+2, y -> 3b+1, z -> 3b.
// Same bit layout as the reference's morton_key
// (FlashKNN/csrc/flash_knn_construction.cu:13-27).
__device__ __forceinline__ uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0xffffu;
  x = (x | (x << 16)) & 0x0000ff0000ffULL;
  x = (x | (x << 8)) & 0x00f00f00f00fULL;
  x = (x | (x << 4)) & 0x0c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x249249249249ULL;
  return x;
}

__device__ __forceinline__ uint32_t compact3(uint64_t x) {
  x &= 0x249249249249ULL;
  x = (x | (x >> 2)) & 0x0c30c30c30c3ULL;
  x = (x | (x >> 4)) & 0x00f00f00f00fULL;
  x = (x | (x >> 8)) & 0x0000ff0000ffULL;
  x = (x | (x >> 16)) & 0xffffULL;
  return static_cast<uint32_t>(x);
}

__device__ __forceinline__ uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
}

// ------------------------------------------------------ squared distance
// dx = candidate - query; FP32 evaluation order fma(dz,dz, fma(dx,dx, dy*dy)).
__device__ __forceinline__ float sq_dist(float cx, float cy, float cz,
                                         float qx, float qy, float qz) {
  const float dx = __fsub_rn(cx, qx);
  const float dy = __fsub_rn(cy, qy);
  const float dz = __fsub_rn(cz, qz);
  return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// ------------------------------------------------ mbarrier + bulk copies
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// One non-blocking probe of the barrier phase; true once `parity` completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait: returns false (and leaves the barrier as is) after `limit`
// probes.  Each try_wait may itself suspend the thread for a short while.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Non-multicast 1-D bulk copy global -> shared memory of the executing CTA
// (a CTA-local shared address is a valid shared::cluster address), completing
// on `bar`.
// dst, src 16-byte aligned; bytes a non-zero multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ------------------------------------------------------ warp primitives
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int warp_inclusive_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    int t = __shfl_up_sync(kFull, v, s);
    if (lane >= s) v += t;
  }
  return v;
}

}  // namespace fknn
