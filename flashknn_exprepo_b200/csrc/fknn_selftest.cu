// Self-test of the bounded-wait failure path.
//
// The query kernel stages candidates with bulk copies that complete on an
// mbarrier, and every wait on that barrier gives up after a bounded number
// of polls, records kStatusTimeout in the workspace's status word and
// returns (fknn_query.cu).  A test cannot make a real copy stall, so this
// kernel builds the stalled state directly: one thread arms a barrier for 16
// bytes that no copy will ever deliver and waits with the same bounded helper.
// No copy is in flight when it gives up, so the CTA can exit at once; the
// host then reads FKNN_DEVICE_TIMEOUT with fknn_read_status.
#include "fknn_common.cuh"
#include "fknn_internal.h"

namespace fknn {

__global__ void k_selftest_wait(Meta* meta, uint32_t limit) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  mbar_init_fence();
  mbar_arrive_expect_tx(&bar, 16u);  // the phase needs 16 bytes that never come
  if (!mbar_wait_bounded(&bar, 0u, limit)) raise_status(&meta->status, kStatusTimeout);
}

int run_selftest_wait(void* ws, size_t ws_bytes, uint32_t limit, cudaStream_t s) {
  if (ws_bytes < sizeof(Meta)) return FKNN_ERR_WORKSPACE;
  Meta* meta = static_cast<Meta*>(ws);
  cudaError_t e = cudaMemsetAsync(meta, 0, sizeof(Meta), s);
  if (e == cudaSuccess) {
    k_selftest_wait<<<1, 32, 0, s>>>(meta, limit);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  return FKNN_OK;
}

}  // namespace fknn
