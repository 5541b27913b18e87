// fknn_query_tables_noalloc: the reference-table query without a workspace.
//
// Who needs it: callers that cannot create device memory for us.  Examples
// are a plugin running inside a host application whose framework owns every
// device allocation through its own pool (a raw cudaMalloc is forbidden
// there), a real-time loop that must not allocate once it has started, and
// a thin binding that only forwards the reference's tensors and has no way
// to size and keep a scratch buffer.  For them this entry point takes the
// same inputs and outputs as fknn_query_tables and keeps its scratch in a
// fixed array that lives in the library itself.
//
// The price of not allocating:
//   * the array has a fixed size (kScratchBytes, about 10 MiB), so problems
//     are limited to kMaxPoints points and kMaxParents parent cells; larger
//     ones are rejected with FKNN_ERR_SCRATCH_LIMIT before anything runs;
//   * every GPU that loads this library holds the array until the process
//     exits;
//   * every call on a device uses the same array: two calls that run on the
//     GPU at the same time (for example on two streams) overwrite each
//     other's scratch and race.  Order such calls on one stream.
// The first call on each device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.  Later calls only launch work on the stream.
// The address is kept for the life of the process: calls after a device
// reset (cudaDeviceReset, which unloads the array) are not supported.
//
// Problems only the device can see (tables naming rows outside the point
// array, a bounded wait that gave up) are OR-ed into a status word at the
// start of the array, as fknn_query_tables does in its workspace; each call
// clears it first.  fknn_query_tables_noalloc_read_status copies it out.
#include <cstdint>
#include <mutex>

#include "../../include/fknn.h"
#include "fknn_internal.h"
#include "fknn_tables.h"

namespace {

constexpr int64_t kMaxPoints = 32768;
constexpr int64_t kMaxParents = 32768;
constexpr size_t kScratchBytes = size_t{10} << 20;
constexpr int kMaxDevices = 64;

// The scratch of every call on a device.  In host code this name is only a
// host-side stand-in for the device array; its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_scratch on the current device, looked up once per device.
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    fknn::note_cuda_error(e);
    return FKNN_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return FKNN_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_scratch_ptr[dev] == nullptr) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
      fknn::note_cuda_error(e);
      return FKNN_ERR_CUDA;
    }
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return FKNN_OK;
}

}  // namespace

extern "C" int fknn_query_tables_noalloc(const float* xyz_sorted, int64_t n,
                                         const int32_t* steps, const int32_t* neigh,
                                         const int32_t* cnt, int64_t p, int32_t k, float cut_r2,
                                         int32_t* idx_out, float* dist_out, void* stream) {
  if (k < 1 || k > 64) return FKNN_ERR_K;
  if (n < 0 || p < 0) return FKNN_ERR_ARG;
  if (n > kMaxPoints || p > kMaxParents) return FKNN_ERR_SCRATCH_LIMIT;
  if ((n > 0 && (!xyz_sorted || !idx_out || !dist_out)) || (p > 0 && (!steps || !neigh || !cnt)))
    return FKNN_ERR_ARG;
  if (fknn::tables_workspace_bytes(n, n, p) > kScratchBytes) return FKNN_ERR_SCRATCH_LIMIT;
  void* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != FKNN_OK) return rc;
  // run_tables clears the scratch's status / counter block on the stream
  // before use; every other scratch buffer is written before it is read.
  const fknn::TablesArgs t{xyz_sorted, n, steps, neigh, cnt, p, nullptr, nullptr, n, k, cut_r2,
                           idx_out, dist_out};
  int launches = 0;
  const int out = fknn::run_tables(t, scratch, kScratchBytes, fknn::resolve_shape(nullptr),
                                   static_cast<cudaStream_t>(stream), &launches);
  if (out == FKNN_OK) fknn::note_launches(launches);
  return out;
}

extern "C" int fknn_query_tables_noalloc_read_status(int* status, void* stream) {
  if (!status) return FKNN_ERR_ARG;
  void* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != FKNN_OK) return rc;
  // the status word is the first int of the scratch, as in every workspace
  return fknn_read_status(scratch, status, stream);
}
