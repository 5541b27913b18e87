// Persistent grid-kNN query kernel for sm_100a.
//
// Semantics follow the reference production kernel
// (FlashKNN/csrc/flash_knn_query_dynamic_load.cu:469-652): every query gets
// the exact K smallest FP32 squared distances among the points of the 27
// candidate runs of its group, strict acceptance d < cut_r2, ascending output,
// (pad index, +inf) padding.  Equal distances are ordered by the lower index
// (the reference leaves their order to its network layout).
//
// Execution model (B200-first, not the reference's block-per-parent loop):
//   * persistent CTAs, one work item per warp at a time, pulled from a device
//     queue (atomicAdd on Meta::queue_head);
//   * the item's candidate runs are staged into the warp's shared-memory tile
//     by non-multicast cp.async.bulk copies (one per run, issued by the lane
//     that owns the run) completing on the warp's mbarrier; groups with more
//     candidates than a tile are streamed tile by tile;
//   * G lanes per query (G * queries <= 32) split the candidates; each lane
//     keeps its K best as packed u64 keys (float bits << 32 | index) in
//     registers, inserted by a branch-free shift network; a warp vote skips
//     the insertion when no lane has an improving candidate;
//   * the G partial lists are merged with xor-shuffle bitonic merges and the
//     row is written straight to the caller's row / index space.
#include "fknn_common.cuh"
#include "fknn_internal.h"

namespace fknn {

constexpr uint64_t kEmpty = ~0ull;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// Insert x into the ascending list L, dropping the largest entry.  Slot j
// becomes min(L[j], max(x, L[j-1])): every slot is computed from the old
// list, so the network has no serial dependency.  x == kEmpty is a no-op.
template <int KCAP>
__device__ __forceinline__ void list_insert(uint64_t (&L)[KCAP], uint64_t x) {
#pragma unroll
  for (int j = KCAP - 1; j >= 1; --j) {
    const bool cj = x < L[j];
    const bool cm = x < L[j - 1];
    L[j] = cj ? (cm ? L[j - 1] : x) : L[j];
  }
  L[0] = x < L[0] ? x : L[0];
}

template <int KCAP>
__device__ __forceinline__ void bitonic_clean_ascending(uint64_t (&L)[KCAP]) {
#pragma unroll
  for (int st = KCAP / 2; st > 0; st >>= 1) {
#pragma unroll
    for (int j = 0; j < KCAP; ++j) {
      if ((j & st) == 0) {
        const uint64_t a = L[j], b = L[j + st];
        const bool sw = b < a;
        L[j] = sw ? b : a;
        L[j + st] = sw ? a : b;
      }
    }
  }
}

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int mask) {
  const uint32_t lo = __shfl_xor_sync(kFull, static_cast<uint32_t>(v), mask);
  const uint32_t hi = __shfl_xor_sync(kFull, static_cast<uint32_t>(v >> 32), mask);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Keep the KCAP smallest of this lane's list and the list of lane ^ mask.
template <int KCAP>
__device__ __forceinline__ void merge_with_lane(uint64_t (&L)[KCAP], int mask) {
  if constexpr (KCAP == 1) {
    L[0] = umin64(L[0], shfl_xor_u64(L[0], mask));
  } else {
#pragma unroll
    for (int j = 0; j < KCAP / 2; ++j) {
      const uint64_t a = L[j], b = L[KCAP - 1 - j];
      const uint64_t pa = shfl_xor_u64(b, mask);  // partner's L[KCAP-1-j]
      const uint64_t pb = shfl_xor_u64(a, mask);  // partner's L[j]
      L[j] = umin64(a, pa);
      L[KCAP - 1 - j] = umin64(b, pb);
    }
    bitonic_clean_ascending<KCAP>(L);
  }
}

__device__ __forceinline__ int ceil_log2(int v) { return v <= 1 ? 0 : 32 - __clz(v - 1); }

template <int KCAP, bool EXACT, typename IdxT>
__global__ void __launch_bounds__(256) k_query(QueryLaunch a, int tile_records,
                                               int min_cands_per_lane) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw) + warp;
  float4* tile = reinterpret_cast<float4*>(smem_raw + 128) +
                 static_cast<size_t>(warp) * tile_records;
  Meta* meta = a.meta;
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  __syncwarp();
  uint32_t phase = 0;
  const int n_items = meta->n_items;
  const int k = a.k;

  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(&meta->queue_head, 1);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n_items) break;
    const int4 it = a.items[item];
    const int q_start = it.y;
    int q_count = it.z;
    if (q_start < 0 || q_count < 0 || q_count > 32 ||
        static_cast<int64_t>(q_start) + q_count > a.n_qrec) {
      if (lane == 0) raise_status(&meta->status, kStatusTable);
      continue;
    }

    // Candidate runs, validated against the support array.
    int2 run = make_int2(0, 0);
    if (lane < kNeighbours) run = a.runs[static_cast<int64_t>(it.x) * kNeighbours + lane];
    if (run.y < 0 || run.x < 0 || static_cast<int64_t>(run.x) + run.y > a.n_support) {
      raise_status(&meta->status, kStatusTable);
      run.y = 0;
    }
    const int incl = warp_inclusive_scan(run.y);
    const int total = __shfl_sync(kFull, incl, 31);
    const int run_off = incl - run.y;

    // Lanes per query: as many as the queries leave free, but each lane
    // should see at least min_cands_per_lane candidates.
    int lg = 5 - ceil_log2(q_count > 0 ? q_count : 1);
    while (lg > 0 && (total >> lg) < min_cands_per_lane) --lg;
    const int G = 1 << lg;
    const int qi = lane >> lg, sub = lane & (G - 1);
    const bool active = qi < q_count;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) q = a.qrec[q_start + qi];

    uint64_t L[KCAP];
#pragma unroll
    for (int j = 0; j < KCAP; ++j) L[j] = kEmpty;
    uint32_t thr = 0xffffffffu;

    bool timed_out = false;
    for (int c0 = 0; c0 < total; c0 += tile_records) {
      const int c1 = min(total, c0 + tile_records);
      __syncwarp();
      fence_proxy_async_smem();  // earlier generic reads of the tile precede the copies
      if (lane == 0) mbar_arrive_expect_tx(bar, static_cast<uint32_t>(c1 - c0) * 16u);
      __syncwarp();
      const int lo = max(run_off, c0), hi = min(run_off + run.y, c1);
      if (hi > lo)
        bulk_copy_g2s(tile + (lo - c0), a.srec + run.x + (lo - run_off),
                      static_cast<uint32_t>(hi - lo) * 16u, bar);
      if (!mbar_wait_bounded(bar, phase, kWaitLimit)) {
        timed_out = true;
        break;
      }
      phase ^= 1u;
      const int cnt = c1 - c0;
      for (int i0 = 0; i0 < cnt; i0 += G) {
        const int i = i0 + sub;
        const bool ok = active && i < cnt;
        const float4 c = ok ? tile[i] : q;
        const float d = sq_dist(c.x, c.y, c.z, q.x, q.y, q.z);
        const uint32_t db = __float_as_uint(d);
        const bool acc = ok && (d < a.cut_r2) && (db <= thr);
        if (__any_sync(kFull, acc)) {
          const uint64_t x =
              acc ? ((static_cast<uint64_t>(db) << 32) | static_cast<uint32_t>(__float_as_int(c.w)))
                  : kEmpty;
          list_insert<KCAP>(L, x);
          // The list holds the exact KCAP best, so its last entry is a valid
          // (if K < KCAP, slightly loose) acceptance bound for the K best.
          thr = static_cast<uint32_t>(L[KCAP - 1] >> 32);
        }
      }
    }
    if (timed_out) {
      if (lane == 0) raise_status(&meta->status, kStatusTimeout);
      // Let this warp's copies land before the CTA may exit.
      mbar_wait_bounded(bar, phase, kWaitLimit);
      return;
    }

    for (int m = 1; m < G; m <<= 1) merge_with_lane<KCAP>(L, m);

    if (active && sub == 0) {
      const int row = __float_as_int(q.w);
      if (row < 0 || row >= a.n_rows) {
        raise_status(&meta->status, kStatusTable);
      } else {
        int64_t pad;
        switch (a.pad_mode) {
          case kPadArray64: pad = static_cast<const int64_t*>(a.pad)[row]; break;
          case kPadArray32: pad = static_cast<const int32_t*>(a.pad)[row]; break;
          case kPadMinusOne: pad = -1; break;
          default: pad = row; break;
        }
        IdxT* io = static_cast<IdxT*>(a.idx_out) + static_cast<int64_t>(row) * k;
        float* dout = a.dist_out + static_cast<int64_t>(row) * k;
        if (EXACT && (KCAP % 4) == 0 && a.vec_ok) {
#pragma unroll
          for (int j = 0; j < KCAP; j += 4) {
            float4 dv;
            IdxT iv[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              const uint64_t e = L[j + t];
              const bool empty = e == kEmpty;
              iv[t] = empty ? static_cast<IdxT>(pad) : static_cast<IdxT>(static_cast<int32_t>(e));
              reinterpret_cast<float*>(&dv)[t] =
                  empty ? __int_as_float(0x7f800000) : __uint_as_float(static_cast<uint32_t>(e >> 32));
            }
            *reinterpret_cast<float4*>(dout + j) = dv;
            if constexpr (sizeof(IdxT) == 4) {
              *reinterpret_cast<int4*>(io + j) = make_int4(iv[0], iv[1], iv[2], iv[3]);
            } else {
              *reinterpret_cast<longlong2*>(io + j) = make_longlong2(iv[0], iv[1]);
              *reinterpret_cast<longlong2*>(io + j + 2) = make_longlong2(iv[2], iv[3]);
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < KCAP; ++j) {
            if (j < k) {
              const uint64_t e = L[j];
              const bool empty = e == kEmpty;
              io[j] = empty ? static_cast<IdxT>(pad) : static_cast<IdxT>(static_cast<int32_t>(e));
              dout[j] = empty ? __int_as_float(0x7f800000) : __uint_as_float(static_cast<uint32_t>(e >> 32));
            }
          }
        }
      }
    }
  }
  // Leave the barrier idle before the CTA exits.
  __syncwarp();
}

// ------------------------------------------------------------------ host

QueryShape resolve_shape(const fknn_config* cfg) {
  QueryShape s{4, 512, 8, 0};
  if (cfg) {
    if (cfg->warps_per_cta) s.warps_per_cta = cfg->warps_per_cta;
    if (cfg->tile_records) s.tile_records = cfg->tile_records;
    if (cfg->min_candidates_per_lane) s.min_candidates_per_lane = cfg->min_candidates_per_lane;
    s.ctas_per_sm = cfg->ctas_per_sm;
  }
  return s;
}

bool shape_valid(const QueryShape& s) {
  const bool warps_ok = s.warps_per_cta == 1 || s.warps_per_cta == 2 ||
                        s.warps_per_cta == 4 || s.warps_per_cta == 8;
  return warps_ok && s.tile_records >= 64 && s.tile_records <= 4096 &&
         s.tile_records % 32 == 0 && s.min_candidates_per_lane >= 1 &&
         s.ctas_per_sm >= 0 && s.ctas_per_sm <= 32 &&
         128 + static_cast<size_t>(s.warps_per_cta) * s.tile_records * 16 <= 227 * 1024;
}

namespace {

template <int KCAP, bool EXACT, typename IdxT>
int launch_t(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s) {
  auto kern = k_query<KCAP, EXACT, IdxT>;
  const int threads = shape.warps_per_cta * 32;
  const size_t smem = 128 + static_cast<size_t>(shape.warps_per_cta) * shape.tile_records * 16;
  // Device properties and occupancy are resolved once per (device, shape) and
  // cached, so a launch inside a CUDA graph capture issues nothing but the
  // kernel itself.
  struct Cached {
    int dev = -1, threads = 0, per_sm = 0, sms = 0;
    size_t smem = 0;
  };
  static Cached cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (cache.dev != dev || cache.threads != threads || cache.smem != smem) {
    Cached c;
    c.dev = dev;
    c.threads = threads;
    c.smem = smem;
    e = cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (smem > 48 * 1024) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem));
      if (e != cudaSuccess) return e;
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (c.per_sm < 1) c.per_sm = 1;
    cache = c;
  }
  const int per_sm = shape.ctas_per_sm > 0 ? shape.ctas_per_sm : cache.per_sm;
  const int grid = cache.sms * per_sm;
  const int slot = profile_start(s);
  kern<<<grid, threads, smem, s>>>(q, shape.tile_records, shape.min_candidates_per_lane);
  e = cudaGetLastError();
  profile_stop(slot, s);
  return e;
}

template <int KCAP>
int launch_k(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s) {
  const bool exact = q.k == KCAP;
  if (q.idx_bits == 64)
    return exact ? launch_t<KCAP, true, int64_t>(q, shape, s)
                 : launch_t<KCAP, false, int64_t>(q, shape, s);
  return exact ? launch_t<KCAP, true, int32_t>(q, shape, s)
               : launch_t<KCAP, false, int32_t>(q, shape, s);
}

}  // namespace

int launch_query(const QueryLaunch& q, const QueryShape& shape, cudaStream_t s) {
  if (q.k <= 1) return launch_k<1>(q, shape, s);
  if (q.k <= 2) return launch_k<2>(q, shape, s);
  if (q.k <= 4) return launch_k<4>(q, shape, s);
  if (q.k <= 8) return launch_k<8>(q, shape, s);
  if (q.k <= 16) return launch_k<16>(q, shape, s);
  if (q.k <= 32) return launch_k<32>(q, shape, s);
  return launch_k<64>(q, shape, s);
}

}  // namespace fknn
