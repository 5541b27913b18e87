// C binding of the reference's CPU kNN baseline (TEST / BASELINE ONLY).
//
// The reference times its GPU kNN against nanoflann: a KD-tree over the
// support cloud with leaf size 20, exact FP32 squared-L2 top-K per query
// through the header's KNNResultSetHeap result set, queries answered one after
// another on one thread
// (Query/ThirdParty/nanoflannkdtree/csrcs/kdtree.cpp:31-63,
//  Query/ThirdParty/nanoflannkdtree/TorchFlann/__init__.py:16-61).
// This file is compiled against the reference's own nanoflann.hpp (a modified
// copy of nanoflann, BSD licence, in that directory) by oracle/build_ref.py
// into oracle/_ref/; it exposes plain C entry points for ctypes and an
// OpenMP loop over the queries of a batch of clouds, so the same code can be
// timed single-threaded (as the reference runs it) and on every host core.
#include <cstddef>
#include <cstdint>
#include <vector>

#include <omp.h>

#include "nanoflann.hpp"

namespace {

// nanoflann's dataset interface over an FP32 [n, 3] array.
struct Cloud {
  const float* xyz;
  size_t n;
  size_t kdtree_get_point_count() const { return n; }
  float kdtree_get_pt(size_t i, size_t d) const { return xyz[3 * i + d]; }
  template <class Box>
  bool kdtree_get_bbox(Box&) const { return false; }
};

using Tree = nanoflann::KDTreeSingleIndexAdaptor<nanoflann::L2_Simple_Adaptor<float, Cloud>,
                                                 Cloud, 3>;

struct Index {
  Cloud cloud;
  Tree tree;
  Index(const float* xyz, size_t n, size_t leaf)
      : cloud{xyz, n}, tree(3, cloud, nanoflann::KDTreeSingleIndexAdaptorParams(leaf)) {}
};

}  // namespace

extern "C" {

// Trees for every cloud of an offset batch (offsets = cumulative ends),
// built in parallel over clouds.  Returns an opaque handle.
void* rnf_build(const float* xyz, const int64_t* offsets, int n_clouds, int leaf, int nthreads) {
  auto* trees = new std::vector<Index*>(static_cast<size_t>(n_clouds), nullptr);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int c = 0; c < n_clouds; ++c) {
    const int64_t start = c ? offsets[c - 1] : 0;
    (*trees)[c] = new Index(xyz + 3 * start, static_cast<size_t>(offsets[c] - start),
                            static_cast<size_t>(leaf));
  }
  return trees;
}

void rnf_free(void* handle) {
  auto* trees = static_cast<std::vector<Index*>*>(handle);
  for (Index* t : *trees) delete t;
  delete trees;
}

// k nearest support points of every query point, queries of cloud c against
// tree c; q_offsets are the queries' cumulative ends.  idx holds indices
// local to the cloud (as the reference returns them); ordered sorts each row
// ascending, as kdtree_knn(..., sorted=true) does.
void rnf_knn(void* handle, const float* q, const int64_t* q_offsets, int n_clouds, int k,
             uint32_t* idx, float* dist, int ordered, int nthreads) {
  auto* trees = static_cast<std::vector<Index*>*>(handle);
  const int64_t m = n_clouds ? q_offsets[n_clouds - 1] : 0;
#pragma omp parallel num_threads(nthreads)
  {
    int c = 0;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < m; ++i) {
      while (q_offsets[c] <= i) ++c;  // clouds are visited in order within a chunk
      while (c > 0 && q_offsets[c - 1] > i) --c;
      nanoflann::KNNResultSetHeap<float, uint32_t> rs(static_cast<size_t>(k), idx + i * k,
                                                      dist + i * k);
      (*trees)[c]->tree.findNeighbors(rs, q + 3 * i);
      if (ordered) rs.sort();
    }
  }
}

}  // extern "C"
