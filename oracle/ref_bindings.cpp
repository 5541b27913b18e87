// pybind11 table for the reference kernels compiled as a GPU oracle
// (TEST INFRASTRUCTURE ONLY).  The functions are the reference's own, from
// FlashKNN/csrc (declarations in flash_knn_query.h and
// flash_knn_construction.h); this file only exposes the subset the parity
// tests call.
#include <torch/extension.h>

#include "flash_knn_construction.h"
#include "flash_knn_query.h"

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("get_cuda_shared_mem", &get_cuda_shared_mem);
  m.def("FlashKNN_Query_Dynamic_Load", &FlashKNN_Query_Dynamic_Load);
  m.def("FlashKNN_Selected_Query_DL", &FlashKNN_Selected_Query_DL);
  m.def("FlashKNN_Nearest_Back_Query_DL", &FlashKNN_Nearest_Back_Query_DL);
  m.def("FlashKNN_Back_Query_DL", &FlashKNN_Back_Query_DL);
  m.def("FlashKNN_Morton_Encode", &FlashKNN_Morton_Encode);
  m.def("FlashKNN_Morton_Neighbor_Keys", &FlashKNN_Morton_Neighbor_Keys);
}
