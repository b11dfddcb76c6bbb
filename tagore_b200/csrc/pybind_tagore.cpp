// pybind_tagore.cpp -- the Python module `Tagore`, a drop-in for the one the
// reference builds (pybind.cu:393-398). It only marshals arguments into the C
// ABI (include/tagore_b200.h); all work happens behind it.
//
// GNN_descent returns the reference's eight device capsules in its order
// (pybind.cu:132-141), each freeing its buffer, plus the FP32 norms as element
// 8. Pruning and Pruning_with_CFS read elements 0-7 only, so tuples from either
// module work with the other's pruning functions.
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "tagore_b200.h"

namespace py = pybind11;

namespace {

void check(int rc) {
  if (rc == TAGORE_OK) return;
  const std::string msg = tagore_last_error();
  if (rc == TAGORE_EINVAL) throw py::value_error(msg);
  if (rc == TAGORE_EIO) throw std::runtime_error("I/O error: " + msg);
  throw std::runtime_error(msg);
}

py::capsule owned(void* p) {
  return py::capsule(p, [](void* q) { tagore_device_free(q); });
}

TagoreKnnState state_from(unsigned K, unsigned POINTS, unsigned DIM, const py::tuple& ptrs) {
  if (ptrs.size() < 8) throw py::value_error("ptrs must hold the 8 buffers GNN_descent returned");
  TagoreKnnState st{};
  st.n = POINTS;
  st.dim = DIM;
  st.k = K;
  void** slots[8] = {&st.graph, &st.reverse_graph, &st.data, &st.nei_distance,
                     &st.reverse_distance, &st.reverse_num, &st.center, &st.hybrid_list};
  for (int i = 0; i < 8; ++i) *slots[i] = ptrs[i].cast<py::capsule>().get_pointer();
  st.owns = 0;
  return st;
}

py::tuple GNN_descent(unsigned K, unsigned POINTS, unsigned DIM, unsigned iter, const std::string& fname) {
  TagoreKnnParams p{};
  p.k = K;
  p.n = POINTS;
  p.dim = DIM;
  p.iters = iter;
  p.mode = TAGORE_KNN_CHOSEN;
  p.rescale = 1;
  p.seed = 0x7A6Eull;
  TagoreKnnState st{};
  uint32_t n = 0, d = 0;
  check(tagore_load_fvecs_header(fname.c_str(), &n, &d));
  std::printf("Points: %u, Dim: %u\n", n, d);
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = tagore_gnn_descent(&p, fname.c_str(), &st);
  }
  check(rc);
  TagoreTimings t{};
  tagore_last_timings(&t);
  std::printf("time of GNN-Descent: %gs\n", t.knn_ms / 1000.0);
  std::fflush(stdout);
  return py::make_tuple(owned(st.graph), owned(st.reverse_graph), owned(st.data),
                        owned(st.nei_distance), owned(st.reverse_distance), owned(st.reverse_num),
                        owned(st.center), owned(st.hybrid_list), owned(st.norms));
}

void Pruning(unsigned K, unsigned POINTS, unsigned DIM, unsigned FINAL_DEGREE, unsigned TOPM,
             py::tuple ptrs, std::string index_type, float thre, std::string index_path) {
  TagoreKnnState st = state_from(K, POINTS, DIM, ptrs);
  TagorePruneParams p{K, POINTS, DIM, FINAL_DEGREE, TOPM, thre};
  std::printf("begin to construct %s\n", index_type.c_str());
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = tagore_pruning(&p, &st, index_type.c_str(), index_path.c_str());
  }
  check(rc);
  TagoreTimings t{};
  tagore_last_timings(&t);
  std::printf("time of pruning: %gs\n", t.prune_ms / 1000.0);
  std::fflush(stdout);
}

void Pruning_with_CFS(unsigned K, unsigned POINTS, unsigned DIM, unsigned FINAL_DEGREE, unsigned TOPM,
                      py::tuple ptrs, std::string mode, std::string metric, float thre) {
  TagoreKnnState st = state_from(K, POINTS, DIM, ptrs);
  TagorePruneParams p{K, POINTS, DIM, FINAL_DEGREE, TOPM, thre};
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = tagore_pruning_cfs(&p, &st, mode.c_str(), metric.c_str());
  }
  check(rc);
  TagoreTimings t{};
  tagore_last_timings(&t);
  std::printf("time of pruning: %gs\n", t.prune_ms / 1000.0);
  std::fflush(stdout);
}

void largeIndex(std::vector<unsigned>& devicelist, unsigned DIM, unsigned K, unsigned cluster_num,
                unsigned max_points, std::string data_prefix, std::string local_prefix,
                std::string index_store_path, unsigned max_degree, unsigned buffer_size,
                unsigned num, std::string centers_path, float thre, unsigned FINAL_DEGREE,
                unsigned TOPM) {
  TagoreLargeParams p{};
  p.dim = DIM;
  p.k = K;
  p.cluster_num = cluster_num;
  p.max_points = max_points;
  p.data_prefix = data_prefix.c_str();
  p.local_prefix = local_prefix.c_str();
  p.index_store_path = index_store_path.c_str();
  p.max_degree = max_degree;
  p.buffer_size = buffer_size;
  p.num = num;
  p.centers_path = centers_path.c_str();
  p.thre = thre;
  p.final_degree = FINAL_DEGREE;
  p.topm = TOPM;
  p.knn_iters = 16;
  p.mode = TAGORE_KNN_CHOSEN;
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = tagore_large_index(&p, devicelist.data(), (int)devicelist.size());
  }
  check(rc);
}

}  // namespace

PYBIND11_MODULE(Tagore, m) {
  m.doc() = "Tagore GPU Indexing (B200 build)";
  m.def("GNN_descent", &GNN_descent, "GNN_descent");
  m.def("Pruning", &Pruning, "Pruning", py::arg("K"), py::arg("POINTS"), py::arg("DIM"),
        py::arg("FINAL_DEGREE"), py::arg("TOPM") = 64, py::arg("ptrs"), py::arg("index_type"),
        py::arg("thre") = 1.0, py::arg("index_path") = "index.data");
  m.def("Pruning_with_CFS", &Pruning_with_CFS, "Pruning_with_CFS");
  m.def("largeIndex", &largeIndex, "largeIndex");
}
