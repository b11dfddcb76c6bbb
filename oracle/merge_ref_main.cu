// merge_ref_main.cu -- runs the reference's own largeIndex host half on given
// local graphs.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.sh (with the reference's
// sources, read in place) into oracle/_ref/merge_ref; tests/test_large_ref_cpu.py
// compares its output with this library's tagore_large_merge. Nothing in the
// product links or runs it.
//
// It reads the cluster assignment as largeIndex does (pybind.cu:314-330),
// orders the clusters with the reference's order_merge_main
// (src/large_index.cu:86-106) and runs its merger order_merge_new (:286-522)
// on one thread while this thread plays gpu_construct's hand-off
// (:255-277): for each cluster in merge order it sets the entry point, waits
// until the merger has a buffer slot for it (has_merged), copies the given
// rows [deg, global ids...] into that slot and marks it built. No device is
// used.
//
// Input file: u32 N, C, K, max_degree, buffer_size; N x (u32 first, u32
// second) cluster ids; for each cluster c (ascending) its |c| x K rows; C
// u32 entry points (global ids). Arguments: input, index path, spill prefix.
// Writes the merge order, one id per line, to stdout after a line "order".
#include <large_index.cuh>

#include <chrono>
#include <cstdio>
#include <thread>

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: merge_ref INPUT INDEX SPILL_PREFIX\n");
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  unsigned hdr[5];
  if (std::fread(hdr, 4, 5, f) != 5) return 4;
  const unsigned N = hdr[0], C = hdr[1], K = hdr[2], max_degree = hdr[3], buffer_size = hdr[4];
  std::vector<unsigned> pairs(2 * (size_t)N);
  if (std::fread(pairs.data(), 4, pairs.size(), f) != pairs.size()) return 5;
  std::vector<unsigned> Centers(N), Centers_second(N);
  for (unsigned i = 0; i < N; i++) {
    Centers[i] = pairs[2 * i];
    Centers_second[i] = pairs[2 * i + 1];
  }
  std::vector<std::vector<unsigned>> clusters(C);
  for (unsigned i = 0; i < N; i++) {
    clusters[Centers[i]].push_back(i);
    clusters[Centers_second[i]].push_back(i);
  }
  size_t max_points = 0;
  std::vector<std::vector<unsigned>> rows(C);
  for (unsigned c = 0; c < C; c++) {
    rows[c].resize(clusters[c].size() * (size_t)K);
    if (std::fread(rows[c].data(), 4, rows[c].size(), f) != rows[c].size()) return 6;
    max_points = std::max(max_points, clusters[c].size());
  }
  std::vector<unsigned> eps(C);
  if (std::fread(eps.data(), 4, C, f) != C) return 7;
  std::fclose(f);

  std::vector<unsigned> results, position(C), metroids(C);
  order_merge_main(Centers, Centers_second, C, N, results, clusters, position, buffer_size);
  std::vector<std::vector<unsigned>> graph_pool(buffer_size);
  for (unsigned i = 0; i < buffer_size; i++) graph_pool[i].resize(max_points * K);
  std::vector<bool> has_built(C, false), has_merged(C, false);

  std::thread merger(order_merge_new, std::ref(clusters), N, C, std::ref(Centers),
                     std::ref(Centers_second), std::ref(results), std::ref(position),
                     std::ref(metroids), std::string(argv[2]), std::string(argv[3]), K,
                     std::ref(graph_pool), std::ref(has_merged), std::ref(has_built), max_degree,
                     buffer_size);
  for (unsigned cid = 0; cid < C; cid++) {
    const unsigned oc = results[cid];
    metroids[cid] = eps[oc];
    while (!has_merged[oc]) std::this_thread::sleep_for(std::chrono::milliseconds(1));
    std::copy(rows[oc].begin(), rows[oc].end(), graph_pool[position[oc]].begin());
    has_built[oc] = true;
  }
  merger.join();
  std::printf("order\n");
  for (unsigned cid = 0; cid < C; cid++) std::printf("%u\n", results[cid]);
  return 0;
}
