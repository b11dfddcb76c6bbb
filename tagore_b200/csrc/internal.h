// internal.h -- host-side interfaces between the C ABI and the kernel files.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/tagore_b200.h"

namespace tagore {

// Records a formatted message for tagore_last_error() and returns `code`.
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define TG_CUDA(call)                                                   \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) return ::tagore::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define TG_TRY(expr)            \
  do {                          \
    int rc_ = (expr);           \
    if (rc_ != TAGORE_OK) return rc_; \
  } while (0)

// ---- launch accounting and stage timing (capi.cu) ----
void count_launch(uint32_t n = 1);
bool profiling();
// Records a start event for stage `name` on `s` (no-op when profiling is off);
// stage_end records the stop event and the stage's algorithmic bytes/items.
void stage_begin(const char* name, cudaStream_t s);
void stage_end(const char* name, cudaStream_t s, uint64_t bytes = 0, uint64_t items = 0);
// Adds bytes/items to a stage after the fact (counts read back from the device).
void stage_add(const char* name, uint64_t bytes, uint64_t items);

// Typed view of the eight reference buffers (capsule order, pybind.cu:132-141).
struct Dev {
  uint32_t n, k, dim;
  uint32_t* graph;     // u32 [n*k]
  uint32_t* rgraph;    // u32 [n*128]
  __half* data;        // f16 [n*dim]
  float* nd;           // f32 [n*k]
  float* rd;           // f32 [n*128]
  uint32_t* rnum;      // u32 [n]
  __half* center;      // f16 [dim]
  uint32_t* hybrid;    // u32 [n*128]
};

inline Dev dev_of(const TagoreKnnState* s) {
  return Dev{s->n, s->k, s->dim, (uint32_t*)s->graph, (uint32_t*)s->reverse_graph,
             (__half*)s->data, (float*)s->nei_distance, (float*)s->reverse_distance,
             (uint32_t*)s->reverse_num, (__half*)s->center, (uint32_t*)s->hybrid_list};
}

// Stream-ordered device scratch that frees itself.
// ---- device memory (capi.cu) ----
// States and scratch come from one memory pool per device that keeps freed
// memory cached, so repeated builds map no new pages;
// tagore_trim_cache() gives the cached memory back.
int pool_alloc(void** p, size_t bytes, cudaStream_t s);
// Counts one allocation (pool_alloc counts its own; pinned host buffers call
// this), reported by tagore_allocation_count().
void count_allocation();
void pool_free(void* p, cudaStream_t s);

// Stream-ordered scratch from the device pool, released on the same stream.
struct Scratch {
  cudaStream_t s;
  void* p = nullptr;
  explicit Scratch(cudaStream_t st) : s(st) {}
  int alloc(size_t bytes) {
    if (bytes == 0) bytes = 16;
    return pool_alloc(&p, bytes, s);
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(p); }
  ~Scratch() {
    if (p) pool_free(p, s);
  }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
};

// ---- prune (prune.cu) ----
struct PruneArgs {
  uint32_t final_degree, topm;
  float thre;
};
// Pruning (pybind.cu:145-229) minus the file write. `type` is NSG, Vamana,
// NSSG, CAGRA or DPG. Writes the entry point to *ep_host for NSG/Vamana.
int prune_index(const Dev& d, const PruneArgs& a, const std::string& type, uint32_t* ep_host,
                cudaStream_t s);
// Pruning_with_CFS (pybind.cu:232-295).
int prune_cfs(const Dev& d, const PruneArgs& a, const std::string& mode, const std::string& metric,
              uint32_t* ep_host, cudaStream_t s);
// Individual stages, exposed for the stage-level parity tests.
int stage_cal_ep(const Dev& d, uint32_t topm, uint32_t* ep_host, cudaStream_t s);
// Opt-in connectivity fix of pruned rows ([deg, ids] stride K): edges are
// appended until every node is reachable from ep (connect.cu).
int connect_graph(const Dev& d, uint32_t ep, uint64_t* added, cudaStream_t s);
// Size of the per-device static scratch of prune_cfs_static.
constexpr size_t kStaticScratchBytes = (size_t)16 << 20;
// prune_cfs for path|2-hop with dist|angle with every temporary carved from
// a static device array of kStaticScratchBytes; larger graphs are rejected.
int prune_cfs_static(const Dev& d, const PruneArgs& a, const std::string& mode,
                     const std::string& metric, uint32_t* ep_host, cudaStream_t s);

// ---- greedy search (search.cu) ----
// tagore_search on stream s; device pointers throughout. search_check is its
// argument validation alone (no device call).
int search_check(const TagoreSearchParams& p, const float* base, uint64_t n, uint32_t dim,
                 const uint64_t* offs, const uint32_t* adj, uint64_t edges, uint32_t ep,
                 const float* queries, uint32_t nq, const uint32_t* out);
int greedy_search(const TagoreSearchParams& p, const float* base, uint64_t n, uint32_t dim,
                  const uint64_t* offs, const uint32_t* adj, uint64_t edges, uint32_t ep,
                  const float* queries, uint32_t nq, uint32_t* out, cudaStream_t s);

// ---- bounded-wait self-test (knn_tc.cu) ----
// k_wait_selftest: *timed_out = 1 when the wait on an mbarrier nothing
// arrives on ran out and the block returned.
namespace knn {
int wait_selftest(int* timed_out, cudaStream_t s);
}

// ---- kNN graph (knn.cu) ----
struct KnnArgs {
  uint32_t k, iters, mode;  // mode: TAGORE_KNN_CHOSEN / _PLAIN / _LEARNED
  uint32_t sample;          // forward samples per list per iteration
  uint32_t per_row;         // proposals kept per join row
  uint64_t seed;
  uint32_t learn_steps;     // training steps of the screen (0: default)
  uint32_t learn_flags;     // TAGORE_LEARN_*
};
// Outcome of the learned screen in the last build on this thread.
struct ScreenStats {
  uint32_t used, steps, screened_iters, per_row, fallback;
  float loss_first, loss_last;
  double last_miss;       // improving pairs the screen did not keep (sampled nodes)
  double last_best_kept;  // share of each row's exact best T the screen kept
};
void set_screen_stats(const ScreenStats& s);
struct KnnStats {
  double ms_total, ms_prep, ms_iters;
  uint64_t proposals, pairs;
};
// Builds the kNN graph over d.data (FP16 base) into d.graph / d.nd.
int knn_build(const Dev& d, const float* norms, const KnnArgs& a, KnnStats* st, cudaStream_t s);

// ---- largeIndex (large_index.cpp) ----
// A local graph's rows: n x K, [deg, global ids..]; entries past a row's
// degree are never read, so resizing leaves them uninitialised.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) {}
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    if constexpr (sizeof...(A) == 0)
      ::new ((void*)p) U;
    else
      ::new ((void*)p) U(std::forward<A>(a)...);
  }
};
using LocalRows = std::vector<uint32_t, NoInitAlloc<uint32_t>>;
// Builds cluster `cid` (global ids `ids`, vectors `data` as the load function
// left them, or null without one) into n x K rows [deg, global ids..] and
// reports its entry point as a global id. `worker` is the builder thread, an
// index into the device list; `stage` is the builder's pinned buffer of
// max_points x K words for the rows' way back (null without a load function).
using LargeBuildFn = std::function<int(const TagoreLargeParams&, uint32_t worker, uint32_t cid,
                                       const std::vector<uint32_t>& ids, const float* data,
                                       uint32_t* stage, LocalRows& rows, uint32_t* medoid)>;
// Reads cluster `cid`'s n vectors (n x dim FP32) into dst, pinned host memory.
using LargeLoadFn =
    std::function<int(const TagoreLargeParams&, uint32_t cid, size_t n, float* dst)>;
// Builder threads (two per device-list entry with a load function, else one)
// each take the next cluster in the merger's order; the host merger consumes
// them in that order. With a load function, each builder reads its next
// cluster on a reader thread into one of two pinned buffers while the current
// cluster builds.
int large_index_run(const TagoreLargeParams& p, const uint32_t* dev_list, int ndev,
                    const LargeBuildFn& build, const LargeLoadFn& load = nullptr);

// ---- base preparation (prep.cu) ----
// FP16 base = raw * factor (as __float2half) and exact FP32 squared norms of
// the FP16 rows, from the FP32 input already on the device.
int prep_base(const float* raw, uint32_t n, uint32_t dim, float factor, __half* data, float* norms,
              cudaStream_t s);
float host_factor(const float* x, uint32_t dim, bool rescale);
void host_center(const float* x, uint32_t n, uint32_t dim, float factor, uint16_t* center_half);
// The same centroid on the device from raw (n x dim FP32 on the device).
int device_center(const float* raw, uint32_t n, uint32_t dim, float factor, __half* center,
                  cudaStream_t s);
// fvecs file -> raw (n x dim FP32 on the device) through pinned chunks;
// *factor = host_factor of vector 0.
int ingest_fvecs(const char* path, uint32_t n, uint32_t dim, bool rescale, float* raw,
                 float* factor, cudaStream_t s);

}  // namespace tagore
