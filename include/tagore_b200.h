/* tagore_b200.h -- C ABI of the B200 graph-index builder.
 *
 * Drop-in boundary for the Python module `Tagore` of ZJU-DAILY/Tagore
 * (pybind.cu:393-398). Every function returns a status code; on failure
 * tagore_last_error() gives a one-line message (thread-local). No function
 * exits the process. Device buffers are plain pointers on the current device.
 */
#ifndef TAGORE_B200_H
#define TAGORE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TAGORE_OK = 0,
  TAGORE_EINVAL = 1,   /* bad argument or unsupported combination */
  TAGORE_EIO = 2,      /* file missing, truncated or unwritable */
  TAGORE_ENOMEM = 3,   /* host or device allocation failed */
  TAGORE_ECUDA = 4,    /* a CUDA call failed */
  TAGORE_ETIMEOUT = 5  /* a bounded wait ran out */
};

/* kNN join modes. CHOSEN: tensor-core screen + exact re-rank where the row
 * width allows (one tile for 16..128 dims in steps of 16; the tile
 * accumulated over 64-dim blocks for 129..1024 dims in steps of 8), the
 * learned screen otherwise; PLAIN: every pair in exact FP32; LEARNED: the
 * learned screen at any width. */
enum { TAGORE_KNN_CHOSEN = 0, TAGORE_KNN_PLAIN = 1, TAGORE_KNN_LEARNED = 2 };

/* learn_flags of TagoreKnnParams (for measuring the screen against itself):
 * FIXED_T keeps the per-row count instead of steering it by the miss rate;
 * NO_TRAIN screens with the untrained start weights. */
enum { TAGORE_LEARN_FIXED_T = 1, TAGORE_LEARN_NO_TRAIN = 2 };

/* The reference's eight device buffers in its capsule order
 * (pybind.cu:132-141), plus project buffers. Ownership: created by
 * tagore_gnn_descent / tagore_state_alloc, released by tagore_state_free. */
typedef struct TagoreKnnState {
  uint32_t n, dim, k;
  int32_t device;
  float norm_factor;        /* power of ten applied to the base (pybind.cu:24-36) */
  uint32_t ep;              /* entry point of the last NSG/Vamana prune */
  void* graph;              /* [0] u32 [n*k]: kNN ids sorted by distance; pruned rows after Pruning */
  void* reverse_graph;      /* [1] u32 [n*128] */
  void* data;               /* [2] f16 [n*dim], scaled by norm_factor */
  void* nei_distance;       /* [3] f32 [n*k] */
  void* reverse_distance;   /* [4] f32 [n*128] */
  void* reverse_num;        /* [5] u32 [n] */
  void* center;             /* [6] f16 [dim], scaled */
  void* hybrid_list;        /* [7] u32 [n*128] */
  void* norms;              /* f32 [n]: exact squared norms of the FP16 base */
  uint32_t owns;            /* 1 when tagore_state_free releases the buffers */
  uint32_t pad_;
} TagoreKnnState;

typedef struct TagoreKnnParams {
  uint32_t k;        /* degree of the kNN graph (K) */
  uint32_t n;        /* POINTS; the fvecs loader takes the count from the file */
  uint32_t dim;      /* DIM */
  uint32_t iters;    /* iterations; the reference runs iters/2 + iters/2 */
  uint32_t mode;     /* TAGORE_KNN_CHOSEN, TAGORE_KNN_PLAIN or TAGORE_KNN_LEARNED */
  uint32_t sample;   /* forward samples per list and iteration (0: 32) */
  uint32_t per_row;  /* proposals kept per local-join row (0: default) */
  uint32_t rescale;  /* 1: power-of-ten rescale as GNN_descent; 0: none (largeIndex) */
  uint64_t seed;
  uint32_t learn_steps;  /* training steps of the learned screen (0: 400) */
  uint32_t learn_flags;  /* TAGORE_LEARN_* */
} TagoreKnnParams;

typedef struct TagorePruneParams {
  uint32_t k, n, dim;
  uint32_t final_degree; /* FINAL_DEGREE */
  uint32_t topm;         /* TOPM (m), default 64 */
  float thre;            /* threshold: alpha for Vamana, cos(angle) for NSSG */
} TagorePruneParams;

typedef struct TagoreLargeParams {
  uint32_t dim, k, cluster_num, max_points;
  const char* data_prefix;        /* cluster files data_prefix + cid: [u32 n][n*dim f32] */
  const char* local_prefix;       /* spill files of evicted local graphs */
  const char* index_store_path;   /* final DiskANN-style index */
  uint32_t max_degree, buffer_size;
  uint32_t num;                   /* total points */
  const char* centers_path;       /* num x (u32 first, u32 second) cluster ids */
  float thre;
  uint32_t final_degree, topm;
  uint32_t knn_iters;             /* GNN-Descent iterations per cluster (reference: 8 + 8) */
  uint32_t mode;                  /* TAGORE_KNN_CHOSEN or TAGORE_KNN_PLAIN */
} TagoreLargeParams;

/* Tagore.GNN_descent(K, POINTS, DIM, iter, fname) (pybind.cu:19-142):
 * loads an fvecs file and builds the kNN graph on the current device. */
int tagore_gnn_descent(const TagoreKnnParams* p, const char* fvecs_path, TagoreKnnState* out);

/* Same as tagore_gnn_descent with the FP32 base in host memory
 * (n x dim, row-major) instead of a file. */
int tagore_gnn_descent_host(const TagoreKnnParams* p, const float* data, uint32_t n, uint32_t dim,
                            TagoreKnnState* out);

/* Tagore.Pruning(K, POINTS, DIM, FINAL_DEGREE, TOPM, ptrs, index_type, thre,
 * index_path) (pybind.cu:145-229): prunes in place and writes the index file
 * (NSG, Vamana, NSSG, CAGRA or DPG layout, src/common.cu:151-248). An empty or
 * NULL index_path skips the file. */
int tagore_pruning(const TagorePruneParams* p, TagoreKnnState* st, const char* index_type,
                   const char* index_path);

/* Tagore.Pruning_with_CFS(K, POINTS, DIM, FINAL_DEGREE, TOPM, ptrs, mode,
 * metric, thre) (pybind.cu:232-295): Collect ('path', '2-hop', '1-hop'),
 * Filter+Store ('dist', 'angle', 'rank'); the result stays in st->graph. */
int tagore_pruning_cfs(const TagorePruneParams* p, TagoreKnnState* st, const char* mode,
                       const char* metric);

/* No counterpart in the reference. Same result as tagore_pruning_cfs for
 * mode 'path' or '2-hop' with metric 'dist' or 'angle', computed without
 * allocating device memory: every temporary comes from one static device
 * array of 16 MiB per device (about 18,000 points at FINAL_DEGREE 32).
 * Graphs whose temporaries do not fit, and other mode/metric pairs, return
 * TAGORE_EINVAL. Work goes to `stream` (a cudaStream_t; NULL is the legacy
 * default stream) and the call returns after it has finished. Calls that
 * overlapped on the GPU would race on the shared array; calls are serialised
 * by a process-wide lock, and each call waits for its work on `stream`
 * before it returns, on error paths too. The first call on a device does its
 * set-up (module load, symbol lookup, kernel attributes) and should come
 * before any stream capture. */
int tagore_pruning_cfs_noalloc(const TagorePruneParams* p, TagoreKnnState* st, const char* mode,
                               const char* metric, void* stream);

/* Tagore.largeIndex(devicelist, DIM, K, cluster_num, max_points, ...)
 * (pybind.cu:298-391). Two builder threads per devicelist entry (1 to 64
 * entries; an id may repeat, which runs more builders on one device) take the
 * clusters in the merger's order; the reference deals them round-robin. */
int tagore_large_index(const TagoreLargeParams* p, const uint32_t* devices, int ndev);

/* The host half of largeIndex alone (reorder + order_merge_new,
 * src/large_index.cu:9-106 and :286-522): the clusters come from
 * p->centers_path as in tagore_large_index, but each cluster's local graph is
 * given: local_rows[cid] holds clusters[cid].size() x p->k rows of
 * [degree, global ids...] and local_medoids[cid] its entry point (a global
 * id). Writes the spill files and p->index_store_path; no device is used.
 * Four builder threads hand the graphs over, as in a multi-device run; the
 * merged bytes do not depend on their schedule. */
int tagore_large_merge(const TagoreLargeParams* p, const uint32_t* const* local_rows,
                       const uint32_t* local_medoids);

/* No counterpart in the reference (opt-in; it changes the edge lists): makes
 * every node of the pruned graph in st->graph ([deg, ids...] rows, stride K)
 * reachable from `ep` by appending edges, in the manner of NSG's tree
 * growing. An unreachable node is attached to the end of a greedy walk from
 * ep toward it. *added receives the number of edges added. Call it after
 * tagore_pruning / tagore_pruning_cfs and before writing an index from the
 * rows. */
int tagore_connect(TagoreKnnState* st, uint32_t ep, uint64_t* added);

/* Greedy search over a graph index, one query per warp: NSG's search
 * (get_neighbors, src/common.cu:65-127) as the recall evaluator of built
 * indexes. The pool holds L candidates sorted by squared L2 distance (ties:
 * earlier arrival first); the first unexpanded one is expanded until none is
 * left. It starts from the entry point's neighbours; with seed != 0 it then
 * tops the pool up to L with seeded random nodes (splitmix64 draws), with
 * seed == 0 the entry point itself goes first. */
typedef struct TagoreSearchParams {
  uint32_t L;         /* pool size */
  uint32_t k;         /* ids written per query; slots past the pool get 0xFFFFFFFF */
  uint64_t seed;      /* 0: entry point first; else seeded random starts */
  uint32_t visit_cap; /* visited-set slots per query, rounded up to a power of two
                         (0: 64 L, at least 16384); a query may visit half of them */
  uint32_t pad_;
} TagoreSearchParams;

/* All pointers are on the current device: base (n x dim FP32), the graph as
 * CSR (offs: n+1 u64, adj: `edges` u32; ids >= n are skipped), queries
 * (nq x dim FP32) and out (nq x k u32). stream may be null (a private
 * stream). Returns TAGORE_EINVAL when a query outgrows the visited set. */
int tagore_search(const TagoreSearchParams* p, const float* base, uint64_t n, uint32_t dim,
                  const uint64_t* offs, const uint32_t* adj, uint64_t edges, uint32_t ep,
                  const float* queries, uint32_t nq, uint32_t* out, void* stream);

/* Index readers, the inverse of the writers below: index_type is NSG, Vamana,
 * NSSG, CAGRA or DPG (the strings Pruning takes, pybind.cu:177-221).
 * tagore_index_info scans the file; tagore_index_read fills the CSR arrays
 * (offs: n+1, adj: edges) for the n and edges it reported. */
typedef struct TagoreIndexInfo {
  uint64_t n;          /* nodes */
  uint64_t edges;      /* adjacency entries over all nodes */
  uint32_t max_degree; /* widest row */
  uint32_t width;      /* header width (NSG, NSSG), max degree (Vamana), 0 (CAGRA, DPG) */
  uint32_t n_eps;      /* entry points stored: NSG and Vamana 1, NSSG its count, else 0 */
  uint32_t eps[16];    /* the first min(n_eps, 16) of them */
  uint32_t pad_;
} TagoreIndexInfo;
int tagore_index_info(const char* path, const char* index_type, TagoreIndexInfo* info);
int tagore_index_read(const char* path, const char* index_type, uint64_t n, uint64_t edges,
                      uint64_t* offs, uint32_t* adj);

/* cal_ep_gpu (src/Tagore_src.cu:1889-2058) alone: entry point of the graph
 * held in st (kNN rows) toward st->center. */
int tagore_entry_point(TagoreKnnState* st, uint32_t topm, uint32_t* ep);

/* Allocates the eight buffers (and norms) for n x dim with degree k on the
 * current device, zero-filled; reverse_num starts at 0 as after GNN_descent. */
int tagore_state_alloc(uint32_t n, uint32_t dim, uint32_t k, TagoreKnnState* out);

/* Releases buffers owned by the state (the capsule destructors of pybind.cu:133-140). */
int tagore_state_free(TagoreKnnState* st);

/* Copies between a host array and one of the state's buffers, by capsule
 * index 0..7 (8 = norms); bytes must not exceed the buffer. */
int tagore_state_upload(TagoreKnnState* st, int which, const void* host, size_t bytes);
int tagore_state_download(const TagoreKnnState* st, int which, void* host, size_t bytes);

/* Byte size of buffer `which` of the state. */
size_t tagore_state_bytes(const TagoreKnnState* st, int which);

/* One whole build from host memory to host memory: rescale + FP16 base,
 * kNN graph (p), CFS 'path'/'dist' prune with final_degree/topm/thre, and the
 * pruned rows copied back as [deg, ids...] stride-k rows into out_graph
 * (n*k u32). *ep_out gets the entry point. Used for the end-to-end timing. */
int tagore_build_index_host(const TagoreKnnParams* p, const float* data, uint32_t n, uint32_t dim,
                            uint32_t final_degree, uint32_t topm, float thre, uint32_t* out_graph,
                            uint32_t* ep_out);

/* Index writers (src/common.cu:151-248), from host rows. */
int tagore_store_nsg(const char* path, const uint32_t* graph, uint32_t width, uint32_t ep,
                     uint32_t n, uint32_t k);
int tagore_store_vamana(const char* path, const uint32_t* graph, uint32_t ep, uint32_t n,
                        uint32_t k);
int tagore_store_nssg(const char* path, const uint32_t* graph, uint32_t width, uint32_t n,
                      uint32_t k);
int tagore_store_dpg(const char* path, const uint32_t* graph, uint32_t n, uint32_t degree);
int tagore_store_cagra(const char* path, const uint32_t* graph, uint32_t n, uint32_t degree);

/* fvecs loader (src/common.cu:6-22): count from the file size, dims from the
 * first record. tagore_load_fvecs_header reports n and dim only. */
int tagore_load_fvecs_header(const char* path, uint32_t* n, uint32_t* dim);
int tagore_load_fvecs(const char* path, float* out, uint32_t n, uint32_t dim);

/* Same as tagore_gnn_descent_host with the FP32 base already on the current
 * device (dev_data). host_data is the same base in host memory: the
 * power-of-ten factor and the centroid are computed from it on host threads,
 * in the reference's order, while the device builds the graph. */
int tagore_gnn_descent_device(const TagoreKnnParams* p, const float* dev_data,
                              const float* host_data, uint32_t n, uint32_t dim,
                              TagoreKnnState* out);

/* Work of later calls on this thread goes to `stream` (a cudaStream_t; NULL
 * restores a private stream per call). Calls still return only when their
 * work has finished. */
int tagore_set_stream(void* stream);

/* Timings of the last build on this thread (milliseconds) and the number of
 * kernels this library launched since the last tagore_reset_counters(). */
typedef struct TagoreTimings {
  double knn_ms, prune_ms, prep_ms, total_ms;
  uint64_t kernel_launches;
} TagoreTimings;
int tagore_last_timings(TagoreTimings* t);
int tagore_reset_counters(void);

/* Per-stage device timing, recorded with CUDA events around each launch on
 * the launching stream while profiling is on. bytes is the stage's
 * algorithmic traffic (rows gathered x row bytes, list and pool traffic). */
typedef struct TagoreStageStat {
  char name[32];
  double ms;
  uint64_t launches;
  uint64_t bytes;
  uint64_t items;
} TagoreStageStat;
int tagore_set_profiling(int on);
int tagore_stage_stats(TagoreStageStat* out, int max, int* count);

/* The learned screen in the last kNN build on this thread: whether it ran,
 * its training steps and loss on the first and last batch, how many
 * iterations it screened, its final per-row count, the miss rate measured on
 * sampled nodes in its last iteration (improving pairs it did not keep) and
 * whether it handed over to the exact join. No counterpart in the reference. */
typedef struct TagoreScreenStats {
  uint32_t used, steps, screened_iters, per_row, fallback, pad_;
  float loss_first, loss_last;
  double last_miss;
  double last_best_kept; /* share of each sampled row's exact best per_row candidates kept */
} TagoreScreenStats;
int tagore_last_screen(TagoreScreenStats* out);

/* Loss and parameter gradients of the screen MLP on a batch, for checking the
 * kernels: rows (n x dim FP16, host), triplets tri (3B row indices a p m,
 * host), params (host, the layout [W1 dim x 128 | b1 128 | W2 128 x 32 | b2
 * 32], FP32); grads receives the same layout. No counterpart in the reference. */
int tagore_mlp_loss_grad(const uint16_t* rows, uint32_t n, uint32_t dim, const uint32_t* tri,
                         uint32_t B, const float* params, float* grads, double* loss);

/* No counterpart in the reference. Checks on the current device that the
 * library's bounded waits end instead of hanging: one block holds TMEM and
 * waits on an mbarrier that nothing ever arrives on, through the same bounded
 * wait as the tensor-core joins (2 s); when the wait runs out it records it,
 * frees the TMEM and returns. *timed_out is 1 when that happened; the device
 * stays usable afterwards. */
int tagore_wait_selftest(int* timed_out);

/* No counterpart in the reference. How many allocations this library has
 * made since it was loaded: device memory from its pools and pinned host
 * buffers. A call that allocates nothing leaves it unchanged. */
uint64_t tagore_allocation_count(void);

/* Frees a device buffer this library allocated (capsule destructor). Like
 * cudaFree it waits for the device's work first. */
int tagore_device_free(void* p);

/* Device memory of states and temporaries comes from a memory pool per
 * device that keeps freed memory for the next build. This returns the
 * current device's cached memory to the system. */
int tagore_trim_cache(void);

const char* tagore_last_error(void);
const char* tagore_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TAGORE_B200_H */
