// capi.cu -- the C ABI (include/tagore_b200.h): argument checks, buffer
// ownership, streams, timings and error reporting around the kernel files.
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"
#include "mlp.cuh"

namespace tagore {

static thread_local std::string g_err;
static thread_local TagoreTimings g_times{};
static thread_local cudaStream_t g_user_stream = nullptr;
static thread_local ScreenStats g_screen{};

void set_screen_stats(const ScreenStats& s) { g_screen = s; }
static std::atomic<uint64_t> g_launches{0};

// ---- stage timing ----
struct StageRec {
  std::string name;
  cudaEvent_t a = nullptr, b = nullptr;
  bool closed = false;
};
static thread_local bool g_prof = false;
static thread_local std::vector<StageRec> g_open;
static thread_local std::vector<TagoreStageStat> g_stats;

static TagoreStageStat& stat_of(const char* name) {
  for (auto& s : g_stats)
    if (std::strncmp(s.name, name, sizeof(s.name)) == 0) return s;
  TagoreStageStat s{};
  std::snprintf(s.name, sizeof(s.name), "%s", name);
  g_stats.push_back(s);
  return g_stats.back();
}

void count_launch(uint32_t n) { g_launches += n; }

// Every device or pinned-host allocation the library makes goes through
// pool_alloc or count_allocation, so this count sees all of them.
static std::atomic<uint64_t> g_allocs{0};
void count_allocation() { ++g_allocs; }
bool profiling() { return g_prof; }

void stage_begin(const char* name, cudaStream_t s) {
  if (!g_prof) return;
  StageRec r;
  r.name = name;
  cudaEventCreate(&r.a);
  cudaEventCreate(&r.b);
  cudaEventRecord(r.a, s);
  g_open.push_back(r);
}

void stage_end(const char* name, cudaStream_t s, uint64_t bytes, uint64_t items) {
  if (!g_prof) return;
  for (auto it = g_open.rbegin(); it != g_open.rend(); ++it)
    if (!it->closed && it->name == name) {
      cudaEventRecord(it->b, s);
      it->closed = true;
      break;
    }
  TagoreStageStat& st = stat_of(name);
  st.launches += 1;
  st.bytes += bytes;
  st.items += items;
}

void stage_add(const char* name, uint64_t bytes, uint64_t items) {
  if (!g_prof) return;
  TagoreStageStat& st = stat_of(name);
  st.bytes += bytes;
  st.items += items;
}

// Resolves recorded events into milliseconds (the stream must be synchronised).
static void stage_flush() {
  for (auto& r : g_open) {
    if (r.closed) {
      float ms = 0.f;
      cudaEventSynchronize(r.b);
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) stat_of(r.name.c_str()).ms += ms;
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_open.clear();
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  const char* base = std::strrchr(file, '/');
  fail(e == cudaErrorMemoryAllocation ? TAGORE_ENOMEM : TAGORE_ECUDA, "%s failed: %s (%s:%d)", what,
       cudaGetErrorString(e), base ? base + 1 : file, line);
  return e == cudaErrorMemoryAllocation ? TAGORE_ENOMEM : TAGORE_ECUDA;
}

// One pool per device, created on first use, with no release threshold: a
// build's states and scratch (several GB at 1M points) are mapped once and
// reused by later builds instead of being unmapped at every synchronisation
// as the default pool does.
static std::mutex g_pool_lock;
static cudaMemPool_t g_pools[64] = {};

static int device_pool(cudaMemPool_t* out) {
  int dev = 0;
  TG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(TAGORE_EINVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> hold(g_pool_lock);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    TG_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;
    TG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return TAGORE_OK;
}

int pool_alloc(void** p, size_t bytes, cudaStream_t s) {
  count_allocation();
  cudaMemPool_t pool = nullptr;
  TG_TRY(device_pool(&pool));
  const cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, s);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
  }
  return TAGORE_OK;
}

void pool_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

namespace {

// The caller's stream (tagore_set_stream) or a non-blocking stream owned by
// one API call.
struct Stream {
  cudaStream_t s = nullptr;
  bool own = false;
  int init() {
    if (g_user_stream) {
      s = g_user_stream;
      return TAGORE_OK;
    }
    TG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    own = true;
    return TAGORE_OK;
  }
  ~Stream() {
    if (s) {
      cudaStreamSynchronize(s);
      stage_flush();
    }
    if (own) cudaStreamDestroy(s);
  }
};

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start(cudaStream_t s) { cudaEventRecord(a, s); }
  double stop(cudaStream_t s) {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
};

size_t buffer_bytes(uint32_t n, uint32_t dim, uint32_t k, int which) {
  switch (which) {
    case 0: return (size_t)n * k * 4;
    case 1: return (size_t)n * 128 * 4;
    case 2: return (size_t)n * dim * 2;
    case 3: return (size_t)n * k * 4;
    case 4: return (size_t)n * 128 * 4;
    case 5: return (size_t)n * 4;
    case 6: return (size_t)dim * 2;
    case 7: return (size_t)n * 128 * 4;
    case 8: return (size_t)n * 4;
    default: return 0;
  }
}

void** slot(TagoreKnnState* st, int which) {
  switch (which) {
    case 0: return &st->graph;
    case 1: return &st->reverse_graph;
    case 2: return &st->data;
    case 3: return &st->nei_distance;
    case 4: return &st->reverse_distance;
    case 5: return &st->reverse_num;
    case 6: return &st->center;
    case 7: return &st->hybrid_list;
    case 8: return &st->norms;
    default: return nullptr;
  }
}

int check_state(const TagoreKnnState* st) {
  if (!st || !st->graph || !st->data || !st->nei_distance || !st->reverse_graph ||
      !st->reverse_distance || !st->reverse_num || !st->center || !st->hybrid_list)
    return fail(TAGORE_EINVAL, "state has missing buffers");
  return TAGORE_OK;
}

int check_prune(const TagorePruneParams* p, TagoreKnnState* st) {
  if (!p) return fail(TAGORE_EINVAL, "null params");
  TG_TRY(check_state(st));
  if (p->k != st->k || p->n != st->n || p->dim != st->dim)
    return fail(TAGORE_EINVAL, "K/POINTS/DIM (%u/%u/%u) differ from the graph's (%u/%u/%u)", p->k,
                p->n, p->dim, st->k, st->n, st->dim);
  return TAGORE_OK;
}

// Builds the state from the FP32 base on the device. The factor and the
// centroid come from host_for_center (the same base in host memory, summed on
// host threads while the device works); with host_for_center null they come
// from `factor` and the device's own sequential centroid.
int build_from_device(const TagoreKnnParams* p, const float* raw_dev, const float* host_for_center,
                      float factor, uint32_t n, uint32_t dim, TagoreKnnState* st, cudaStream_t s) {
  const bool rescale = p->rescale != 0;
  st->norm_factor = host_for_center ? host_factor(host_for_center, dim, rescale) : factor;
  Timer t0;
  t0.start(s);
  TG_TRY(prep_base(raw_dev, n, dim, st->norm_factor, (__half*)st->data, (float*)st->norms, s));
  std::vector<uint16_t> center(dim);
  std::thread cth;
  if (host_for_center)
    cth = std::thread(host_center, host_for_center, n, dim, st->norm_factor, center.data());
  else
    TG_TRY(device_center(raw_dev, n, dim, st->norm_factor, (__half*)st->center, s));
  KnnArgs a{p->k,       p->iters, p->mode,        p->sample,
            p->per_row, p->seed,  p->learn_steps, p->learn_flags};
  KnnStats ks{};
  const auto w0 = std::chrono::steady_clock::now();
  const int rc = knn_build(dev_of(st), (const float*)st->norms, a, &ks, s);
  g_times.knn_ms = t0.stop(s);
  const auto w1 = std::chrono::steady_clock::now();
  if (cth.joinable()) cth.join();
  const auto w2 = std::chrono::steady_clock::now();
  g_times.prep_ms = std::chrono::duration<double, std::milli>(w2 - w1).count();  // centroid wait
  g_times.total_ms = std::chrono::duration<double, std::milli>(w2 - w0).count();
  TG_TRY(rc);
  if (host_for_center)
    TG_CUDA(cudaMemcpyAsync(st->center, center.data(), (size_t)dim * 2, cudaMemcpyHostToDevice, s));
  TG_CUDA(cudaStreamSynchronize(s));
  return TAGORE_OK;
}

}  // namespace
}  // namespace tagore

using namespace tagore;

extern "C" {

const char* tagore_last_error(void) { return g_err.c_str(); }
const char* tagore_version(void) { return "tagore_b200 0.1 (sm_100a)"; }

int tagore_last_timings(TagoreTimings* t) {
  if (!t) return fail(TAGORE_EINVAL, "null timings");
  *t = g_times;
  t->kernel_launches = g_launches.load();
  return TAGORE_OK;
}

uint64_t tagore_allocation_count(void) { return g_allocs.load(); }

int tagore_reset_counters(void) {
  g_launches = 0;
  g_stats.clear();
  return TAGORE_OK;
}

int tagore_set_stream(void* stream) {
  g_user_stream = reinterpret_cast<cudaStream_t>(stream);
  return TAGORE_OK;
}

int tagore_set_profiling(int on) {
  g_prof = on != 0;
  return TAGORE_OK;
}

int tagore_stage_stats(TagoreStageStat* out, int max, int* count) {
  if (!count) return fail(TAGORE_EINVAL, "null count");
  stage_flush();
  const int n = (int)g_stats.size();
  for (int i = 0; i < n && i < max && out; ++i) out[i] = g_stats[i];
  *count = n;
  return TAGORE_OK;
}

size_t tagore_state_bytes(const TagoreKnnState* st, int which) {
  return st ? buffer_bytes(st->n, st->dim, st->k, which) : 0;
}

int tagore_state_alloc(uint32_t n, uint32_t dim, uint32_t k, TagoreKnnState* out) {
  if (!out) return fail(TAGORE_EINVAL, "null state");
  if (n == 0 || dim == 0 || k == 0) return fail(TAGORE_EINVAL, "n, dim and k must be positive");
  std::memset(out, 0, sizeof(*out));
  out->n = n;
  out->dim = dim;
  out->k = k;
  out->norm_factor = 1.0f;
  out->owns = 1;
  cudaGetDevice(&out->device);
  Stream s;
  TG_TRY(s.init());
  for (int w = 0; w <= 8; ++w) {
    void** p = slot(out, w);
    const size_t b = buffer_bytes(n, dim, k, w);
    int rc = pool_alloc(p, b, s.s);
    if (rc == TAGORE_OK) {
      const cudaError_t e = cudaMemsetAsync(*p, 0, b, s.s);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemsetAsync(state)", __FILE__, __LINE__);
    }
    if (rc != TAGORE_OK) {
      cudaStreamSynchronize(s.s);
      tagore_state_free(out);
      return rc;
    }
  }
  TG_CUDA(cudaStreamSynchronize(s.s));  // zero fill done before work on any stream
  return TAGORE_OK;
}

// Buffers go back to the pool once all work on the device has finished, as
// cudaFree would wait for it.
int tagore_device_free(void* p) {
  if (!p) return TAGORE_OK;
  TG_CUDA(cudaDeviceSynchronize());
  TG_CUDA(cudaFreeAsync(p, nullptr));
  return TAGORE_OK;
}

int tagore_state_free(TagoreKnnState* st) {
  if (!st) return TAGORE_OK;
  if (st->owns) {
    cudaDeviceSynchronize();
    for (int w = 0; w <= 8; ++w) {
      void** p = slot(st, w);
      if (*p) cudaFreeAsync(*p, nullptr);
      *p = nullptr;
    }
  }
  st->owns = 0;
  return TAGORE_OK;
}

int tagore_last_screen(TagoreScreenStats* out) {
  if (!out) return fail(TAGORE_EINVAL, "null stats");
  std::memset(out, 0, sizeof(*out));
  out->used = g_screen.used;
  out->steps = g_screen.steps;
  out->screened_iters = g_screen.screened_iters;
  out->per_row = g_screen.per_row;
  out->fallback = g_screen.fallback;
  out->loss_first = g_screen.loss_first;
  out->loss_last = g_screen.loss_last;
  out->last_miss = g_screen.last_miss;
  out->last_best_kept = g_screen.last_best_kept;
  return TAGORE_OK;
}

int tagore_mlp_loss_grad(const uint16_t* rows, uint32_t n, uint32_t dim, const uint32_t* tri,
                         uint32_t B, const float* params, float* grads, double* loss) {
  if (!rows || !tri || !params || !grads || !loss || n == 0 || B == 0 || dim == 0)
    return fail(TAGORE_EINVAL, "bad screen-gradient arguments");
  for (size_t i = 0; i < (size_t)3 * B; ++i)
    if (tri[i] >= n) return fail(TAGORE_EINVAL, "triplet row %u >= %u", tri[i], n);
  Stream s;
  TG_TRY(s.init());
  Scratch dev(s.s), work(s.s);
  TG_TRY(dev.alloc((size_t)n * dim * 2 + (size_t)3 * B * 4 + 16));
  __half* x = dev.as<__half>();
  uint32_t* t = reinterpret_cast<uint32_t*>(x + (size_t)n * dim + ((size_t)n * dim & 1));
  TG_CUDA(cudaMemcpyAsync(x, rows, (size_t)n * dim * 2, cudaMemcpyHostToDevice, s.s));
  TG_CUDA(cudaMemcpyAsync(t, tri, (size_t)3 * B * 4, cudaMemcpyHostToDevice, s.s));
  mlp::Net net;
  TG_TRY(net.init(dim, 1, s.s));
  TG_TRY(net.set_params(params, s.s));
  TG_TRY(net.loss_grad(t, B, x, work, loss, s.s));
  TG_TRY(net.get(nullptr, grads, s.s));
  return TAGORE_OK;
}

int tagore_trim_cache(void) {
  cudaMemPool_t pool = nullptr;
  TG_TRY(device_pool(&pool));
  TG_CUDA(cudaDeviceSynchronize());
  TG_CUDA(cudaMemPoolTrimTo(pool, 0));
  return TAGORE_OK;
}

int tagore_state_upload(TagoreKnnState* st, int which, const void* host, size_t bytes) {
  if (!st || !host || which < 0 || which > 8 || !*slot(st, which))
    return fail(TAGORE_EINVAL, "bad upload arguments");
  if (bytes > buffer_bytes(st->n, st->dim, st->k, which))
    return fail(TAGORE_EINVAL, "upload of %zu bytes exceeds buffer %d", bytes, which);
  TG_CUDA(cudaMemcpy(*slot(st, which), host, bytes, cudaMemcpyHostToDevice));
  return TAGORE_OK;
}

int tagore_state_download(const TagoreKnnState* st, int which, void* host, size_t bytes) {
  if (!st || !host || which < 0 || which > 8)
    return fail(TAGORE_EINVAL, "bad download arguments");
  void* p = *slot(const_cast<TagoreKnnState*>(st), which);
  if (!p) return fail(TAGORE_EINVAL, "buffer %d is not allocated", which);
  if (bytes > buffer_bytes(st->n, st->dim, st->k, which))
    return fail(TAGORE_EINVAL, "download of %zu bytes exceeds buffer %d", bytes, which);
  TG_CUDA(cudaMemcpy(host, p, bytes, cudaMemcpyDeviceToHost));
  return TAGORE_OK;
}

int tagore_gnn_descent_host(const TagoreKnnParams* p, const float* data, uint32_t n, uint32_t dim,
                            TagoreKnnState* out) {
  if (!p || !data || !out) return fail(TAGORE_EINVAL, "null argument");
  if (dim != p->dim) return fail(TAGORE_EINVAL, "DIM %u differs from the data's %u", p->dim, dim);
  if (dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", dim);
  if (p->k == 0 || p->k >= n) return fail(TAGORE_EINVAL, "need POINTS > K >= 1");
  Stream st;
  TG_TRY(st.init());
  TG_TRY(tagore_state_alloc(n, dim, p->k, out));
  float* raw = nullptr;
  int rc = pool_alloc((void**)&raw, (size_t)n * dim * 4, st.s);
  if (rc != TAGORE_OK) {
    tagore_state_free(out);
    return rc;
  }
  const cudaError_t e = cudaMemcpyAsync(raw, data, (size_t)n * dim * 4, cudaMemcpyHostToDevice, st.s);
  if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpyAsync(raw)", __FILE__, __LINE__);
  if (rc == TAGORE_OK) rc = build_from_device(p, raw, data, 1.0f, n, dim, out, st.s);
  pool_free(raw, st.s);
  cudaStreamSynchronize(st.s);
  if (rc != TAGORE_OK) tagore_state_free(out);
  return rc;
}

int tagore_gnn_descent_device(const TagoreKnnParams* p, const float* dev_data,
                              const float* host_data, uint32_t n, uint32_t dim,
                              TagoreKnnState* out) {
  if (!p || !dev_data || !host_data || !out) return fail(TAGORE_EINVAL, "null argument");
  if (dim != p->dim) return fail(TAGORE_EINVAL, "DIM %u differs from the data's %u", p->dim, dim);
  if (dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", dim);
  if (p->k == 0 || p->k >= n) return fail(TAGORE_EINVAL, "need POINTS > K >= 1");
  Stream st;
  TG_TRY(st.init());
  TG_TRY(tagore_state_alloc(n, dim, p->k, out));
  const int rc = build_from_device(p, dev_data, host_data, 1.0f, n, dim, out, st.s);
  if (rc != TAGORE_OK) tagore_state_free(out);
  return rc;
}

// GNN_descent's file path (pybind.cu:19-105) with the parsing on the device:
// the file streams through pinned chunks, the device strips each record's
// count and checks it, and the factor, FP16 base, norms and centroid are made
// on the device.
int tagore_gnn_descent(const TagoreKnnParams* p, const char* fvecs_path, TagoreKnnState* out) {
  if (!p || !fvecs_path || !out) return fail(TAGORE_EINVAL, "null argument");
  uint32_t n = 0, dim = 0;
  TG_TRY(tagore_load_fvecs_header(fvecs_path, &n, &dim));
  if (dim != p->dim) return fail(TAGORE_EINVAL, "file DIM %u differs from DIM %u", dim, p->dim);
  if (dim % 4) return fail(TAGORE_EINVAL, "DIM must be a multiple of 4 (got %u)", dim);
  if (p->k == 0 || p->k >= n) return fail(TAGORE_EINVAL, "need POINTS > K >= 1");
  Stream st;
  TG_TRY(st.init());
  TG_TRY(tagore_state_alloc(n, dim, p->k, out));
  float* raw = nullptr;
  float factor = 1.0f;
  int rc = pool_alloc((void**)&raw, (size_t)n * dim * 4, st.s);
  if (rc == TAGORE_OK) rc = ingest_fvecs(fvecs_path, n, dim, p->rescale != 0, raw, &factor, st.s);
  if (rc == TAGORE_OK) rc = build_from_device(p, raw, nullptr, factor, n, dim, out, st.s);
  if (raw) pool_free(raw, st.s);
  cudaStreamSynchronize(st.s);
  if (rc != TAGORE_OK) tagore_state_free(out);
  return rc;
}

int tagore_connect(TagoreKnnState* st, uint32_t ep, uint64_t* added) {
  TG_TRY(check_state(st));
  Stream s;
  TG_TRY(s.init());
  return connect_graph(dev_of(st), ep, added, s.s);
}

int tagore_entry_point(TagoreKnnState* st, uint32_t topm, uint32_t* ep) {
  TG_TRY(check_state(st));
  if (!ep || topm == 0) return fail(TAGORE_EINVAL, "bad entry-point arguments");
  Stream s;
  TG_TRY(s.init());
  return stage_cal_ep(dev_of(st), topm, ep, s.s);
}

int tagore_wait_selftest(int* timed_out) {
  if (!timed_out) return fail(TAGORE_EINVAL, "null argument");
  Stream s;
  TG_TRY(s.init());
  return knn::wait_selftest(timed_out, s.s);
}

int tagore_search(const TagoreSearchParams* p, const float* base, uint64_t n, uint32_t dim,
                  const uint64_t* offs, const uint32_t* adj, uint64_t edges, uint32_t ep,
                  const float* queries, uint32_t nq, uint32_t* out, void* stream) {
  if (!p) return fail(TAGORE_EINVAL, "null search parameters");
  TG_TRY(search_check(*p, base, n, dim, offs, adj, edges, ep, queries, nq, out));
  if (nq == 0) return TAGORE_OK;
  if (stream) return greedy_search(*p, base, n, dim, offs, adj, edges, ep, queries, nq, out,
                                   static_cast<cudaStream_t>(stream));
  Stream s;
  TG_TRY(s.init());
  return greedy_search(*p, base, n, dim, offs, adj, edges, ep, queries, nq, out, s.s);
}

int tagore_pruning_cfs(const TagorePruneParams* p, TagoreKnnState* st, const char* mode,
                       const char* metric) {
  TG_TRY(check_prune(p, st));
  if (!mode || !metric) return fail(TAGORE_EINVAL, "null mode/metric");
  Stream s;
  TG_TRY(s.init());
  Timer t;
  t.start(s.s);
  PruneArgs a{p->final_degree, p->topm, p->thre};
  uint32_t ep = 0;
  TG_TRY(prune_cfs(dev_of(st), a, mode, metric, &ep, s.s));
  g_times.prune_ms = t.stop(s.s);
  st->ep = ep;
  return TAGORE_OK;
}

// For callers that may not allocate device memory while they prune: a
// serving process that has handed all of HBM to its own arena (resident
// shards, caches) where a library allocation would fail or grow a pool
// behind the arena's back, and code that must not synchronise the device the
// way cudaFree can. The temporaries live in one static device array per
// device; the lock keeps calls from overlapping on it.
int tagore_pruning_cfs_noalloc(const TagorePruneParams* p, TagoreKnnState* st, const char* mode,
                               const char* metric, void* stream) {
  static std::mutex lock;
  TG_TRY(check_prune(p, st));
  if (!mode || !metric) return fail(TAGORE_EINVAL, "null mode/metric");
  std::lock_guard<std::mutex> hold(lock);
  PruneArgs a{p->final_degree, p->topm, p->thre};
  uint32_t ep = 0;
  TG_TRY(prune_cfs_static(dev_of(st), a, mode, metric, &ep, static_cast<cudaStream_t>(stream)));
  st->ep = ep;
  return TAGORE_OK;
}

int tagore_pruning(const TagorePruneParams* p, TagoreKnnState* st, const char* index_type,
                   const char* index_path) {
  TG_TRY(check_prune(p, st));
  if (!index_type) return fail(TAGORE_EINVAL, "null index_type");
  const std::string type(index_type);
  Stream s;
  TG_TRY(s.init());
  Timer t;
  t.start(s.s);
  PruneArgs a{p->final_degree, p->topm, p->thre};
  uint32_t ep = 0;
  TG_TRY(prune_index(dev_of(st), a, type, &ep, s.s));
  g_times.prune_ms = t.stop(s.s);
  st->ep = ep;
  if (!index_path || !*index_path) return TAGORE_OK;
  const uint32_t n = st->n, K = st->k, d = p->final_degree;
  std::vector<uint32_t> rows((size_t)n * K);
  TG_CUDA(cudaMemcpy(rows.data(), st->graph, rows.size() * 4, cudaMemcpyDeviceToHost));
  if (type == "NSG") return tagore_store_nsg(index_path, rows.data(), d, ep, n, K);
  if (type == "Vamana") return tagore_store_vamana(index_path, rows.data(), ep, n, K);
  if (type == "NSSG") return tagore_store_nssg(index_path, rows.data(), d, n, K);
  if (type == "CAGRA") return tagore_store_cagra(index_path, rows.data(), n, d);
  return tagore_store_dpg(index_path, rows.data(), n, d);
}

int tagore_build_index_host(const TagoreKnnParams* p, const float* data, uint32_t n, uint32_t dim,
                            uint32_t final_degree, uint32_t topm, float thre, uint32_t* out_graph,
                            uint32_t* ep_out) {
  if (!out_graph) return fail(TAGORE_EINVAL, "null output");
  TagoreKnnState st{};
  TG_TRY(tagore_gnn_descent_host(p, data, n, dim, &st));
  TagorePruneParams pp{p->k, n, dim, final_degree, topm, thre};
  int rc = tagore_pruning_cfs(&pp, &st, "path", "dist");
  if (rc == TAGORE_OK) {
    cudaError_t e = cudaMemcpy(out_graph, st.graph, (size_t)n * p->k * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpy(graph)", __FILE__, __LINE__);
    if (ep_out) *ep_out = st.ep;
  }
  tagore_state_free(&st);
  return rc;
}

int tagore_large_merge(const TagoreLargeParams* p, const uint32_t* const* local_rows,
                       const uint32_t* local_medoids) {
  if (!p || !local_rows || !local_medoids) return fail(TAGORE_EINVAL, "null argument");
  LargeBuildFn given = [&](const TagoreLargeParams& q, uint32_t, uint32_t cid,
                           const std::vector<uint32_t>& ids, const float*, uint32_t*,
                           LocalRows& rows, uint32_t* medoid) -> int {
    if (!local_rows[cid]) return fail(TAGORE_EINVAL, "no local graph for cluster %u", cid);
    rows.assign(local_rows[cid], local_rows[cid] + ids.size() * (size_t)q.k);
    *medoid = local_medoids[cid];
    return TAGORE_OK;
  };
  // Four builder threads hand the given graphs to the merger: the schedule of
  // a multi-device run, whose merged bytes must not depend on it.
  const uint32_t workers[4] = {0, 0, 0, 0};
  return large_index_run(*p, workers, 4, given);
}

int tagore_large_index(const TagoreLargeParams* p, const uint32_t* devices, int ndev) {
  if (!p || !devices) return fail(TAGORE_EINVAL, "null argument");
  // gpu_construct (src/large_index.cu:130-279) for one cluster: read
  // [u32 n][n x dim f32], kNN graph without rescale, CFS path/dist prune with
  // alpha = thre, rows back to the host with local ids mapped to global ones.
  // The cluster file [u32 n][n x dim f32] into pinned memory, on the
  // builder's reader thread.
  LargeLoadFn load = [](const TagoreLargeParams& q, uint32_t cid, size_t n, float* dst) -> int {
    const std::string path = std::string(q.data_prefix) + std::to_string(cid);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(TAGORE_EIO, "cannot open cluster file '%s'", path.c_str());
    uint32_t n_file = 0;
    const size_t cnt = n * q.dim;
    const bool ok = std::fread(&n_file, 4, 1, f) == 1 && std::fread(dst, 4, cnt, f) == cnt;
    std::fclose(f);
    if (!ok) return fail(TAGORE_EIO, "'%s' holds fewer than %zu vectors", path.c_str(), n);
    return TAGORE_OK;
  };
  LargeBuildFn build = [devices](const TagoreLargeParams& q, uint32_t worker, uint32_t cid,
                                 const std::vector<uint32_t>& ids, const float* x,
                                 uint32_t* stage, LocalRows& rows, uint32_t* medoid) -> int {
    TG_CUDA(cudaSetDevice((int)devices[worker]));
    const uint32_t n = (uint32_t)ids.size(), dim = q.dim;
    TagoreKnnParams kp{};
    kp.k = q.k;
    kp.n = n;
    kp.dim = dim;
    kp.iters = q.knn_iters ? q.knn_iters : 16;
    kp.mode = q.mode;
    kp.rescale = 0;
    kp.seed = 0x7A6Eull + cid;
    TagoreKnnState st{};
    TG_TRY(tagore_gnn_descent_host(&kp, x, n, dim, &st));
    TagorePruneParams pp{q.k, n, dim, q.final_degree, q.topm, q.thre};
    int rc = tagore_pruning_cfs(&pp, &st, "path", "dist");
    // The rows come back in one contiguous copy into the builder's pinned
    // buffer and are mapped to global ids on their way into the stride-K
    // rows; a pruned row holds at most min(final_degree, K - 1) ids.
    const uint32_t W = std::min(q.final_degree, q.k - 1) + 1;
    if (rc == TAGORE_OK) {
      cudaError_t e = cudaMemcpy(stage, st.graph, (size_t)n * q.k * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpy(cluster rows)", __FILE__, __LINE__);
      *medoid = ids[st.ep];
    }
    tagore_state_free(&st);
    TG_TRY(rc);
    rows.resize((size_t)n * q.k);
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t* src = stage + (size_t)i * q.k;
      uint32_t* r = rows.data() + (size_t)i * q.k;
      const uint32_t deg = src[0];
      if (deg >= W) return fail(TAGORE_ECUDA, "cluster %u row %u holds %u ids (> %u)", cid, i, deg, W - 1);
      r[0] = deg;
      for (uint32_t j = 1; j <= deg; ++j) r[j] = ids[src[j]];
    }
    return TAGORE_OK;
  };
  return large_index_run(*p, devices, ndev, build, load);
}

}  // extern "C"
