// large_index.cpp -- largeIndex (pybind.cu:298-391,
// src/large_index.cu): every point sits in two clusters; each cluster's local
// graph is built on the GPU (kNN graph without rescale, CFS path prune with
// alpha = thre), remapped to global ids and handed to a host merger that keeps
// `buffer_size` local graphs in memory, merges the two copies of a point when
// both are resident, spills evicted local graphs to local_prefix + cid, and
// finally streams the DiskANN-style index.
//
// Two builder threads per entry of the device list (one when the local
// graphs are given) take the clusters in the merger's order from a shared
// counter, so uneven clusters balance over the devices as they come (the
// reference deals them round-robin, src/large_index.cu:175); the builders run
// at most two clusters per builder ahead of the merger (a host thread). Every wait between them is bounded and
// ends in TAGORE_ETIMEOUT. The merged bytes equal a sequential run of the reference's
// merger (order_merge_new, :286-522) over the same local graphs.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace tagore {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// Greedy cluster order of reorder() (src/large_index.cu:9-83, "Algorithm 4"):
// fill the buffer with the clusters overlapping most with those already
// chosen, then repeatedly pick the cluster and the slot whose eviction keeps
// the largest overlap. Defined here where the reference reads an unset index
// (no positive overlap anywhere): the smallest unchosen cluster, slot 0.
void cluster_order(const std::vector<uint32_t>& inter, uint32_t C, uint32_t bs,
                   std::vector<uint32_t>& order, std::vector<uint32_t>& position) {
  order.clear();
  position.assign(C, 0);
  std::vector<uint8_t> visited(C, 0);
  std::vector<uint32_t> buffer;
  order.push_back(0);
  visited[0] = 1;
  buffer.push_back(0);
  position[0] = 0;
  auto first_free = [&]() {
    for (uint32_t j = 0; j < C; ++j)
      if (!visited[j]) return j;
    return kNone;
  };
  for (uint32_t i = 1; i < bs; ++i) {
    uint64_t max_sum = 0;
    uint32_t max_id = kNone;
    for (uint32_t j = 0; j < C; ++j) {
      if (visited[j]) continue;
      uint64_t t = 0;
      for (uint32_t r : order) t += inter[(size_t)j * C + r];
      if (t > max_sum) {
        max_sum = t;
        max_id = j;
      }
    }
    if (max_id == kNone) max_id = first_free();
    order.push_back(max_id);
    buffer.push_back(max_id);
    position[max_id] = i;
    visited[max_id] = 1;
  }
  for (uint32_t i = 0; i + bs < C; ++i) {
    uint64_t max_sum = 0;
    uint32_t max_id = kNone, max_evict = 0;
    for (uint32_t j = 0; j < C; ++j) {
      if (visited[j]) continue;
      uint64_t total = 0;
      for (uint32_t k = 0; k < bs; ++k) total += inter[(size_t)j * C + buffer[k]];
      uint64_t best = 0;
      uint32_t best_k = kNone;
      for (uint32_t k = 0; k < bs; ++k) {
        const uint64_t t = total - inter[(size_t)j * C + buffer[k]];  // all slots but k
        if (t > best) {
          best = t;
          best_k = k;
        }
      }
      if (best > max_sum) {
        max_sum = best;
        max_id = j;
        max_evict = best_k;
      }
    }
    if (max_id == kNone) {
      max_id = first_free();
      max_evict = 0;
    }
    buffer[max_evict] = max_id;
    order.push_back(max_id);
    visited[max_id] = 1;
    position[max_id] = max_evict;
  }
}

// Membership of the up to 2K ids of two rows without an N-sized array: open
// addressing over at least 4K slots (load <= 1/2), cleared in O(1) by a
// generation tag.
struct IdSet {
  std::vector<uint32_t> key, tag;
  uint32_t mask = 0, shift = 0, gen = 0;
  explicit IdSet(uint32_t K) {
    uint32_t bits = 6;
    while ((1u << bits) < 4u * K) ++bits;
    key.assign(1u << bits, 0);
    tag.assign(1u << bits, 0);
    mask = (1u << bits) - 1u;
    shift = 32 - bits;
  }
  void clear() {
    if (++gen == 0) {  // the tags wrapped: reset them once
      std::fill(tag.begin(), tag.end(), 0u);
      gen = 1;
    }
  }
  // Inserts id; false if it was already there.
  bool insert(uint32_t id) {
    uint32_t h = (id * 0x9E3779B1u) >> shift;
    while (tag[h] == gen) {
      if (key[h] == id) return false;
      h = (h + 1) & mask;
    }
    tag[h] = gen;
    key[h] = id;
    return true;
  }
};

struct Built {
  LocalRows rows;  // n x K, [deg, global ids...]
  uint32_t medoid = 0;
  bool ready = false;
};

struct Shared {
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Built> built;  // by processing index
  uint32_t consumed = 0;     // clusters the merger has taken
  int error = TAGORE_OK;
  std::string msg;
};

bool wait_for(Shared& sh, std::unique_lock<std::mutex>& lk, const std::function<bool()>& pred) {
  return sh.cv.wait_for(lk, std::chrono::seconds(1800), [&] { return pred() || sh.error; });
}

struct Writer {
  FILE* f = nullptr;
  std::vector<char> buf;
  explicit Writer(const std::string& p) {
    f = std::fopen(p.c_str(), "wb");
    if (f) {
      buf.resize(8u << 20);
      std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    }
  }
  bool put(const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }
  bool close() {
    const bool ok = f && std::fclose(f) == 0;
    f = nullptr;
    return ok;
  }
  ~Writer() {
    if (f) std::fclose(f);
  }
};

struct Reader {
  FILE* f = nullptr;
  std::vector<char> buf;
  bool open(const std::string& p, size_t buffer = 1u << 20, uint64_t at = 0) {
    f = std::fopen(p.c_str(), "rb");
    if (f) {
      buf.resize(buffer);
      std::setvbuf(f, buf.data(), _IOFBF, buf.size());
      if (at && std::fseek(f, (long)at, SEEK_SET) != 0) {
        std::fclose(f);
        f = nullptr;
      }
    }
    return f != nullptr;
  }
  bool get(void* p, size_t n) { return n == 0 || std::fread(p, 1, n, f) == n; }
  ~Reader() {
    if (f) std::fclose(f);
  }
};

// The merger of order_merge_new (src/large_index.cu:286-522), sequentially.
int merge_all(const TagoreLargeParams& p, const std::vector<std::vector<uint32_t>>& clusters,
              const std::vector<uint32_t>& centers, const std::vector<uint32_t>& second,
              const std::vector<uint32_t>& order, const std::vector<uint32_t>& position,
              Shared& sh) {
  const uint32_t C = (uint32_t)clusters.size(), N = p.num, K = p.k, bs = p.buffer_size;
  const uint32_t maxd = p.max_degree;
  std::vector<LocalRows> pool(bs);
  std::vector<uint32_t> buffer(bs, kNone), pointers(N, 0), medoids(C, 0);
  std::vector<uint8_t> visited(N, 0), node_set(N, 0), cached(N, 0);
  std::vector<uint32_t> nhood;
  // The final pass runs over point ranges [lo(r), lo(r + 1)) in parallel;
  // spill() records where each range starts in each local index file
  // (members are in ascending global id).
  const uint32_t R = std::max(1u, std::min({16u, std::thread::hardware_concurrency(),
                                            N / 4096u + 1u}));
  auto lo = [&](uint32_t r) { return (uint32_t)((uint64_t)r * N / R); };
  std::vector<uint64_t> part_off((size_t)C * (R + 1), 0);
  auto take = [&](uint32_t i) -> int {
    std::unique_lock<std::mutex> lk(sh.mu);
    if (!wait_for(sh, lk, [&] { return sh.built[i].ready; }))
      return fail(TAGORE_ETIMEOUT, "largeIndex: cluster %u was not built in time", order[i]);
    if (sh.error) return sh.error;
    pool[position[order[i]]].swap(sh.built[i].rows);
    medoids[i] = sh.built[i].medoid;
    sh.consumed = i + 1;
    sh.cv.notify_all();
    return TAGORE_OK;
  };
  auto row = [&](uint32_t cid, uint32_t j) { return pool[position[cid]].data() + (size_t)j * K; };
  auto spill = [&](uint32_t cid) -> int {
    Writer w(std::string(p.local_prefix) + std::to_string(cid));
    if (!w.f) return fail(TAGORE_EIO, "cannot create local index for cluster %u", cid);
    uint64_t* offs = part_off.data() + (size_t)cid * (R + 1);
    uint64_t at = 0;
    uint32_t part = 0;
    for (uint32_t j = 0; j < clusters[cid].size(); ++j) {
      const uint32_t* r = row(cid, j);
      while (part < R && clusters[cid][j] >= lo(part)) offs[part++] = at;
      if (!w.put(r, 4) || !w.put(r + 1, 4ull * r[0]))
        return fail(TAGORE_EIO, "write of local index %u failed", cid);
      at += 4ull * (1 + r[0]);
      visited[clusters[cid][j]] = 1;
      pointers[clusters[cid][j]] = kNone;
    }
    while (part <= R) offs[part++] = at;
    if (!w.close()) return fail(TAGORE_EIO, "write of local index %u failed", cid);
    return TAGORE_OK;
  };
  TG_TRY(take(0));
  for (uint32_t j = 0; j < clusters[order[0]].size(); ++j) {
    visited[clusters[order[0]][j]] = 1;
    pointers[clusters[order[0]][j]] = j;
  }
  buffer[0] = order[0];
  for (uint32_t i = 1; i < C; ++i) {
    TG_TRY(take(i));
    const uint32_t cur = order[i];
    for (uint32_t j = 0; j < clusters[cur].size(); ++j) {
      const uint32_t node = clusters[cur][j];
      if (!visited[node]) {
        visited[node] = 1;
        pointers[node] = j;
        continue;
      }
      if (pointers[node] == kNone) continue;  // the other copy went to disk
      const uint32_t ano = centers[node] == cur ? second[node] : centers[node];
      uint32_t* old_r = row(ano, pointers[node]);
      uint32_t* new_r = row(cur, j);
      // the copy in the point's first cluster goes first (:332-368)
      const uint32_t* first = centers[node] != cur ? old_r : new_r;
      const uint32_t* then = centers[node] != cur ? new_r : old_r;
      nhood.clear();
      for (uint32_t k = 1; k <= first[0]; ++k) {
        node_set[first[k]] = 1;
        nhood.push_back(first[k]);
      }
      for (uint32_t k = 1; k <= then[0]; ++k)
        if (!node_set[then[k]]) {
          node_set[then[k]] = 1;
          nhood.push_back(then[k]);
        }
      const uint32_t deg = std::min<uint32_t>((uint32_t)nhood.size(), maxd);
      for (uint32_t k = 1; k <= deg; ++k) old_r[k] = nhood[k - 1];
      old_r[0] = deg;
      new_r[0] = 0;
      for (uint32_t v : nhood) node_set[v] = 0;
      cached[node] = 1;
    }
    buffer[position[cur]] = cur;
    if (i + 1 >= bs && i + 1 < C) {
      const uint32_t evict = buffer[position[order[i + 1]]];
      if (evict != kNone) TG_TRY(spill(evict));
    }
  }
  for (uint32_t s = 0; s < bs; ++s)
    if (buffer[s] != kNone) TG_TRY(spill(buffer[s]));
  pool.clear();

  // Final merge into the index file (:447-520). Point i's record comes
  // from the local indexes of its two clusters, read in member order; each
  // range of points is merged by its own thread from its own file positions
  // into its own buffer, and the buffers are written in order.
  std::vector<std::vector<uint32_t>> part_out(R);
  std::vector<int> part_rc(R, TAGORE_OK);
  std::vector<std::string> part_msg(R);  // the library's error text is per thread
  auto final_part = [&](uint32_t r) {
    std::vector<Reader> shard(C);
    IdSet seen(K);
    std::vector<uint32_t> a(K), b(K), nh;
    std::vector<uint32_t>& o = part_out[r];
    auto reader = [&](uint32_t c) -> Reader* {
      if (!shard[c].f &&
          !shard[c].open(std::string(p.local_prefix) + std::to_string(c), 64u << 10,
                         part_off[(size_t)c * (R + 1) + r]))
        return nullptr;
      return &shard[c];
    };
    for (uint32_t i = lo(r); i < lo(r + 1); ++i) {
      Reader* f1 = reader(centers[i]);
      Reader* f2 = reader(second[i]);
      if (!f1 || !f2) {
        part_rc[r] = fail(TAGORE_EIO, "cannot open local index of cluster %u",
                          f1 ? second[i] : centers[i]);
        part_msg[r] = tagore_last_error();
        return;
      }
      uint32_t d1 = 0, d2 = 0;
      bool ok;
      if (cached[i]) {
        Reader* src = f1;
        ok = f1->get(&d1, 4);
        if (ok && d1 == 0) {
          src = f2;
          ok = f2->get(&d1, 4);
        } else if (ok) {
          ok = f2->get(&d2, 4);
        }
        ok = ok && d1 <= K && src->get(a.data(), 4ull * d1);
        if (ok) {
          o.push_back(d1);
          o.insert(o.end(), a.begin(), a.begin() + d1);
        }
      } else {
        ok = f1->get(&d1, 4) && d1 <= K && f1->get(a.data(), 4ull * d1) && f2->get(&d2, 4) &&
             d2 <= K && f2->get(b.data(), 4ull * d2);
        if (ok) {
          nh.clear();
          seen.clear();
          for (uint32_t j = 0; j < d1; ++j) {  // the first row whole, as the reference
            seen.insert(a[j]);
            nh.push_back(a[j]);
          }
          for (uint32_t j = 0; j < d2; ++j)
            if (seen.insert(b[j])) nh.push_back(b[j]);
          const uint32_t deg = std::min<uint32_t>((uint32_t)nh.size(), maxd);
          o.push_back(deg);
          o.insert(o.end(), nh.begin(), nh.begin() + deg);
        }
      }
      if (!ok) {
        part_rc[r] = fail(TAGORE_EIO, "reading the local indexes failed (point %u)", i);
        part_msg[r] = tagore_last_error();
        return;
      }
    }
  };
  {
    std::vector<std::thread> th;
    for (uint32_t r = 1; r < R; ++r) th.emplace_back(final_part, r);
    final_part(0);
    for (auto& t : th) t.join();
  }
  for (uint32_t r = 0; r < R; ++r)
    if (part_rc[r] != TAGORE_OK) return fail(part_rc[r], "%s", part_msg[r].c_str());
  Writer out(p.index_store_path);
  if (!out.f) return fail(TAGORE_EIO, "cannot create '%s'", p.index_store_path);
  uint64_t index_size = 0;
  bool ok = out.put(&index_size, 8) && out.put(&maxd, 4) && out.put(&maxd, 4) && out.put(&index_size, 8);
  for (uint32_t r = 0; ok && r < R; ++r) {
    ok = out.put(part_out[r].data(), part_out[r].size() * 4);
    index_size += part_out[r].size() * 4ull;
    std::vector<uint32_t>().swap(part_out[r]);
  }
  if (!ok) return fail(TAGORE_EIO, "writing '%s' failed", p.index_store_path);
  index_size += 24;
  // header: size, max degree, medoid of the last cluster built (:516-519)
  if (std::fflush(out.f) != 0 || std::fseek(out.f, 0, SEEK_SET) != 0 || !out.put(&index_size, 8) ||
      !out.put(&maxd, 4) || !out.put(&medoids[C - 1], 4) || !out.close())
    return fail(TAGORE_EIO, "write to '%s' failed", p.index_store_path);
  return TAGORE_OK;
}

}  // namespace

int large_index_run(const TagoreLargeParams& p, const uint32_t* dev_list, int ndev,
                    const LargeBuildFn& build, const LargeLoadFn& load) {
  if (!p.data_prefix || !p.local_prefix || !p.index_store_path || !p.centers_path)
    return fail(TAGORE_EINVAL, "largeIndex: null path");
  if (ndev < 1 || ndev > 64 || !dev_list)
    return fail(TAGORE_EINVAL, "largeIndex: devicelist must hold 1 to 64 device ids");
  const uint32_t C = p.cluster_num, N = p.num;
  if (C == 0 || N == 0 || p.buffer_size == 0 || p.k == 0 || p.max_degree == 0 || p.max_degree >= p.k)
    return fail(TAGORE_EINVAL, "largeIndex: need clusters, points, buffer_size > 0 and max_degree < K");
  FILE* f = std::fopen(p.centers_path, "rb");
  if (!f) return fail(TAGORE_EIO, "cannot open '%s'", p.centers_path);
  std::vector<uint32_t> cc((size_t)N * 2);
  const size_t got = std::fread(cc.data(), 4, cc.size(), f);
  std::fclose(f);
  if (got != cc.size()) return fail(TAGORE_EIO, "'%s' holds fewer than %u center pairs", p.centers_path, N);
  std::vector<uint32_t> centers(N), second(N);
  std::vector<std::vector<uint32_t>> clusters(C);
  for (uint32_t i = 0; i < N; ++i) {
    centers[i] = cc[2 * i];
    second[i] = cc[2 * i + 1];
    if (centers[i] >= C || second[i] >= C) return fail(TAGORE_EINVAL, "point %u names a cluster >= %u", i, C);
  }
  for (uint32_t i = 0; i < N; ++i) {
    clusters[centers[i]].push_back(i);
    clusters[second[i]].push_back(i);
  }
  for (uint32_t c = 0; c < C; ++c) {
    if (clusters[c].size() > p.max_points)
      return fail(TAGORE_EINVAL,
                  "cluster %u holds %zu points > max_points %u (the reference splits it into "
                  "clusters that have no data file)",
                  c, clusters[c].size(), p.max_points);
    if (clusters[c].size() <= p.k)
      return fail(TAGORE_EINVAL, "cluster %u holds %zu points, not more than K = %u", c,
                  clusters[c].size(), p.k);
  }
  std::vector<uint32_t> inter((size_t)C * C, 0);  // order_merge_main (:86-106)
  for (uint32_t i = 0; i < N; ++i) {
    ++inter[(size_t)centers[i] * C + second[i]];
    ++inter[(size_t)second[i] * C + centers[i]];
  }
  TagoreLargeParams q = p;
  q.buffer_size = std::min(p.buffer_size, C);
  std::vector<uint32_t> order, position;
  cluster_order(inter, C, q.buffer_size, order, position);

  Shared sh;
  sh.built.resize(C);
  int merge_rc = TAGORE_OK;
  std::string merge_msg;
  std::thread merger([&]() {
    merge_rc = merge_all(q, clusters, centers, second, order, position, sh);
    if (merge_rc != TAGORE_OK) merge_msg = tagore_last_error();
    std::lock_guard<std::mutex> g(sh.mu);
    if (merge_rc != TAGORE_OK && !sh.error) sh.error = merge_rc;
    sh.cv.notify_all();
  });
  // With a load function (clusters built on devices), two builders share each
  // device entry: while one copies its rows back and maps them to global
  // ids, the other's kernels keep the device busy.
  const uint32_t per_device = load ? 2u : 1u;
  const uint32_t workers = (uint32_t)ndev * per_device;
  const uint32_t ahead = 2 * workers;  // clusters claimed but not yet merged
  uint32_t next = 0;                   // next cluster (merge order) to hand out, under sh.mu
  size_t largest = 0;
  for (uint32_t c = 0; c < C; ++c) largest = std::max(largest, clusters[c].size());
  auto record = [&](int rc) {  // under sh.mu: the first error wins, with its message
    if (rc != TAGORE_OK && !sh.error) {
      sh.error = rc;
      sh.msg = tagore_last_error();
    }
  };
  // The next cluster if the merger window has room now (no wait).
  auto try_claim = [&](uint32_t* out) -> bool {
    std::lock_guard<std::mutex> g(sh.mu);
    if (sh.error || next >= C || sh.consumed + ahead <= next) return false;
    *out = next++;
    return true;
  };
  auto claim = [&](uint32_t* out) -> bool {
    std::unique_lock<std::mutex> lk(sh.mu);
    if (!wait_for(sh, lk, [&] { return next >= C || sh.consumed + ahead > next; })) {
      if (!sh.error) {
        sh.error = TAGORE_ETIMEOUT;
        sh.msg = "largeIndex: merger stalled";
      }
      sh.cv.notify_all();
      return false;
    }
    if (sh.error || next >= C) return false;
    *out = next++;
    return true;
  };
  // A reader thread fills one pinned buffer with a cluster's vectors while
  // the builder works on the other.
  struct Prefetch {
    std::thread t;
    int rc = TAGORE_OK;
    std::string msg;
    void start(const LargeLoadFn& fn, const TagoreLargeParams& q, uint32_t cid, size_t n,
               float* dst) {
      rc = TAGORE_OK;
      msg.clear();
      t = std::thread([this, &fn, &q, cid, n, dst] {
        rc = fn(q, cid, n, dst);
        if (rc != TAGORE_OK) msg = tagore_last_error();
      });
    }
    int wait() {
      if (t.joinable()) t.join();
      if (rc != TAGORE_OK) fail(rc, "%s", msg.c_str());
      return rc;
    }
    ~Prefetch() {
      if (t.joinable()) t.join();
    }
  };
  auto builder = [&](uint32_t w) {
    // two load buffers (n x dim floats) and the rows' staging buffer
    void* pinned[3] = {nullptr, nullptr, nullptr};
    struct Free {
      void** p;
      ~Free() {
        for (int b = 0; b < 3; ++b)
          if (p[b]) cudaFreeHost(p[b]);
      }
    } release{pinned};
    if (load) {
      const size_t bytes[3] = {std::max<size_t>(largest, 1) * q.dim * sizeof(float),
                               std::max<size_t>(largest, 1) * q.dim * sizeof(float),
                               std::max<size_t>(largest, 1) * q.k * sizeof(uint32_t)};
      for (int b = 0; b < 3; ++b) {
        count_allocation();
        if (cudaMallocHost(&pinned[b], bytes[b]) != cudaSuccess) {
          pinned[b] = nullptr;
          std::lock_guard<std::mutex> g(sh.mu);
          record(fail(TAGORE_ENOMEM, "largeIndex: no pinned buffer of %zu bytes", bytes[b]));
          sh.cv.notify_all();
          return;
        }
      }
    }
    float* const bufs[2] = {static_cast<float*>(pinned[0]), static_cast<float*>(pinned[1])};
    uint32_t* const stage = static_cast<uint32_t*>(pinned[2]);
    uint32_t i = 0;
    if (!claim(&i)) return;
    Prefetch pf[2];
    int buf = 0;
    if (load) pf[buf].start(load, q, order[i], clusters[order[i]].size(), bufs[buf]);
    while (true) {
      const uint32_t cid = order[i];
      int rc = load ? pf[buf].wait() : TAGORE_OK;
      // the next cluster's file is read while this one builds, when the
      // merger window already has room for it; otherwise it is claimed
      // (waiting for the window) after the build, as without a reader
      uint32_t j = 0;
      const bool ahead_claimed = rc == TAGORE_OK && load && try_claim(&j);
      if (ahead_claimed)
        pf[buf ^ 1].start(load, q, order[j], clusters[order[j]].size(), bufs[buf ^ 1]);
      LocalRows rows;
      uint32_t medoid = 0;
      if (rc == TAGORE_OK)
        rc = build(q, w % (uint32_t)ndev, cid, clusters[cid], load ? bufs[buf] : nullptr, stage,
                   rows, &medoid);
      {
        std::lock_guard<std::mutex> g(sh.mu);
        if (rc != TAGORE_OK) {
          record(rc);
        } else {
          sh.built[i].rows.swap(rows);
          sh.built[i].medoid = medoid;
          sh.built[i].ready = true;
        }
        sh.cv.notify_all();
      }
      if (rc != TAGORE_OK) return;
      if (!ahead_claimed) {
        if (!claim(&j)) return;
        if (load) pf[buf ^ 1].start(load, q, order[j], clusters[order[j]].size(), bufs[buf ^ 1]);
      }
      i = j;
      buf ^= 1;
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t w = 1; w < workers; ++w) pool.emplace_back(builder, w);
  builder(0);  // the calling thread is builder 0
  for (auto& t : pool) t.join();
  merger.join();
  // the first error recorded wins: a builder's (with its message), else the merger's
  int rc;
  std::string msg;
  {
    std::lock_guard<std::mutex> g(sh.mu);
    rc = sh.error;
    msg = sh.msg;
  }
  if (rc == TAGORE_OK) rc = merge_rc;
  if (rc != TAGORE_OK) return fail(rc, "%s", msg.empty() ? merge_msg.c_str() : msg.c_str());
  return TAGORE_OK;
}

}  // namespace tagore
