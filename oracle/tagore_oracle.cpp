// tagore_oracle.cpp -- CPU restatement of Tagore's graph-index build path.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity checker for the CUDA
// product in tagore_b200/ and the timed CPU baseline of bench.py. Nothing in
// the product links, loads or calls it.
//
// Parity pin: the restatement is checked (a) against hand-derived answers on
// tiny graphs in tests/test_oracle_*.py and (b) against golden fixtures made by
// running the reference Tagore module itself (tests/golden/make_golden.py).
// Rows of the reference that are nondeterministic (atomic append order, races)
// are pinned under the fixed legal schedule documented below.
//
// Semantics restated (file:line refer to ZJU-DAILY/Tagore):
//  * distances: FP32 arithmetic on the FP16 base in the reference's lane order
//    (src/Tagore_src.cu:1429-1443): lane l owns 4-dim chunks j = l (mod 32);
//    accumulator x takes dims 4j and 4j+2, y takes 4j+1 and 4j+3, each as a
//    fused multiply-add of the difference; then a shuffle-down tree over
//    offsets 16,8,4,2,1; result x + y.
//  * sorts: the reference's block-wide bitonic network (src/Tagore_src.cu:26-147)
//    executed on the same positions, so ties resolve exactly as it does.
//  * schedule: cross-thread append order (rings, reverse lists, unions) is the
//    ascending order of the appending index; cross-block reverse inserts run in
//    ascending source-node order; blocks read the kNN graph as it was before the
//    kernel started (a read-only snapshot; the reference rewrites rows in place
//    while other blocks read them, src/Tagore_src.cu:1280,1358 vs :1463,1477).
//  * the few reads of uninitialised memory in the reference get the value its
//    code evidently means; each is marked "defined here" below.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#include <omp.h>

namespace {

constexpr uint32_t kReserve = 128;       // RESERVENUM, include/Tagore_src.cuh:29
constexpr uint32_t kSelectCand = 480;    // SELECT_CAND, include/Tagore_src.cuh:36
constexpr float kInfDis = 10000000.0f;   // INF_DIS, include/Tagore_src.cuh:35
constexpr uint32_t kInv = 0xFFFFFFFFu;
constexpr uint32_t kSample = 32;         // SAMPLE, include/Tagore_src.cuh:34

enum Status { OK = 0, EINVAL_ = 1 };

inline float h2f(uint16_t h) {
  _Float16 v;
  std::memcpy(&v, &h, 2);
  return (float)v;
}

inline uint16_t f2h(float f) {
  _Float16 v = (_Float16)f;  // round to nearest even, as __float2half
  uint16_t h;
  std::memcpy(&h, &v, 2);
  return h;
}

// FP32 squared L2 in the reference's lane order, see header.
float dist_ref(const uint16_t* a, const uint16_t* b, uint32_t dim) {
  float lx[32], ly[32];
  for (int l = 0; l < 32; ++l) lx[l] = ly[l] = 0.0f;
  const uint32_t chunks = dim / 4;
  for (uint32_t j = 0; j < chunks; ++j) {
    const int l = j & 31;
    const float d0 = h2f(a[4 * j + 0]) - h2f(b[4 * j + 0]);
    const float d1 = h2f(a[4 * j + 1]) - h2f(b[4 * j + 1]);
    const float d2 = h2f(a[4 * j + 2]) - h2f(b[4 * j + 2]);
    const float d3 = h2f(a[4 * j + 3]) - h2f(b[4 * j + 3]);
    lx[l] = std::fma(d0, d0, lx[l]);
    ly[l] = std::fma(d1, d1, ly[l]);
    lx[l] = std::fma(d2, d2, lx[l]);
    ly[l] = std::fma(d3, d3, ly[l]);
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int l = 0; l < off; ++l) {
      lx[l] = lx[l] + lx[l + off];
      ly[l] = ly[l] + ly[l + off];
    }
  return lx[0] + ly[0];
}

// The reference's bitonic network (src/Tagore_src.cu:29-44): strides 1,2,4..,
// steps stride..1, the first step of each merge mirrored, pairs beyond len
// skipped. gt(u,d) decides the swap; sw(u,d) performs it.
template <class Gt, class Sw>
void ref_network(uint32_t len, Gt gt, Sw sw) {
  for (uint32_t stride = 1; stride < len; stride <<= 1)
    for (uint32_t step = stride; step > 0; step >>= 1)
      for (uint32_t k = 0; k < len / 2; ++k) {
        const uint32_t a = 2 * step * (k / step), b = k % step;
        const uint32_t u = (step == stride) ? (a + step - 1 - b) : (a + b);
        const uint32_t d = a + b + step;
        if (d < len && gt(u, d)) sw(u, d);
      }
}

// Membership in a sorted id array; the reference's branchless search
// (src/Tagore_src.cu:1282-1290) is an exact membership test.
inline bool sorted_contains(const uint32_t* a, uint32_t len, uint32_t key) {
  return std::binary_search(a, a + len, key);
}

struct State {
  uint32_t n, k, dim;
  uint32_t* graph;
  uint32_t* reverse_graph;
  const uint16_t* data;
  float* nei_distance;
  float* reverse_distance;
  uint32_t* reverse_num;
  const uint16_t* center;
  uint32_t* hybrid_list;
};

inline const uint16_t* vec(const State& s, uint32_t id) { return s.data + (size_t)id * s.dim; }

// distance_filter (src/Tagore_src.cu:1488-1490), `threshold*res - dis`, which
// nvcc contracts to one fused multiply-add; angle_filter (:1493-1495).
inline bool pruned_by(int metric, float res, float dis, float cur, float thre) {
  if (metric == 0) return std::fma(thre, res, -dis) < 0.0f;
  float v = (dis + cur) - res;
  v = v / 2.0f;
  v = v / std::sqrt(dis * cur);
  return (thre - v) < 0.0f;
}

// Beam search shared by cal_ep_gpu (src/Tagore_src.cu:1905-2047) and
// collect_path (:1211-1335). Appends every scored node to the 480-slot ring in
// ascending neighbour order. Returns top_M_Cand[0].
uint32_t beam(const State& s, const uint32_t* G, const uint16_t* query, uint32_t start,
              uint32_t topm, uint32_t iters, uint32_t* ring_id, float* ring_dis,
              uint32_t* ring_count) {
  const uint32_t K = s.k, W = topm + K;
  std::vector<uint32_t> id(W, kInv), id2(W);
  std::vector<float> dis(W, kInfDis);
  std::vector<uint8_t> ex(W, 1);
  for (uint32_t t = 0; t < K; ++t) {
    id[topm + t] = G[(size_t)start * K + t];
    ex[topm + t] = 0;
  }
  uint32_t curr = K;  // curr_of_candset starts at K (:1217, :1911)
  for (uint32_t i = 0; i < K; ++i) {
    dis[topm + i] = dist_ref(query, vec(s, id[topm + i]), s.dim);
    if (ring_id) {
      ring_id[i % kSelectCand] = id[topm + i];
      ring_dis[i % kSelectCand] = dis[topm + i];
    }
  }
  {
    float* D = dis.data() + topm;
    uint32_t* I = id.data() + topm;
    uint8_t* E = ex.data() + topm;
    ref_network(K, [&](uint32_t u, uint32_t d) { return D[u] > D[d]; },
                [&](uint32_t u, uint32_t d) {
                  std::swap(D[u], D[d]);
                  std::swap(I[u], I[d]);
                  std::swap(E[u], E[d]);
                });
  }
  for (uint32_t i = 0; i < topm; ++i) {
    if (topm + i < W) {
      id[i] = id[topm + i];
      dis[i] = dis[topm + i];
      ex[i] = ex[topm + i];
    } else {  // defined here: beam slots past the K seeds start empty (the
              // reference reads uninitialised shared memory when TOPM > K)
      id[i] = kInv;
      dis[i] = kInfDis;
      ex[i] = 1;
    }
  }
  auto rebuild_id2 = [&]() {
    id2 = id;
    ref_network(W, [&](uint32_t u, uint32_t d) { return id2[u] > id2[d]; },
                [&](uint32_t u, uint32_t d) { std::swap(id2[u], id2[d]); });
  };
  rebuild_id2();
  uint32_t to_explore = kInv;
  for (uint32_t it = 0; it < iters; ++it) {
    // The reference's "none left" test (`j == TOPM` inside the j < TOPM loop,
    // :1270) never fires, so an exhausted beam re-expands the previous node.
    for (uint32_t j = 0; j < topm; ++j)
      if (!ex[j]) {
        to_explore = id[j];
        ex[j] = 1;
        break;
      }
    if (to_explore == kInv) break;
    for (uint32_t j = 0; j < K; ++j) {
      const uint32_t a = G[(size_t)to_explore * K + j];
      dis[topm + j] = sorted_contains(id2.data(), W, a) ? kInfDis : 0.0f;
      id[topm + j] = a;
      ex[topm + j] = 0;
    }
    for (uint32_t j = 0; j < K; ++j) {
      if (dis[topm + j] < 1.0f) {
        dis[topm + j] = dist_ref(query, vec(s, id[topm + j]), s.dim);
        if (ring_id) {
          ring_id[curr % kSelectCand] = id[topm + j];
          ring_dis[curr % kSelectCand] = dis[topm + j];
        }
        ++curr;
      }
    }
    ref_network(W, [&](uint32_t u, uint32_t d) { return dis[u] > dis[d]; },
                [&](uint32_t u, uint32_t d) {
                  std::swap(dis[u], dis[d]);
                  std::swap(id[u], id[d]);
                  std::swap(ex[u], ex[d]);
                });
    rebuild_id2();
  }
  if (ring_count) *ring_count = curr;
  return id[0];
}

// Sort a candidate list by distance with the reference network and mark
// adjacent repeats (src/Tagore_src.cu:1345-1348, :1391-1395, :1562-1565). The
// repeat test reads the sorted ids before any are marked.
void sort_and_mark(uint32_t* cand, float* dis, uint32_t len) {
  ref_network(len, [&](uint32_t u, uint32_t d) { return dis[u] > dis[d]; },
              [&](uint32_t u, uint32_t d) {
                std::swap(dis[u], dis[d]);
                std::swap(cand[u], cand[d]);
              });
  std::vector<uint32_t> orig(cand, cand + len);
  for (uint32_t i = 1; i < len; ++i)
    if (orig[i] == orig[i - 1]) cand[i] = kInv;
}

// Filter stage (Filter_path, src/Tagore_src.cu:1399-1460; the same loop in
// filter_reverse :1567-1621). Returns the number of ids the reference stores,
// which is one less than the number of selection steps taken (:1462, :1623).
uint32_t filter(const State& s, uint32_t bid, uint32_t* cand, const float* dis, uint32_t len,
                uint32_t fd, int metric, float thre, uint32_t* fin, float* fdis) {
  uint32_t tmp = 0;
  while (tmp < len && (cand[tmp] == bid || cand[tmp] == kInv)) ++tmp;
  if (tmp >= len) return 0;  // defined here: the reference reads past the list
  std::vector<uint32_t> sel(fd + 1);
  std::vector<float> seld(fd + 1);
  sel[0] = cand[tmp];
  seld[0] = dis[tmp];
  float cur_dis = dis[tmp];
  uint32_t cur = 1;
  ++tmp;
  while (cur < fd) {
    const uint32_t p = sel[cur - 1];
    for (uint32_t i = tmp; i < len; ++i) {
      if (cand[i] == kInv || cand[i] == p) {
        cand[i] = kInv;
        continue;
      }
      const float res = dist_ref(vec(s, p), vec(s, cand[i]), s.dim);
      if (pruned_by(metric, res, dis[i], cur_dis, thre)) cand[i] = kInv;
    }
    while (tmp < len && cand[tmp] == kInv) ++tmp;
    if (tmp < len) {
      sel[cur] = cand[tmp];
      seld[cur] = dis[tmp];
      cur_dis = dis[tmp];
    }
    ++cur;
    ++tmp;
    if (tmp >= len) break;
  }
  const uint32_t stored = cur - 1;
  for (uint32_t i = 0; i < stored; ++i) {
    fin[i] = sel[i];
    fdis[i] = seld[i];
  }
  return stored;
}

// Sequential reverse insert with the reference's replacement rule
// (src/Tagore_src.cu:1465-1475): the c-th insert into t's list takes slot c
// while c < cap, later ones replace slot c % cap when strictly closer.
void reverse_insert_dist(State& s, uint32_t t, uint32_t src, float d) {
  const uint32_t K = s.k;
  const uint32_t c = s.reverse_num[t]++;
  if (c < K) {
    s.reverse_graph[(size_t)t * K + c] = src;
    s.reverse_distance[(size_t)t * kReserve + c] = d;
  } else if (d < s.reverse_distance[(size_t)t * kReserve + (c % K)]) {
    s.reverse_graph[(size_t)t * K + (c % K)] = src;
    s.reverse_distance[(size_t)t * kReserve + (c % K)] = d;
  }
}

struct Pruned {
  std::vector<uint32_t> ids;   // [n * fd]
  std::vector<float> dis;      // [n * fd]
  std::vector<uint32_t> cnt;   // [n]
};

// Shared tail of select_path / select_2hop: write rows, then reverse inserts in
// ascending source order (:1462-1477, :1477 writes the degree).
void store_selected(State& s, const Pruned& P, uint32_t fd) {
  const uint32_t K = s.k;
  for (uint32_t b = 0; b < s.n; ++b) {
    const uint32_t c = P.cnt[b];
    for (uint32_t i = 0; i < c; ++i) {
      s.graph[(size_t)b * K + i + 1] = P.ids[(size_t)b * fd + i];
      s.nei_distance[(size_t)b * K + i] = P.dis[(size_t)b * fd + i];
    }
    s.graph[(size_t)b * K] = c;
  }
  for (uint32_t b = 0; b < s.n; ++b)
    for (uint32_t i = 0; i < P.cnt[b]; ++i)
      reverse_insert_dist(s, P.ids[(size_t)b * fd + i], b, P.dis[(size_t)b * fd + i]);
}

}  // namespace

extern "C" {

typedef struct {
  uint32_t n, k, dim;
  uint32_t* graph;
  uint32_t* reverse_graph;
  const uint16_t* data;
  float* nei_distance;
  float* reverse_distance;
  uint32_t* reverse_num;
  const uint16_t* center;
  uint32_t* hybrid_list;
} OrcState;

static State to_state(const OrcState* o) {
  return State{o->n, o->k, o->dim, o->graph, o->reverse_graph, o->data, o->nei_distance,
               o->reverse_distance, o->reverse_num, o->center, o->hybrid_list};
}

float orc_dist(const uint16_t* a, const uint16_t* b, uint32_t dim) { return dist_ref(a, b, dim); }

// Batch form: out[i] = dist(data[ia[i]], data[ib[i]]).
void orc_dist_pairs(const uint16_t* data, uint32_t dim, const uint32_t* ia, const uint32_t* ib,
                    uint64_t m, float* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i)
    out[i] = dist_ref(data + (size_t)ia[i] * dim, data + (size_t)ib[i] * dim, dim);
}

uint16_t orc_f2h(float f) { return f2h(f); }
float orc_h2f(uint16_t h) { return h2f(h); }

// Sorts `vals` (with payload) by the reference network; used by unit tests.
void orc_network_sort_u32(uint32_t* keys, uint32_t* payload, uint32_t len) {
  ref_network(len, [&](uint32_t u, uint32_t d) { return keys[u] > keys[d]; },
              [&](uint32_t u, uint32_t d) {
                std::swap(keys[u], keys[d]);
                if (payload) std::swap(payload[u], payload[d]);
              });
}

// cal_ep_gpu (src/Tagore_src.cu:1889-2058): one beam of 30 expansions from
// node 0's neighbours toward the FP16 centre.
int orc_cal_ep(const OrcState* o, uint32_t topm, uint32_t* ep) {
  State s = to_state(o);
  *ep = beam(s, s.graph, s.center, 0, topm, 30, nullptr, nullptr, nullptr);
  return OK;
}

// select_path = collect_path + Filter_path(distance_filter) (:1498-1517).
int orc_select_path(OrcState* o, uint32_t ep, uint32_t fd, uint32_t topm, float thre) {
  State s = to_state(o);
  const uint32_t K = s.k, L = kSelectCand + K;
  if (fd > K || fd == 0) return EINVAL_;
  std::vector<uint32_t> G(s.graph, s.graph + (size_t)s.n * K);           // snapshot
  std::vector<float> ND(s.nei_distance, s.nei_distance + (size_t)s.n * K);
  Pruned P{std::vector<uint32_t>((size_t)s.n * fd), std::vector<float>((size_t)s.n * fd),
           std::vector<uint32_t>(s.n)};
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t bb = 0; bb < (int64_t)s.n; ++bb) {
    const uint32_t b = (uint32_t)bb;
    std::vector<uint32_t> cand(L);
    std::vector<float> dis(L);
    uint32_t curr = 0;
    beam(s, G.data(), vec(s, b), ep, topm, 10, cand.data() + K, dis.data() + K, &curr);
    for (uint32_t i = curr; i < kSelectCand; ++i) {  // :1336-1339
      cand[K + i] = kInv;
      dis[K + i] = kInfDis;
    }
    for (uint32_t i = 0; i < K; ++i) {  // :1340-1343
      cand[i] = G[(size_t)b * K + i];
      dis[i] = ND[(size_t)b * K + i];
    }
    sort_and_mark(cand.data(), dis.data(), L);
    P.cnt[b] = filter(s, b, cand.data(), dis.data(), L, fd, 0, thre, &P.ids[(size_t)b * fd],
                      &P.dis[(size_t)b * fd]);
  }
  store_selected(s, P, fd);
  return OK;
}

// select_2hop = collect_2hop + Filter_path(angle_filter) (:1520-1534).
int orc_select_2hop(OrcState* o, uint32_t fd, float thre) {
  State s = to_state(o);
  const uint32_t K = s.k, L = kSelectCand + K;
  if (fd > K || fd == 0 || K * K < kSelectCand) return EINVAL_;
  std::vector<uint32_t> G(s.graph, s.graph + (size_t)s.n * K);
  std::vector<float> ND(s.nei_distance, s.nei_distance + (size_t)s.n * K);
  Pruned P{std::vector<uint32_t>((size_t)s.n * fd), std::vector<float>((size_t)s.n * fd),
           std::vector<uint32_t>(s.n)};
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t bb = 0; bb < (int64_t)s.n; ++bb) {
    const uint32_t b = (uint32_t)bb;
    std::vector<uint32_t> cand(L);
    std::vector<float> dis(L);
    for (uint32_t i = 0; i < K; ++i) {  // :1353-1356
      cand[i] = G[(size_t)b * K + i];
      dis[i] = ND[(size_t)b * K + i];
    }
    for (uint32_t i = 0; i < kSelectCand; ++i) {  // :1357-1359, 1367-1389
      const uint32_t hop = G[(size_t)b * K + i / K];
      cand[K + i] = G[(size_t)hop * K + i % K];
      dis[K + i] = dist_ref(vec(s, b), vec(s, cand[K + i]), s.dim);
    }
    sort_and_mark(cand.data(), dis.data(), L);
    P.cnt[b] = filter(s, b, cand.data(), dis.data(), L, fd, 1, thre, &P.ids[(size_t)b * fd],
                      &P.dis[(size_t)b * fd]);
  }
  store_selected(s, P, fd);
  return OK;
}

// filter_reverse (:1537-1657). metric 0 = distance_filter, 1 = angle_filter.
// Defined here: the angle rule's d(u, last kept) (`cur_nei_dis`, never
// assigned in this kernel) is the distance of the most recent selection.
int orc_filter_reverse(OrcState* o, uint32_t fd, int metric, float thre) {
  State s = to_state(o);
  const uint32_t K = s.k;
  if (fd > K || fd == 0) return EINVAL_;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t bb = 0; bb < (int64_t)s.n; ++bb) {
    const uint32_t b = (uint32_t)bb;
    uint32_t* row = s.graph + (size_t)b * K;
    const uint32_t cur_num = row[0];
    const uint32_t rn = std::min(K, s.reverse_num[b]);
    const uint32_t len = cur_num + rn;
    std::vector<uint32_t> cand(len);
    std::vector<float> dis(len);
    for (uint32_t i = 0; i < cur_num; ++i) {
      cand[i] = row[i + 1];
      dis[i] = s.nei_distance[(size_t)b * K + i];
    }
    for (uint32_t i = 0; i < rn; ++i) {
      cand[cur_num + i] = s.reverse_graph[(size_t)b * K + i];
      dis[cur_num + i] = s.reverse_distance[(size_t)b * kReserve + i];
    }
    if (len > fd) {
      sort_and_mark(cand.data(), dis.data(), len);
      std::vector<uint32_t> fin(fd);
      std::vector<float> fdis(fd);
      const uint32_t stored =
          filter(s, b, cand.data(), dis.data(), len, fd, metric, thre, fin.data(), fdis.data());
      for (uint32_t i = 0; i < stored; ++i) row[i + 1] = fin[i];
      row[0] = stored;
    } else {
      uint32_t dup = 0;  // union in ascending reverse-slot order (:1636-1645)
      for (uint32_t i = 0; i < rn; ++i) {
        bool found = false;
        for (uint32_t j = 0; j < cur_num; ++j)
          if (cand[j] == cand[cur_num + i]) {
            found = true;
            break;
          }
        // Defined here: a stride-K row holds at most K-1 ids; with FINAL_DEGREE == K
        // the reference would spill its last union id into the next row.
        if (!found && cur_num + dup + 1 < K) row[cur_num + 1 + dup++] = cand[cur_num + i];
      }
      row[0] = cur_num + dup;
    }
  }
  return OK;
}

// select_1hop_cagra = collect_1hop + filter_cagra (:1660-1710, :1787-1797).
int orc_select_1hop_cagra(OrcState* o, uint32_t d) {
  State s = to_state(o);
  const uint32_t K = s.k;
  if (d > K || d == 0 || 2 * d > kReserve) return EINVAL_;
  std::vector<uint32_t> nei((size_t)s.n * K), det((size_t)s.n * K);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t bb = 0; bb < (int64_t)s.n; ++bb) {
    const uint32_t b = (uint32_t)bb;
    uint32_t* nei0 = &nei[(size_t)b * K];
    uint32_t* detour = &det[(size_t)b * K];
    for (uint32_t j = 0; j < K; ++j) {
      nei0[j] = s.graph[(size_t)b * K + j];
      detour[j] = 0;
    }
    for (uint32_t i = 0; i < K / 2; ++i) {
      const uint32_t* nei1 = s.graph + (size_t)s.graph[(size_t)b * K + i] * K;
      const uint32_t* nei2 = s.graph + (size_t)s.graph[(size_t)b * K + K - 1 - i] * K;
      for (uint32_t t = 0; t + 1 < K; ++t) {
        const bool first = t < K - 1 - i;
        const uint32_t key = first ? nei0[i + 1 + t] : nei0[t + 1];
        const uint32_t* lst = first ? nei1 : nei2;
        const uint32_t my = first ? (i + 1 + t) : (t + 1);
        for (uint32_t j = 0; j < K; ++j)
          if (lst[j] == key) {
            ++detour[my];
            break;
          }
      }
    }
    ref_network(K, [&](uint32_t u, uint32_t v) { return detour[u] > detour[v]; },
                [&](uint32_t u, uint32_t v) {
                  std::swap(detour[u], detour[v]);
                  std::swap(nei0[u], nei0[v]);
                });
  }
  for (uint32_t b = 0; b < s.n; ++b)  // reverse (id, detour) pairs, :1696-1709
    for (uint32_t i = 0; i < d; ++i) {
      const uint32_t t = nei[(size_t)b * K + i], dt = det[(size_t)b * K + i];
      const uint32_t c = s.reverse_num[t]++;
      uint32_t* pr = s.reverse_graph + (size_t)t * d * 2;
      if (c < d) {
        pr[c * 2] = b;
        pr[c * 2 + 1] = dt;
      } else if (pr[(c % d) * 2 + 1] > dt) {
        pr[(c % d) * 2] = b;
        pr[(c % d) * 2 + 1] = dt;
      }
      s.hybrid_list[(size_t)b * K + i] = t;
    }
  return OK;
}

// select_1hop_dpg = collect_1hop + filter_dpg (:1713-1785, :1799-1809).
// Defined here: each warp compares against its own staged vector (the four
// warps of the reference share one staging buffer, :1714-1720). Rejected when
// the reference's direct-slot bound K-d-1 exceeds d (its writes then spill into
// the next node's pair list).
int orc_select_1hop_dpg(OrcState* o, uint32_t d) {
  State s = to_state(o);
  const uint32_t K = s.k;
  if (d == 0 || 2 * d > kReserve || K < d + 1 || K - d - 1 > d) return EINVAL_;
  const uint32_t direct = K - d - 1;
  std::vector<uint32_t> nei((size_t)s.n * K), det((size_t)s.n * K);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t bb = 0; bb < (int64_t)s.n; ++bb) {
    const uint32_t b = (uint32_t)bb;
    uint32_t* nei0 = &nei[(size_t)b * K];
    uint32_t* detour = &det[(size_t)b * K];
    for (uint32_t j = 0; j < K; ++j) {
      nei0[j] = s.graph[(size_t)b * K + j];
      detour[j] = 0;
    }
    for (uint32_t i = 0; i < K / 2; ++i) {
      const uint32_t n1 = nei0[i], n2 = nei0[K - 1 - i];
      for (uint32_t j = i + 1; j < K; ++j)
        if (dist_ref(vec(s, n1), vec(s, nei0[j]), s.dim) < s.nei_distance[(size_t)b * K + j])
          ++detour[j];
      for (uint32_t j = K - i; j < K; ++j)
        if (dist_ref(vec(s, n2), vec(s, nei0[j]), s.dim) < s.nei_distance[(size_t)b * K + j])
          ++detour[j];
    }
    ref_network(K, [&](uint32_t u, uint32_t v) { return detour[u] > detour[v]; },
                [&](uint32_t u, uint32_t v) {
                  std::swap(detour[u], detour[v]);
                  std::swap(nei0[u], nei0[v]);
                });
  }
  for (uint32_t b = 0; b < s.n; ++b)
    for (uint32_t i = 0; i < d; ++i) {
      const uint32_t t = nei[(size_t)b * K + i], dt = det[(size_t)b * K + i];
      const uint32_t c = s.reverse_num[t]++;
      uint32_t* pr = s.reverse_graph + (size_t)t * d * 2;
      if (c < direct) {
        pr[c * 2] = b;
        pr[c * 2 + 1] = dt;
      } else if (pr[(c % d) * 2 + 1] > dt) {
        pr[(c % d) * 2] = b;
        pr[(c % d) * 2 + 1] = dt;
      }
      s.hybrid_list[(size_t)b * K + i] = t;
    }
  return OK;
}

// filter_reverse_1hop (:1812-1886): rank merge into dense stride-d rows.
int orc_filter_reverse_1hop(OrcState* o, uint32_t d) {
  State s = to_state(o);
  const uint32_t K = s.k;
  if (d > K || d == 0 || 2 * d > kReserve) return EINVAL_;
  std::vector<uint32_t> out((size_t)s.n * d);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t bb = 0; bb < (int64_t)s.n; ++bb) {
    const uint32_t b = (uint32_t)bb;
    const uint32_t rn = std::min(d, s.reverse_num[b]);
    std::vector<uint32_t> rev(rn), rdet(rn), nid(d);
    for (uint32_t i = 0; i < rn; ++i) {
      rev[i] = s.reverse_graph[(size_t)b * d * 2 + i * 2];
      rdet[i] = s.reverse_graph[(size_t)b * d * 2 + i * 2 + 1];
    }
    for (uint32_t i = 0; i < d; ++i) nid[i] = s.hybrid_list[(size_t)b * K + i];
    ref_network(rn, [&](uint32_t u, uint32_t v) { return rev[u] > rev[v]; },
                [&](uint32_t u, uint32_t v) {
                  std::swap(rev[u], rev[v]);
                  std::swap(rdet[u], rdet[v]);
                });
    for (uint32_t i = 1; i < rn; ++i)
      if (rev[i] == rev[i - 1]) rdet[i] = kInv;
    uint32_t* row = &out[(size_t)b * d];
    for (uint32_t i = 0; i < d / 2; ++i) row[i] = nid[i];
    ref_network(rn, [&](uint32_t u, uint32_t v) { return rdet[u] > rdet[v]; },
                [&](uint32_t u, uint32_t v) {
                  std::swap(rdet[u], rdet[v]);
                  std::swap(rev[u], rev[v]);
                });
    uint32_t cnt = 0;
    if (rn < d / 2) {
      for (uint32_t i = 0; i < rn; ++i) {
        bool flag = false;
        for (uint32_t j = 0; j < d - rn; ++j)
          if (rev[i] == nid[j]) {
            flag = true;
            break;
          }
        if (!flag) row[d / 2 + cnt++] = rev[i];
      }
      for (uint32_t i = 0; i < d / 2 - cnt; ++i) row[d / 2 + cnt + i] = nid[i + d / 2];
    } else {
      for (uint32_t i = 0; i < rn && cnt < d / 2; ++i) {
        bool flag = false;
        for (uint32_t j = 0; j < d / 2; ++j)
          if (rev[i] == nid[j]) {
            flag = true;
            break;
          }
        if (!flag) row[d / 2 + cnt++] = rev[i];
      }
      const uint32_t m = std::min(cnt, d / 2);
      for (uint32_t i = 0; i < d / 2 - m; ++i) row[m + d / 2 + i] = nid[i + d / 2];
    }
  }
  // Write the dense rows back over the graph buffer as the reference does
  // (graph[bid * d + i], :1836,1851,1856,1871,1876); untouched slots keep the
  // old contents.
  const uint32_t written = 2 * (d / 2);  // with odd d the last slot is untouched
  for (uint32_t b = 0; b < s.n; ++b) {
    for (uint32_t i = 0; i < written; ++i) s.graph[(size_t)b * d + i] = out[(size_t)b * d + i];
  }
  return OK;
}

// Pruning (pybind.cu:145-229) minus the file write, which the caller does from
// the returned graph. Returns the entry point through ep_out for NSG/Vamana.
int orc_prune(OrcState* o, uint32_t fd, uint32_t topm, const char* index_type, float thre,
              uint32_t* ep_out) {
  const std::string t(index_type);
  uint32_t ep = 0;
  int rc = OK;
  if (t == "NSG" || t == "Vamana") {
    const float th = (t == "NSG") ? 1.0f : thre;
    if ((rc = orc_cal_ep(o, topm, &ep))) return rc;
    if ((rc = orc_select_path(o, ep, fd, topm, th))) return rc;
    rc = orc_filter_reverse(o, fd, 0, th);
  } else if (t == "NSSG") {
    if ((rc = orc_select_2hop(o, fd, thre))) return rc;
    rc = orc_filter_reverse(o, fd, 1, thre);
  } else if (t == "CAGRA") {
    if ((rc = orc_select_1hop_cagra(o, fd))) return rc;
    rc = orc_filter_reverse_1hop(o, fd);
  } else if (t == "DPG") {
    if ((rc = orc_select_1hop_dpg(o, fd))) return rc;
    rc = orc_filter_reverse_1hop(o, fd);
  } else {
    return EINVAL_;
  }
  if (ep_out) *ep_out = ep;
  return rc;
}

// Pruning_with_CFS (pybind.cu:232-295) for the well-defined combinations.
int orc_prune_cfs(OrcState* o, uint32_t fd, uint32_t topm, const char* mode, const char* metric,
                  float thre, uint32_t* ep_out) {
  const std::string m(mode), me(metric);
  uint32_t ep = 0;
  int rc = OK;
  const bool dist_like = (me == "dist" || me == "angle");
  if (m == "path" && dist_like) {
    if ((rc = orc_cal_ep(o, topm, &ep))) return rc;
    if ((rc = orc_select_path(o, ep, fd, topm, thre))) return rc;
  } else if (m == "2-hop" && dist_like) {
    if ((rc = orc_select_2hop(o, fd, thre))) return rc;
  } else if (m == "1-hop" && me == "rank") {
    if ((rc = orc_select_1hop_cagra(o, fd))) return rc;
  } else {
    return EINVAL_;
  }
  if (me == "dist") rc = orc_filter_reverse(o, fd, 0, thre);
  else if (me == "angle") rc = orc_filter_reverse(o, fd, 1, thre);
  else rc = orc_filter_reverse_1hop(o, fd);
  if (ep_out) *ep_out = ep;
  return rc;
}

// ---------------------------------------------------------------------------
// Host preparation of GNN_descent (pybind.cu:20-61): power-of-ten rescale from
// vector 0, centroid by a sequential float sum, FP16 base and centre.
int orc_host_prep(const float* data, uint32_t n, uint32_t dim, uint16_t* data_half,
                  uint16_t* center_half, float* norm_out) {
  float ave = 0.0f;
  for (uint32_t i = 0; i < dim; ++i) ave += std::fabs(data[i]);
  ave /= (float)dim;
  float norm = 1.0f;
  if (ave > 0.0f && std::isfinite(ave)) {
    while (ave < 0.5f) {
      ave *= 10;
      norm *= 10;
    }
    while (ave > 5) {
      ave /= 10;
      norm /= 10;
    }
  }
  std::vector<float> c(dim, 0.0f);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = 0; j < dim; ++j) c[j] += data[(size_t)i * dim + j];
  for (uint32_t j = 0; j < dim; ++j) {
    c[j] /= (float)n;
    center_half[j] = f2h(c[j] * norm);
  }
  for (size_t i = 0; i < (size_t)n * dim; ++i) data_half[i] = f2h(data[i] * norm);
  *norm_out = norm;
  return OK;
}

// ---------------------------------------------------------------------------
// Brute-force kNN ground truth (squared L2, FP32), OpenMP over queries.
int orc_bruteforce_knn(const float* base, uint32_t n, uint32_t dim, const float* q, uint32_t nq,
                       uint32_t k, const uint32_t* exclude_self, uint32_t* out) {
#pragma omp parallel
  {
    std::vector<std::pair<float, uint32_t>> best;
#pragma omp for schedule(dynamic, 16)
    for (int64_t qi = 0; qi < (int64_t)nq; ++qi) {
      best.clear();
      const float* x = q + (size_t)qi * dim;
      const uint32_t self = exclude_self ? exclude_self[qi] : kInv;
      for (uint32_t i = 0; i < n; ++i) {
        if (i == self) continue;
        const float* y = base + (size_t)i * dim;
        float acc = 0.0f;
        for (uint32_t j = 0; j < dim; ++j) {
          const float t = x[j] - y[j];
          acc += t * t;
        }
        if (best.size() < k) {
          best.emplace_back(acc, i);
          std::push_heap(best.begin(), best.end());
        } else if (acc < best.front().first) {
          std::pop_heap(best.begin(), best.end());
          best.back() = {acc, i};
          std::push_heap(best.begin(), best.end());
        }
      }
      std::sort_heap(best.begin(), best.end());
      for (uint32_t j = 0; j < k; ++j) out[(size_t)qi * k + j] = j < best.size() ? best[j].second : kInv;
    }
  }
  return OK;
}

// Greedy best-first search over an index (the NSG search loop the reference
// keeps as dead code, src/common.cu:65-127), with a visited bitmap and pool
// size L. As there, the pool starts from ep's adjacency filled up to L with
// random unvisited ids (:74-82); the ids come from a splitmix64 stream of
// (seed, query index) instead of rand(), so two indexes over the same base
// are searched from the same starts. seed == 0 starts from ep and its
// adjacency alone. Adjacency is CSR (offsets, ids).
int orc_greedy_search(const float* base, uint32_t n, uint32_t dim, const uint64_t* offs,
                      const uint32_t* adj, uint32_t ep, const float* q, uint32_t nq, uint32_t L,
                      uint32_t k, uint64_t seed, uint32_t* out) {
#pragma omp parallel
  {
    std::vector<uint8_t> seen(n);
    std::vector<uint32_t> touched;
    struct C {
      float d;
      uint32_t id;
      bool open;
    };
    std::vector<C> pool;
#pragma omp for schedule(dynamic, 8)
    for (int64_t qi = 0; qi < (int64_t)nq; ++qi) {
      const float* x = q + (size_t)qi * dim;
      auto dist = [&](uint32_t id) {
        const float* y = base + (size_t)id * dim;
        float acc = 0.0f;
        for (uint32_t j = 0; j < dim; ++j) {
          const float t = x[j] - y[j];
          acc += t * t;
        }
        return acc;
      };
      pool.clear();
      for (uint32_t id : touched) seen[id] = 0;
      touched.clear();
      auto visit = [&](uint32_t id) {
        if (id >= n || seen[id]) return;
        seen[id] = 1;
        touched.push_back(id);
        C c{dist(id), id, true};
        if (pool.size() >= L && c.d >= pool.back().d) return;
        auto it = std::upper_bound(pool.begin(), pool.end(), c,
                                   [](const C& a, const C& b) { return a.d < b.d; });
        pool.insert(it, c);
        if (pool.size() > L) pool.pop_back();
      };
      if (seed == 0) visit(ep);
      for (uint64_t e = offs[ep]; e < offs[ep + 1]; ++e) visit(adj[e]);
      if (seed != 0) {
        uint64_t z = seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(qi + 1));
        auto next = [&]() {
          z += 0x9E3779B97F4A7C15ull;
          uint64_t x = z;
          x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
          x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
          return x ^ (x >> 31);
        };
        const uint32_t want = std::min<uint32_t>(L, n);
        while (touched.size() < want) visit((uint32_t)(next() % n));
      }
      while (true) {
        size_t idx = 0;
        while (idx < pool.size() && !pool[idx].open) ++idx;
        if (idx >= pool.size()) break;
        pool[idx].open = false;
        const uint32_t u = pool[idx].id;
        for (uint64_t e = offs[u]; e < offs[u + 1]; ++e) visit(adj[e]);
      }
      for (uint32_t j = 0; j < k; ++j) out[(size_t)qi * k + j] = j < pool.size() ? pool[j].id : kInv;
    }
  }
  return OK;
}

// ---------------------------------------------------------------------------
// OpenMP NN-Descent (Dong et al., WWW 2011) on FP32 vectors: the CPU baseline.
// Each node keeps K (dist, id, new) sorted; per iteration it samples up to S
// new and S old forward neighbours plus reverse samples, then joins new x new
// and new x old under per-node spin locks.
int orc_nndescent(const float* base, uint32_t n, uint32_t dim, uint32_t K, uint32_t iters,
                  uint32_t S, uint64_t seed, uint32_t* out_ids, float* out_dis) {
  if (K == 0 || K >= n) return EINVAL_;
  struct E {
    float d;
    uint32_t id;
    uint8_t is_new;
  };
  std::vector<E> nb((size_t)n * K);
  std::vector<std::atomic_flag> locks(n);
  for (auto& l : locks) l.clear();
  auto dist = [&](uint32_t a, uint32_t b) {
    const float* x = base + (size_t)a * dim;
    const float* y = base + (size_t)b * dim;
    float acc = 0.0f;
    for (uint32_t j = 0; j < dim; ++j) {
      const float t = x[j] - y[j];
      acc += t * t;
    }
    return acc;
  };
#pragma omp parallel for schedule(static)
  for (int64_t uu = 0; uu < (int64_t)n; ++uu) {
    const uint32_t u = (uint32_t)uu;
    std::mt19937_64 rng(seed ^ (0x9E3779B97F4A7C15ull * (u + 1)));
    E* row = &nb[(size_t)u * K];
    uint32_t c = 0;
    while (c < K) {
      const uint32_t v = (uint32_t)(rng() % n);
      if (v == u) continue;
      bool dup = false;
      for (uint32_t j = 0; j < c; ++j) dup |= row[j].id == v;
      if (dup) continue;
      row[c++] = E{dist(u, v), v, 1};
    }
    std::sort(row, row + K, [](const E& a, const E& b) { return a.d < b.d; });
  }
  auto insert = [&](uint32_t u, uint32_t v, float d) -> int {
    E* row = &nb[(size_t)u * K];
    if (d >= row[K - 1].d) return 0;
    while (locks[u].test_and_set(std::memory_order_acquire)) {
    }
    int changed = 0;
    if (d < row[K - 1].d) {
      bool dup = false;
      for (uint32_t j = 0; j < K; ++j)
        if (row[j].id == v) {
          dup = true;
          break;
        }
      if (!dup) {
        uint32_t pos = K - 1;
        while (pos > 0 && row[pos - 1].d > d) {
          row[pos] = row[pos - 1];
          --pos;
        }
        row[pos] = E{d, v, 1};
        changed = 1;
      }
    }
    locks[u].clear(std::memory_order_release);
    return changed;
  };
  std::vector<std::vector<uint32_t>> nw(n), ol(n), rnw(n), rol(n);
  std::vector<std::atomic_flag> rlocks(n);
  for (auto& l : rlocks) l.clear();
  for (uint32_t it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(static)
    for (int64_t uu = 0; uu < (int64_t)n; ++uu) {
      const uint32_t u = (uint32_t)uu;
      nw[u].clear();
      ol[u].clear();
      rnw[u].clear();
      rol[u].clear();
      E* row = &nb[(size_t)u * K];
      for (uint32_t j = 0; j < K; ++j) {
        if (row[j].is_new) {
          if (nw[u].size() < S) {
            nw[u].push_back(row[j].id);
            row[j].is_new = 0;
          }
        } else if (ol[u].size() < S) {
          ol[u].push_back(row[j].id);
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (int64_t uu = 0; uu < (int64_t)n; ++uu) {
      const uint32_t u = (uint32_t)uu;
      for (uint32_t v : nw[u]) {
        while (rlocks[v].test_and_set(std::memory_order_acquire)) {
        }
        if (rnw[v].size() < S) rnw[v].push_back(u);
        rlocks[v].clear(std::memory_order_release);
      }
      for (uint32_t v : ol[u]) {
        while (rlocks[v].test_and_set(std::memory_order_acquire)) {
        }
        if (rol[v].size() < S) rol[v].push_back(u);
        rlocks[v].clear(std::memory_order_release);
      }
    }
    long updates = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : updates)
    for (int64_t uu = 0; uu < (int64_t)n; ++uu) {
      const uint32_t u = (uint32_t)uu;
      std::vector<uint32_t> N = nw[u], O = ol[u];
      N.insert(N.end(), rnw[u].begin(), rnw[u].end());
      O.insert(O.end(), rol[u].begin(), rol[u].end());
      std::sort(N.begin(), N.end());
      N.erase(std::unique(N.begin(), N.end()), N.end());
      std::sort(O.begin(), O.end());
      O.erase(std::unique(O.begin(), O.end()), O.end());
      for (size_t i = 0; i < N.size(); ++i) {
        for (size_t j = i + 1; j < N.size(); ++j) {
          const float d = dist(N[i], N[j]);
          updates += insert(N[i], N[j], d) + insert(N[j], N[i], d);
        }
        for (uint32_t y : O) {
          if (y == N[i]) continue;
          const float d = dist(N[i], y);
          updates += insert(N[i], y, d) + insert(y, N[i], d);
        }
      }
    }
    (void)updates;
  }
  for (size_t i = 0; i < (size_t)n * K; ++i) {
    out_ids[i] = nb[i].id;
    out_dis[i] = nb[i].d;
  }
  return OK;
}

int orc_num_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
