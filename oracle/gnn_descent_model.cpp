// gnn_descent_model.cpp -- CPU restatement of the reference's GNN_descent.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: a model of ZJU-DAILY/Tagore's
// two-phase GNN-Descent (pybind.cu:103-124) used to compare the kNN recall
// this project's GPU build reaches with the recall of the reference's own
// algorithm at equal iterations, on inputs the reference module does not run
// on here. Nothing in the product links, loads or calls it.
//
// What is restated, kernel by kernel (src/Tagore_src.cu):
//  * initialize_graph (:158-166): K uniform random ids per node, distance
//    INF_DIS, visit flags cleared (seeded here; the reference seeds by clock());
//  * cal_power (:1164-1184): squared norms in FP16, a shuffle-down tree per
//    32 dimensions and a sequential FP16 sum of the warp results;
//  * phase 1, iter/2 rounds: nn_descent_opt_sample (:531-594),
//    nn_descent_opt_reverse_sample (:603-674, including its binary searches
//    over lists that are not sorted), nn_descent_opt_cal (:684-1033: FP16 Gram
//    tiles with FP32 accumulation, the -INF/INF thresholds at 0.01, the row
//    and column minima of each 16x16 tile with the lane layout and tie rules
//    of its shuffles, appends into lists of RESERVENUM), nn_descent_opt_merge
//    (:1043-1161) with the reference's bitonic network on its positions;
//  * do_reverse_graph and reset_visit_reversenum (:1187-1206);
//  * phase 2, iter/2 rounds of sample_kernel6 (:178-403): four unvisited
//    neighbours, 64 forward plus 64 random reverse neighbours of each, id
//    sort and dedupe, FP16 distances with __hfma2 accumulation and the FP16
//    shuffle tree, merge and reverse inserts with the replacement rule;
//  * merge_reverse_plus (:420-512).
// FP16 operations are emulated exactly: each one is computed exactly in
// double and rounded once to FP16 (round to nearest even). The tensor-core
// tile's accumulation order is not specified by the hardware; each 16-wide
// k-step is added to the FP32 accumulator with one rounding here.
//
// Schedule: nodes run in parallel with atomic counters, as the reference's
// blocks do, so appends land in a data-dependent order and rows that other
// nodes rewrite are read as they stand; like the reference, two runs need not
// agree bit for bit. Within a node the block's threads are executed in
// ascending thread order. Reads of uninitialised shared memory see 0xFFFFFFFF.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

constexpr uint32_t kRes = 128;        // RESERVENUM
constexpr uint32_t kS = 32;           // SAMPLE
constexpr uint32_t kMaxP = 512;       // MAX_P
constexpr float kInf = 10000000.0f;   // INF_DIS
constexpr uint32_t kNone = 0xFFFFFFFFu;

using h16 = _Float16;

inline h16 hround(double v) { return (h16)v; }  // one correctly rounded conversion
inline h16 hsub(h16 a, h16 b) { return hround((double)a - (double)b); }
inline h16 hadd(h16 a, h16 b) { return hround((double)a + (double)b); }
inline h16 hmul(h16 a, h16 b) { return hround((double)a * (double)b); }
inline h16 hfma(h16 a, h16 b, h16 c) { return hround((double)a * (double)b + (double)c); }

inline uint64_t mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

inline uint32_t fetch_add(uint32_t* p) { return __atomic_fetch_add(p, 1u, __ATOMIC_RELAXED); }

// The reference's block bitonic network (src/Tagore_src.cu:26-147): strides
// 1,2,4,.., steps stride..1, first step of each merge mirrored, pairs past
// len skipped.
template <class Gt, class Sw>
void network(uint32_t len, Gt gt, Sw sw) {
  for (uint32_t stride = 1; stride < len; stride <<= 1)
    for (uint32_t step = stride; step > 0; step >>= 1)
      for (uint32_t k = 0; k < len / 2; ++k) {
        const uint32_t a = 2 * step * (k / step), b = k % step;
        const uint32_t u = step == stride ? a + step - 1 - b : a + b;
        const uint32_t d = a + b + step;
        if (d < len && gt(u, d)) sw(u, d);
      }
}

// Binary search of the reference's merge kernels: count of entries < v (or
// <= v) in a[0, n) with its halving loop; reads a[n] like the reference.
template <bool kLe, class T>
uint32_t bsearch_pos(const T* a, uint32_t n, T v) {
  uint32_t tmp = n, r = 0;
  while (tmp > 1) {
    const uint32_t h = tmp / 2;
    const T c = a[r + h];
    r += (kLe ? c <= v : c < v) ? h : 0;
    tmp -= h;
  }
  const T c = a[r];
  r += (kLe ? c <= v : c < v) ? 1 : 0;
  return r;
}

struct Model {
  uint32_t n, d, K;
  const h16* x;        // FP16 base
  std::vector<float> xf;  // the same values as float (exact)
  std::vector<uint32_t> graph, rgraph, hybrid, rnum, rnum_old, new_num, old_num;
  std::vector<float> nd, rd, power;
  std::vector<uint8_t> visit;

  const float* row(uint32_t i) const { return xf.data() + (size_t)i * d; }

  float fp16_dist(const h16* q, uint32_t c) const {
    // sample_kernel6 :261-286: lane l takes half4 chunks j = l (mod 32)
    h16 vx[32], vy[32];
    for (int l = 0; l < 32; ++l) vx[l] = vy[l] = (h16)0.0f;
    const h16* b = x + (size_t)c * d;
    for (uint32_t j = 0; j < d / 4; ++j) {
      const int l = j & 31;
      const h16 d0 = hsub(q[4 * j], b[4 * j]), d1 = hsub(q[4 * j + 1], b[4 * j + 1]);
      vx[l] = hfma(d0, d0, vx[l]);
      vy[l] = hfma(d1, d1, vy[l]);
      const h16 d2 = hsub(q[4 * j + 2], b[4 * j + 2]), d3 = hsub(q[4 * j + 3], b[4 * j + 3]);
      vx[l] = hfma(d2, d2, vx[l]);
      vy[l] = hfma(d3, d3, vy[l]);
    }
    for (int m = 16; m > 0; m >>= 1)
      for (int l = 0; l < m; ++l) {
        vx[l] = hadd(vx[l], vx[l + m]);
        vy[l] = hadd(vy[l], vy[l + m]);
      }
    return (float)hadd(vx[0], vy[0]);
  }

  void init(uint64_t seed) {
    // one extra zeroed row: at K < 64 sample_kernel6 reads 64 forward
    // neighbours, past the end of the last row (the reference reads on into
    // whatever follows its allocation)
    graph.assign((size_t)n * K + 64, 0);
    nd.assign((size_t)n * K, kInf);
    visit.assign((size_t)n * K, 0);
    rgraph.assign((size_t)n * kRes, 0);
    rd.assign((size_t)n * kRes, 0.0f);
    hybrid.assign((size_t)n * kRes, 0);
    rnum.assign(n, 0);
    rnum_old.assign(n, 0);
    new_num.assign(n, 0);
    old_num.assign(n, 0);
    power.assign(n, 0.0f);
#pragma omp parallel for schedule(static)
    for (int64_t uu = 0; uu < (int64_t)n; ++uu) {
      const uint32_t u = (uint32_t)uu;
      for (uint32_t i = 0; i < K; ++i)
        graph[(size_t)u * K + i] = (uint32_t)(mix(seed ^ ((uint64_t)u * K + i)) % n);
      // cal_power: per-warp FP16 tree, then a sequential FP16 sum
      const h16* r = x + (size_t)u * d;
      const uint32_t warps = (d + 31) / 32;
      h16 tot = (h16)0.0f;
      for (uint32_t w = 0; w < warps; ++w) {
        h16 v[32];
        for (int l = 0; l < 32; ++l) {
          const uint32_t t = w * 32 + l;
          v[l] = t < d ? hmul(r[t], r[t]) : (h16)0.0f;
        }
        // shuffle-down tree: lanes past the warp end add their own value
        for (int m = 16; m > 0; m >>= 1)
          for (int l = 0; l < 32; ++l) v[l] = hadd(v[l], l + m < 32 ? v[l + m] : v[l]);
        tot = hadd(tot, v[0]);
      }
      power[u] = (float)tot;
    }
  }

  // ---- phase 1 ----
  void sample(uint32_t u) {
    const size_t o = (size_t)u * K;
    uint32_t nn[kS], on[kS], nc = 0, oc = 0, p = 0;
    while (nc < kS && oc < kS && p < K) {
      if (!visit[o + p]) {
        nn[nc++] = graph[o + p];
        visit[o + p] = 1;
      } else {
        on[oc++] = graph[o + p];
      }
      ++p;
    }
    while (oc < kS && p < K) {
      if (visit[o + p]) on[oc++] = graph[o + p];
      ++p;
    }
    while (nc < kS && p < K) {
      if (!visit[o + p]) {
        nn[nc++] = graph[o + p];
        visit[o + p] = 1;
      }
      ++p;
    }
    for (uint32_t i = 0; i < nc; ++i) {
      const uint32_t t = fetch_add(&rnum[nn[i]]);
      if (t < kS) rgraph[(size_t)nn[i] * K + t] = u;
      hybrid[(size_t)u * kRes + i] = nn[i];
    }
    for (uint32_t i = 0; i < oc; ++i) {
      const uint32_t t = fetch_add(&rnum_old[on[i]]);
      if (t < kS) rgraph[(size_t)on[i] * K + kS + t] = u;
      hybrid[(size_t)u * kRes + 2 * kS + i] = on[i];
    }
    new_num[u] = nc;
    old_num[u] = oc;
  }

  void reverse_sample(uint32_t u) {
    uint32_t nn[kS + 1], on[kS + 1];
    std::fill(nn, nn + kS + 1, kNone);
    std::fill(on, on + kS + 1, kNone);
    const uint32_t nnum = new_num[u], onum = old_num[u];
    for (uint32_t i = 0; i < nnum; ++i) nn[i] = hybrid[(size_t)u * kRes + i];
    for (uint32_t i = 0; i < onum; ++i) on[i] = hybrid[(size_t)u * kRes + 2 * kS + i];
    const uint32_t nr = std::min(rnum[u], kS), orv = std::min(rnum_old[u], kS);
    for (uint32_t i = 0; i < nr; ++i) {
      const uint32_t v = rgraph[(size_t)u * K + i];
      const uint32_t r = bsearch_pos<false>(nn, nnum, v);
      if (nn[r] == v) rgraph[(size_t)u * K + i] = kNone;
      else hybrid[(size_t)u * kRes + new_num[u]++] = v;
    }
    for (uint32_t i = 0; i < orv; ++i) {
      const uint32_t v = rgraph[(size_t)u * K + kS + i];
      const uint32_t r = bsearch_pos<false>(on, onum, v);
      if (on[r] == v) rgraph[(size_t)u * K + kS + i] = kNone;
      else hybrid[(size_t)u * kRes + 2 * kS + old_num[u]++] = v;
    }
  }

  void append(uint32_t owner, uint32_t id, float v) {
    const uint32_t t = fetch_add(&rnum[owner]);
    if (t < kRes) {
      rgraph[(size_t)owner * kRes + t] = id;
      rd[(size_t)owner * kRes + t] = v;
    }
  }

  // One 64x64 tile of FP32 Gram values between the rows listed in a and b
  // (zero rows past na / nb), 16-wide k-steps each added with one rounding.
  void gram(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, float* g) const {
    for (uint32_t i = 0; i < 64; ++i)
      for (uint32_t j = 0; j < 64; ++j) {
        float acc = 0.0f;
        if (i < na && j < nb) {
          const float* p = row(a[i]);
          const float* q = row(b[j]);
          for (uint32_t k0 = 0; k0 < d; k0 += 16) {
            double s = 0.0;
            for (uint32_t k = k0; k < std::min(d, k0 + 16); ++k) s += (double)p[k] * (double)q[k];
            acc = (float)((double)acc + s);
          }
        }
        g[i * 64 + j] = acc;
      }
  }

  // The 8 accumulator values of lane l of warp tile (wx, wy), with the
  // thresholds and norms applied (:745-757): slot 0/1 row r, cols 2c, 2c+1;
  // 2/3 row r+8; 4/5 row r, cols 2c+8, 2c+9; 6/7 row r+8, cols 2c+8, 2c+9.
  void lane_vals(const float* g, const uint32_t* A, const uint32_t* B, uint32_t wx, uint32_t wy,
                 int l, float v[8]) const {
    const uint32_t r = wx * 16 + l / 4, c = wy * 16 + (l % 4) * 2;
    const uint32_t rows[8] = {r, r, r + 8, r + 8, r, r, r + 8, r + 8};
    const uint32_t cols[8] = {c, c + 1, c, c + 1, c + 8, c + 9, c + 8, c + 9};
    for (int s = 0; s < 8; ++s) {
      float a = g[rows[s] * 64 + cols[s]];
      if (a < 0.01f) a = -kInf;
      float t = std::fma(-2.0f, a, power[A[rows[s]]] + power[B[cols[s]]]);
      if (t < 0.01f) t = kInf;
      v[s] = t;
    }
  }

  // Row minima of the tile (one per row r, r+8 of lane group l/4), with the
  // reference's compare order and shuffles (:759-789).
  void row_mins(const float vals[32][8], const uint32_t* B, uint32_t wy, float mv[32][2],
                uint32_t mi[32][2]) const {
    for (int l = 0; l < 32; ++l) {
      const uint32_t c = wy * 16 + (l % 4) * 2;
      const float* v = vals[l];
      for (int h = 0; h < 2; ++h) {
        const int s = 2 * h;  // 0 (row r) or 2 (row r+8)
        uint32_t id = v[s] < v[s + 1] ? B[c] : B[c + 1];
        float m = std::min(v[s], v[s + 1]);
        id = m < v[s + 4] ? id : B[c + 8];
        m = std::min(m, v[s + 4]);
        id = m < v[s + 5] ? id : B[c + 9];
        m = std::min(m, v[s + 5]);
        mv[l][h] = m;
        mi[l][h] = id;
      }
    }
    for (int off : {2, 1}) {
      float nv[32][2];
      uint32_t ni[32][2];
      for (int l = 0; l < 32; ++l)
        for (int h = 0; h < 2; ++h) {
          const int src = l + off < 32 ? l + off : l;
          const float tv = mv[src][h];
          const uint32_t ti = mi[src][h];
          ni[l][h] = mv[l][h] < tv ? mi[l][h] : ti;
          nv[l][h] = std::min(mv[l][h], tv);
        }
      std::memcpy(mv, nv, sizeof(nv));
      std::memcpy(mi, ni, sizeof(ni));
    }
  }

  // Column minima over the tile's 16 rows (:810-893): pairs (slot a, slot b)
  // of rows r and r+8, then seven shuffles down by 4.
  void col_mins(const float vals[32][8], const uint32_t* A, uint32_t wx, int sa, int sb,
                float out_v[4], uint32_t out_i[4]) const {
    float mv[32];
    uint32_t mi[32];
    for (int l = 0; l < 32; ++l) {
      const uint32_t r = wx * 16 + l / 4;
      mi[l] = vals[l][sa] < vals[l][sb] ? A[r] : A[r + 8];
      mv[l] = std::min(vals[l][sa], vals[l][sb]);
    }
    for (int it = 0; it < 7; ++it) {
      float nv[32];
      uint32_t ni[32];
      for (int l = 0; l < 32; ++l) {
        const int src = l + 4 < 32 ? l + 4 : l;
        ni[l] = mv[l] < mv[src] ? mi[l] : mi[src];
        nv[l] = std::min(mv[l], mv[src]);
      }
      std::memcpy(mv, nv, sizeof(nv));
      std::memcpy(mi, ni, sizeof(ni));
    }
    for (int l = 0; l < 4; ++l) {
      out_v[l] = mv[l];
      out_i[l] = mi[l];
    }
  }

  void cal(uint32_t u, std::vector<float>& g) {
    uint32_t nn[64], on[64];
    const uint32_t nnum = new_num[u], onum = old_num[u];
    for (uint32_t i = 0; i < 64; ++i) {
      nn[i] = i < nnum ? hybrid[(size_t)u * kRes + i] : 0u;
      on[i] = i < onum ? hybrid[(size_t)u * kRes + 2 * kS + i] : 0u;
    }
    float vals[32][8], mv[32][2];
    uint32_t mi[32][2];
    if (onum > 0) {
      gram(nn, nnum, on, onum, g.data());
      for (uint32_t wx = 0; wx < 4; ++wx)
        for (uint32_t wy = 0; wy < 4; ++wy) {
          for (int l = 0; l < 32; ++l) lane_vals(g.data(), nn, on, wx, wy, l, vals[l]);
          row_mins(vals, on, wy, mv, mi);
          for (int l = 0; l < 32; l += 4)
            for (int h = 0; h < 2; ++h) {
              const uint32_t r = wx * 16 + l / 4 + 8 * h;
              if (r < nnum && mv[l][h] < kInf) append(nn[r], mi[l][h], mv[l][h]);
            }
          // columns 2c, 2c+1 (slots 0/2, 1/3), then 2c+8, 2c+9 (4/6, 5/7)
          const int pairs[4][2] = {{0, 2}, {1, 3}, {4, 6}, {5, 7}};
          const uint32_t add[4] = {0, 1, 8, 9};
          for (int q = 0; q < 4; ++q) {
            float cv[4];
            uint32_t ci[4];
            col_mins(vals, nn, wx, pairs[q][0], pairs[q][1], cv, ci);
            for (int l = 0; l < 4; ++l) {
              const uint32_t col = wy * 16 + l * 2 + add[q];
              if (col < onum && cv[l] < kInf) append(on[col], ci[l], cv[l]);
            }
          }
        }
    }
    gram(nn, nnum, nn, nnum, g.data());
    for (uint32_t wx = 0; wx < 4; ++wx)
      for (uint32_t wy = wx; wy < 4; ++wy) {
        for (int l = 0; l < 32; ++l) lane_vals(g.data(), nn, nn, wx, wy, l, vals[l]);
        row_mins(vals, nn, wy, mv, mi);
        for (int l = 0; l < 32; l += 4)
          for (int h = 0; h < 2; ++h) {
            const uint32_t r = wx * 16 + l / 4 + 8 * h;
            if (r < nnum) append(nn[r], mi[l][h], mv[l][h]);
          }
      }
  }

  // The merge shared by nn_descent_opt_merge, sample_kernel6 and
  // merge_reverse_plus: cand (ids, dists) sorted by distance, pos[] their
  // insertion points (K for dropped ones); own rows from the snapshot.
  // `rev` adds the reverse inserts of sample_kernel6 for every written entry.
  void merge_into(uint32_t u, const uint32_t* own_id, const float* own_d, const uint8_t* own_v,
                  const uint32_t* cid, const float* cd, const uint32_t* pos, uint32_t cnt,
                  bool keep_visit, bool rev) {
    if (cnt == 0) return;
    const size_t o = (size_t)u * K;
    for (uint32_t e = 0; e < K + cnt; ++e) {
      uint32_t r, id;
      float v;
      uint8_t vis = 0;
      if (e < (K / 32) * 32) {
        v = own_d[e];
        id = own_id[e];
        vis = own_v ? own_v[e] : 0;
        r = bsearch_pos<true>(cd, cnt, v) + e;
      } else {
        const uint32_t q = e - K;
        if (e < K || q >= cnt) continue;
        v = cd[q];
        id = cid[q];
        r = pos[q] + q;
      }
      if (r >= K) continue;
      nd[o + r] = v;
      graph[o + r] = id;
      if (keep_visit) visit[o + r] = vis;
      if (rev) {
        const uint32_t t = fetch_add(&rnum[id]);
        if (t < K) {
          rgraph[(size_t)id * K + t] = u;
          rd[(size_t)id * kRes + t] = v;
        } else if (v < rd[(size_t)id * kRes + (t % K)]) {
          rgraph[(size_t)id * K + t % K] = u;
          rd[(size_t)id * kRes + (t % K)] = v;
        }
      }
    }
  }

  // Insertion points of the candidates into the own row by distance, repeats
  // of an own (id, distance) marked INF with point K (:1084-1105).
  void positions(const uint32_t* own_id, const float* own_d, const uint32_t* cid, float* cd,
                 uint32_t* pos, uint32_t cnt, bool skip_marked) const {
    for (uint32_t i = 0; i < cnt; ++i) {
      if (skip_marked && pos[i] == K) continue;
      uint32_t r = bsearch_pos<false>(own_d, K, cd[i]);
      for (uint32_t t = 0; r + t < K && own_d[r + t] == cd[i]; ++t)
        if (own_id[r + t] == cid[i]) {
          cd[i] = kInf;
          r = K;
          break;
        }
      pos[i] = r;
    }
  }

  void sort_by_dist(float* cd, uint32_t* cid, uint32_t* pos, uint32_t cnt) const {
    network(cnt, [&](uint32_t a, uint32_t b) { return cd[a] > cd[b]; },
            [&](uint32_t a, uint32_t b) {
              std::swap(cd[a], cd[b]);
              std::swap(cid[a], cid[b]);
              std::swap(pos[a], pos[b]);
            });
  }

  void merge1(uint32_t u) {
    const size_t o = (size_t)u * K;
    const float min_ele = nd[o + K - 1];
    const uint32_t cnt_all = std::min(kRes, rnum[u]);
    uint32_t cid[kRes + 1], pos[kRes + 1];
    float cd[kRes + 1];
    std::fill(cid, cid + kRes + 1, kNone);
    std::fill(cd, cd + kRes + 1, kInf);
    uint32_t cnt = 0;
    for (uint32_t i = 0; i < cnt_all; ++i)
      if (rd[(size_t)u * kRes + i] < min_ele) {
        cid[cnt] = rgraph[(size_t)u * kRes + i];
        cd[cnt++] = rd[(size_t)u * kRes + i];
      }
    std::vector<uint32_t> own_id(graph.begin() + o, graph.begin() + o + K);
    std::vector<float> own_d(nd.begin() + o, nd.begin() + o + K);
    std::vector<uint8_t> own_v(visit.begin() + o, visit.begin() + o + K);
    own_d.push_back(kInf);  // the slot past the row the searches may read
    own_id.push_back(kNone);
    std::fill(pos, pos + kRes + 1, 0u);
    network(cnt, [&](uint32_t a, uint32_t b) { return cid[a] > cid[b]; },
            [&](uint32_t a, uint32_t b) {
              std::swap(cd[a], cd[b]);
              std::swap(cid[a], cid[b]);
            });
    for (uint32_t i = 0; i < cnt; ++i)
      if ((i > 0 && cid[i] == cid[i - 1]) || cid[i] == u) {
        pos[i] = K;
        cd[i] = kInf;
      }
    positions(own_id.data(), own_d.data(), cid, cd, pos, cnt, true);
    sort_by_dist(cd, cid, pos, cnt);
    merge_into(u, own_id.data(), own_d.data(), own_v.data(), cid, cd, pos, cnt, true, false);
  }

  void reverse_graph(uint32_t u) {
    for (uint32_t i = 0; i < K; ++i) {
      const uint32_t v = graph[(size_t)u * K + i];
      const uint32_t t = fetch_add(&rnum[v]);
      if (t < K) {
        rgraph[(size_t)v * K + t] = u;
        rd[(size_t)v * kRes + t] = nd[(size_t)u * K + i];
      }
    }
  }

  void reset_visit(uint32_t u) {
    for (uint32_t i = 0; i < K; ++i) {
      visit[(size_t)u * K + i] = 0;
      if (rgraph[(size_t)u * K + i] > n) rgraph[(size_t)u * K + i] = 0;
    }
    rnum[u] = 0;
  }

  // ---- phase 2 ----
  void sample2(uint32_t u, uint32_t it, uint64_t seed) {
    const size_t o = (size_t)u * K;
    uint32_t fetch[4];
    for (uint32_t g = 0; g < 4; ++g) {  // the lock hands slots to the groups in turn
      uint32_t t = g;
      while (t < K && visit[o + t]) ++t;
      if (t < K) visit[o + t] = 1;
      fetch[g] = t % K;
    }
    std::vector<uint32_t> cand(kMaxP);
    for (uint32_t tid = 0; tid < kMaxP; ++tid) {
      const uint32_t y = tid / 32, lane = tid % 32, g = y / 4;
      const uint32_t s = graph[o + fetch[g]];
      if (y % 4 < 2) cand[tid] = graph[(size_t)s * K + lane + (y % 4) * 32];
      else
        cand[tid] = rgraph[(size_t)s * K +
                           (uint32_t)(mix(seed ^ mix(((uint64_t)u << 24) ^ (it << 16) ^ tid)) % K)];
    }
    std::vector<uint32_t> own_sorted(kMaxP, kNone);
    for (uint32_t i = 0; i < K; ++i) own_sorted[i] = graph[o + i];
    network(kMaxP, [&](uint32_t a, uint32_t b) { return cand[a] > cand[b]; },
            [&](uint32_t a, uint32_t b) { std::swap(cand[a], cand[b]); });
    network(K, [&](uint32_t a, uint32_t b) { return own_sorted[a] > own_sorted[b]; },
            [&](uint32_t a, uint32_t b) { std::swap(own_sorted[a], own_sorted[b]); });
    std::vector<float> cdis(kMaxP);
    for (uint32_t i = 0; i < kMaxP; ++i)
      cdis[i] = (i > 0 && cand[i] == cand[i - 1]) || cand[i] == u ? kInf : 0.0f;
    for (uint32_t i = 0; i < kMaxP; ++i) {
      if (cdis[i] > 1.0f) continue;
      const uint32_t r = bsearch_pos<false>(own_sorted.data(), K, cand[i]);
      if (own_sorted[r] == cand[i]) cdis[i] = kInf;
    }
    const h16* q = x + (size_t)u * d;
    for (uint32_t i = 0; i < kMaxP; ++i)
      if (cdis[i] < 1.0f) cdis[i] = fp16_dist(q, cand[i]);
    const float min_ele = nd[o + K - 1];
    std::vector<uint32_t> cid, pos;
    std::vector<float> cd;
    for (uint32_t i = 0; i < kMaxP; ++i)
      if (cdis[i] < min_ele) {
        cid.push_back(cand[i]);
        cd.push_back(cdis[i]);
      }
    const uint32_t cnt = (uint32_t)cid.size();
    std::vector<uint32_t> own_id(graph.begin() + o, graph.begin() + o + K);
    std::vector<float> own_d(nd.begin() + o, nd.begin() + o + K);
    std::vector<uint8_t> own_v(visit.begin() + o, visit.begin() + o + K);
    own_d.push_back(kInf);
    own_id.push_back(kNone);
    pos.assign(cnt + 1, 0u);
    cd.push_back(kInf);
    cid.push_back(kNone);
    positions(own_id.data(), own_d.data(), cid.data(), cd.data(), pos.data(), cnt, false);
    sort_by_dist(cd.data(), cid.data(), pos.data(), cnt);
    merge_into(u, own_id.data(), own_d.data(), own_v.data(), cid.data(), cd.data(), pos.data(),
               cnt, true, true);
  }

  void merge_reverse(uint32_t u) {
    const size_t o = (size_t)u * K;
    const uint32_t cnt = std::min(K, rnum[u]);
    std::vector<uint32_t> own_id(graph.begin() + o, graph.begin() + o + K);
    std::vector<float> own_d(nd.begin() + o, nd.begin() + o + K);
    own_d.push_back(kInf);
    own_id.push_back(kNone);
    std::vector<uint32_t> rid(K + 1, kNone), pos(K + 1, 0u);
    std::vector<float> rdist(K + 1, kInf);
    for (uint32_t i = 0; i < cnt; ++i) {
      rid[i] = rgraph[o + i];
      rdist[i] = rd[(size_t)u * kRes + i];
    }
    network(cnt, [&](uint32_t a, uint32_t b) { return rid[a] > rid[b]; },
            [&](uint32_t a, uint32_t b) {
              std::swap(rdist[a], rdist[b]);
              std::swap(rid[a], rid[b]);
            });
    for (uint32_t i = 0; i < K; ++i) {
      const uint32_t r = bsearch_pos<false>(rid.data(), cnt, own_id[i]);
      if (rid[r] == own_id[i]) {
        pos[r] = K;
        rdist[r] = kInf;
      }
    }
    for (uint32_t i = 0; i < cnt; ++i) {
      uint32_t r = bsearch_pos<false>(own_d.data(), K, rdist[i]);
      for (uint32_t t = 0; r + t < K && std::fabs(own_d[r + t] - rdist[i]) < 0.1f; ++t)
        if (own_id[r + t] == rid[i]) {
          rdist[i] = kInf;
          r = K;
          break;
        }
      pos[i] = r;
    }
    sort_by_dist(rdist.data(), rid.data(), pos.data(), cnt);
    merge_into(u, own_id.data(), own_d.data(), nullptr, rid.data(), rdist.data(), pos.data(), cnt,
               false, false);
  }
};

}  // namespace

extern "C" {

// The reference's GNN_descent on an FP16 base (data_half, n x dim, already
// scaled), K neighbours, `iters` iterations split iter/2 + iter/2 as the
// reference does. Writes the final graph and distances (n x K).
int orc_gnn_descent_model(const uint16_t* data_half, uint32_t n, uint32_t dim, uint32_t K,
                          uint32_t iters, uint64_t seed, uint32_t* out_ids, float* out_dis) {
  if (K == 0 || K > 96 || K % 32 != 0 || dim % 4 != 0 || n <= K) return 1;
  Model m;
  m.n = n;
  m.d = dim;
  m.K = K;
  m.x = reinterpret_cast<const h16*>(data_half);
  m.xf.resize((size_t)n * dim);
  for (size_t i = 0; i < m.xf.size(); ++i) m.xf[i] = (float)m.x[i];
  m.init(seed);
  const uint32_t p1 = iters / 2, p2 = iters / 2;
  const int64_t N = n;
  for (uint32_t it = 0; it < p1; ++it) {
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < N; ++u) m.sample((uint32_t)u);
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < N; ++u) m.reverse_sample((uint32_t)u);
    std::fill(m.rnum.begin(), m.rnum.end(), 0u);
    std::fill(m.rnum_old.begin(), m.rnum_old.end(), 0u);
#pragma omp parallel
    {
      std::vector<float> g(64 * 64);
#pragma omp for schedule(dynamic, 256)
      for (int64_t u = 0; u < N; ++u) m.cal((uint32_t)u, g);
    }
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < N; ++u) m.merge1((uint32_t)u);
    std::fill(m.rnum.begin(), m.rnum.end(), 0u);
  }
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < N; ++u) m.reverse_graph((uint32_t)u);
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < N; ++u) m.reset_visit((uint32_t)u);
  for (uint32_t it = 0; it < p2; ++it) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t u = 0; u < N; ++u) m.sample2((uint32_t)u, it, seed);
    if (it + 1 < p2) std::fill(m.rnum.begin(), m.rnum.end(), 0u);
  }
#pragma omp parallel for schedule(static)
  for (int64_t u = 0; u < N; ++u) m.merge_reverse((uint32_t)u);
  std::copy(m.graph.begin(), m.graph.begin() + (size_t)n * K, out_ids);
  std::copy(m.nd.begin(), m.nd.end(), out_dis);
  return 0;
}

}  // extern "C"
