// io.cpp -- fvecs loader and the five index writers, byte-compatible with the
// reference (src/common.cu:6-22 and :151-248). Errors are returned, never
// exit()ed.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace tagore {
namespace {

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) { f = std::fopen(path, mode); }
  ~File() {
    if (f) std::fclose(f);
  }
  bool write(const void* p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }
  bool close() {
    const bool ok = f && std::fclose(f) == 0;
    f = nullptr;
    return ok;
  }
};

// Writes `[deg][deg ids]` records of stride-k rows whose slot 0 is the degree.
bool write_rows(File& out, const uint32_t* graph, uint32_t n, uint32_t k, uint64_t* bytes,
                uint32_t* max_deg) {
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t gk = graph[(size_t)i * k];
    if (gk >= k) return false;  // a stride-k row holds at most k-1 ids
    if (!out.write(&gk, 4) || !out.write(graph + (size_t)i * k + 1, (size_t)gk * 4)) return false;
    if (bytes) *bytes += 4ull * (gk + 1);
    if (max_deg && gk > *max_deg) *max_deg = gk;
  }
  return true;
}

// Parses one of the five index layouts into CSR: a counting pass leaves offs
// and adj null; a filling pass writes at most n_cap rows and e_cap ids.
constexpr uint32_t kMaxRowDegree = 1u << 24;  // larger rows mean a corrupt file

int read_index(const char* path, const char* type_c, TagoreIndexInfo* info, uint64_t n_cap,
               uint64_t e_cap, uint64_t* offs, uint32_t* adj) {
  if (!path || !type_c || !info) return fail(TAGORE_EINVAL, "index reader: null argument");
  const std::string type(type_c);
  const bool nsg = type == "NSG", vamana = type == "Vamana", nssg = type == "NSSG",
             cagra = type == "CAGRA", dpg = type == "DPG";
  if (!nsg && !vamana && !nssg && !cagra && !dpg)
    return fail(TAGORE_EINVAL, "unknown index type '%s'", type_c);
  File in(path, "rb");
  if (!in.f) return fail(TAGORE_EIO, "cannot open '%s'", path);
  auto rd = [&](void* p, size_t bytes) { return std::fread(p, 1, bytes, in.f) == bytes; };
  TagoreIndexInfo r;
  std::memset(&r, 0, sizeof(r));
  uint64_t vamana_size = 0, dpg_rows = 0;
  if (nsg || nssg) {
    if (!rd(&r.width, 4)) return fail(TAGORE_EIO, "'%s': truncated header", path);
    if (nsg) {
      r.n_eps = 1;
      if (!rd(&r.eps[0], 4)) return fail(TAGORE_EIO, "'%s': truncated header", path);
    } else {
      if (!rd(&r.n_eps, 4)) return fail(TAGORE_EIO, "'%s': truncated header", path);
      for (uint32_t i = 0; i < r.n_eps; ++i) {
        uint32_t e;
        if (!rd(&e, 4)) return fail(TAGORE_EIO, "'%s': truncated entry points", path);
        if (i < 16) r.eps[i] = e;
      }
    }
  } else if (vamana) {
    uint64_t frozen = 0;
    r.n_eps = 1;
    if (!rd(&vamana_size, 8) || !rd(&r.width, 4) || !rd(&r.eps[0], 4) || !rd(&frozen, 8))
      return fail(TAGORE_EIO, "'%s': truncated header", path);
  } else if (dpg) {
    char magic[8];
    uint32_t major = 0, minor = 0, cnt = 0;
    if (!rd(magic, 8) || !rd(&major, 4) || !rd(&minor, 4) || !rd(&cnt, 4))
      return fail(TAGORE_EIO, "'%s': truncated header", path);
    if (std::memcmp(magic, "KNNGRAPH", 8) != 0) return fail(TAGORE_EIO, "'%s': not a KNNGRAPH file", path);
    dpg_rows = cnt;
  }
  uint64_t n = 0, edges = 0;
  if (offs) offs[0] = 0;
  std::vector<uint32_t> row;
  while (!dpg || n < dpg_rows) {
    uint32_t deg = 0;
    const size_t got = std::fread(&deg, 1, 4, in.f);
    if (got == 0 && !dpg) break;  // end of the rows
    if (got != 4) return fail(TAGORE_EIO, "'%s': truncated at row %llu", path, (unsigned long long)n);
    if (dpg) {
      uint32_t valid = 0;  // KGraph's second count; the row holds `deg` ids
      if (!rd(&valid, 4)) return fail(TAGORE_EIO, "'%s': truncated at row %llu", path, (unsigned long long)n);
    }
    if (deg > kMaxRowDegree)
      return fail(TAGORE_EIO, "'%s': row %llu claims %u ids", path, (unsigned long long)n, deg);
    row.resize(deg);
    if (!rd(row.data(), 4ull * deg))
      return fail(TAGORE_EIO, "'%s': truncated at row %llu", path, (unsigned long long)n);
    if (offs) {
      if (n >= n_cap || edges + deg > e_cap)
        return fail(TAGORE_EINVAL, "'%s': more rows or ids than the arrays hold", path);
      std::memcpy(adj + edges, row.data(), 4ull * deg);
      offs[n + 1] = edges + deg;
    }
    edges += deg;
    if (deg > r.max_degree) r.max_degree = deg;
    ++n;
  }
  if (vamana) {
    const long long end = std::ftell(in.f);
    if (end < 0 || (uint64_t)end != vamana_size)
      return fail(TAGORE_EIO, "'%s': header size %llu, file holds %lld bytes", path,
                  (unsigned long long)vamana_size, end);
  }
  if (offs && (n != n_cap || edges != e_cap))
    return fail(TAGORE_EINVAL, "'%s': holds %llu rows and %llu ids, not %llu and %llu", path,
                (unsigned long long)n, (unsigned long long)edges, (unsigned long long)n_cap,
                (unsigned long long)e_cap);
  r.n = n;
  r.edges = edges;
  *info = r;
  return TAGORE_OK;
}

}  // namespace
}  // namespace tagore

using namespace tagore;

extern "C" {

// load_data (src/common.cu:6-22): [int32 d][d floats] per vector; the count
// comes from the file size.
int tagore_load_fvecs_header(const char* path, uint32_t* n, uint32_t* dim) {
  File in(path, "rb");
  if (!in.f) return fail(TAGORE_EIO, "cannot open '%s'", path);
  uint32_t d = 0;
  if (std::fread(&d, 4, 1, in.f) != 1 || d == 0) return fail(TAGORE_EIO, "'%s': bad fvecs header", path);
  if (std::fseek(in.f, 0, SEEK_END) != 0) return fail(TAGORE_EIO, "'%s': seek failed", path);
  const long long sz = std::ftell(in.f);
  const unsigned long long rec = 4ull * (d + 1);
  if (sz <= 0 || (unsigned long long)sz % rec != 0)
    return fail(TAGORE_EIO, "'%s': size %lld is not a whole number of %u-dim records", path, sz, d);
  *n = (uint32_t)((unsigned long long)sz / rec);
  *dim = d;
  return TAGORE_OK;
}

int tagore_load_fvecs(const char* path, float* out, uint32_t n, uint32_t dim) {
  File in(path, "rb");
  if (!in.f) return fail(TAGORE_EIO, "cannot open '%s'", path);
  std::vector<char> buf(4ull * (dim + 1) * 4096);
  uint32_t done = 0;
  while (done < n) {
    const uint32_t cnt = std::min<uint32_t>(4096, n - done);
    const size_t bytes = 4ull * (dim + 1) * cnt;
    if (std::fread(buf.data(), 1, bytes, in.f) != bytes)
      return fail(TAGORE_EIO, "'%s': truncated at vector %u", path, done);
    for (uint32_t i = 0; i < cnt; ++i) {
      uint32_t d;
      std::memcpy(&d, buf.data() + 4ull * (dim + 1) * i, 4);
      if (d != dim) return fail(TAGORE_EIO, "'%s': vector %u has dim %u, expected %u", path, done + i, d, dim);
      std::memcpy(out + (size_t)(done + i) * dim, buf.data() + 4ull * (dim + 1) * i + 4, 4ull * dim);
    }
    done += cnt;
  }
  return TAGORE_OK;
}

int tagore_index_info(const char* path, const char* index_type, TagoreIndexInfo* info) {
  return read_index(path, index_type, info, 0, 0, nullptr, nullptr);
}

int tagore_index_read(const char* path, const char* index_type, uint64_t n, uint64_t edges,
                      uint64_t* offs, uint32_t* adj) {
  if (!offs || (!adj && edges)) return fail(TAGORE_EINVAL, "index reader: null output array");
  TagoreIndexInfo info;
  uint32_t dummy = 0;
  return read_index(path, index_type, &info, n, edges, offs, adj ? adj : &dummy);
}

// StoreNSG (src/common.cu:151-162): [u32 width][u32 ep] then [deg][ids] rows.
int tagore_store_nsg(const char* path, const uint32_t* graph, uint32_t width, uint32_t ep,
                     uint32_t n, uint32_t k) {
  File out(path, "wb");
  if (!out.f) return fail(TAGORE_EIO, "cannot create '%s'", path);
  if (!out.write(&width, 4) || !out.write(&ep, 4) || !write_rows(out, graph, n, k, nullptr, nullptr) ||
      !out.close())
    return fail(TAGORE_EIO, "write to '%s' failed", path);
  return TAGORE_OK;
}

// StoreVamana (src/common.cu:165-192): [u64 size][u32 max_degree][u32 ep]
// [u64 frozen = 0] then rows; size and max_degree are patched at the end.
int tagore_store_vamana(const char* path, const uint32_t* graph, uint32_t ep, uint32_t n,
                        uint32_t k) {
  File out(path, "wb");
  if (!out.f) return fail(TAGORE_EIO, "cannot create '%s'", path);
  uint64_t size = 24, frozen = 0;
  uint32_t maxd = 0;
  if (!out.write(&size, 8) || !out.write(&maxd, 4) || !out.write(&ep, 4) || !out.write(&frozen, 8) ||
      !write_rows(out, graph, n, k, &size, &maxd))
    return fail(TAGORE_EIO, "write to '%s' failed", path);
  if (std::fseek(out.f, 0, SEEK_SET) != 0 || !out.write(&size, 8) || !out.write(&maxd, 4) || !out.close())
    return fail(TAGORE_EIO, "write to '%s' failed", path);
  return TAGORE_OK;
}

// StoreNSSG (src/common.cu:195-216): [u32 width][u32 10][10 entry ids] then
// rows. The entry ids are the first ten of a std::random_shuffle of 0..n-1,
// which draws from the C library's rand() like the reference.
int tagore_store_nssg(const char* path, const uint32_t* graph, uint32_t width, uint32_t n,
                      uint32_t k) {
  File out(path, "wb");
  if (!out.f) return fail(TAGORE_EIO, "cannot create '%s'", path);
  std::vector<uint32_t> ids(n);
  for (uint32_t i = 0; i < n; ++i) ids[i] = i;
  for (uint32_t i = 1; i < n; ++i) {  // libstdc++'s random_shuffle loop
    const uint32_t j = (uint32_t)(std::rand() % (int)(i + 1));
    if (i != j) std::swap(ids[i], ids[j]);
  }
  const uint32_t n_ep = 10;
  std::vector<uint32_t> eps(n_ep, 0);
  for (uint32_t i = 0; i < n_ep && i < n; ++i) eps[i] = ids[i];
  if (!out.write(&width, 4) || !out.write(&n_ep, 4) || !out.write(eps.data(), 4 * n_ep) ||
      !write_rows(out, graph, n, k, nullptr, nullptr) || !out.close())
    return fail(TAGORE_EIO, "write to '%s' failed", path);
  return TAGORE_OK;
}

// StoreDPG (src/common.cu:219-237): "KNNGRAPH", u32 2, u32 0, u32 N, then per
// node [u32 deg][u32 deg][ids]. The reference reads stride-K rows from the
// dense stride-d rows filter_reverse_1hop wrote (pybind.cu:219-221); this
// writer takes the dense rows, deg = d.
int tagore_store_dpg(const char* path, const uint32_t* graph, uint32_t n, uint32_t degree) {
  File out(path, "wb");
  if (!out.f) return fail(TAGORE_EIO, "cannot create '%s'", path);
  const uint32_t major = 2, minor = 0;
  bool ok = out.write("KNNGRAPH", 8) && out.write(&major, 4) && out.write(&minor, 4) && out.write(&n, 4);
  for (uint32_t i = 0; ok && i < n; ++i)
    ok = out.write(&degree, 4) && out.write(&degree, 4) && out.write(graph + (size_t)i * degree, 4ull * degree);
  if (!ok || !out.close()) return fail(TAGORE_EIO, "write to '%s' failed", path);
  return TAGORE_OK;
}

// StoreCAGRA (src/common.cu:240-248): per node [u32 d][d ids] of dense rows.
int tagore_store_cagra(const char* path, const uint32_t* graph, uint32_t n, uint32_t degree) {
  File out(path, "wb");
  if (!out.f) return fail(TAGORE_EIO, "cannot create '%s'", path);
  bool ok = true;
  for (uint32_t i = 0; ok && i < n; ++i)
    ok = out.write(&degree, 4) && out.write(graph + (size_t)i * degree, 4ull * degree);
  if (!ok || !out.close()) return fail(TAGORE_EIO, "write to '%s' failed", path);
  return TAGORE_OK;
}

}  // extern "C"
