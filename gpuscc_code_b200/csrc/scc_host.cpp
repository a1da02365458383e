// Host graph I/O for the SCC engine: load()-compatible reader, CSR builder,
// deterministic generators and the CPU decomposition behind the -t flag.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "scc_capi.h"
#include "scc_gen.h"
#include "scc_internal.h"

namespace {

unsigned hw_threads() {
  unsigned t = std::thread::hardware_concurrency();
  if (t == 0) t = 1;
  if (t > 64) t = 64;
  return t;
}

template <class F>
void parallel_for(uint64_t n, F &&f) {
  const unsigned nt = n < 65536 ? 1u : hw_threads();
  if (nt == 1) {
    f(0ull, n, 0u);
    return;
  }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t) {
    const uint64_t b = n * t / nt, e = n * (t + 1) / nt;
    th.emplace_back([&, b, e, t] { f(b, e, t); });
  }
  for (auto &x : th) x.join();
}

// sort each bucket, drop duplicates (and self-loops if asked), compact in place
void finish_lists(uint32_t n, std::vector<uint32_t> &off, std::vector<uint32_t> &adj, const uint32_t *owner_is,
                  bool drop_self) {
  (void)owner_is;
  std::vector<uint32_t> newdeg(n + 2, 0);
  parallel_for(n, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t i = b; i < e; ++i) {
      const uint32_t v = (uint32_t)i + 1;
      uint32_t *lo = adj.data() + off[v], *hi = adj.data() + off[v + 1];
      std::sort(lo, hi);
      uint32_t *w = lo;
      for (uint32_t *r = lo; r < hi; ++r) {
        if (drop_self && *r == v) continue;
        if (w != lo && *(w - 1) == *r) continue;
        *w++ = *r;
      }
      newdeg[v] = (uint32_t)(w - lo);
    }
  });
  // compact
  uint32_t pos = 0;
  for (uint32_t v = 1; v <= n; ++v) {
    const uint32_t b = off[v];
    const uint32_t d = newdeg[v];
    if (pos != b) std::memmove(adj.data() + pos, adj.data() + b, d * sizeof(uint32_t));
    off[v] = pos;
    pos += d;
  }
  off[n + 1] = pos;
  off[0] = 0;
  adj.resize(pos);
}

uint32_t *dup_array(const std::vector<uint32_t> &v, size_t extra) {
  uint32_t *p = (uint32_t *)std::malloc((v.size() + extra) * sizeof(uint32_t));
  if (!p) return nullptr;
  std::memcpy(p, v.data(), v.size() * sizeof(uint32_t));
  for (size_t i = 0; i < extra; ++i) p[v.size() + i] = 0;
  return p;
}

// ------------------------------------------------------------ loader helpers
constexpr char kBinMagic[8] = {'S', 'C', 'C', 'B', 'C', 'S', 'R', '1'};
// edge sections at least this long are parsed by all host threads
constexpr size_t kParallelParseBytes = 8u << 20;

struct BinHeader {
  char magic[8];
  uint32_t n, m, nnz_header;
  int32_t symmetric, sorted_unique, pad;
};

// Edge lines of a text graph split into one chunk per thread at line
// boundaries; each chunk is parsed on its own, then the first nnz non-blank
// lines are kept in file order, exactly as the serial reader would take them
// (a malformed line after those is never looked at, as in load.cpp).
int parse_edges_parallel(const char *path, const char *p, const char *end, uint32_t n, long long nnz,
                         bool symmetric, std::vector<uint32_t> &src, std::vector<uint32_t> &dst,
                         long long &count_edges) {
  const unsigned nt = hw_threads();
  std::vector<const char *> cut(nt + 1);
  cut[0] = p;
  cut[nt] = end;
  for (unsigned t = 1; t < nt; ++t) {
    const char *c = p + (size_t)(end - p) * t / nt;
    if (c < cut[t - 1]) c = cut[t - 1];
    while (c < end && c[-1] != '\n') ++c;
    cut[t] = c;
  }
  struct Part {
    std::vector<uint32_t> d, s;  // one entry per line (symmetric copies added later)
    long long bad_line = -1;     // first malformed or out-of-range line in this chunk
    int bad_kind = 0;            // 1 = unparsable, 2 = vertex out of range
  };
  std::vector<Part> parts(nt);
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t) {
    th.emplace_back([&, t] {
      Part &pt = parts[t];
      const char *q = cut[t], *qe = cut[t + 1];
      auto skip_ws = [&] {
        while (q < qe && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
      };
      auto read_int = [&](long long &x) -> bool {
        skip_ws();
        bool neg = false;
        if (q < qe && (*q == '-' || *q == '+')) neg = *q++ == '-';
        if (q >= qe || *q < '0' || *q > '9') return false;
        long long v = 0;
        while (q < qe && *q >= '0' && *q <= '9') v = v * 10 + (*q++ - '0');
        x = neg ? -v : v;
        return true;
      };
      while (q < qe) {
        skip_ws();
        if (q < qe && *q == '\n') {
          ++q;
          continue;
        }
        if (q >= qe) break;
        long long d = 0, sv = 0;
        const bool ok = read_int(d) && read_int(sv);
        while (q < qe && *q != '\n') ++q;
        if (q < qe) ++q;
        if (pt.bad_line < 0 && (!ok || d < 1 || d > n || sv < 1 || sv > n)) {
          pt.bad_line = (long long)pt.d.size();
          pt.bad_kind = ok ? 2 : 1;
        }
        pt.d.push_back(ok ? (uint32_t)d : 0u);
        pt.s.push_back(ok ? (uint32_t)sv : 0u);
      }
    });
  }
  for (auto &x : th) x.join();
  long long seen = 0;
  for (unsigned t = 0; t < nt && seen < nnz; ++t) {
    const Part &pt = parts[t];
    const long long take = std::min<long long>((long long)pt.d.size(), nnz - seen);
    if (pt.bad_line >= 0 && pt.bad_line < take) {
      const long long line = seen + pt.bad_line + 1;
      if (pt.bad_kind == 1) return sccb::set_error(SCC_ERR_IO, "%s: bad edge line %lld", path, line);
      return sccb::set_error(SCC_ERR_IO, "%s: edge line %lld names a vertex outside 1..%u", path, line, n);
    }
    for (long long i = 0; i < take; ++i) {
      const uint32_t d = pt.d[i], sv = pt.s[i];
      src.push_back(sv);  // edge src -> dst (load.cpp:78-93)
      dst.push_back(d);
      if (symmetric && d != sv) {
        src.push_back(d);
        dst.push_back(sv);
        ++count_edges;
      }
    }
    seen += take;
  }
  if (seen < nnz) return sccb::set_error(SCC_ERR_IO, "%s: %lld edge lines expected, %lld found", path, nnz, seen);
  return SCC_OK;
}

int load_binary(const char *path, const std::string &buf, scc_host_csr *out) {
  BinHeader h;
  if (buf.size() < sizeof(h)) return sccb::set_error(SCC_ERR_IO, "%s: truncated binary CSR", path);
  std::memcpy(&h, buf.data(), sizeof(h));
  const uint64_t words = 2ull * (h.n + 2ull) + 2ull * h.m;
  if (h.n >= (1u << 30) || buf.size() != sizeof(h) + words * 4)
    return sccb::set_error(SCC_ERR_IO, "%s: binary CSR size does not match its header", path);
  const uint32_t *w = reinterpret_cast<const uint32_t *>(buf.data() + sizeof(h));
  std::vector<uint32_t> off(w, w + h.n + 2), adj(w + h.n + 2, w + h.n + 2 + h.m);
  std::vector<uint32_t> offT(w + h.n + 2 + h.m, w + 2 * (h.n + 2) + h.m), adjT(w + 2 * (h.n + 2) + h.m, w + words);
  if (off[h.n + 1] != h.m || offT[h.n + 1] != h.m) return sccb::set_error(SCC_ERR_IO, "%s: binary CSR offsets corrupt", path);
  std::memset(out, 0, sizeof(*out));
  out->n = h.n;
  out->m = h.m;
  out->nnz_header = h.nnz_header;
  out->sorted_unique = h.sorted_unique;
  out->owned = 1;
  out->nodes = dup_array(off, 0);
  out->edges = dup_array(adj, 1);
  if (h.symmetric) {
    out->nodesT = out->nodes;
    out->edgesT = out->edges;
    out->symmetric = 1;
  } else {
    out->nodesT = dup_array(offT, 0);
    out->edgesT = dup_array(adjT, 1);
  }
  if (!out->nodes || !out->edges || !out->nodesT || !out->edgesT) {
    scc_host_csr_free(out);
    return sccb::set_error(SCC_ERR_NOMEM, "host allocation of %u-vertex CSR failed", h.n);
  }
  return SCC_OK;
}

}  // namespace

namespace sccb {

// Builds the reference layout (load.cpp:144-191) from 1-based pairs.
int build_csr(uint32_t n, uint64_t ne, const uint32_t *src, const uint32_t *dst, bool drop_self, scc_host_csr *out) {
  if (ne >= 0xffffffffull) return set_error(SCC_ERR_CAPACITY, "more than 2^32-1 edges");
  std::vector<uint32_t> off(n + 2, 0), adj(ne);
  for (uint64_t i = 0; i < ne; ++i) {
    if (src[i] < 1 || src[i] > n || dst[i] < 1 || dst[i] > n)
      return set_error(SCC_ERR_INVALID, "edge %llu (%u -> %u) outside 1..%u", (unsigned long long)i, src[i], dst[i], n);
    ++off[src[i] + 1];
  }
  // off[v+1] holds deg(v); exclusive scan so that off[v] = start of v
  off[0] = 0;
  off[1] = 0;
  for (uint32_t v = 1; v <= n; ++v) off[v + 1] += off[v];
  {
    std::vector<uint32_t> fill(off.begin(), off.end());
    for (uint64_t i = 0; i < ne; ++i) adj[fill[src[i]]++] = dst[i];
  }
  finish_lists(n, off, adj, nullptr, drop_self);
  const uint32_t m = off[n + 1];
  // transpose by counting; sources visited in increasing order keep lists sorted
  std::vector<uint32_t> offT(n + 2, 0), adjT(m);
  for (uint32_t i = 0; i < m; ++i) ++offT[adj[i] + 1];
  offT[0] = 0;
  offT[1] = 0;
  for (uint32_t v = 1; v <= n; ++v) offT[v + 1] += offT[v];
  {
    std::vector<uint32_t> fill(offT.begin(), offT.end());
    for (uint32_t v = 1; v <= n; ++v)
      for (uint32_t i = off[v]; i < off[v + 1]; ++i) adjT[fill[adj[i]]++] = v;
  }
  std::memset(out, 0, sizeof(*out));
  out->n = n;
  out->m = m;
  out->nnz_header = m;
  out->symmetric = 0;
  out->sorted_unique = 1;
  out->owned = 1;
  out->nodes = dup_array(off, 0);
  out->edges = dup_array(adj, 1);
  out->nodesT = dup_array(offT, 0);
  out->edgesT = dup_array(adjT, 1);
  if (!out->nodes || !out->edges || !out->nodesT || !out->edgesT) {
    scc_host_csr_free(out);
    return set_error(SCC_ERR_NOMEM, "host allocation of %u-vertex CSR failed", n);
  }
  return SCC_OK;
}

int plan_batch(uint32_t count, uint32_t n_lo, uint32_t n_hi, uint32_t deg_lo_milli, uint32_t deg_hi_milli,
               uint64_t seed, std::vector<sccg::BatchGraph> *plan) {
  if (count == 0 || n_lo < 2 || n_hi < n_lo || deg_hi_milli < deg_lo_milli)
    return set_error(SCC_ERR_INVALID, "bad batch arguments");
  plan->resize(count);
  const double ln_lo = std::log((double)n_lo), ln_hi = std::log((double)n_hi);
  for (uint32_t g = 0; g < count; ++g) {
    const uint64_t h = sccg::mix64(seed ^ sccg::mix64((uint64_t)g ^ 0x4241544348ull));
    const double u1 = (double)(h & 0xffffffffull) / 4294967296.0;
    const double u2 = (double)((h >> 32) & 0x7fffffffull) / 2147483648.0;
    sccg::BatchGraph b{};
    uint32_t n = (uint32_t)std::floor(std::exp(ln_lo + u1 * (ln_hi - ln_lo)));
    b.n = n < n_lo ? n_lo : (n > n_hi ? n_hi : n);
    b.type = (uint32_t)(h >> 63);
    b.scale = 1;
    while ((1u << b.scale) < b.n) ++b.scale;
    const double deg = (deg_lo_milli + u2 * (double)(deg_hi_milli - deg_lo_milli)) / 1000.0;
    b.samples = (uint64_t)std::llround(deg * b.n);
    b.seed = sccg::mix64(seed + g + 1);
    (*plan)[g] = b;
  }
  return SCC_OK;
}

}  // namespace sccb

using sccb::set_error;

extern "C" {

void scc_host_csr_free(scc_host_csr *c) {
  if (!c) return;
  if (c->owned) {
    const bool same = c->nodesT == c->nodes;
    std::free(c->nodes);
    std::free(c->edges);
    if (!same) {
      std::free(c->nodesT);
      std::free(c->edgesT);
    }
  }
  std::memset(c, 0, sizeof(*c));
}

int scc_batch_pack(uint32_t count, const scc_host_csr *graphs, scc_host_csr *out, uint32_t *seg_first) {
  sccb::clear_error();
  if (!out || !seg_first || (count && !graphs)) return set_error(SCC_ERR_INVALID, "null argument");
  uint64_t N = 0, M = 0;
  bool sorted = true;
  for (uint32_t g = 0; g < count; ++g) {
    const scc_host_csr &c = graphs[g];
    if (!c.nodes || !c.nodesT || (c.m && (!c.edges || !c.edgesT)))
      return set_error(SCC_ERR_INVALID, "graph %u: arrays missing", g);
    if (c.nodes[c.n + 1] != c.m || c.nodesT[c.n + 1] != c.m)
      return set_error(SCC_ERR_INVALID, "graph %u: offsets end at %u/%u, expected m = %u", g, c.nodes[c.n + 1],
                       c.nodesT[c.n + 1], c.m);
    N += c.n;
    M += c.m;
    sorted = sorted && c.sorted_unique;
  }
  if (N >= (1ull << 30) || M >= (1ull << 32)) return set_error(SCC_ERR_CAPACITY, "packed batch exceeds 32-bit ids");
  std::vector<uint32_t> off(N + 2), offT(N + 2), adj(M + 1), adjT(M + 1);
  uint32_t vb = 0, eb = 0;
  seg_first[0] = 1;
  for (uint32_t g = 0; g < count; ++g) {
    const scc_host_csr &c = graphs[g];
    for (uint32_t v = 1; v <= c.n + 1; ++v) {  // entry n+1 equals the next graph's first
      off[vb + v] = c.nodes[v] + eb;
      offT[vb + v] = c.nodesT[v] + eb;
    }
    for (uint32_t j = 0; j < c.m; ++j) {
      adj[eb + j] = c.edges[j] + vb;
      adjT[eb + j] = c.edgesT[j] + vb;
    }
    vb += c.n;
    eb += c.m;
    seg_first[g + 1] = vb + 1;
  }
  off[N + 1] = offT[N + 1] = (uint32_t)M;
  std::memset(out, 0, sizeof(*out));
  out->n = (uint32_t)N;
  out->m = (uint32_t)M;
  out->nnz_header = (uint32_t)M;
  out->sorted_unique = sorted ? 1 : 0;
  out->owned = 1;
  out->nodes = dup_array(off, 0);
  out->edges = dup_array(adj, 0);
  out->nodesT = dup_array(offT, 0);
  out->edgesT = dup_array(adjT, 0);
  if (!out->nodes || !out->edges || !out->nodesT || !out->edgesT) {
    scc_host_csr_free(out);
    return set_error(SCC_ERR_NOMEM, "host allocation of the packed batch failed");
  }
  return SCC_OK;
}

int scc_csr_from_edges(uint32_t n, uint64_t n_edges, const uint32_t *src, const uint32_t *dst, int drop_self_loops,
                       scc_host_csr *out) {
  sccb::clear_error();
  if (!out || (n_edges && (!src || !dst))) return set_error(SCC_ERR_INVALID, "null argument");
  if (n >= (1u << 30)) return set_error(SCC_ERR_CAPACITY, "n must be below 2^30");
  return sccb::build_csr(n, n_edges, src, dst, drop_self_loops != 0, out);
}

// ---------------------------------------------------------------- loader
// load.cpp:18-207, same semantics, linear-time parsing.
int scc_save(const char *path, const scc_host_csr *g) {
  sccb::clear_error();
  if (!path || !g || !g->nodes || !g->nodesT || (g->m && (!g->edges || !g->edgesT)))
    return set_error(SCC_ERR_INVALID, "null argument");
  FILE *f = std::fopen(path, "wb");
  if (!f) return set_error(SCC_ERR_IO, "cannot create %s", path);
  BinHeader h{};
  std::memcpy(h.magic, kBinMagic, 8);
  h.n = g->n;
  h.m = g->m;
  h.nnz_header = g->nnz_header;
  h.symmetric = g->symmetric;
  h.sorted_unique = g->sorted_unique;
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  ok = ok && std::fwrite(g->nodes, 4, (size_t)g->n + 2, f) == (size_t)g->n + 2;
  ok = ok && std::fwrite(g->edges, 4, g->m, f) == g->m;
  ok = ok && std::fwrite(g->nodesT, 4, (size_t)g->n + 2, f) == (size_t)g->n + 2;
  ok = ok && std::fwrite(g->edgesT, 4, g->m, f) == g->m;
  ok = std::fclose(f) == 0 && ok;
  return ok ? SCC_OK : set_error(SCC_ERR_IO, "writing %s failed", path);
}

int scc_load(const char *path, int header, scc_host_csr *out) {
  (void)header;  // load.cpp ignores it as well
  sccb::clear_error();
  if (!path || !out) return set_error(SCC_ERR_INVALID, "null argument");
  std::memset(out, 0, sizeof(*out));
  FILE *f = std::fopen(path, "rb");
  if (!f) return set_error(SCC_ERR_IO, "cannot open %s", path);
  std::string buf;
  {
    char tmp[1 << 16];
    size_t r;
    while ((r = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, r);
    std::fclose(f);
  }
  size_t pos = 0;
  auto next_line = [&](std::string &line) -> bool {
    if (pos >= buf.size()) return false;
    size_t e = buf.find('\n', pos);
    if (e == std::string::npos) e = buf.size();
    line.assign(buf, pos, e - pos);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    pos = e + 1;
    return true;
  };
  if (buf.size() >= 8 && std::memcmp(buf.data(), kBinMagic, 8) == 0) return load_binary(path, buf, out);
  std::string line;
  if (!next_line(line)) return set_error(SCC_ERR_IO, "%s: empty file", path);
  const bool pattern = std::strstr(line.c_str(), "pattern") != nullptr;
  const bool symmetric = std::strstr(line.c_str(), "symmetric") != nullptr;
  (void)pattern;  // the weight column, if any, is ignored either way
  while (!line.empty() && line[0] == '%') {
    if (!next_line(line)) return set_error(SCC_ERR_IO, "%s: no header line", path);
  }
  long long m0 = -1, n0 = -1, nnz = -1;
  if (std::strstr(path, ".mtx")) {
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &m0, &n0, &nnz) != 3)
      return set_error(SCC_ERR_IO, "%s: bad MatrixMarket size line", path);
    if (m0 != n0) return set_error(SCC_ERR_IO, "%s: matrix is %lld x %lld, not square", path, m0, n0);
  } else {
    if (std::sscanf(line.c_str(), "%lld %lld", &m0, &nnz) != 2)
      return set_error(SCC_ERR_IO, "%s: bad header line", path);
  }
  if (m0 < 0 || nnz < 0) return set_error(SCC_ERR_IO, "%s: negative sizes", path);
  if (m0 >= (1ll << 30)) return set_error(SCC_ERR_CAPACITY, "%s: %lld vertices exceed 2^30", path, m0);
  const uint32_t n = (uint32_t)m0;
  std::vector<uint32_t> src, dst;
  src.reserve((size_t)nnz * (symmetric ? 2 : 1));
  dst.reserve((size_t)nnz * (symmetric ? 2 : 1));
  long long count_edges = nnz;
  const char *p = buf.c_str() + pos;
  const char *end = buf.c_str() + buf.size();
  auto skip_ws = [&]() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  };
  auto read_int = [&](long long &x) -> bool {
    skip_ws();
    bool neg = false;
    if (p < end && (*p == '-' || *p == '+')) neg = *p++ == '-';
    if (p >= end || *p < '0' || *p > '9') return false;
    long long v = 0;
    while (p < end && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
    x = neg ? -v : v;
    return true;
  };
  if ((size_t)(end - p) >= kParallelParseBytes && hw_threads() > 1) {
    int prc = parse_edges_parallel(path, p, end, n, nnz, symmetric, src, dst, count_edges);
    if (prc != SCC_OK) return prc;
  } else
  for (long long i = 0; i < nnz;) {
    // skip blank lines
    skip_ws();
    if (p < end && *p == '\n') {
      ++p;
      continue;
    }
    if (p >= end) return set_error(SCC_ERR_IO, "%s: %lld edge lines expected, %lld found", path, nnz, i);
    long long d = 0, s = 0;
    if (!read_int(d) || !read_int(s)) return set_error(SCC_ERR_IO, "%s: bad edge line %lld", path, i + 1);
    while (p < end && *p != '\n') ++p;  // weight / rest of line
    if (p < end) ++p;
    if (d < 1 || d > n || s < 1 || s > n)
      return set_error(SCC_ERR_IO, "%s: edge line %lld names a vertex outside 1..%u", path, i + 1, n);
    // edge src -> dst (load.cpp:78-93)
    src.push_back((uint32_t)s);
    dst.push_back((uint32_t)d);
    if (symmetric && d != s) {
      src.push_back((uint32_t)d);
      dst.push_back((uint32_t)s);
      ++count_edges;
    }
    ++i;
  }
  int rc = sccb::build_csr(n, src.size(), src.data(), dst.data(), false, out);
  if (rc != SCC_OK) return rc;
  out->nnz_header = (uint32_t)count_edges;
  if (symmetric) {
    // load.cpp:199-202: the transpose is the graph itself
    std::free(out->nodesT);
    std::free(out->edgesT);
    out->nodesT = out->nodes;
    out->edgesT = out->edges;
    out->symmetric = 1;
  }
  return SCC_OK;
}

// ------------------------------------------------------------- generators
int scc_gen_rmat(uint32_t scale, uint64_t samples, uint32_t a_ppm, uint32_t b_ppm, uint32_t c_ppm, uint64_t seed,
                 int permute, scc_host_csr *out) {
  sccb::clear_error();
  if (!out || scale > 29 || (uint64_t)a_ppm + b_ppm + c_ppm > 1000000ull)
    return set_error(SCC_ERR_INVALID, "bad R-MAT arguments");
  const uint32_t n = 1u << scale;
  std::vector<uint32_t> src(samples), dst(samples);
  const sccg::Rmat r = sccg::make_rmat(scale, a_ppm, b_ppm, c_ppm, seed);
  const sccg::Perm pm = sccg::make_perm(scale, seed);
  parallel_for(samples, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t i = b; i < e; ++i) {
      uint32_t s, d;
      r.draw(i, s, d);
      if (permute) {
        s = pm(s);
        d = pm(d);
      }
      src[i] = s + 1;
      dst[i] = d + 1;
    }
  });
  return sccb::build_csr(n, samples, src.data(), dst.data(), true, out);
}

int scc_gen_er(uint32_t n, uint64_t samples, uint64_t seed, scc_host_csr *out) {
  sccb::clear_error();
  if (!out || n == 0 || n >= (1u << 30)) return set_error(SCC_ERR_INVALID, "bad ER arguments");
  std::vector<uint32_t> src(samples), dst(samples);
  parallel_for(samples, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t i = b; i < e; ++i) {
      uint32_t s, d;
      sccg::er_draw(seed, i, n, s, d);
      src[i] = s + 1;
      dst[i] = d + 1;
    }
  });
  return sccb::build_csr(n, samples, src.data(), dst.data(), true, out);
}

int scc_gen_grid(uint32_t side, uint32_t bidir_ppm, uint32_t longrange_ppm, uint64_t seed, scc_host_csr *out) {
  sccb::clear_error();
  if (!out || side < 2 || (uint64_t)side * side >= (1ull << 30)) return set_error(SCC_ERR_INVALID, "bad grid side");
  const uint32_t n = side * side;
  const uint64_t ge = 2ull * side * (side - 1);
  const uint64_t lr = ge * longrange_ppm / 1000000ull;
  std::vector<uint32_t> src(2 * ge + lr), dst(2 * ge + lr);
  std::vector<uint8_t> cnt(ge);
  parallel_for(ge, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t i = b; i < e; ++i) {
      uint32_t s[2], d[2];
      const uint32_t k = sccg::grid_edge(seed, side, i, bidir_ppm, s, d);
      cnt[i] = (uint8_t)k;
      for (uint32_t j = 0; j < 2; ++j) {
        src[2 * i + j] = j < k ? s[j] + 1 : 0;
        dst[2 * i + j] = j < k ? d[j] + 1 : 0;
      }
    }
  });
  uint64_t w = 0;
  for (uint64_t i = 0; i < 2 * ge; ++i)
    if (src[i]) {
      src[w] = src[i];
      dst[w] = dst[i];
      ++w;
    }
  for (uint64_t k = 0; k < lr; ++k) {
    uint32_t s, d;
    sccg::grid_longrange(seed, n, k, s, d);
    src[w] = s + 1;
    dst[w] = d + 1;
    ++w;
  }
  return sccb::build_csr(n, w, src.data(), dst.data(), true, out);
}

int scc_gen_batch(uint32_t count, uint32_t n_lo, uint32_t n_hi, uint32_t deg_lo_milli, uint32_t deg_hi_milli,
                  uint64_t seed, scc_host_csr *out, uint32_t *seg_first) {
  sccb::clear_error();
  if (!out || !seg_first) return set_error(SCC_ERR_INVALID, "null output");
  std::vector<sccg::BatchGraph> plan;
  int rc = sccb::plan_batch(count, n_lo, n_hi, deg_lo_milli, deg_hi_milli, seed, &plan);
  if (rc) return rc;
  std::vector<uint64_t> draw_base(count + 1, 0);
  seg_first[0] = 1;
  for (uint32_t g = 0; g < count; ++g) {
    draw_base[g + 1] = draw_base[g] + plan[g].samples;
    seg_first[g + 1] = seg_first[g] + plan[g].n;
  }
  const uint64_t total = draw_base[count];
  const uint64_t n = (uint64_t)seg_first[count] - 1;
  if (n >= (1u << 30)) return set_error(SCC_ERR_CAPACITY, "batch has %llu vertices", (unsigned long long)n);
  std::vector<uint32_t> src(total), dst(total);
  parallel_for(count, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t g = b; g < e; ++g) {
      const uint32_t base = seg_first[g];
      for (uint64_t i = 0; i < plan[g].samples; ++i) {
        uint32_t s, d;
        sccg::batch_draw(plan[g], i, s, d);
        src[draw_base[g] + i] = base + s;
        dst[draw_base[g] + i] = base + d;
      }
    }
  });
  return sccb::build_csr((uint32_t)n, total, src.data(), dst.data(), true, out);
}

// ------------------------------------------------------------ -t Tarjan
// The CPU decomposition the apps run for -t (tarjan.h:5, tarjan.cpp:72-240):
// sequential, one host thread.  Iterative Tarjan with an explicit
// (vertex, next-edge) call stack, so the stack is O(n) rather than O(m).
int scc_tarjan(const scc_host_csr *g, uint32_t *labels, uint32_t *nscc, double *secs) {
  sccb::clear_error();
  if (!g || (g->n && (!g->nodes || !g->edges))) return set_error(SCC_ERR_INVALID, "null graph");
  const auto t0 = std::chrono::steady_clock::now();
  const uint32_t n = g->n;
  std::vector<uint32_t> index(n + 1, 0), low(n + 1, 0), comp(n + 1, 0);
  std::vector<uint32_t> stk;
  std::vector<std::pair<uint32_t, uint32_t>> call;
  stk.reserve(1024);
  call.reserve(1024);
  std::vector<uint8_t> onstk(n + 1, 0);
  uint32_t next = 1, count = 0;
  for (uint32_t root = 1; root <= n; ++root) {
    if (index[root]) continue;
    call.emplace_back(root, g->nodes[root]);
    index[root] = low[root] = next++;
    stk.push_back(root);
    onstk[root] = 1;
    while (!call.empty()) {
      const uint32_t v = call.back().first;
      uint32_t &ei = call.back().second;
      if (ei < g->nodes[v + 1]) {
        const uint32_t u = g->edges[ei++];
        if (!index[u]) {
          index[u] = low[u] = next++;
          stk.push_back(u);
          onstk[u] = 1;
          call.emplace_back(u, g->nodes[u]);
        } else if (onstk[u] && index[u] < low[v]) {
          low[v] = index[u];
        }
        continue;
      }
      if (low[v] == index[v]) {
        uint32_t mn = v, w;
        const size_t top = stk.size();
        size_t i = top;
        do {
          w = stk[--i];
          mn = w < mn ? w : mn;
        } while (w != v);
        for (size_t j = i; j < top; ++j) {
          comp[stk[j]] = mn;
          onstk[stk[j]] = 0;
        }
        stk.resize(i);
        ++count;
      }
      call.pop_back();
      if (!call.empty()) {
        const uint32_t p = call.back().first;
        if (low[v] < low[p]) low[p] = low[v];
      }
    }
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (labels) {
    labels[0] = 0;
    for (uint32_t v = 1; v <= n; ++v) labels[v] = comp[v];
  }
  if (nscc) *nscc = count;
  if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
  return SCC_OK;
}

}  // extern "C"
