// Deterministic synthetic graph generators shared by host and device code.
//
// Every draw is a pure function of (seed, sample index, draw index) built on
// the splitmix64 finaliser, so a graph is identical whether it is produced by
// the host threads or by a device kernel, and independent of thread count.
// Probabilities are integer thresholds on 32-bit draws (no floating point).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define SCCG_HD __host__ __device__ __forceinline__
#else
#define SCCG_HD inline
#endif

namespace sccg {

SCCG_HD uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

SCCG_HD uint32_t mulhi32(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * (uint64_t)n) >> 32); }

// parts-per-million -> threshold on a uniform 32-bit draw
SCCG_HD uint64_t ppm_threshold(uint32_t ppm) { return ((uint64_t)ppm << 32) / 1000000ull; }

// Seeded bijection of [0, 2^bits): 4-round balanced Feistel network over
// 2*ceil(bits/2) bits with cycle walking back into range.
struct Perm {
  uint32_t bits, half;
  uint64_t key;
  SCCG_HD uint32_t round_f(uint32_t r, uint32_t i) const {
    return (uint32_t)mix64(key ^ ((uint64_t)i << 40) ^ r) & ((1u << half) - 1u);
  }
  SCCG_HD uint32_t once(uint32_t x) const {
    const uint32_t mask = (1u << half) - 1u;
    uint32_t l = x >> half, r = x & mask;
    for (uint32_t i = 0; i < 4; ++i) {
      const uint32_t t = l ^ round_f(r, i);
      l = r;
      r = t;
    }
    return (l << half) | r;
  }
  SCCG_HD uint32_t operator()(uint32_t x) const {
    if (bits == 0) return 0;
    const uint64_t lim = 1ull << bits;
    do {
      x = once(x);
    } while ((uint64_t)x >= lim);
    return x;
  }
};

SCCG_HD Perm make_perm(uint32_t bits, uint64_t seed) {
  Perm p;
  p.bits = bits;
  p.half = (bits + 1) / 2;
  if (p.half == 0) p.half = 1;
  p.key = mix64(seed ^ 0x7065726d75746174ull);
  return p;
}

// R-MAT draw of sample `i`: 0-based (src, dst) over 2^scale vertices.
// a,b,c thresholds are cumulative on a 32-bit draw: quadrant a = (0,0),
// b = (0,1), c = (1,0), d = (1,1); bits are fixed from the most significant.
struct Rmat {
  uint32_t scale;
  uint64_t seed;
  uint64_t ta, tb, tc;  // cumulative thresholds
  SCCG_HD void draw(uint64_t i, uint32_t &src, uint32_t &dst) const {
    const uint64_t base = mix64(seed ^ mix64(i ^ 0x524d4154ull));
    uint32_t s = 0, d = 0;
    uint64_t h = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      if ((l & 1u) == 0) h = mix64(base + (uint64_t)(l >> 1) * 0x9e3779b97f4a7c15ull);
      const uint64_t r = (l & 1u) ? (h >> 32) : (h & 0xffffffffull);
      uint32_t sb, db;
      if (r < ta) { sb = 0; db = 0; }
      else if (r < tb) { sb = 0; db = 1; }
      else if (r < tc) { sb = 1; db = 0; }
      else { sb = 1; db = 1; }
      s = (s << 1) | sb;
      d = (d << 1) | db;
    }
    src = s;
    dst = d;
  }
};

SCCG_HD Rmat make_rmat(uint32_t scale, uint32_t a_ppm, uint32_t b_ppm, uint32_t c_ppm, uint64_t seed) {
  Rmat r;
  r.scale = scale;
  r.seed = seed;
  r.ta = ppm_threshold(a_ppm);
  r.tb = ppm_threshold(a_ppm + b_ppm);
  r.tc = ppm_threshold(a_ppm + b_ppm + c_ppm);
  return r;
}

// Uniform directed draw over n vertices (0-based).
SCCG_HD void er_draw(uint64_t seed, uint64_t i, uint32_t n, uint32_t &src, uint32_t &dst) {
  const uint64_t h = mix64(seed ^ mix64(i ^ 0x4552ull));
  src = mulhi32((uint32_t)h, n);
  dst = mulhi32((uint32_t)(h >> 32), n);
}

// Grid edge `e` of a side x side grid: horizontal edges first
// ((i,j)-(i,j+1), e = i*(side-1)+j), then vertical ((i,j)-(i+1,j)).
// Each is oriented by a coin flip; with probability bidir_ppm it is kept in
// both directions.  Writes up to two 0-based directed edges, returns count.
SCCG_HD uint32_t grid_edge(uint64_t seed, uint32_t side, uint64_t e, uint32_t bidir_ppm, uint32_t *src,
                           uint32_t *dst) {
  const uint64_t hcount = (uint64_t)side * (side - 1);
  uint32_t a, b;
  if (e < hcount) {
    const uint32_t i = (uint32_t)(e / (side - 1)), j = (uint32_t)(e % (side - 1));
    a = i * side + j;
    b = a + 1;
  } else {
    const uint64_t f = e - hcount;
    const uint32_t i = (uint32_t)(f / side), j = (uint32_t)(f % side);
    a = i * side + j;
    b = a + side;
  }
  const uint64_t h = mix64(seed ^ mix64(e ^ 0x47524944ull));
  if ((h & 0xffffffffull) < ppm_threshold(bidir_ppm)) {
    src[0] = a; dst[0] = b;
    src[1] = b; dst[1] = a;
    return 2;
  }
  if ((h >> 32) & 1ull) { src[0] = a; dst[0] = b; }
  else { src[0] = b; dst[0] = a; }
  return 1;
}

// One graph of a batch of independent graphs (see plan_batch in scc_host.cpp).
struct BatchGraph {
  uint32_t n;        // vertices
  uint32_t type;     // 0 = Erdos-Renyi draws, 1 = R-MAT (0.57, 0.19, 0.19, 0.05)
  uint32_t scale;    // ceil(log2 n) for R-MAT
  uint32_t pad;
  uint64_t samples;  // edge draws
  uint64_t seed;
};

// Draw i of batch graph g: 0-based local (src, dst).  R-MAT draws over
// 2^scale ids are permuted by the graph's bijection and folded into [0, n).
SCCG_HD void batch_draw(const BatchGraph &g, uint64_t i, uint32_t &src, uint32_t &dst) {
  if (g.type == 0) {
    er_draw(g.seed, i, g.n, src, dst);
    return;
  }
  const Rmat r = make_rmat(g.scale, 570000, 190000, 190000, g.seed);
  const Perm p = make_perm(g.scale, g.seed);
  uint32_t s, d;
  r.draw(i, s, d);
  src = p(s) % g.n;
  dst = p(d) % g.n;
}

// Long-range edge k of the grid graph: uniform src, dst over side^2 vertices.
SCCG_HD void grid_longrange(uint64_t seed, uint32_t nverts, uint64_t k, uint32_t &src, uint32_t &dst) {
  er_draw(seed ^ 0x4c4f4e47ull, k, nverts, src, dst);
}

}  // namespace sccg
