// Device-side construction of the synthetic R-MAT graph: the same draws as
// the host generator (scc_gen.h), sorted and deduplicated with CUB radix
// sort, laid out as the reference's 1-based CSR plus transpose.  This is
// input preparation, not part of the SCC path.
#include <cub/cub.cuh>

#include <cstdint>
#include <vector>

#include "scc_gen.h"

namespace sccb {

namespace {

__global__ void rmat_keys_kernel(sccg::Rmat r, sccg::Perm pm, int permute, uint64_t samples,
                                 unsigned long long *keys) {
  const uint32_t scale = r.scale;
  const unsigned long long all = (1ull << (2 * scale)) - 1ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < samples;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s, d;
    r.draw(i, s, d);
    if (permute) {
      s = pm(s);
      d = pm(d);
    }
    keys[i] = s == d ? all : (((unsigned long long)s << scale) | d);
  }
}

// keep first copy of each key, drop self-loops (the sentinel is one)
__global__ void unique_flags_kernel(const unsigned long long *keys, uint64_t cnt, uint32_t scale, uint8_t *keep) {
  const unsigned long long mask = (1ull << scale) - 1ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    const bool self = (k >> scale) == (k & mask);
    keep[i] = !self && (i == 0 || keys[i - 1] != k);
  }
}

// adjacency (1-based low half) and degree histogram of the high half
__global__ void split_kernel(const unsigned long long *keys, uint32_t m, uint32_t scale, uint32_t *adj,
                             uint32_t *deg) {
  const unsigned long long mask = (1ull << scale) - 1ull;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    adj[i] = (uint32_t)(k & mask) + 1u;
    atomicAdd(deg + (uint32_t)(k >> scale) + 1u, 1u);  // deg[v+1] for 1-based v = hi+1 -> index hi+2 after shift
  }
}

__global__ void swap_kernel(const unsigned long long *keys, uint32_t m, uint32_t scale, unsigned long long *out) {
  const unsigned long long mask = (1ull << scale) - 1ull;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    out[i] = ((k & mask) << scale) | (k >> scale);
  }
}

struct Tmp {
  void *p = nullptr;
  size_t n = 0;
  ~Tmp() {
    if (p) cudaFree(p);
  }
  cudaError_t get(size_t b) {
    if (b <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, b ? b : 16);
    if (e == cudaSuccess) n = b;
    return e;
  }
};

#define GCK(x)                              \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

// sorted unique keys -> off (n+2, 1-based layout) and adj (m)
cudaError_t keys_to_csr(const unsigned long long *keys, uint32_t m, uint32_t scale, uint32_t n, uint32_t *off,
                        uint32_t *adj, Tmp &tmp, cudaStream_t st) {
  // deg: n+2 entries where deg[v+1] = out-degree of 1-based v
  GCK(cudaMemsetAsync(off, 0, ((size_t)n + 2) * 4, st));
  if (m) split_kernel<<<148 * 8, 256, 0, st>>>(keys, m, scale, adj, off + 1);
  GCK(cudaGetLastError());
  // off[v] = sum_{u < v} deg(u): inclusive scan of off[1..n+1] shifted
  // after split: off[1 + hi + 1] = deg of (hi+1) -> off[v+1] = deg(v); off[1] = 0
  size_t tb = 0;
  GCK(cub::DeviceScan::InclusiveSum(nullptr, tb, off + 1, off + 1, (int)(n + 1), st));
  GCK(tmp.get(tb));
  GCK(cub::DeviceScan::InclusiveSum(tmp.p, tb, off + 1, off + 1, (int)(n + 1), st));
  return cudaSuccess;
}

}  // namespace

namespace {

// Sorted-unique keys pipeline shared by the generators: A holds `samples`
// keys (src << bits | dst, 0-based, self-loops already replaced by the all-ones
// sentinel, itself a self-loop).  Produces the 1-based CSR + transpose of the
// n-vertex graph in freshly cudaMalloc'ed arrays.
cudaError_t keys_pipeline(Tmp &ka, Tmp &kb, uint64_t samples, uint32_t bits, uint32_t n, cudaStream_t st,
                          uint32_t **d_off, uint32_t **d_adj, uint32_t **d_offT, uint32_t **d_adjT, uint32_t *m_out) {
  unsigned long long *A = (unsigned long long *)ka.p, *B = (unsigned long long *)kb.p;
  Tmp flags, tmp, nsel;
  const int end_bit = 2 * (int)bits;
  size_t tb = 0;
  GCK(cub::DeviceRadixSort::SortKeys(nullptr, tb, A, B, (int)samples, 0, end_bit, st));
  GCK(tmp.get(tb));
  GCK(cub::DeviceRadixSort::SortKeys(tmp.p, tb, A, B, (int)samples, 0, end_bit, st));
  // B sorted; flag uniques and compact into A
  GCK(flags.get(samples));
  unique_flags_kernel<<<148 * 16, 256, 0, st>>>(B, samples, bits, (uint8_t *)flags.p);
  GCK(cudaGetLastError());
  GCK(nsel.get(16));
  GCK(cub::DeviceSelect::Flagged(nullptr, tb, B, (uint8_t *)flags.p, A, (int *)nsel.p, (int)samples, st));
  GCK(tmp.get(tb));
  GCK(cub::DeviceSelect::Flagged(tmp.p, tb, B, (uint8_t *)flags.p, A, (int *)nsel.p, (int)samples, st));
  int mi = 0;
  GCK(cudaMemcpyAsync(&mi, nsel.p, 4, cudaMemcpyDeviceToHost, st));
  GCK(cudaStreamSynchronize(st));
  const uint32_t m = (uint32_t)mi;
  uint32_t *off = nullptr, *adj = nullptr, *offT = nullptr, *adjT = nullptr;
  auto cleanup = [&]() {
    if (off) cudaFree(off);
    if (adj) cudaFree(adj);
    if (offT) cudaFree(offT);
    if (adjT) cudaFree(adjT);
  };
  cudaError_t e = cudaMalloc(&off, ((size_t)n + 2) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&adj, ((size_t)m + 1) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&offT, ((size_t)n + 2) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&adjT, ((size_t)m + 1) * 4);
  if (e == cudaSuccess) e = keys_to_csr(A, m, bits, n, off, adj, tmp, st);
  // transpose: swap halves, sort, split
  if (e == cudaSuccess && m) {
    swap_kernel<<<148 * 16, 256, 0, st>>>(A, m, bits, B);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(nullptr, tb, B, A, (int)m, 0, end_bit, st);
  if (e == cudaSuccess) e = tmp.get(tb);
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(tmp.p, tb, B, A, (int)m, 0, end_bit, st);
  if (e == cudaSuccess) e = keys_to_csr(A, m, bits, n, offT, adjT, tmp, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(adj + m, 0, 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(adjT + m, 0, 4, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cleanup();
    return e;
  }
  *d_off = off;
  *d_adj = adj;
  *d_offT = offT;
  *d_adjT = adjT;
  *m_out = m;
  return cudaSuccess;
}

// keys of every draw of every graph of a batch, ids made global by the
// graph's vertex base
__global__ void batch_keys_kernel(const sccg::BatchGraph *plan, const unsigned long long *draw_base,
                                  const uint32_t *vbase, uint32_t count, uint64_t total, uint32_t bits,
                                  unsigned long long *keys) {
  const unsigned long long all = (1ull << (2 * bits)) - 1ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = count - 1;  // graph: largest g with draw_base[g] <= i
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (draw_base[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    const sccg::BatchGraph g = plan[lo];
    uint32_t s, d;
    sccg::batch_draw(g, i - draw_base[lo], s, d);
    keys[i] = s == d ? all : (((unsigned long long)(vbase[lo] + s) << bits) | (vbase[lo] + d));
  }
}

}  // namespace

cudaError_t gen_rmat_device(uint32_t scale, uint64_t samples, uint32_t a_ppm, uint32_t b_ppm, uint32_t c_ppm,
                            uint64_t seed, int permute, cudaStream_t st, uint32_t **d_off, uint32_t **d_adj,
                            uint32_t **d_offT, uint32_t **d_adjT, uint32_t *m_out) {
  if (scale < 1 || scale > 29 || samples >= (1ull << 31)) return cudaErrorInvalidValue;
  const sccg::Rmat r = sccg::make_rmat(scale, a_ppm, b_ppm, c_ppm, seed);
  const sccg::Perm pm = sccg::make_perm(scale, seed);
  Tmp ka, kb;
  GCK(ka.get(samples * 8));
  GCK(kb.get(samples * 8));
  rmat_keys_kernel<<<148 * 16, 256, 0, st>>>(r, pm, permute, samples, (unsigned long long *)ka.p);
  GCK(cudaGetLastError());
  return keys_pipeline(ka, kb, samples, scale, 1u << scale, st, d_off, d_adj, d_offT, d_adjT, m_out);
}

cudaError_t gen_batch_device(const sccg::BatchGraph *plan, uint32_t count, cudaStream_t st, uint32_t **d_off,
                             uint32_t **d_adj, uint32_t **d_offT, uint32_t **d_adjT, uint32_t *n_out,
                             uint32_t *m_out) {
  if (count == 0) return cudaErrorInvalidValue;
  std::vector<unsigned long long> draw_base(count + 1, 0);
  std::vector<uint32_t> vbase(count + 1, 0);
  for (uint32_t g = 0; g < count; ++g) {
    draw_base[g + 1] = draw_base[g] + plan[g].samples;
    vbase[g + 1] = vbase[g] + plan[g].n;
  }
  const uint64_t total = draw_base[count];
  const uint32_t n = vbase[count];
  if (total >= (1ull << 31) || n >= (1u << 30)) return cudaErrorInvalidValue;
  uint32_t bits = 1;
  while ((1ull << bits) < (unsigned long long)n) ++bits;
  Tmp dplan, dbase, dv, ka, kb;
  GCK(dplan.get(sizeof(sccg::BatchGraph) * count));
  GCK(dbase.get(8ull * (count + 1)));
  GCK(dv.get(4ull * (count + 1)));
  GCK(cudaMemcpyAsync(dplan.p, plan, sizeof(sccg::BatchGraph) * count, cudaMemcpyHostToDevice, st));
  GCK(cudaMemcpyAsync(dbase.p, draw_base.data(), 8ull * (count + 1), cudaMemcpyHostToDevice, st));
  GCK(cudaMemcpyAsync(dv.p, vbase.data(), 4ull * (count + 1), cudaMemcpyHostToDevice, st));
  GCK(ka.get(total * 8 + 8));
  GCK(kb.get(total * 8 + 8));
  batch_keys_kernel<<<148 * 16, 256, 0, st>>>((const sccg::BatchGraph *)dplan.p, (const unsigned long long *)dbase.p,
                                             (const uint32_t *)dv.p, count, total, bits, (unsigned long long *)ka.p);
  GCK(cudaGetLastError());
  *n_out = n;
  return keys_pipeline(ka, kb, total, bits, n, st, d_off, d_adj, d_offT, d_adjT, m_out);
}

}  // namespace sccb
