// Graph statistics for the strategy network: one pass over the offsets of the
// CSR and its transpose (degree moments, extremes, trim-1 yield of the first
// sweep), a sampled reciprocity test, and the sizes of the first three
// breadth-first levels from the highest-degree vertex.  All integer work on
// the device; the 16 floats are formed on the host from the accumulators.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "scc_engine.h"
#include "scc_features.h"

namespace sccb {
namespace {

struct FeatAcc {
  unsigned long long sum_out;
  unsigned long long hub_key;  // (in+out degree) << 32 | ~id: max picks the hub, ties to the smaller id
  double sumsq_out;
  uint32_t max_out, max_in;
  uint32_t z_out, z_in, z_any, one_out, one_in, low;
  uint32_t recip, recip_n;
  uint32_t lvl[4];  // sizes of BFS levels 0..3
  uint32_t pad[2];
};

constexpr uint32_t kSamples = 1u << 16;

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long x) {
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ double warp_sumd(double x) {
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ unsigned long long warp_max64(unsigned long long x) {
  for (int o = 16; o; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
    x = y > x ? y : x;
  }
  return x;
}

__global__ void degree_kernel(EngGraph g, FeatAcc *acc) {
  unsigned long long s = 0, hub = 0;
  double sq = 0.0;
  uint32_t mo = 0, mi = 0, zo = 0, zi = 0, za = 0, oo = 0, oi = 0, lo = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  // the loop bound is rounded up to a whole warp so every lane reaches the shuffles
  const uint32_t n_pad = (g.n + 31u) & ~31u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
    if (i < g.n) {
      const uint32_t v = i + 1;
      const uint32_t od = g.off[v + 1] - g.off[v];
      const uint32_t id = g.offT[v + 1] - g.offT[v];
      s += od;
      sq += (double)od * (double)od;
      mo = od > mo ? od : mo;
      mi = id > mi ? id : mi;
      zo += od == 0;
      zi += id == 0;
      za += (od == 0) | (id == 0);
      oo += od == 1;
      oi += id == 1;
      lo += (od <= 2) & (id <= 2);
      const unsigned long long key = ((unsigned long long)(od + id) << 32) | (0xffffffffu - v);
      hub = key > hub ? key : hub;
    }
  }
  s = warp_sum64(s);
  sq = warp_sumd(sq);
  hub = warp_max64(hub);
  mo = __reduce_max_sync(0xffffffffu, mo);
  mi = __reduce_max_sync(0xffffffffu, mi);
  zo = __reduce_add_sync(0xffffffffu, zo);
  zi = __reduce_add_sync(0xffffffffu, zi);
  za = __reduce_add_sync(0xffffffffu, za);
  oo = __reduce_add_sync(0xffffffffu, oo);
  oi = __reduce_add_sync(0xffffffffu, oi);
  lo = __reduce_add_sync(0xffffffffu, lo);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc->sum_out, s);
    atomicAdd(&acc->sumsq_out, sq);
    atomicMax(&acc->hub_key, hub);
    atomicMax(&acc->max_out, mo);
    atomicMax(&acc->max_in, mi);
    atomicAdd(&acc->z_out, zo);
    atomicAdd(&acc->z_in, zi);
    atomicAdd(&acc->z_any, za);
    atomicAdd(&acc->one_out, oo);
    atomicAdd(&acc->one_in, oi);
    atomicAdd(&acc->low, lo);
  }
}

// Does the sorted (or, if not sorted, scanned up to 4096 entries) list
// adj[b, e) contain x?
__device__ bool list_has(const uint32_t *adj, uint32_t b, uint32_t e, uint32_t x, bool sorted) {
  if (sorted) {
    while (b < e) {
      const uint32_t mid = b + (e - b) / 2;
      const uint32_t y = adj[mid];
      if (y == x) return true;
      if (y < x) b = mid + 1;
      else e = mid;
    }
    return false;
  }
  const uint32_t lim = e - b > 4096u ? b + 4096u : e;
  for (uint32_t j = b; j < lim; ++j)
    if (adj[j] == x) return true;
  return false;
}

// Sampled reciprocity: edge k*m/S (k < S); its source by binary search over
// the offsets; counts u->w with w->u also present (self-loops not sampled).
__global__ void recip_kernel(EngGraph g, uint32_t samples, FeatAcc *acc) {
  uint32_t hit = 0, cnt = 0;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < samples) {
    const uint32_t e = (uint32_t)(((unsigned long long)t * g.m) / samples);
    uint32_t lo = 1, hi = g.n;  // largest v with off[v] <= e
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if (g.off[mid] <= e) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t u = lo, w = g.adj[e];
    if (w != u && w >= 1 && w <= g.n) {
      cnt = 1;
      hit = list_has(g.adj, g.off[w], g.off[w + 1], u, g.sorted_unique != 0) ? 1u : 0u;
    }
  }
  hit = __reduce_add_sync(0xffffffffu, hit);
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if ((threadIdx.x & 31) == 0 && cnt) {
    atomicAdd(&acc->recip, hit);
    atomicAdd(&acc->recip_n, cnt);
  }
}

__global__ void bfs_seed_kernel(FeatAcc *acc, uint32_t *vis, uint32_t *list) {
  const uint32_t hub = 0xffffffffu - (uint32_t)(acc->hub_key & 0xffffffffu);
  list[0] = hub;
  atomicOr(&vis[hub >> 5], 1u << (hub & 31));
  acc->lvl[0] = 1;
}

// One level: a warp per frontier vertex, lanes over its out-edges; newly
// visited vertices are appended to the next list with one atomic per warp.
__global__ void bfs_level_kernel(EngGraph g, const uint32_t *cur, const uint32_t *cur_n, uint32_t *nxt,
                                 uint32_t *nxt_n, uint32_t *vis) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t count = *cur_n;
  for (uint32_t i = warp; i < count; i += nwarps) {
    const uint32_t v = cur[i];
    const uint32_t b = g.off[v], e = g.off[v + 1];
    for (uint32_t j0 = b; j0 < e; j0 += 32) {
      const uint32_t j = j0 + lane;
      bool fresh = false;
      uint32_t w = 0;
      if (j < e) {
        w = g.adj[j];
        const uint32_t bit = 1u << (w & 31);
        if (!(__ldcg(&vis[w >> 5]) & bit)) fresh = !(atomicOr(&vis[w >> 5], bit) & bit);
      }
      const uint32_t mask = __ballot_sync(0xffffffffu, fresh);
      if (mask) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(nxt_n, __popc(mask));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (fresh) nxt[base + __popc(mask & ((1u << lane) - 1u))] = w;
      }
    }
  }
}

}  // namespace

size_t features_scratch_bytes(uint32_t n) {
  const size_t words = ((size_t)n + 32) / 32 + 4;
  return sizeof(FeatAcc) + words * 4 + 2 * ((size_t)n + 1) * 4 + 64;
}

size_t features_acc_bytes() { return sizeof(FeatAcc); }

cudaError_t graph_features_launch(const EngGraph &g, void *scratch, size_t scratch_bytes, void *host_acc,
                                  cudaStream_t st) {
  if (g.n == 0) return cudaSuccess;  // graph_features_finish gives zeros
  if (scratch_bytes < features_scratch_bytes(g.n)) return cudaErrorInvalidValue;
  const size_t words = ((size_t)g.n + 32) / 32 + 4;
  FeatAcc *acc = reinterpret_cast<FeatAcc *>(scratch);
  uint32_t *vis = reinterpret_cast<uint32_t *>(acc + 1);
  uint32_t *la = vis + words, *lb = la + g.n + 1;
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(FeatAcc) + words * 4, st);
  if (e != cudaSuccess) return e;
  const uint32_t blocks = (g.n + 255) / 256 < 148u * 8 ? (g.n + 255) / 256 : 148u * 8;
  degree_kernel<<<blocks, 256, 0, st>>>(g, acc);
  const uint32_t samples = g.m < kSamples ? g.m : kSamples;
  if (samples) recip_kernel<<<(samples + 255) / 256, 256, 0, st>>>(g, samples, acc);
  bfs_seed_kernel<<<1, 1, 0, st>>>(acc, vis, la);
  // levels 1..3 alternate between the two lists; sizes land in acc->lvl[1..3]
  bfs_level_kernel<<<148 * 8, 256, 0, st>>>(g, la, &acc->lvl[0], lb, &acc->lvl[1], vis);
  bfs_level_kernel<<<148 * 8, 256, 0, st>>>(g, lb, &acc->lvl[1], la, &acc->lvl[2], vis);
  bfs_level_kernel<<<148 * 8, 256, 0, st>>>(g, la, &acc->lvl[2], lb, &acc->lvl[3], vis);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return cudaMemcpyAsync(host_acc, acc, sizeof(FeatAcc), cudaMemcpyDeviceToHost, st);
}

void graph_features_finish(uint32_t n, uint32_t m, const void *host_acc, float *feat) {
  std::memset(feat, 0, sizeof(float) * kFeatures);
  if (n == 0) return;
  const FeatAcc &h = *reinterpret_cast<const FeatAcc *>(host_acc);
  features_from_counts(n, m, h.sum_out, h.sumsq_out, h.max_out, h.max_in, h.z_out, h.z_in, h.z_any, h.one_out,
                       h.one_in, h.low, h.recip, h.recip_n, h.lvl, feat);
}

cudaError_t graph_features(const EngGraph &g, void *scratch, size_t scratch_bytes, float *feat,
                           cudaStream_t st) {
  FeatAcc h{};
  cudaError_t e = graph_features_launch(g, scratch, scratch_bytes, &h, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  graph_features_finish(g.n, g.m, &h, feat);
  return cudaSuccess;
}

void features_from_counts(uint32_t n, uint32_t m, unsigned long long sum_out, double sumsq_out, uint32_t max_out,
                          uint32_t max_in, uint32_t z_out, uint32_t z_in, uint32_t z_any, uint32_t one_out,
                          uint32_t one_in, uint32_t low, uint32_t recip, uint32_t recip_n, const uint32_t lvl[4],
                          float *f) {
  const double dn = n ? (double)n : 1.0;
  const double mean = (double)sum_out / dn;
  double var = sumsq_out / dn - mean * mean;
  if (var < 0) var = 0;
  const double ln = std::log2(dn + 1.0);
  f[0] = (float)std::log2(dn);
  f[1] = (float)std::log2((double)m + 1.0);
  f[2] = (float)mean;
  f[3] = (float)std::log2(1.0 + var);
  f[4] = (float)std::log2(1.0 + max_out);
  f[5] = (float)std::log2(1.0 + max_in);
  f[6] = (float)(z_out / dn);
  f[7] = (float)(z_in / dn);
  f[8] = (float)(z_any / dn);
  f[9] = (float)(one_out / dn);
  f[10] = (float)(one_in / dn);
  f[11] = (float)(low / dn);
  f[12] = recip_n ? (float)((double)recip / recip_n) : 0.f;
  f[13] = (float)(std::log2(1.0 + lvl[1]) / ln);
  f[14] = (float)(std::log2(1.0 + lvl[2]) / ln);
  f[15] = (float)(std::log2(1.0 + lvl[3]) / ln);
}

}  // namespace sccb
