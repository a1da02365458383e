// scc_solve_noalloc: the whole decomposition without any device allocation.
//
// Some callers cannot call cudaMalloc: plugins hosted by a framework that
// owns the whole device-memory budget and forbids side allocations (the
// framework's allocator, not the plugin, decides what lives on the device),
// and latency-critical host loops that must not hit the allocator's implicit
// device synchronisation.  For them this entry point runs the same
// persistent solve kernel as scc_solve_device, with every scratch buffer
// (labels, partitions, component sizes, bitmaps, worklists, election slots,
// control block) carved out of one file-scope device array instead of
// context-owned allocations.  The caller still passes the graph and the
// label output as device pointers.  The call returns once the solve has
// finished: it waits for `stream` to read back the result.
//
// Limits: at most kMaxN vertices and kMaxM edges per graph (the array is
// about 5 MB; every GPU that loads this library holds it until the process
// exits).  All calls share the array and it keeps the last call's contents;
// each call resets what must start fresh.  Calls that overlap on the GPU (two
// streams, two host threads) race on it and must be serialised by the caller.
// The first call on a device performs a one-time set-up for that device
// (looking up the array's device address with cudaGetSymbolAddress while the
// device is current).  cudaDeviceReset unloads the module that holds the
// array, so the address found by the set-up is no longer valid afterwards:
// a process that resets a device must not call this entry point on that
// device again (scc_solve_device has no such restriction).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "scc_capi.h"
#include "scc_engine.h"
#include "scc_internal.h"

namespace {

constexpr uint32_t kMaxN = 1u << 16;  // vertices
constexpr uint32_t kMaxM = 1u << 22;  // edges (each direction)
constexpr size_t a256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr uint32_t kWords = sccb::bitmap_words(kMaxN) + sccb::kBitmapSlack;
constexpr size_t kVec = a256(size_t(kMaxN + 1) * 4);        // one u32 per vertex
constexpr size_t kBitmaps = a256(size_t(kWords) * 4 * 7);   // elim, fvis, bvis, fexp, bexp, tflag, queued
constexpr size_t kSlots = a256(size_t(kMaxN + 1) * (3 * 8 + 8));  // election slots + asynchronous reach queue
constexpr uint32_t kHeavyCap = kMaxM / 256u + 2u;
constexpr size_t kHeavy = a256(size_t(kHeavyCap) * 5 * 4);
constexpr size_t kCtl = a256(sizeof(sccb::Ctl));
constexpr size_t kFlag = 256;  // CSR check flag
constexpr size_t kScratchBytes = 11 * kVec + kBitmaps + kSlots + kHeavy + kCtl + kFlag;

}  // namespace

// The scratch.  In host code `g_noalloc_scratch` is only a stand-in symbol:
// its device address comes from cudaGetSymbolAddress (below), once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// Set-up, done by the first call on each device with that device current.
int scratch_for_current_device(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sccb::set_error(SCC_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return sccb::set_error(SCC_ERR_CAPACITY, "device %d beyond %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return sccb::set_error(SCC_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return SCC_OK;
}

}  // namespace

extern "C" int scc_solve_noalloc(const scc_dev_csr *g, const scc_opts *opts, uint32_t *d_labels, uint32_t *nscc,
                                 void *stream) {
  sccb::clear_error();
  if (!g || !g->nodes || !g->nodesT || (g->m && (!g->edges || !g->edgesT)))
    return sccb::set_error(SCC_ERR_INVALID, "null graph");
  if (g->n > kMaxN || g->m > kMaxM)
    return sccb::set_error(SCC_ERR_CAPACITY,
                           "scc_solve_noalloc handles at most %u vertices and %u edges (got %u and %u); "
                           "use scc_solve_device for larger graphs",
                           kMaxN, kMaxM, g->n, g->m);
  scc_opts o;
  scc_opts_default(&o);
  if (opts) o = *opts;
  int rc = sccb::check_opts(&o);  // the same option set as the context entry points
  if (rc) return rc;
  // an error left by the caller's earlier work would otherwise surface as this solve's
  cudaError_t pending = cudaGetLastError();
  if (pending != cudaSuccess)
    return sccb::set_error(SCC_ERR_CUDA, "pending CUDA error before the solve: %s", cudaGetErrorString(pending));
  unsigned char *base = nullptr;
  rc = scratch_for_current_device(&base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t n = g->n;

  // carve the scratch (same roles as the context-owned buffers)
  sccb::Params p{};
  p.g.n = n;
  p.g.m = g->m;
  p.g.sorted_unique = g->sorted_unique ? 1u : 0u;
  p.g.off = g->nodes;
  p.g.adj = g->edges;
  p.g.offT = g->nodesT;
  p.g.adjT = g->edgesT;
  unsigned char *cur = base;
  auto vec = [&]() {
    uint32_t *r = reinterpret_cast<uint32_t *>(cur);
    cur += kVec;
    return r;
  };
  sccb::EngState &s = p.s;
  s.label = vec();
  s.range = vec();
  s.rpivot = vec();
  s.aux = vec();
  s.sccsize = vec();
  s.qa = vec();
  s.qb = vec();
  s.act[0] = vec();
  s.act[1] = vec();
  s.piv = vec();
  s.pivkey = vec();
  uint32_t *bm = reinterpret_cast<uint32_t *>(cur);
  cur += kBitmaps;
  s.elim = bm;
  s.fvis = bm + 1 * (size_t)kWords;
  s.bvis = bm + 2 * (size_t)kWords;
  s.fexp = bm + 3 * (size_t)kWords;
  s.bexp = bm + 4 * (size_t)kWords;
  s.tflag = bm + 5 * (size_t)kWords;
  s.queued = bm + 6 * (size_t)kWords;
  s.slot = reinterpret_cast<unsigned long long *>(cur);
  s.aq = reinterpret_cast<uint32_t *>(s.slot + 3 * ((size_t)n + 1));
  cur += kSlots;
  uint32_t *h = reinterpret_cast<uint32_t *>(cur);
  cur += kHeavy;
  s.hv = h;
  s.hbeg = h + (size_t)kHeavyCap;
  s.hdeg = h + 2 * (size_t)kHeavyCap;
  s.htag = h + 3 * (size_t)kHeavyCap;
  s.hbase = h + 4 * (size_t)kHeavyCap;
  s.ctl = reinterpret_cast<sccb::Ctl *>(cur);
  cur += kCtl;
  uint32_t *flag = reinterpret_cast<uint32_t *>(cur);
  s.seg = nullptr;
  s.out_labels = d_labels;
  s.nwords = sccb::bitmap_words(n);
  s.qcap = n + 1;
  s.hcap = kHeavyCap;
  s.nseg = 1;
  sccb::EngOpts &e = p.o;
  e.alg = (uint32_t)o.alg;
  e.wcc = o.wcc ? 1u : 0u;
  e.trim2 = o.trim2 ? 1u : 0u;
  e.trim_first = o.trim_first ? 1u : 0u;
  e.pivot_rule = (uint32_t)o.pivot_rule;
  e.switch_thr = (uint32_t)((uint64_t)n * (uint64_t)o.switch_permille / 1000ull);
  e.trim_depth = o.trim_depth;
  e.pull_alpha = o.pull_alpha;
  e.pull_beta = o.pull_beta;
  e.warp_degree = o.warp_degree ? o.warp_degree : 32u;
  e.heavy_degree = o.heavy_degree ? o.heavy_degree : 4096u;
  e.max_iters = o.max_iters ? o.max_iters : (1u << 20);
  e.timeout_ns = (unsigned long long)(o.timeout_ms ? o.timeout_ms : 10000u) * 1000000ull;
  e.trim_first_depth = o.trim_first_depth;
  e.async_depth = o.async_depth ? o.async_depth : 4;
  e.test_stall_ns = (unsigned long long)o.test_stall_us * 1000ull;
  if (o.test_queue_cap && o.test_queue_cap < s.qcap) s.qcap = o.test_queue_cap;
  if (d_labels) s.label = d_labels;  // labels go straight to the caller's buffer

  // the array keeps the previous call's contents: reset what must start fresh
  cudaError_t err = cudaMemsetAsync(s.ctl, 0, sizeof(sccb::Ctl), st);
  if (err == cudaSuccess) err = cudaMemsetAsync(s.slot, 0xff, ((size_t)n + 1) * (3 * 8 + 8), st);
  if (err != cudaSuccess) return sccb::set_error(SCC_ERR_CUDA, "scratch reset: %s", cudaGetErrorString(err));
  for (int t = 0; t < 2; ++t) {
    uint32_t bad = 0;
    err = sccb::check_device_csr(t ? g->nodesT : g->nodes, t ? g->edgesT : g->edges, n, g->m, flag, &bad, st);
    if (err != cudaSuccess) return sccb::set_error(SCC_ERR_CUDA, "CSR check: %s", cudaGetErrorString(err));
    if (bad) return sccb::set_error(SCC_ERR_INVALID, "device %s is malformed", t ? "transpose" : "graph");
  }
  err = sccb::launch_init(p, st);
  if (err == cudaSuccess) {
    uint32_t grid = 0;
    err = sccb::launch_phase(p, sccb::PH_SOLVE, 0, 0, 0, o.block_size ? o.block_size : 256, o.grid_blocks, st, &grid,
                             o.occupancy);
  }
  sccb::Ctl hc;
  if (err == cudaSuccess) err = cudaMemcpyAsync(&hc, s.ctl, sizeof(hc), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) return sccb::set_error(SCC_ERR_CUDA, "solve launch: %s", cudaGetErrorString(err));
  if (hc.gs.err) return sccb::set_error(SCC_ERR_TIMEOUT, "device-side wait or iteration cap ran out (0x%x)", hc.gs.err);
  if (hc.phase_ret) return sccb::set_error(SCC_ERR_STATE, "%u vertices left without a component", hc.phase_ret);
  if (nscc) *nscc = hc.nscc;
  return SCC_OK;
}
