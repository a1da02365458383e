// C ABI of the SCC engine: contexts, device residency, the whole-solve
// launch and the phase-level entry points (see include/scc_capi.h).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "scc_capi.h"
#include "scc_engine.h"
#include "scc_features.h"
#include "scc_internal.h"

namespace sccb {

static thread_local char g_err[1024] = "";

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}
void clear_error() { g_err[0] = 0; }

}  // namespace sccb

using sccb::set_error;

namespace {

struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b) {
    if (b == 0) b = 16;
    if (b <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T *as() const {
    return reinterpret_cast<T *>(p);
  }
};

}  // namespace

struct scc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  scc_opts opts{};
  // bound graph
  uint32_t n = 0, m = 0;
  int sorted_unique = 0;
  bool have_graph = false;
  const uint32_t *d_off = nullptr, *d_adj = nullptr, *d_offT = nullptr, *d_adjT = nullptr;
  DBuf g_off, g_adj, g_offT, g_adjT;  // owned graph storage
  // per-vertex state
  uint32_t cap_n = 0, cap_h = 0;
  bool have_state = false;
  DBuf label, range, rpivot, aux, sccsize, bitmaps, qa, qb, act0, act1, piv, pivkey, slot, heavy, ctl, seg;
  DBuf feat;  // scratch of scc_graph_features
  uint32_t nwords = 0;
  bool slot_dirty = true;
  uint32_t nseg = 0;
  std::vector<uint32_t> seg_host;
  bool phase_ready = false;
  sccb::Ctl *h_ctl = nullptr;  // pinned
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint32_t grid_used = 0;
  uint32_t launches = 0;
  uint32_t *enq_labels = nullptr;
  cudaGraphExec_t solve_exec = nullptr;  // captured solve (scc_solve_capture)
};

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  return set_error(e == cudaErrorMemoryAllocation ? SCC_ERR_NOMEM : SCC_ERR_CUDA, "%s: %s", what,
                   cudaGetErrorString(e));
}
#define CK(call, what)                          \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

int use_device(scc_ctx *c) {
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  return SCC_OK;
}

}  // namespace

namespace sccb {

int check_opts(const scc_opts *o) {
  if (o->alg < SCC_ALG_QUADRATIC || o->alg > SCC_ALG_BEST) return set_error(SCC_ERR_INVALID, "unknown alg %d", o->alg);
  if (o->block_size != 0 && o->block_size != 128 && o->block_size != 256 && o->block_size != 512 &&
      o->block_size != 1024)
    return set_error(SCC_ERR_INVALID, "block_size must be 128, 256, 512 or 1024 (got %d)", o->block_size);
  if (o->pivot_rule < 0 || o->pivot_rule > 1) return set_error(SCC_ERR_INVALID, "unknown pivot rule %d", o->pivot_rule);
  if (o->switch_permille < 0 || o->switch_permille > 1000)
    return set_error(SCC_ERR_INVALID, "switch_permille must be in 0..1000");
  if (o->heavy_degree != 0 && o->heavy_degree < 256) return set_error(SCC_ERR_INVALID, "heavy_degree must be >= 256");
  if (o->occupancy != 0 && (o->occupancy < 3 || o->occupancy > 6))
    return set_error(SCC_ERR_INVALID, "occupancy must be 0 or 3..6");
  if (o->test_stall_us > 10000000u) return set_error(SCC_ERR_INVALID, "test_stall_us must be at most 10 s");
  return SCC_OK;
}

}  // namespace sccb

namespace {

using sccb::check_opts;

int ensure_state(scc_ctx *c) {
  const uint32_t n = c->n;
  const uint32_t hcap = c->m / 256u + 2u;
  if (c->have_state && n <= c->cap_n && hcap <= c->cap_h) return SCC_OK;
  const uint32_t cn = n > c->cap_n ? n : c->cap_n;
  const uint32_t ch = hcap > c->cap_h ? hcap : c->cap_h;
  const size_t vb = ((size_t)cn + 1) * 4;
  const uint32_t nw = sccb::bitmap_words(cn) + sccb::kBitmapSlack;
  CK(c->label.ensure(vb), "alloc labels");
  CK(c->range.ensure(vb), "alloc ranges");
  CK(c->rpivot.ensure(vb), "alloc pivots");
  CK(c->aux.ensure(vb), "alloc aux");
  CK(c->sccsize.ensure(vb), "alloc component sizes");
  CK(c->bitmaps.ensure((size_t)nw * 4 * 7), "alloc bitmaps");
  CK(c->qa.ensure(vb), "alloc queue");
  CK(c->qb.ensure(vb), "alloc queue");
  CK(c->act0.ensure(vb), "alloc active list");
  CK(c->act1.ensure(vb), "alloc active list");
  CK(c->piv.ensure(vb), "alloc pivot list");
  CK(c->pivkey.ensure(vb), "alloc pivot keys");
  // election slots, then the asynchronous reach queue (2(n+1) entries: both
  // directions): both all ones between uses
  const size_t slot_bytes = ((size_t)cn + 1) * 3 * 8 + ((size_t)cn + 1) * 8;
  if (slot_bytes > c->slot.bytes) c->slot_dirty = true;
  CK(c->slot.ensure(slot_bytes), "alloc election slots");
  CK(c->heavy.ensure((size_t)ch * 5 * 4), "alloc heavy list");
  CK(c->ctl.ensure(sizeof(sccb::Ctl)), "alloc control block");
  if (c->slot_dirty) {
    CK(cudaMemsetAsync(c->slot.p, 0xff, c->slot.bytes, c->stream), "init election slots");
    c->slot_dirty = false;
  }
  c->cap_n = cn;
  c->cap_h = ch;
  c->nwords = nw;
  c->have_state = true;
  return SCC_OK;
}

sccb::Params make_params(scc_ctx *c, uint32_t *out_labels) {
  sccb::Params p{};
  p.g.n = c->n;
  p.g.m = c->m;
  p.g.sorted_unique = c->sorted_unique ? 1u : 0u;
  p.g.off = c->d_off;
  p.g.adj = c->d_adj;
  p.g.offT = c->d_offT;
  p.g.adjT = c->d_adjT;
  sccb::EngState &s = p.s;
  s.label = c->label.as<uint32_t>();
  s.range = c->range.as<uint32_t>();
  s.rpivot = c->rpivot.as<uint32_t>();
  s.aux = c->aux.as<uint32_t>();
  s.sccsize = c->sccsize.as<uint32_t>();
  // bitmaps sized for this graph (words beyond it are never touched)
  const uint32_t nw = sccb::bitmap_words(c->n);
  uint32_t *bm = c->bitmaps.as<uint32_t>();
  const uint32_t stride = c->nwords;
  s.elim = bm + 0 * (size_t)stride;
  s.fvis = bm + 1 * (size_t)stride;
  s.bvis = bm + 2 * (size_t)stride;
  s.fexp = bm + 3 * (size_t)stride;
  s.bexp = bm + 4 * (size_t)stride;
  s.tflag = bm + 5 * (size_t)stride;
  s.queued = bm + 6 * (size_t)stride;
  s.qa = c->qa.as<uint32_t>();
  s.qb = c->qb.as<uint32_t>();
  s.act[0] = c->act0.as<uint32_t>();
  s.act[1] = c->act1.as<uint32_t>();
  s.piv = c->piv.as<uint32_t>();
  s.pivkey = c->pivkey.as<uint32_t>();
  s.slot = c->slot.as<unsigned long long>();
  s.aq = reinterpret_cast<uint32_t *>(s.slot + 3 * ((size_t)c->cap_n + 1));
  uint32_t *h = c->heavy.as<uint32_t>();
  s.hv = h;
  s.hbeg = h + (size_t)c->cap_h;
  s.hdeg = h + 2 * (size_t)c->cap_h;
  s.htag = h + 3 * (size_t)c->cap_h;
  s.hbase = h + 4 * (size_t)c->cap_h;
  s.seg = c->nseg > 1 ? c->seg.as<uint32_t>() : nullptr;
  s.out_labels = out_labels;
  s.ctl = c->ctl.as<sccb::Ctl>();
  s.nwords = nw;
  s.qcap = c->n + 1;
  s.hcap = c->cap_h;
  s.nseg = c->nseg > 1 ? c->nseg : 1;
  const scc_opts &o = c->opts;
  sccb::EngOpts &e = p.o;
  e.alg = (uint32_t)o.alg;
  e.wcc = o.wcc ? 1u : 0u;
  e.trim2 = o.trim2 ? 1u : 0u;
  e.trim_first = o.trim_first ? 1u : 0u;
  e.pivot_rule = (uint32_t)o.pivot_rule;
  e.switch_thr = (uint32_t)((uint64_t)c->n * (uint64_t)o.switch_permille / 1000ull);
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
  // a test cap only shortens the usable part of the (n+1)-entry worklists
  if (o.test_queue_cap && o.test_queue_cap < s.qcap) s.qcap = o.test_queue_cap;
  // labels are written straight into the caller's device buffer when given
  if (out_labels) s.label = out_labels;
  return p;
}

int block_size_of(const scc_ctx *c) { return c->opts.block_size ? c->opts.block_size : 256; }

int need_graph(scc_ctx *c) {
  if (!c) return set_error(SCC_ERR_INVALID, "null context");
  if (!c->have_graph) return set_error(SCC_ERR_STATE, "no graph bound to the context");
  if (c->nseg > 1 && c->seg_host.back() != c->n + 1)
    return set_error(SCC_ERR_INVALID, "segments end at %u but the graph has %u vertices", c->seg_host.back() - 1, c->n);
  if (c->nseg > 1 && c->nseg > c->n)
    return set_error(SCC_ERR_INVALID, "%u segments for %u vertices (partition ids must stay below n+1)", c->nseg, c->n);
  return SCC_OK;
}

int read_ctl(scc_ctx *c) {
  CK(cudaMemcpyAsync(c->h_ctl, c->ctl.p, sizeof(sccb::Ctl), cudaMemcpyDeviceToHost, c->stream), "read control block");
  CK(cudaStreamSynchronize(c->stream), "synchronise");
  if (c->h_ctl->gs.err) {
    c->slot_dirty = true;
    c->phase_ready = false;
    const uint32_t e = c->h_ctl->gs.err;
    return set_error(SCC_ERR_TIMEOUT, "device-side %s (flags 0x%x, at barrier %u)",
                     (e & 1u) ? "barrier wait timed out" : (e & 2u) ? "iteration cap reached" : "queue overflow", e,
                     c->h_ctl->gs.err_where);
  }
  return SCC_OK;
}

// A segmented graph must hold independent graphs: no edge may leave its
// source's segment (the first FB round relies on it and runs unranged).
// Checked on the device whenever a caller's segment table and a graph are
// both bound; on a violation the segments are dropped.
int verify_segments(scc_ctx *c) {
  if (c->nseg <= 1 || !c->have_graph || c->seg_host.back() != c->n + 1) return SCC_OK;
  CK(c->ctl.ensure(sizeof(sccb::Ctl)), "alloc control block");
  for (int t = 0; t < 2; ++t) {
    uint32_t bad = 0;
    CK(sccb::check_segments(t ? c->d_offT : c->d_off, t ? c->d_adjT : c->d_adj, c->n, c->seg.as<uint32_t>(), c->nseg,
                            c->ctl.as<uint32_t>(), &bad, c->stream),
       "segment check");
    if (bad) {
      c->nseg = 0;
      c->seg_host.clear();
      return set_error(SCC_ERR_INVALID, "an edge of the %s leaves its segment (segments must be independent graphs)",
                       t ? "transpose" : "graph");
    }
  }
  return SCC_OK;
}

// fresh_ctl: the control block (barrier arrivals included) was just cleared
// by the init kernel, so no separate clear is enqueued
int launch(scc_ctx *c, uint32_t phase, uint32_t a0 = 0, uint32_t a1 = 0, uint32_t a2 = 0,
           uint32_t *out_labels = nullptr, bool fresh_ctl = false) {
  const sccb::Params p = make_params(c, out_labels);
  // the grid barrier counts arrivals from zero in every launch
  if (!fresh_ctl)
    CK(cudaMemsetAsync(&p.s.ctl->gs.arrived, 0, sizeof(p.s.ctl->gs.arrived), c->stream), "clear barrier");
  CK(sccb::launch_phase(p, phase, a0, a1, a2, block_size_of(c), c->opts.grid_blocks, c->stream, &c->grid_used,
                        c->opts.occupancy),
     "cooperative launch");
  ++c->launches;
  return SCC_OK;
}

int reset_state(scc_ctx *c) {
  int rc = ensure_state(c);
  if (rc) return rc;
  CK(cudaGetLastError(), "pending CUDA error before the solve");
  // the init kernel also clears the control block
  const sccb::Params p = make_params(c, nullptr);
  CK(sccb::launch_init(p, c->stream), "init launch");
  ++c->launches;
  return SCC_OK;
}

void fill_stats(scc_ctx *c, scc_stats *st, float ms) {
  if (!st) return;
  const sccb::Ctl &k = *c->h_ctl;
  std::memset(st, 0, sizeof(*st));
  st->steps = k.steps;
  st->fwd_depth = k.fwd_depth;
  st->bwd_depth = k.bwd_depth;
  st->trim_iters = k.trim_iters;
  st->wcc_iters = k.wcc_iters;
  st->wcc_step = k.wcc_step;
  st->n_trimmed = k.n_trimmed;
  st->n_trim2 = k.n_trim2;
  st->n_fb_elim = k.n_fbe + k.n_trim2;
  st->nscc = k.nscc;
  // trim-1 removes singletons, trim-2 pairs; F∩B components were counted per pivot
  uint32_t largest = k.largest_fb;
  if (k.n_trim2 && largest < 2u) largest = 2u;
  if (k.n_trimmed && largest < 1u) largest = 1u;
  st->largest_scc = largest;
  st->pull_sweeps = k.pull_sweeps;
  st->grid_blocks = c->grid_used;
  st->block_size = (uint32_t)block_size_of(c);
  st->kernel_launches = c->launches;
  st->ms_total = ms;
  st->ms_trim = k.ns_trim * 1e-6;
  st->ms_fwd = k.ns_fwd * 1e-6;
  st->ms_bwd = k.ns_bwd * 1e-6;
  st->ms_update = k.ns_update * 1e-6;
  st->ms_wcc = k.ns_wcc * 1e-6;
}

}  // namespace

// checked and unchecked variants of binding and segment tables (defined below)
extern "C" {
static int bind_device_impl(scc_ctx *c, const scc_dev_csr *g, bool verify);
static int set_segments_impl(scc_ctx *c, uint32_t nseg, const uint32_t *seg_first, bool verify);
}

extern "C" {

const char *scc_last_error(void) { return sccb::g_err; }
const char *scc_version(void) { return "gpuscc_b200 1.0 (sm_100a)"; }

void scc_opts_default(scc_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->alg = SCC_ALG_TOPO;  // scc.cu:80
  o->wcc = 0;
  o->trim2 = 0;
  o->trim_first = 1;  // scc.cu:38 TRIM_FIRST
  o->block_size = 256;  // scc.cu:82
  o->warp_size = 32;  // scc.cu:81
  o->pivot_rule = SCC_PIVOT_MIN_ID;
  o->switch_permille = 10;  // n/100 (scc.cu:507)
  o->trim_depth = 0;
  o->pull_alpha = 0;
  o->pull_beta = 0;
  o->trim_first_depth = 1;
}

int scc_ctx_create(int device, const scc_opts *opts, scc_ctx **out) {
  sccb::clear_error();
  if (!out) return set_error(SCC_ERR_INVALID, "null output");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(SCC_ERR_NODEVICE, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return set_error(SCC_ERR_INVALID, "device %d out of range (have %d)", device, ndev);
  scc_opts o;
  scc_opts_default(&o);
  if (opts) o = *opts;
  int rc = check_opts(&o);
  if (rc) return rc;
  scc_ctx *c = new scc_ctx();
  c->device = device;
  c->opts = o;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_ctl, sizeof(sccb::Ctl));
  if (e == cudaSuccess) std::memset(c->h_ctl, 0, sizeof(sccb::Ctl));
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e != cudaSuccess) {
    scc_ctx_destroy(c);
    return cuda_fail(e, "context setup");
  }
  *out = c;
  return SCC_OK;
}

int scc_ctx_destroy(scc_ctx *c) {
  if (!c) return SCC_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (DBuf *b : {&c->g_off, &c->g_adj, &c->g_offT, &c->g_adjT, &c->label, &c->range, &c->rpivot, &c->aux, &c->sccsize,
                  &c->bitmaps, &c->qa, &c->qb, &c->act0, &c->act1, &c->piv, &c->pivkey, &c->slot, &c->heavy,
                  &c->ctl, &c->seg, &c->feat})
    b->release();
  if (c->h_ctl) cudaFreeHost(c->h_ctl);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->solve_exec) cudaGraphExecDestroy(c->solve_exec);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SCC_OK;
}

int scc_ctx_set_opts(scc_ctx *c, const scc_opts *o) {
  sccb::clear_error();
  if (!c || !o) return set_error(SCC_ERR_INVALID, "null argument");
  int rc = check_opts(o);
  if (rc) return rc;
  c->opts = *o;
  return SCC_OK;
}

int scc_ctx_get_opts(const scc_ctx *c, scc_opts *o) {
  if (!c || !o) return set_error(SCC_ERR_INVALID, "null argument");
  *o = c->opts;
  return SCC_OK;
}

void *scc_ctx_stream(scc_ctx *c) { return c ? (void *)c->stream : nullptr; }

int scc_ctx_upload(scc_ctx *c, const scc_host_csr *g) {
  sccb::clear_error();
  if (!c || !g) return set_error(SCC_ERR_INVALID, "null argument");
  if (g->n >= (1u << 30)) return set_error(SCC_ERR_CAPACITY, "n must be below 2^30");
  if (!g->nodes || !g->nodesT || (g->m && (!g->edges || !g->edgesT))) return set_error(SCC_ERR_INVALID, "null arrays");
  if (g->nodes[g->n + 1] != g->m || g->nodesT[g->n + 1] != g->m)
    return set_error(SCC_ERR_INVALID, "nodes[n+1] (%u) / nodesT[n+1] (%u) differ from m (%u)", g->nodes[g->n + 1],
                     g->nodesT[g->n + 1], g->m);
  int rc = use_device(c);
  if (rc) return rc;
  const size_t ob = ((size_t)g->n + 2) * 4, eb = ((size_t)g->m + 1) * 4;
  CK(c->g_off.ensure(ob), "alloc graph");
  CK(c->g_adj.ensure(eb), "alloc graph");
  CK(cudaMemcpyAsync(c->g_off.p, g->nodes, ob, cudaMemcpyHostToDevice, c->stream), "upload nodes");
  if (g->m) CK(cudaMemcpyAsync(c->g_adj.p, g->edges, (size_t)g->m * 4, cudaMemcpyHostToDevice, c->stream), "upload edges");
  c->d_off = c->g_off.as<uint32_t>();
  c->d_adj = c->g_adj.as<uint32_t>();
  if (g->nodesT == g->nodes && g->edgesT == g->edges) {
    c->d_offT = c->d_off;
    c->d_adjT = c->d_adj;
  } else {
    CK(c->g_offT.ensure(ob), "alloc graph");
    CK(c->g_adjT.ensure(eb), "alloc graph");
    CK(cudaMemcpyAsync(c->g_offT.p, g->nodesT, ob, cudaMemcpyHostToDevice, c->stream), "upload nodesT");
    if (g->m)
      CK(cudaMemcpyAsync(c->g_adjT.p, g->edgesT, (size_t)g->m * 4, cudaMemcpyHostToDevice, c->stream), "upload edgesT");
    c->d_offT = c->g_offT.as<uint32_t>();
    c->d_adjT = c->g_adjT.as<uint32_t>();
  }
  // the kernels trust the layout: reject anything that would index outside it
  CK(c->ctl.ensure(sizeof(sccb::Ctl)), "alloc control block");
  for (int t = 0; t < 2; ++t) {
    uint32_t bad = 0;
    CK(sccb::check_device_csr(t ? c->d_offT : c->d_off, t ? c->d_adjT : c->d_adj, g->n, g->m, c->ctl.as<uint32_t>(),
                              &bad, c->stream),
       "CSR check");
    if (bad) {
      c->have_graph = false;
      return set_error(SCC_ERR_INVALID, "%s: %s", t ? "transpose" : "graph",
                       (bad & 1u) ? "offsets are not monotone from 0 to m" : "a neighbour id is outside 1..n");
    }
  }
  c->n = g->n;
  c->m = g->m;
  c->sorted_unique = g->sorted_unique;
  c->have_graph = true;
  c->phase_ready = false;
  int rs = ensure_state(c);
  return rs ? rs : verify_segments(c);
}

int scc_gen_rmat_device(scc_ctx *c, uint32_t scale, uint64_t samples, uint32_t a_ppm, uint32_t b_ppm,
                        uint32_t c_ppm, uint64_t seed, int permute, scc_dev_csr *out) {
  sccb::clear_error();
  if (!c) return set_error(SCC_ERR_INVALID, "null context");
  if (scale < 1 || scale > 29 || samples >= (1ull << 31) || (uint64_t)a_ppm + b_ppm + c_ppm > 1000000ull)
    return set_error(SCC_ERR_INVALID, "bad R-MAT arguments");
  int rc = use_device(c);
  if (rc) return rc;
  for (DBuf *b : {&c->g_off, &c->g_adj, &c->g_offT, &c->g_adjT}) b->release();
  c->have_graph = false;
  uint32_t *off = nullptr, *adj = nullptr, *offT = nullptr, *adjT = nullptr, m = 0;
  CK(sccb::gen_rmat_device(scale, samples, a_ppm, b_ppm, c_ppm, seed, permute, c->stream, &off, &adj, &offT, &adjT, &m),
     "device R-MAT build");
  const uint32_t n = 1u << scale;
  c->g_off.p = off;
  c->g_off.bytes = ((size_t)n + 2) * 4;
  c->g_adj.p = adj;
  c->g_adj.bytes = ((size_t)m + 1) * 4;
  c->g_offT.p = offT;
  c->g_offT.bytes = ((size_t)n + 2) * 4;
  c->g_adjT.p = adjT;
  c->g_adjT.bytes = ((size_t)m + 1) * 4;
  c->d_off = off;
  c->d_adj = adj;
  c->d_offT = offT;
  c->d_adjT = adjT;
  c->n = n;
  c->m = m;
  c->sorted_unique = 1;
  c->have_graph = true;
  c->phase_ready = false;
  if (out) {
    out->n = n;
    out->m = m;
    out->sorted_unique = 1;
    out->nodes = off;
    out->edges = adj;
    out->nodesT = offT;
    out->edgesT = adjT;
  }
  return ensure_state(c);
}

int scc_gen_batch_device(scc_ctx *c, uint32_t count, uint32_t n_lo, uint32_t n_hi, uint32_t deg_lo_milli,
                         uint32_t deg_hi_milli, uint64_t seed, scc_dev_csr *out, uint32_t *seg_first) {
  sccb::clear_error();
  if (!c || !seg_first) return set_error(SCC_ERR_INVALID, "null argument");
  std::vector<sccg::BatchGraph> plan;
  int rc = sccb::plan_batch(count, n_lo, n_hi, deg_lo_milli, deg_hi_milli, seed, &plan);
  if (rc) return rc;
  rc = use_device(c);
  if (rc) return rc;
  for (DBuf *b : {&c->g_off, &c->g_adj, &c->g_offT, &c->g_adjT}) b->release();
  c->have_graph = false;
  uint32_t *off = nullptr, *adj = nullptr, *offT = nullptr, *adjT = nullptr, n = 0, m = 0;
  CK(sccb::gen_batch_device(plan.data(), count, c->stream, &off, &adj, &offT, &adjT, &n, &m), "device batch build");
  c->g_off.p = off;
  c->g_off.bytes = ((size_t)n + 2) * 4;
  c->g_adj.p = adj;
  c->g_adj.bytes = ((size_t)m + 1) * 4;
  c->g_offT.p = offT;
  c->g_offT.bytes = ((size_t)n + 2) * 4;
  c->g_adjT.p = adjT;
  c->g_adjT.bytes = ((size_t)m + 1) * 4;
  c->d_off = off;
  c->d_adj = adj;
  c->d_offT = offT;
  c->d_adjT = adjT;
  c->n = n;
  c->m = m;
  c->sorted_unique = 1;
  c->have_graph = true;
  c->phase_ready = false;
  seg_first[0] = 1;
  for (uint32_t g = 0; g < count; ++g) seg_first[g + 1] = seg_first[g] + plan[g].n;
  if (out) {
    out->n = n;
    out->m = m;
    out->sorted_unique = 1;
    out->nodes = off;
    out->edges = adj;
    out->nodesT = offT;
    out->edgesT = adjT;
  }
  rc = ensure_state(c);
  if (rc) return rc;
  return set_segments_impl(c, count, seg_first, false);  // built here: no edge crosses segments
}

static int bind_device_impl(scc_ctx *c, const scc_dev_csr *g, bool verify) {
  sccb::clear_error();
  if (!c || !g) return set_error(SCC_ERR_INVALID, "null argument");
  if (g->n >= (1u << 30)) return set_error(SCC_ERR_CAPACITY, "n must be below 2^30");
  if (!g->nodes || !g->nodesT || (g->m && (!g->edges || !g->edgesT))) return set_error(SCC_ERR_INVALID, "null arrays");
  int rc = use_device(c);
  if (rc) return rc;
  CK(c->ctl.ensure(sizeof(sccb::Ctl)), "alloc control block");
  if (!c->h_ctl) return set_error(SCC_ERR_STATE, "context not initialised");
  for (int t = 0; verify && t < 2; ++t) {
    uint32_t bad = 0;
    CK(sccb::check_device_csr(t ? g->nodesT : g->nodes, t ? g->edgesT : g->edges, g->n, g->m, c->ctl.as<uint32_t>(),
                              &bad, c->stream),
       "device CSR check");
    if (bad)
      return set_error(SCC_ERR_INVALID, "device %s: %s", t ? "transpose" : "graph",
                       (bad & 1u) ? "offsets are not monotone from 0 to m" : "a neighbour id is outside 1..n");
  }
  c->d_off = g->nodes;
  c->d_adj = g->edges;
  c->d_offT = g->nodesT;
  c->d_adjT = g->edgesT;
  c->n = g->n;
  c->m = g->m;
  c->sorted_unique = g->sorted_unique;
  c->have_graph = true;
  c->phase_ready = false;
  rc = ensure_state(c);
  return (rc || !verify) ? rc : verify_segments(c);
}

int scc_ctx_bind_device(scc_ctx *c, const scc_dev_csr *g) { return bind_device_impl(c, g, true); }

int scc_ctx_download(scc_ctx *c, scc_host_csr *out) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  if (!out) return set_error(SCC_ERR_INVALID, "null output");
  rc = use_device(c);
  if (rc) return rc;
  std::memset(out, 0, sizeof(*out));
  const size_t ob = ((size_t)c->n + 2) * 4, eb = ((size_t)c->m + 1) * 4;
  out->nodes = (uint32_t *)std::malloc(ob);
  out->edges = (uint32_t *)std::malloc(eb);
  out->nodesT = (uint32_t *)std::malloc(ob);
  out->edgesT = (uint32_t *)std::malloc(eb);
  out->owned = 1;
  if (!out->nodes || !out->edges || !out->nodesT || !out->edgesT) {
    scc_host_csr_free(out);
    return set_error(SCC_ERR_NOMEM, "host allocation failed");
  }
  CK(cudaMemcpy(out->nodes, c->d_off, ob, cudaMemcpyDeviceToHost), "download");
  CK(cudaMemcpy(out->nodesT, c->d_offT, ob, cudaMemcpyDeviceToHost), "download");
  if (c->m) {
    CK(cudaMemcpy(out->edges, c->d_adj, (size_t)c->m * 4, cudaMemcpyDeviceToHost), "download");
    CK(cudaMemcpy(out->edgesT, c->d_adjT, (size_t)c->m * 4, cudaMemcpyDeviceToHost), "download");
  }
  out->edges[c->m] = 0;
  out->edgesT[c->m] = 0;
  out->nodes[0] = 0;
  out->nodesT[0] = 0;
  out->n = c->n;
  out->m = c->m;
  out->nnz_header = c->m;
  out->sorted_unique = c->sorted_unique;
  return SCC_OK;
}

int scc_ctx_download_into(scc_ctx *c, uint32_t *nodes, uint32_t *edges, uint32_t *nodesT, uint32_t *edgesT) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  if (!nodes || !nodesT || (c->m && (!edges || !edgesT))) return set_error(SCC_ERR_INVALID, "null output");
  rc = use_device(c);
  if (rc) return rc;
  const size_t ob = ((size_t)c->n + 2) * 4, eb = (size_t)c->m * 4;
  CK(cudaMemcpyAsync(nodes, c->d_off, ob, cudaMemcpyDeviceToHost, c->stream), "download");
  CK(cudaMemcpyAsync(nodesT, c->d_offT, ob, cudaMemcpyDeviceToHost, c->stream), "download");
  if (eb) {
    CK(cudaMemcpyAsync(edges, c->d_adj, eb, cudaMemcpyDeviceToHost, c->stream), "download");
    CK(cudaMemcpyAsync(edgesT, c->d_adjT, eb, cudaMemcpyDeviceToHost, c->stream), "download");
  }
  CK(cudaStreamSynchronize(c->stream), "download");
  nodes[0] = 0;
  nodesT[0] = 0;
  return SCC_OK;
}

static int set_segments_impl(scc_ctx *c, uint32_t nseg, const uint32_t *seg_first, bool verify) {
  sccb::clear_error();
  if (!c) return set_error(SCC_ERR_INVALID, "null context");
  if (nseg == 0) {
    c->nseg = 0;
    c->seg_host.clear();
    return SCC_OK;
  }
  if (!seg_first) return set_error(SCC_ERR_INVALID, "null segment table");
  if (seg_first[0] != 1) return set_error(SCC_ERR_INVALID, "seg_first[0] must be 1");
  for (uint32_t s = 0; s < nseg; ++s)
    if (seg_first[s + 1] < seg_first[s]) return set_error(SCC_ERR_INVALID, "segment table not monotone at %u", s);
  int rc = use_device(c);
  if (rc) return rc;
  c->seg_host.assign(seg_first, seg_first + nseg + 1);
  CK(c->seg.ensure(((size_t)nseg + 1) * 4), "alloc segments");
  CK(cudaMemcpyAsync(c->seg.p, c->seg_host.data(), ((size_t)nseg + 1) * 4, cudaMemcpyHostToDevice, c->stream),
     "upload segments");
  c->nseg = nseg;
  c->phase_ready = false;
  return verify ? verify_segments(c) : SCC_OK;
}

int scc_ctx_set_segments(scc_ctx *c, uint32_t nseg, const uint32_t *seg_first) {
  return set_segments_impl(c, nseg, seg_first, true);
}

int scc_solve_enqueue(scc_ctx *c, uint32_t *d_labels) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  rc = use_device(c);
  if (rc) return rc;
  c->launches = 0;
  rc = reset_state(c);
  if (rc) return rc;
  // ms_total: the persistent kernel alone.  Not recorded while the sequence
  // is being captured (a replay times the whole graph launch instead).
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->stream, &cs), "capture status");
  const bool timed = cs == cudaStreamCaptureStatusNone;
  if (timed) CK(cudaEventRecord(c->ev0, c->stream), "event");
  rc = launch(c, sccb::PH_SOLVE, 0, 0, 0, d_labels, true);
  if (rc) return rc;
  if (timed) CK(cudaEventRecord(c->ev1, c->stream), "event");
  c->enq_labels = d_labels;
  c->phase_ready = false;
  return SCC_OK;
}

int scc_solve_collect(scc_ctx *c, uint32_t *nscc, scc_stats *st) {
  if (!c) return set_error(SCC_ERR_INVALID, "null context");
  int rc = read_ctl(c);
  if (rc) return rc;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1), "solve timing events");
  if (c->h_ctl->phase_ret != 0)
    return set_error(SCC_ERR_STATE, "%u vertices left without a component", c->h_ctl->phase_ret);
  if (nscc) *nscc = c->h_ctl->nscc;
  fill_stats(c, st, ms);
  return SCC_OK;
}

int scc_solve_capture(scc_ctx *c, uint32_t *d_labels) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  rc = use_device(c);
  if (rc) return rc;
  CK(cudaGetLastError(), "pending CUDA error at capture entry");
  rc = ensure_state(c);  // allocations and the slot reset happen before capture
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream), "pre-capture sync");
  if (c->solve_exec) {
    cudaGraphExecDestroy(c->solve_exec);
    c->solve_exec = nullptr;
  }
  CK(cudaGetLastError(), "pending CUDA error before capture");
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  CK(cudaGetLastError(), "pending CUDA error after begin capture");
  rc = scc_solve_enqueue(c, d_labels);
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ee != cudaSuccess) return cuda_fail(ee, "end capture");
  const cudaError_t ie = cudaGraphInstantiate(&c->solve_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    c->solve_exec = nullptr;
    return cuda_fail(ie, "instantiate captured solve");
  }
  return SCC_OK;
}

int scc_solve_replay(scc_ctx *c, uint32_t *nscc, scc_stats *st) {
  sccb::clear_error();
  if (!c || !c->solve_exec) return set_error(SCC_ERR_STATE, "no captured solve (call scc_solve_capture)");
  int rc = use_device(c);
  if (rc) return rc;
  if (c->slot_dirty) {  // an earlier failure left election slots set: restore them outside the graph
    CK(cudaMemsetAsync(c->slot.p, 0xff, c->slot.bytes, c->stream), "reset election slots");
    c->slot_dirty = false;
  }
  CK(cudaEventRecord(c->ev0, c->stream), "event");  // ms_total: the whole replayed graph
  CK(cudaGraphLaunch(c->solve_exec, c->stream), "graph launch");
  CK(cudaEventRecord(c->ev1, c->stream), "event");
  c->launches = 2;
  return scc_solve_collect(c, nscc, st);
}

int scc_read_labels(scc_ctx *c, uint32_t *labels) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  if (!labels) return set_error(SCC_ERR_INVALID, "null output");
  rc = use_device(c);
  if (rc) return rc;
  CK(cudaMemcpyAsync(labels, c->label.p, ((size_t)c->n + 1) * 4, cudaMemcpyDeviceToHost, c->stream), "labels D2H");
  CK(cudaStreamSynchronize(c->stream), "labels D2H");
  labels[0] = 0;
  return SCC_OK;
}

int scc_solve_device(scc_ctx *c, uint32_t *d_labels, uint32_t *nscc, scc_stats *st) {
  int rc = scc_solve_enqueue(c, d_labels);
  if (rc) return rc;
  return scc_solve_collect(c, nscc, st);
}

int scc_solve(scc_ctx *c, uint32_t *labels, uint32_t *nscc, scc_stats *st) {
  int rc = scc_solve_device(c, nullptr, nscc, st);
  if (rc) return rc;
  if (labels) {
    CK(cudaMemcpyAsync(labels, c->label.p, ((size_t)c->n + 1) * 4, cudaMemcpyDeviceToHost, c->stream), "labels D2H");
    CK(cudaStreamSynchronize(c->stream), "labels D2H");
    labels[0] = 0;
  }
  return SCC_OK;
}

int scc_batch_solve(scc_ctx *c, uint32_t count, const scc_host_csr *graphs, uint32_t *const *labels,
                    uint32_t *nscc) {
  sccb::clear_error();
  if (!c || (count && !graphs)) return set_error(SCC_ERR_INVALID, "null argument");
  if (count == 0) return SCC_OK;
  std::vector<uint32_t> seg(count + 1);
  scc_host_csr packed;
  int rc = scc_batch_pack(count, graphs, &packed, seg.data());
  if (rc) return rc;
  std::vector<uint32_t> all((size_t)packed.n + 1);
  scc_ctx_set_segments(c, 0, nullptr);  // no stale table is checked against the packed graph
  rc = scc_ctx_upload(c, &packed);
  if (!rc) rc = set_segments_impl(c, count, seg.data(), false);  // packed here: no edge crosses segments
  uint32_t total = 0;
  if (!rc) rc = scc_solve(c, all.data(), &total, nullptr);
  scc_ctx_set_segments(c, 0, nullptr);
  scc_host_csr_free(&packed);
  if (rc) return rc;
  // global ids -> each graph's own ids; a component's label is its smallest id
  for (uint32_t g = 0; g < count; ++g) {
    const uint32_t base = seg[g] - 1, n = graphs[g].n;
    uint32_t roots = 0;
    for (uint32_t v = 1; v <= n; ++v) {
      const uint32_t l = all[base + v] - base;
      roots += l == v;
      if (labels && labels[g]) labels[g][v] = l;
    }
    if (labels && labels[g]) labels[g][0] = 0;
    if (nscc) nscc[g] = roots;
  }
  return SCC_OK;
}

int scc_get_profile(scc_ctx *c, double *ms, uint32_t *counts) {
  sccb::clear_error();
  if (!c) return set_error(SCC_ERR_INVALID, "null context");
  for (int i = 0; i < 16; ++i) {
    if (ms) ms[i] = c->h_ctl->prof_ns[i] * 1e-6;
    if (counts) counts[i] = c->h_ctl->prof_cnt[i];
  }
  return SCC_OK;
}

int scc_get_trace(scc_ctx *c, uint32_t *n, uint32_t *slot, uint32_t *a, uint32_t *b, double *ms) {
  sccb::clear_error();
  if (!c || !n) return set_error(SCC_ERR_INVALID, "null argument");
  const uint32_t cnt = c->h_ctl->trace_n < sccb::kTrace ? c->h_ctl->trace_n : sccb::kTrace;
  *n = cnt;
  for (uint32_t i = 0; i < cnt; ++i) {
    if (slot) slot[i] = c->h_ctl->trace_slot[i];
    if (a) a[i] = c->h_ctl->trace_a[i];
    if (b) b[i] = c->h_ctl->trace_b[i];
    if (ms) ms[i] = c->h_ctl->trace_ns[i] * 1e-6;
  }
  return SCC_OK;
}

// ------------------------------------------------------------- phases
static int phase_prologue(scc_ctx *c) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  rc = use_device(c);
  if (rc) return rc;
  if (!c->phase_ready) return set_error(SCC_ERR_STATE, "call scc_phase_begin first");
  return SCC_OK;
}

static int run_phase(scc_ctx *c, uint32_t phase, uint32_t a0 = 0, uint32_t a1 = 0, uint32_t a2 = 0) {
  int rc = phase_prologue(c);
  if (rc) return rc;
  rc = launch(c, phase, a0, a1, a2);
  if (rc) return rc;
  return read_ctl(c);
}

int scc_phase_begin(scc_ctx *c) {
  sccb::clear_error();
  int rc = need_graph(c);
  if (rc) return rc;
  rc = use_device(c);
  if (rc) return rc;
  rc = reset_state(c);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream), "phase begin");
  c->phase_ready = true;
  return SCC_OK;
}

int scc_trim1(scc_ctx *c, uint32_t *it) {
  int rc = run_phase(c, sccb::PH_TRIM1);
  if (!rc && it) *it = c->h_ctl->phase_ret;
  return rc;
}
int scc_trim(scc_ctx *c, uint32_t *it) {
  int rc = run_phase(c, sccb::PH_TRIM);
  if (!rc && it) *it = c->h_ctl->phase_ret;
  return rc;
}
int scc_trim2(scc_ctx *c, uint32_t *removed) {
  int rc = run_phase(c, sccb::PH_TRIM2);
  if (!rc && removed) *removed = c->h_ctl->phase_ret;
  return rc;
}
int scc_select_pivots(scc_ctx *c, uint32_t *np) {
  int rc = run_phase(c, sccb::PH_SELECT);
  if (!rc && np) *np = c->h_ctl->piv_count;
  return rc;
}
int scc_reach(scc_ctx *c, int dir, int variant, int first_step, uint32_t *depth) {
  if (dir != 0 && dir != 1) return set_error(SCC_ERR_INVALID, "dir must be 0 (forward) or 1 (backward)");
  if (variant != SCC_ALG_QUADRATIC && variant != SCC_ALG_TOPO && variant != SCC_ALG_DATA &&
      variant != SCC_ALG_LINEAR && variant != SCC_ALG_BEST)
    return set_error(SCC_ERR_INVALID, "reach variant must be q, t, d, l or b");
  int rc = run_phase(c, sccb::PH_REACH, (uint32_t)dir, (uint32_t)variant, first_step ? 0u : 1u);
  if (!rc && depth) *depth = c->h_ctl->phase_ret;
  return rc;
}
int scc_update(scc_ctx *c, int32_t *has_pivot) {
  int rc = run_phase(c, sccb::PH_UPDATE);
  if (!rc && has_pivot) *has_pivot = c->h_ctl->piv_count > 0;
  return rc;
}
int scc_count_elimmed(scc_ctx *c, uint32_t *ne) {
  int rc = phase_prologue(c);
  if (rc) return rc;
  rc = read_ctl(c);
  if (!rc && ne) *ne = c->h_ctl->n_fbe + c->h_ctl->n_trim2;
  return rc;
}
int scc_unset_pivots(scc_ctx *c) { return run_phase(c, sccb::PH_UNSET); }
int scc_update_wcc(scc_ctx *c, uint32_t *depth, int32_t *has_pivot) {
  int rc = run_phase(c, sccb::PH_WCC);
  if (!rc) {
    if (depth) *depth = c->h_ctl->phase_ret;
    if (has_pivot) *has_pivot = c->h_ctl->piv_count > 0;
  }
  return rc;
}
int scc_get_states(scc_ctx *c, uint8_t *states) {
  int rc = phase_prologue(c);
  if (rc) return rc;
  if (!states) return set_error(SCC_ERR_INVALID, "null output");
  void *d = nullptr;
  CK(cudaMalloc(&d, (size_t)c->n + 1), "alloc");
  const sccb::Params p = make_params(c, nullptr);
  cudaError_t e = sccb::launch_states(p, (uint8_t *)d, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(states, d, (size_t)c->n + 1, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "states export");
  return SCC_OK;
}
int scc_get_ranges(scc_ctx *c, uint32_t *ranges) {
  int rc = phase_prologue(c);
  if (rc) return rc;
  if (!ranges) return set_error(SCC_ERR_INVALID, "null output");
  void *d = nullptr;
  CK(cudaMalloc(&d, ((size_t)c->n + 1) * 4), "alloc");
  const sccb::Params p = make_params(c, nullptr);
  cudaError_t e = sccb::launch_ranges(p, (uint32_t *)d, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ranges, d, ((size_t)c->n + 1) * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "ranges export");
  return SCC_OK;
}
int scc_graph_features(scc_ctx *c, float *feat) {
  sccb::clear_error();
  if (!c || !feat) return set_error(SCC_ERR_INVALID, "null argument");
  int rc = use_device(c);
  if (!rc) rc = need_graph(c);
  if (rc) return rc;
  CK(c->feat.ensure(sccb::features_scratch_bytes(c->n)), "alloc feature scratch");
  sccb::EngGraph g{};
  g.n = c->n;
  g.m = c->m;
  g.sorted_unique = c->sorted_unique ? 1u : 0u;
  g.off = c->d_off;
  g.adj = c->d_adj;
  g.offT = c->d_offT;
  g.adjT = c->d_adjT;
  CK(sccb::graph_features(g, c->feat.p, c->feat.bytes, feat, c->stream), "graph features");
  return SCC_OK;
}

int scc_get_labels(scc_ctx *c, uint32_t *labels, uint32_t *nscc) {
  int rc = run_phase(c, sccb::PH_FINALIZE);
  if (rc) return rc;
  if (c->h_ctl->phase_ret != 0)
    return set_error(SCC_ERR_STATE, "%u vertices are not assigned to a component yet", c->h_ctl->phase_ret);
  if (nscc) *nscc = c->h_ctl->nscc;
  if (labels) {
    CK(cudaMemcpy(labels, c->label.p, ((size_t)c->n + 1) * 4, cudaMemcpyDeviceToHost), "labels D2H");
    labels[0] = 0;
  }
  return SCC_OK;
}

}  // extern "C"

namespace sccb {
// For graphs packed by this library (valid by construction, or checked when
// they were uploaded): no device checks, no host synchronisation.
int ctx_bind_unchecked(scc_ctx *c, const scc_dev_csr *g) { return bind_device_impl(c, g, false); }
int ctx_set_segments_unchecked(scc_ctx *c, uint32_t nseg, const uint32_t *seg_first) {
  return set_segments_impl(c, nseg, seg_first, false);
}
}  // namespace sccb
