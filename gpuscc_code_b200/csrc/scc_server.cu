// Request loop with continuous batching on one device.
//
// Three parties share the request table under one mutex:
//  * callers: scc_server_submit appends a request (rejected at once when its
//    CSR alone exceeds the memory budget) and poll/wait read its result;
//  * the admission thread takes requests in arrival order, waits until the
//    resident bytes plus the request's CSR fit the budget, allocates the CSR
//    from the stream-ordered pool and uploads it on the copy stream while
//    the solver is busy with earlier batches;
//  * the solver thread, whenever the device is free, takes every uploaded
//    request (oldest first) whose options match the oldest one's, up to the
//    batch limits, packs them into one segmented CSR with a device kernel (a
//    single graph is bound in place), runs one persistent solve, unpacks each
//    segment's labels back to local ids and copies them to the caller's
//    buffer, then frees the request's device memory.
// With a strategy network loaded, the admission thread also launches each
// request's feature pass on a stream of its own (behind the upload, never in
// front of the next one); the solver reads the features when it forms a
// batch and lets the network pick the options of all new requests at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "scc_capi.h"
#include "scc_engine.h"
#include "scc_features.h"
#include "scc_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct PackDesc {
  const uint32_t *off, *adj, *offT, *adjT;
  uint32_t n, m, vbase, ebase;
};

// blockIdx.y = graph; ids shift by vbase, edge offsets by ebase.  Each graph
// also writes the entry after its last vertex (equal to the next graph's
// first entry, or m_total for the last graph).
__global__ void pack_kernel(const PackDesc *__restrict__ d, uint32_t *off, uint32_t *adj, uint32_t *offT,
                            uint32_t *adjT) {
  const PackDesc g = d[blockIdx.y];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= g.n; i += stride) {
    const uint32_t v = i + 1;
    off[g.vbase + v] = g.off[v] + g.ebase;
    offT[g.vbase + v] = g.offT[v] + g.ebase;
  }
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < g.m; j += stride) {
    adj[g.ebase + j] = g.adj[j] + g.vbase;
    adjT[g.ebase + j] = g.adjT[j] + g.vbase;
  }
}

// labels of graph y: global -> local ids, in place; counts the roots.
__global__ void unpack_kernel(const PackDesc *__restrict__ d, uint32_t *labels, uint32_t *nscc) {
  const PackDesc g = d[blockIdx.y];
  uint32_t roots = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t n_pad = (g.n + 31u) & ~31u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
    if (i < g.n) {
      const uint32_t v = i + 1;
      const uint32_t l = labels[g.vbase + v] - g.vbase;
      labels[g.vbase + v] = l;
      roots += l == v;
    }
  }
  roots = __reduce_add_sync(0xffffffffu, roots);
  if ((threadIdx.x & 31) == 0 && roots) atomicAdd(&nscc[blockIdx.y], roots);
}

enum ReqState { RQ_QUEUED, RQ_UPLOADING, RQ_READY, RQ_RUNNING, RQ_DONE };

struct Request {
  uint64_t id = 0;
  scc_host_csr g{};
  uint32_t *labels = nullptr;
  uint64_t bytes = 0;
  ReqState state = RQ_QUEUED;
  Clock::time_point t_submit, t_admit, t_done;
  void *dmem = nullptr;  // one allocation: off | offT | adj | adjT
  cudaEvent_t uploaded = nullptr;
  bool have_choice = false;
  int32_t choice[3] = {0, 0, 0};
  void *h_acc = nullptr;  // page-locked slot receiving the feature accumulators
  bool feat_pending = false;
  cudaEvent_t featured = nullptr;  // features of this request done (feature stream)
  scc_request_info info{};
  const uint32_t *d_off() const { return static_cast<const uint32_t *>(dmem); }
  const uint32_t *d_offT() const { return d_off() + pad4(g.n + 2); }
  const uint32_t *d_adj() const { return d_offT() + pad4(g.n + 2); }
  const uint32_t *d_adjT() const { return d_adj() + pad4(g.m); }
  static uint64_t pad4(uint64_t x) { return (x + 3) & ~uint64_t(3); }
  static uint64_t csr_bytes(uint32_t n, uint32_t m) { return (2 * pad4(n + 2) + 2 * pad4(m)) * 4; }
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct scc_server {
  scc_server_cfg cfg{};
  scc_ctx *ctx = nullptr;
  cudaStream_t solve_st = nullptr, copy_st = nullptr;
  cudaStream_t feat_st = nullptr;  // feature passes: behind their upload, never in front of the next one
  cudaMemPool_t pool = nullptr;
  // packed batch CSR and its scratch
  uint32_t *p_off = nullptr, *p_offT = nullptr, *p_adj = nullptr, *p_adjT = nullptr;
  uint32_t *d_labels = nullptr;
  uint32_t labels_cap = 0;
  PackDesc *d_desc = nullptr;
  uint32_t *d_nscc = nullptr;
  scc_mlp *mlp = nullptr;

  std::mutex mu;
  std::condition_variable cv_admit, cv_solve, cv_done;
  std::deque<Request *> admit_q;
  std::map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  bool stopping = false;
  scc_server_stats st{};
  std::thread admit_thr, solve_thr;

  void admit_loop();
  void solve_loop();
  int run_batch(std::vector<Request *> &batch);
  int choose(std::vector<Request *> &ready);
  // page-locked slots for feature accumulators (one per request in flight)
  std::mutex acc_mu;
  std::vector<void *> acc_free, acc_chunks;
  void *get_acc();
  void put_acc(void *p);
  void finish(Request *r, int status);
};

namespace {

int srv_fail(cudaError_t e, const char *what) {
  return sccb::set_error(e == cudaErrorMemoryAllocation ? SCC_ERR_NOMEM : SCC_ERR_CUDA, "%s: %s", what,
                         cudaGetErrorString(e));
}
#define SCK(call, what)                                \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return srv_fail(e_, what);  \
  } while (0)

}  // namespace

void scc_server::admit_loop() {
  cudaSetDevice(cfg.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_admit.wait(lk, [&] {
      if (admit_q.empty()) return stopping;
      return st.resident_bytes + admit_q.front()->bytes <= st.budget_bytes;
    });
    if (admit_q.empty()) return;  // stopping and drained
    Request *r = admit_q.front();
    admit_q.pop_front();
    st.resident_bytes += r->bytes;
    st.peak_resident_bytes = std::max(st.peak_resident_bytes, st.resident_bytes);
    r->state = RQ_UPLOADING;
    r->t_admit = Clock::now();
    lk.unlock();
    cudaError_t e = cudaMallocFromPoolAsync(&r->dmem, r->bytes, pool, copy_st);
    if (e == cudaSuccess) {
      uint32_t *o = const_cast<uint32_t *>(r->d_off());
      const size_t nb = ((size_t)r->g.n + 2) * 4, mb = (size_t)r->g.m * 4;
      e = cudaMemcpyAsync(o, r->g.nodes, nb, cudaMemcpyHostToDevice, copy_st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(const_cast<uint32_t *>(r->d_offT()), r->g.nodesT, nb, cudaMemcpyHostToDevice, copy_st);
      if (e == cudaSuccess && mb)
        e = cudaMemcpyAsync(const_cast<uint32_t *>(r->d_adj()), r->g.edges, mb, cudaMemcpyHostToDevice, copy_st);
      if (e == cudaSuccess && mb)
        e = cudaMemcpyAsync(const_cast<uint32_t *>(r->d_adjT()), r->g.edgesT, mb, cudaMemcpyHostToDevice, copy_st);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->uploaded, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventRecord(r->uploaded, copy_st);
      // with a network loaded, the graph's features are computed on their own
      // stream behind the upload, with nothing waiting for them (the next
      // uploads go on): the solver reads the accumulators when it forms the
      // batch that may take r
      if (e == cudaSuccess && mlp) {
        void *scratch = nullptr;
        const size_t fb = sccb::features_scratch_bytes(r->g.n);
        r->h_acc = get_acc();
        e = r->h_acc ? cudaStreamWaitEvent(feat_st, r->uploaded, 0) : cudaErrorMemoryAllocation;
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&scratch, fb, pool, feat_st);
        if (e == cudaSuccess) {
          sccb::EngGraph g{};
          g.n = r->g.n;
          g.m = r->g.m;
          g.sorted_unique = r->g.sorted_unique ? 1u : 0u;
          g.off = r->d_off();
          g.adj = r->d_adj();
          g.offT = r->d_offT();
          g.adjT = r->d_adjT();
          e = sccb::graph_features_launch(g, scratch, fb, r->h_acc, feat_st);
          cudaFreeAsync(scratch, feat_st);
          if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->featured, cudaEventDisableTiming);
          if (e == cudaSuccess) e = cudaEventRecord(r->featured, feat_st);
          r->feat_pending = e == cudaSuccess;
        }
      }
    }
    lk.lock();
    if (e != cudaSuccess) {
      sccb::set_error(SCC_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
      cudaStreamSynchronize(copy_st);  // nothing may still write into the allocation when it is freed
      cudaStreamSynchronize(feat_st);
      lk.unlock();
      finish(r, e == cudaErrorMemoryAllocation ? SCC_ERR_NOMEM : SCC_ERR_CUDA);
      lk.lock();
      continue;
    }
    r->state = RQ_READY;
    cv_solve.notify_one();
  }
}

// Marks r done with the given status, releases its device memory (ordered
// after the solve stream's work) and wakes waiters.
void scc_server::finish(Request *r, int status) {
  if (r->uploaded) cudaStreamWaitEvent(solve_st, r->uploaded, 0);  // the upload may still be in flight
  if (r->featured) cudaStreamWaitEvent(solve_st, r->featured, 0);  // and the feature pass reading the graph
  if (r->h_acc) {
    if (r->featured) cudaEventSynchronize(r->featured);  // the accumulator copy lands in the slot
    put_acc(r->h_acc);
    r->h_acc = nullptr;
  }
  if (r->featured) cudaEventDestroy(r->featured);
  r->featured = nullptr;
  if (r->dmem) cudaFreeAsync(r->dmem, solve_st);
  r->dmem = nullptr;
  if (r->uploaded) cudaEventDestroy(r->uploaded);
  r->uploaded = nullptr;
  std::lock_guard<std::mutex> lk(mu);
  st.resident_bytes -= r->bytes;
  r->t_done = Clock::now();
  r->info.status = status;
  r->info.queue_ms = ms_between(r->t_submit, r->t_admit);
  r->info.latency_ms = ms_between(r->t_submit, r->t_done);
  std::memcpy(r->info.choice, r->choice, sizeof(r->choice));
  r->state = RQ_DONE;
  ++st.completed;
  cv_done.notify_all();
  cv_admit.notify_one();
}

// Features + network choice for the ready requests that have none yet.
void *scc_server::get_acc() {
  std::lock_guard<std::mutex> lk(acc_mu);
  if (acc_free.empty()) {
    constexpr size_t kSlot = 256, kSlots = 256;
    void *chunk = nullptr;
    if (cudaMallocHost(&chunk, kSlot * kSlots) != cudaSuccess) return nullptr;
    acc_chunks.push_back(chunk);
    for (size_t i = 0; i < kSlots; ++i) acc_free.push_back(static_cast<char *>(chunk) + i * kSlot);
  }
  void *p = acc_free.back();
  acc_free.pop_back();
  return p;
}

void scc_server::put_acc(void *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(acc_mu);
  acc_free.push_back(p);
}

// Choices for the ready requests that have none: their features were
// launched at admission; one forward pass of the network covers them all.
// Without a network (or without features) a request keeps choice (0,0,0),
// the plain method.
int scc_server::choose(std::vector<Request *> &ready) {
  std::vector<Request *> todo;
  for (Request *r : ready) {
    if (r->have_choice) continue;
    if (!mlp || !r->feat_pending) {
      r->have_choice = true;
      continue;
    }
    todo.push_back(r);
  }
  if (todo.empty()) return SCC_OK;
  std::vector<float> x(todo.size() * sccb::kFeatures);
  for (size_t i = 0; i < todo.size(); ++i) {
    Request *r = todo[i];
    SCK(cudaEventSynchronize(r->featured), "features");
    sccb::graph_features_finish(r->g.n, r->g.m, r->h_acc, &x[i * sccb::kFeatures]);
  }
  std::vector<int32_t> ch(todo.size() * 3);
  int rc = scc_mlp_predict(mlp, x.data(), (uint32_t)todo.size(), ch.data());
  if (rc) return rc;
  for (size_t i = 0; i < todo.size(); ++i) {
    std::memcpy(todo[i]->choice, &ch[i * 3], sizeof(todo[i]->choice));
    todo[i]->have_choice = true;
  }
  return SCC_OK;
}

int scc_server::run_batch(std::vector<Request *> &batch) {
  scc_opts o = cfg.opts;
  if (mlp) {
    int rc = scc_mlp_apply(batch[0]->choice, &o);
    if (rc) return rc;
  }
  int rc = scc_ctx_set_opts(ctx, &o);
  if (rc) return rc;
  for (Request *r : batch) SCK(cudaStreamWaitEvent(solve_st, r->uploaded, 0), "wait upload");
  uint64_t N = 0, M = 0;
  std::vector<PackDesc> desc(batch.size());
  for (size_t i = 0; i < batch.size(); ++i) {
    Request *r = batch[i];
    desc[i] = PackDesc{r->d_off(), r->d_adj(), r->d_offT(), r->d_adjT(), r->g.n, r->g.m, (uint32_t)N, (uint32_t)M};
    N += r->g.n;
    M += r->g.m;
  }
  if (N + 1 > labels_cap) {
    if (d_labels) cudaFree(d_labels);
    d_labels = nullptr;
    labels_cap = 0;
    SCK(cudaMalloc(&d_labels, (N + 1) * 4), "alloc labels");
    labels_cap = (uint32_t)(N + 1);
  }
  SCK(cudaMemcpyAsync(d_desc, desc.data(), desc.size() * sizeof(PackDesc), cudaMemcpyHostToDevice, solve_st),
      "descriptors");
  scc_dev_csr dg{};
  dg.n = (uint32_t)N;
  dg.m = (uint32_t)M;
  if (batch.size() == 1) {
    Request *r = batch[0];
    dg.sorted_unique = r->g.sorted_unique;
    dg.nodes = r->d_off();
    dg.nodesT = r->d_offT();
    dg.edges = r->d_adj();
    dg.edgesT = r->d_adjT();
    rc = scc_ctx_set_segments(ctx, 0, nullptr);
  } else {
    int su = 1;
    for (Request *r : batch) su &= r->g.sorted_unique ? 1 : 0;
    SCK(cudaMemsetAsync(p_off, 0, 8, solve_st), "pack");
    SCK(cudaMemsetAsync(p_offT, 0, 8, solve_st), "pack");
    pack_kernel<<<dim3(64, (unsigned)batch.size()), 256, 0, solve_st>>>(d_desc, p_off, p_adj, p_offT, p_adjT);
    SCK(cudaGetLastError(), "pack launch");
    dg.sorted_unique = su;
    dg.nodes = p_off;
    dg.nodesT = p_offT;
    dg.edges = p_adj;
    dg.edgesT = p_adjT;
    std::vector<uint32_t> seg(batch.size() + 1);
    for (size_t i = 0; i < batch.size(); ++i) seg[i] = desc[i].vbase + 1;
    seg[batch.size()] = (uint32_t)N + 1;
    rc = 0;
    // segments are set after binding (binding checks the CSR on the solve stream)
    int brc = scc_ctx_bind_device(ctx, &dg);
    if (brc) return brc;
    rc = scc_ctx_set_segments(ctx, (uint32_t)batch.size(), seg.data());
    if (rc) return rc;
  }
  if (batch.size() == 1) {
    rc = scc_ctx_bind_device(ctx, &dg);
    if (rc) return rc;
  }
  uint32_t nscc = 0;
  scc_stats stats{};
  rc = scc_solve_device(ctx, d_labels, &nscc, &stats);
  if (rc) return rc;
  SCK(cudaMemsetAsync(d_nscc, 0, batch.size() * 4, solve_st), "unpack");
  if (batch.size() > 1) {
    unpack_kernel<<<dim3(16, (unsigned)batch.size()), 256, 0, solve_st>>>(d_desc, d_labels, d_nscc);
    SCK(cudaGetLastError(), "unpack launch");
  }
  std::vector<uint32_t> counts(batch.size());
  if (batch.size() > 1)
    SCK(cudaMemcpyAsync(counts.data(), d_nscc, batch.size() * 4, cudaMemcpyDeviceToHost, solve_st), "counts");
  else
    counts[0] = nscc;
  for (size_t i = 0; i < batch.size(); ++i) {
    Request *r = batch[i];
    // labels[0] is overwritten below; slot vbase belongs to the previous graph
    SCK(cudaMemcpyAsync(r->labels + 1, d_labels + desc[i].vbase + 1, (size_t)r->g.n * 4, cudaMemcpyDeviceToHost,
                        solve_st),
        "labels");
  }
  SCK(cudaStreamSynchronize(solve_st), "solve stream");
  for (size_t i = 0; i < batch.size(); ++i) {
    Request *r = batch[i];
    r->labels[0] = 0;
    r->info.nscc = counts[i];
    r->info.batch_graphs = (uint32_t)batch.size();
    r->info.solve_ms = stats.ms_total;
  }
  return SCC_OK;
}

void scc_server::solve_loop() {
  cudaSetDevice(cfg.device);
  const uint32_t max_g = cfg.batching ? (cfg.max_batch_graphs ? cfg.max_batch_graphs : 256) : 1;
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_solve.wait(lk, [&] {
      if (stopping && admit_q.empty()) {
        bool busy = false;
        for (auto &kv : reqs)
          if (kv.second->state == RQ_UPLOADING || kv.second->state == RQ_READY) busy = true;
        if (!busy) return true;
      }
      for (auto &kv : reqs)
        if (kv.second->state == RQ_READY) return true;
      return false;
    });
    std::vector<Request *> ready;
    for (auto &kv : reqs)
      if (kv.second->state == RQ_READY) ready.push_back(kv.second.get());  // ids ascend: oldest first
    if (ready.empty()) return;  // stopping, nothing left
    lk.unlock();
    int rc = choose(ready);
    std::vector<Request *> batch;
    if (rc == SCC_OK) {
      uint64_t nv = 0, ne = 0;
      for (Request *r : ready) {
        if (batch.size() >= max_g) break;
        if (!batch.empty() && batch[0]->g.n > cfg.solo_vertices) break;  // a large graph goes alone
        if (!batch.empty() && r->g.n > cfg.solo_vertices) continue;
        if (!batch.empty() && std::memcmp(r->choice, batch[0]->choice, sizeof(r->choice)) != 0) continue;
        if (!batch.empty() && (nv + r->g.n > cfg.max_batch_vertices || ne + r->g.m > cfg.max_batch_edges)) continue;
        batch.push_back(r);
        nv += r->g.n;
        ne += r->g.m;
      }
      lk.lock();
      for (Request *r : batch) r->state = RQ_RUNNING;
      ++st.batches;
      st.graphs_batched += batch.size();
      lk.unlock();
      rc = run_batch(batch);
    } else {
      batch = ready;
    }
    for (Request *r : batch) finish(r, rc);
    lk.lock();
  }
}

extern "C" {

void scc_server_cfg_default(scc_server_cfg *cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->batching = 1;
  cfg->max_batch_graphs = 256;
  cfg->max_batch_vertices = 1u << 24;
  cfg->max_batch_edges = 1u << 27;
  cfg->solo_vertices = 1u << 18;
  scc_opts_default(&cfg->opts);
  cfg->opts.alg = SCC_ALG_HYBRID;
  cfg->opts.wcc = 1;
  cfg->opts.trim2 = 1;
}

int scc_server_start(const scc_server_cfg *cfg, scc_server **out) {
  sccb::clear_error();
  if (!cfg || !out) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  *out = nullptr;
  std::unique_ptr<scc_server> s(new scc_server());
  s->cfg = *cfg;
  if (!s->cfg.max_batch_graphs) s->cfg.max_batch_graphs = 256;
  if (!s->cfg.max_batch_vertices) s->cfg.max_batch_vertices = 1u << 24;
  if (!s->cfg.max_batch_edges) s->cfg.max_batch_edges = 1u << 27;
  if (!s->cfg.solo_vertices) s->cfg.solo_vertices = 1u << 18;
  if (s->cfg.max_batch_vertices >= (1u << 30)) return sccb::set_error(SCC_ERR_INVALID, "max_batch_vertices >= 2^30");
  if (sccb::features_acc_bytes() > 256) return sccb::set_error(SCC_ERR_STATE, "feature accumulator slot too small");
  SCK(cudaSetDevice(cfg->device), "cudaSetDevice");
  int rc = scc_ctx_create(cfg->device, &cfg->opts, &s->ctx);
  if (rc) return rc;
  s->solve_st = static_cast<cudaStream_t>(scc_ctx_stream(s->ctx));
  auto cleanup = [&](int code) {
    scc_server *p = s.release();
    p->stopping = true;
    scc_server_stop(p);
    return code;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&s->copy_st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->feat_st, cudaStreamNonBlocking);
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = cfg->device;
  if (e == cudaSuccess) e = cudaMemPoolCreate(&s->pool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = ~0ull;  // keep freed request memory in the pool for the next uploads
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  const uint64_t nv = s->cfg.max_batch_vertices, ne = s->cfg.max_batch_edges;
  if (e == cudaSuccess && s->cfg.batching) {
    e = cudaMalloc(&s->p_off, (nv + 2) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->p_offT, (nv + 2) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->p_adj, ne * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->p_adjT, ne * 4);
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->d_desc, s->cfg.max_batch_graphs * sizeof(PackDesc));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_nscc, s->cfg.max_batch_graphs * 4);
  if (e != cudaSuccess) {
    srv_fail(e, "server setup");
    return cleanup(e == cudaErrorMemoryAllocation ? SCC_ERR_NOMEM : SCC_ERR_CUDA);
  }
  if (cfg->mem_budget) {
    s->st.budget_bytes = cfg->mem_budget;
  } else {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->st.budget_bytes = fr / 2;
  }
  s->admit_thr = std::thread([p = s.get()] { p->admit_loop(); });
  s->solve_thr = std::thread([p = s.get()] { p->solve_loop(); });
  *out = s.release();
  return SCC_OK;
}

int scc_server_set_model(scc_server *s, const float *params, const float *mean, const float *scale) {
  sccb::clear_error();
  if (!s) return sccb::set_error(SCC_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto &kv : s->reqs)
    if (kv.second->state != RQ_DONE)
      return sccb::set_error(SCC_ERR_BUSY, "set the model while no request is in flight");
  if (!params) {
    if (s->mlp) scc_mlp_destroy(s->mlp);
    s->mlp = nullptr;
    return SCC_OK;
  }
  if (!mean || !scale) return sccb::set_error(SCC_ERR_INVALID, "normalisation missing");
  if (!s->mlp) {
    int rc = scc_mlp_create(s->cfg.device, 0, &s->mlp);
    if (rc) return rc;
  }
  int rc = scc_mlp_params(s->mlp, const_cast<float *>(params), 0);
  if (!rc) rc = scc_mlp_norm(s->mlp, const_cast<float *>(mean), const_cast<float *>(scale), 0);
  return rc;
}

int scc_server_submit(scc_server *s, const scc_host_csr *g, uint32_t *labels, uint64_t *id) {
  sccb::clear_error();
  if (!s || !g || !labels || !id) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  if (!g->nodes || !g->nodesT || (g->m && (!g->edges || !g->edgesT)))
    return sccb::set_error(SCC_ERR_INVALID, "graph arrays missing");
  if (g->n >= (1u << 30)) return sccb::set_error(SCC_ERR_CAPACITY, "n must be below 2^30");
  if (g->nodes[g->n + 1] != g->m || g->nodesT[g->n + 1] != g->m)
    return sccb::set_error(SCC_ERR_INVALID, "offsets end at %u/%u, expected m = %u", g->nodes[g->n + 1],
                           g->nodesT[g->n + 1], g->m);
  std::unique_ptr<Request> r(new Request());
  r->g = *g;
  r->labels = labels;
  r->bytes = Request::csr_bytes(g->n, g->m);
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return sccb::set_error(SCC_ERR_STATE, "server is stopping");
  ++s->st.submitted;
  if (r->bytes > s->st.budget_bytes) {
    ++s->st.rejected;
    return sccb::set_error(SCC_ERR_REJECTED, "graph needs %llu bytes, the budget is %llu",
                           (unsigned long long)r->bytes, (unsigned long long)s->st.budget_bytes);
  }
  if (!s->cfg.batching && g->n + 1 > (1u << 30)) return sccb::set_error(SCC_ERR_CAPACITY, "graph too large");
  r->id = s->next_id++;
  *id = r->id;
  s->admit_q.push_back(r.get());
  s->reqs.emplace(r->id, std::move(r));
  s->cv_admit.notify_one();
  return SCC_OK;
}

static int retire(scc_server *s, std::map<uint64_t, std::unique_ptr<Request>>::iterator it, scc_request_info *info) {
  Request *r = it->second.get();
  if (info) *info = r->info;
  const int status = r->info.status;
  s->reqs.erase(it);
  if (status) return sccb::set_error(status, "request failed with status %d", status);
  return SCC_OK;
}

int scc_server_poll(scc_server *s, uint64_t id, scc_request_info *info) {
  sccb::clear_error();
  if (!s) return sccb::set_error(SCC_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sccb::set_error(SCC_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
  if (it->second->state != RQ_DONE) return SCC_ERR_BUSY;
  return retire(s, it, info);
}

int scc_server_wait(scc_server *s, uint64_t id, uint32_t timeout_ms, scc_request_info *info) {
  sccb::clear_error();
  if (!s) return sccb::set_error(SCC_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sccb::set_error(SCC_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
  Request *r = it->second.get();
  auto done = [&] { return r->state == RQ_DONE; };
  if (timeout_ms) {
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return SCC_ERR_BUSY;
  } else {
    s->cv_done.wait(lk, done);
  }
  return retire(s, s->reqs.find(id), info);
}

int scc_server_get_stats(scc_server *s, scc_server_stats *st) {
  sccb::clear_error();
  if (!s || !st) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->st;
  return SCC_OK;
}

int scc_server_stop(scc_server *s) {
  if (!s) return SCC_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv_admit.notify_all();
    s->cv_solve.notify_all();
  }
  if (s->admit_thr.joinable()) s->admit_thr.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->cv_solve.notify_all();
  }
  if (s->solve_thr.joinable()) s->solve_thr.join();
  cudaSetDevice(s->cfg.device);
  if (s->solve_st) cudaStreamSynchronize(s->solve_st);
  if (s->copy_st) cudaStreamSynchronize(s->copy_st);
  if (s->feat_st) cudaStreamSynchronize(s->feat_st);
  for (auto &kv : s->reqs) {
    Request *r = kv.second.get();
    if (r->dmem) cudaFree(r->dmem);
    if (r->uploaded) cudaEventDestroy(r->uploaded);
    if (r->featured) cudaEventDestroy(r->featured);
  }
  for (void *p : {(void *)s->p_off, (void *)s->p_offT, (void *)s->p_adj, (void *)s->p_adjT, (void *)s->d_labels,
                  (void *)s->d_desc, (void *)s->d_nscc})
    if (p) cudaFree(p);
  for (void *c : s->acc_chunks) cudaFreeHost(c);
  if (s->mlp) scc_mlp_destroy(s->mlp);
  if (s->ctx) scc_ctx_destroy(s->ctx);
  if (s->copy_st) cudaStreamDestroy(s->copy_st);
  if (s->feat_st) cudaStreamDestroy(s->feat_st);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
  return SCC_OK;
}

}  // extern "C"
