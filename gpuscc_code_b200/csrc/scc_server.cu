// Request loop with continuous batching on one device.
//
// Three parties share the request table under one mutex:
//  * callers: scc_server_register uploads a graph once and keeps its CSR
//    resident under a handle; scc_server_submit_resident queues a solve of a
//    resident graph (no upload), scc_server_submit one of a host graph
//    (uploaded for that request only); poll/wait read the result;
//  * the admission thread takes the requests that need an upload in arrival
//    order (host graphs, and resident graphs whose device copy was evicted),
//    waits until the resident bytes plus the upload fit the budget -- evicting
//    resident graphs that no request uses, least recently used first --
//    allocates from the stream-ordered pool and uploads on the copy stream
//    while the solver is busy with earlier batches;
//  * the solver thread, whenever the device is free, takes every ready
//    request (oldest first) whose options match the oldest one's, up to the
//    batch limits, packs them into one segmented CSR with a device kernel (a
//    single graph is bound in place), runs one persistent solve, unpacks each
//    segment's labels back to local ids and copies them to the caller's
//    buffer, then frees a host graph's device copy (a resident one stays).
// With a strategy network loaded, each uploaded graph's feature pass runs on
// a stream of its own (behind the upload, never in front of the next one);
// the solver reads the features when it forms a batch and lets the network
// pick the options of all new requests at once (once per resident graph).
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

uint64_t pad4(uint64_t x) { return (x + 3) & ~uint64_t(3); }

// A graph's device copy: one allocation off | offT | adj | adjT, its upload
// event and, with a network loaded, its feature pass.
struct DevGraph {
  scc_host_csr g{};
  uint64_t bytes = 0;
  void *dmem = nullptr;
  cudaEvent_t uploaded = nullptr;
  void *h_acc = nullptr;  // page-locked slot receiving the feature accumulators
  bool feat_pending = false;
  cudaEvent_t featured = nullptr;  // features done (feature stream)
  bool have_choice = false;
  int32_t choice[3] = {0, 0, 0};
  const uint32_t *d_off() const { return static_cast<const uint32_t *>(dmem); }
  const uint32_t *d_offT() const { return d_off() + pad4(g.n + 2); }
  const uint32_t *d_adj() const { return d_offT() + pad4(g.n + 2); }
  const uint32_t *d_adjT() const { return d_adj() + pad4(g.m); }
  static uint64_t csr_bytes(uint32_t n, uint32_t m) { return (2 * pad4(n + 2) + 2 * pad4(m)) * 4; }
  // the allocation also holds the 16-byte flag of the upload's CSR check
  static uint64_t alloc_bytes(uint32_t n, uint32_t m) { return csr_bytes(n, m) + 16; }
  uint32_t *check_flag() const {
    return reinterpret_cast<uint32_t *>(static_cast<char *>(dmem) + csr_bytes(g.n, g.m));
  }
};

// A registered graph: the caller's host arrays (valid until unregistered)
// and, while resident, its device copy.  pending counts the requests that
// name it and are not finished; only a graph with none may be evicted.
struct Resident {
  uint64_t handle = 0;
  DevGraph dg;
  uint32_t pending = 0;
  uint64_t last_use = 0;         // LRU clock of the last request
  bool uploading = false;
  cudaEvent_t released = nullptr;  // solve-stream point after the last finished request
};

struct Request {
  uint64_t id = 0;
  DevGraph own;              // a host graph's per-request copy
  Resident *res = nullptr;   // or the resident graph it names
  uint32_t *labels = nullptr;
  ReqState state = RQ_QUEUED;
  Clock::time_point t_submit, t_admit, t_done;
  bool have_choice = false;
  int32_t choice[3] = {0, 0, 0};
  scc_request_info info{};
  DevGraph &dev() { return res ? res->dg : own; }
  const scc_host_csr &g() { return dev().g; }
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
  std::map<uint64_t, std::unique_ptr<Resident>> residents;
  uint64_t next_id = 1, next_handle = 1, lru_clock = 0;
  bool stopping = false;
  scc_server_stats st{};
  std::thread admit_thr, solve_thr;

  void admit_loop();
  void solve_loop();
  int run_batch(std::vector<Request *> &batch);
  int choose(std::vector<Request *> &ready);
  cudaError_t upload(DevGraph &d, bool *invalid);
  cudaError_t start_features(DevGraph &d);
  bool make_room(uint64_t bytes);
  void evict(Resident *r);
  void release_dev(DevGraph &d, cudaStream_t order);
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

// Pool allocation + upload of d's host arrays on the copy stream; with a
// network loaded, the graph's feature pass follows on its own stream.
// Called without the lock; d.dmem is published by the caller.
cudaError_t scc_server::upload(DevGraph &d, bool *invalid) {
  void *mem = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&mem, d.bytes, pool, copy_st);
  if (e != cudaSuccess) return e;
  d.dmem = mem;
  const size_t nb = ((size_t)d.g.n + 2) * 4, mb = (size_t)d.g.m * 4;
  e = cudaMemcpyAsync(const_cast<uint32_t *>(d.d_off()), d.g.nodes, nb, cudaMemcpyHostToDevice, copy_st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(const_cast<uint32_t *>(d.d_offT()), d.g.nodesT, nb, cudaMemcpyHostToDevice, copy_st);
  if (e == cudaSuccess && mb)
    e = cudaMemcpyAsync(const_cast<uint32_t *>(d.d_adj()), d.g.edges, mb, cudaMemcpyHostToDevice, copy_st);
  if (e == cudaSuccess && mb)
    e = cudaMemcpyAsync(const_cast<uint32_t *>(d.d_adjT()), d.g.edgesT, mb, cudaMemcpyHostToDevice, copy_st);
  if (e == cudaSuccess && !d.uploaded) e = cudaEventCreateWithFlags(&d.uploaded, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(d.uploaded, copy_st);
  // the kernels trust the layout: each uploaded copy is checked once here,
  // so the solver binds it (and batches packed from it) without checks
  *invalid = false;
  for (int t = 0; e == cudaSuccess && t < 2; ++t) {
    uint32_t bad = 0;
    e = sccb::check_device_csr(t ? d.d_offT() : d.d_off(), t ? d.d_adjT() : d.d_adj(), d.g.n, d.g.m, d.check_flag(),
                               &bad, copy_st);
    if (e == cudaSuccess && bad) *invalid = true;
  }
  if (*invalid) return e;
  // the features are computed behind the upload with nothing waiting for them
  // (the next uploads go on): the solver reads the accumulators when it forms
  // the batch that takes the graph
  if (e == cudaSuccess && mlp && !d.feat_pending) e = start_features(d);
  return e;
}

cudaError_t scc_server::start_features(DevGraph &d) {
  void *scratch = nullptr;
  const size_t fb = sccb::features_scratch_bytes(d.g.n);
  if (!d.h_acc) d.h_acc = get_acc();
  cudaError_t e = d.h_acc ? cudaStreamWaitEvent(feat_st, d.uploaded, 0) : cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&scratch, fb, pool, feat_st);
  if (e != cudaSuccess) return e;
  sccb::EngGraph g{};
  g.n = d.g.n;
  g.m = d.g.m;
  g.sorted_unique = d.g.sorted_unique ? 1u : 0u;
  g.off = d.d_off();
  g.adj = d.d_adj();
  g.offT = d.d_offT();
  g.adjT = d.d_adjT();
  e = sccb::graph_features_launch(g, scratch, fb, d.h_acc, feat_st);
  cudaFreeAsync(scratch, feat_st);
  if (e == cudaSuccess && !d.featured) e = cudaEventCreateWithFlags(&d.featured, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(d.featured, feat_st);
  d.feat_pending = e == cudaSuccess;
  return e;
}

// Frees d's device copy in stream order: after `order`'s pending work (the
// solve stream, or the copy stream behind a recorded release point), after
// the upload and the feature pass that read it.
void scc_server::release_dev(DevGraph &d, cudaStream_t order) {
  if (d.uploaded) cudaStreamWaitEvent(order, d.uploaded, 0);
  if (d.featured) cudaStreamWaitEvent(order, d.featured, 0);
  if (d.h_acc) {
    if (d.featured) cudaEventSynchronize(d.featured);  // the accumulator copy lands in the slot
    put_acc(d.h_acc);
    d.h_acc = nullptr;
  }
  d.feat_pending = false;
  if (d.dmem) cudaFreeAsync(d.dmem, order);
  d.dmem = nullptr;
}

// Evicts resident graph r (lock held; no request names it).
void scc_server::evict(Resident *r) {
  if (r->released) cudaStreamWaitEvent(copy_st, r->released, 0);
  release_dev(r->dg, copy_st);
  st.resident_bytes -= r->dg.bytes;
  ++st.evictions;
}

// Makes `bytes` fit the budget by evicting resident graphs that no request
// names, least recently used first (lock held).  False, evicting nothing,
// when even all of those would not free enough.
bool scc_server::make_room(uint64_t bytes) {
  if (st.resident_bytes + bytes <= st.budget_bytes) return true;
  uint64_t evictable = 0;
  for (auto &kv : residents) {
    const Resident *r = kv.second.get();
    if (!r->uploading && !r->pending && r->dg.dmem) evictable += r->dg.bytes;
  }
  if (st.resident_bytes - evictable + bytes > st.budget_bytes) return false;
  while (st.resident_bytes + bytes > st.budget_bytes) {
    Resident *victim = nullptr;
    for (auto &kv : residents) {
      Resident *r = kv.second.get();
      if (!r->uploading && !r->pending && r->dg.dmem && (!victim || r->last_use < victim->last_use)) victim = r;
    }
    evict(victim);
  }
  return true;
}

void scc_server::admit_loop() {
  cudaSetDevice(cfg.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_admit.wait(lk, [&] {
      if (admit_q.empty()) return stopping;
      Request *r = admit_q.front();
      if (r->res) return !r->res->uploading && (r->res->dg.dmem != nullptr || make_room(r->res->dg.bytes));
      return make_room(r->own.bytes);
    });
    if (admit_q.empty()) return;  // stopping and drained
    Request *r = admit_q.front();
    admit_q.pop_front();
    r->t_admit = Clock::now();
    if (r->res && r->res->dg.dmem) {  // uploaded meanwhile (another request of the same graph, or register)
      r->state = RQ_READY;
      cv_solve.notify_one();
      continue;
    }
    DevGraph &d = r->dev();
    if (r->res) {
      r->res->uploading = true;
      ++st.reuploads;
    }
    st.resident_bytes += d.bytes;
    st.peak_resident_bytes = std::max(st.peak_resident_bytes, st.resident_bytes);
    r->state = RQ_UPLOADING;
    lk.unlock();
    bool invalid = false;
    const cudaError_t e = upload(d, &invalid);
    lk.lock();
    if (r->res) {
      r->res->uploading = false;
      cv_admit.notify_all();
    }
    if (e != cudaSuccess || invalid) {
      if (invalid) sccb::set_error(SCC_ERR_INVALID, "uploaded graph is malformed");
      else sccb::set_error(SCC_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
      cudaStreamSynchronize(copy_st);  // nothing may still write into the allocation when it is freed
      cudaStreamSynchronize(feat_st);
      release_dev(d, copy_st);
      if (r->res) st.resident_bytes -= d.bytes;  // a host graph's bytes are returned by finish
      lk.unlock();
      finish(r, invalid ? SCC_ERR_INVALID : e == cudaErrorMemoryAllocation ? SCC_ERR_NOMEM : SCC_ERR_CUDA);
      lk.lock();
      continue;
    }
    r->state = RQ_READY;
    cv_solve.notify_one();
  }
}

// Marks r done with the given status, releases a host graph's device copy
// (ordered after the solve stream's work; a resident graph keeps its copy and
// records where the solve stream stopped using it) and wakes waiters.
void scc_server::finish(Request *r, int status) {
  if (!r->res) {
    release_dev(r->own, solve_st);
    if (r->own.uploaded) cudaEventDestroy(r->own.uploaded);
    if (r->own.featured) cudaEventDestroy(r->own.featured);
    r->own.uploaded = r->own.featured = nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (r->res) {
    Resident *res = r->res;
    if (!res->released) cudaEventCreateWithFlags(&res->released, cudaEventDisableTiming);
    if (res->released) cudaEventRecord(res->released, solve_st);
    --res->pending;
  } else if (r->state != RQ_QUEUED) {
    st.resident_bytes -= r->own.bytes;
  }
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
// launched at upload (or, for a resident graph uploaded before the network
// was loaded, are launched now); one forward pass of the network covers all
// of them, and a resident graph keeps its choice for its later requests.
// Without a network a request keeps choice (0,0,0), the plain method.
int scc_server::choose(std::vector<Request *> &ready) {
  std::vector<DevGraph *> todo;
  for (Request *r : ready) {
    if (r->have_choice) continue;
    DevGraph &d = r->dev();
    if (!mlp || d.have_choice) {
      if (mlp) std::memcpy(r->choice, d.choice, sizeof(r->choice));
      r->have_choice = true;
      continue;
    }
    if (!d.feat_pending) {
      cudaError_t e = start_features(d);
      if (e != cudaSuccess) {  // the plain method stays the fallback
        r->have_choice = true;
        continue;
      }
    }
    if (std::find(todo.begin(), todo.end(), &d) == todo.end()) todo.push_back(&d);
  }
  if (!todo.empty()) {
    std::vector<float> x(todo.size() * sccb::kFeatures);
    for (size_t i = 0; i < todo.size(); ++i) {
      DevGraph *d = todo[i];
      SCK(cudaEventSynchronize(d->featured), "features");
      sccb::graph_features_finish(d->g.n, d->g.m, d->h_acc, &x[i * sccb::kFeatures]);
    }
    std::vector<int32_t> ch(todo.size() * 3);
    int rc = scc_mlp_predict(mlp, x.data(), (uint32_t)todo.size(), ch.data());
    if (rc) return rc;
    for (size_t i = 0; i < todo.size(); ++i) {
      std::memcpy(todo[i]->choice, &ch[i * 3], sizeof(todo[i]->choice));
      todo[i]->have_choice = true;
    }
  }
  for (Request *r : ready) {
    if (r->have_choice) continue;
    std::memcpy(r->choice, r->dev().choice, sizeof(r->choice));
    r->have_choice = true;
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
  for (Request *r : batch) SCK(cudaStreamWaitEvent(solve_st, r->dev().uploaded, 0), "wait upload");
  uint64_t N = 0, M = 0;
  std::vector<PackDesc> desc(batch.size());
  for (size_t i = 0; i < batch.size(); ++i) {
    const DevGraph &d = batch[i]->dev();
    desc[i] = PackDesc{d.d_off(), d.d_adj(), d.d_offT(), d.d_adjT(), d.g.n, d.g.m, (uint32_t)N, (uint32_t)M};
    N += d.g.n;
    M += d.g.m;
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
    const DevGraph &d = batch[0]->dev();
    dg.sorted_unique = d.g.sorted_unique;
    dg.nodes = d.d_off();
    dg.nodesT = d.d_offT();
    dg.edges = d.d_adj();
    dg.edgesT = d.d_adjT();
    rc = sccb::ctx_set_segments_unchecked(ctx, 0, nullptr);
  } else {
    int su = 1;
    for (Request *r : batch) su &= r->g().sorted_unique ? 1 : 0;
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
    // every member was checked at its upload and the pack kernel keeps each
    // graph on its own ids: bind and segment without device checks
    int brc = sccb::ctx_bind_unchecked(ctx, &dg);
    if (brc) return brc;
    rc = sccb::ctx_set_segments_unchecked(ctx, (uint32_t)batch.size(), seg.data());
    if (rc) return rc;
  }
  if (batch.size() == 1) {
    rc = sccb::ctx_bind_unchecked(ctx, &dg);
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
    SCK(cudaMemcpyAsync(r->labels + 1, d_labels + desc[i].vbase + 1, (size_t)r->g().n * 4, cudaMemcpyDeviceToHost,
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

// at most four edges per vertex: the deep, thin graphs (grids) of a stream
static bool is_thin(uint32_t n, uint32_t m) { return (uint64_t)m <= 4ull * n; }

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
        const uint32_t gn = r->g().n, gm = r->g().m;
        if (!batch.empty() && batch[0]->g().n > cfg.solo_vertices) break;  // a large graph goes alone
        if (!batch.empty() && gn > cfg.solo_vertices) continue;
        if (!batch.empty() && std::memcmp(r->choice, batch[0]->choice, sizeof(r->choice)) != 0) continue;
        // a batch runs as many rounds and levels as its deepest graph: thin
        // graphs (grids: thousands of levels) are batched only with each other
        if (!batch.empty() && is_thin(r->g().n, gm) != is_thin(batch[0]->g().n, batch[0]->g().m)) continue;
        if (!batch.empty() && (nv + gn > cfg.max_batch_vertices || ne + gm > cfg.max_batch_edges)) continue;
        batch.push_back(r);
        nv += gn;
        ne += gm;
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
  for (auto &kv : s->residents) kv.second->dg.have_choice = false;  // picks belong to the old network
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

static int check_host_graph(const scc_host_csr *g) {
  if (!g->nodes || !g->nodesT || (g->m && (!g->edges || !g->edgesT)))
    return sccb::set_error(SCC_ERR_INVALID, "graph arrays missing");
  if (g->n >= (1u << 30)) return sccb::set_error(SCC_ERR_CAPACITY, "n must be below 2^30");
  if (g->nodes[g->n + 1] != g->m || g->nodesT[g->n + 1] != g->m)
    return sccb::set_error(SCC_ERR_INVALID, "offsets end at %u/%u, expected m = %u", g->nodes[g->n + 1],
                           g->nodesT[g->n + 1], g->m);
  return SCC_OK;
}

int scc_server_register(scc_server *s, const scc_host_csr *g, uint64_t *handle) {
  sccb::clear_error();
  if (!s || !g || !handle) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  int rc = check_host_graph(g);
  if (rc) return rc;
  std::unique_ptr<Resident> res(new Resident());
  res->dg.g = *g;
  res->dg.bytes = DevGraph::alloc_bytes(g->n, g->m);
  Resident *r = res.get();
  {
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stopping) return sccb::set_error(SCC_ERR_STATE, "server is stopping");
    if (r->dg.bytes > s->st.budget_bytes) {
      ++s->st.rejected;
      return sccb::set_error(SCC_ERR_REJECTED, "graph needs %llu bytes, the budget is %llu",
                             (unsigned long long)r->dg.bytes, (unsigned long long)s->st.budget_bytes);
    }
    // room comes from evicting idle resident graphs or from requests finishing
    s->cv_done.wait(lk, [&] { return s->stopping || s->make_room(r->dg.bytes); });
    if (s->stopping) return sccb::set_error(SCC_ERR_STATE, "server is stopping");
    s->st.resident_bytes += r->dg.bytes;
    s->st.peak_resident_bytes = std::max(s->st.peak_resident_bytes, s->st.resident_bytes);
    r->handle = s->next_handle++;
    r->uploading = true;
    r->last_use = ++s->lru_clock;
    s->residents.emplace(r->handle, std::move(res));
  }
  cudaSetDevice(s->cfg.device);
  bool invalid = false;
  cudaError_t e = s->upload(r->dg, &invalid);
  if (e == cudaSuccess && !invalid) e = cudaEventSynchronize(r->dg.uploaded);
  std::lock_guard<std::mutex> lk(s->mu);
  r->uploading = false;
  s->cv_admit.notify_all();
  if (e != cudaSuccess || invalid) {
    cudaStreamSynchronize(s->copy_st);
    cudaStreamSynchronize(s->feat_st);
    s->release_dev(r->dg, s->copy_st);
    s->st.resident_bytes -= r->dg.bytes;
    if (r->dg.uploaded) cudaEventDestroy(r->dg.uploaded);
    if (r->dg.featured) cudaEventDestroy(r->dg.featured);
    s->residents.erase(r->handle);
    if (invalid) return sccb::set_error(SCC_ERR_INVALID, "graph is malformed (offsets or neighbour ids)");
    return srv_fail(e, "register upload");
  }
  ++s->st.registered;
  *handle = r->handle;
  return SCC_OK;
}

int scc_server_submit_resident(scc_server *s, uint64_t handle, uint32_t *labels, uint64_t *id) {
  sccb::clear_error();
  if (!s || !labels || !id) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return sccb::set_error(SCC_ERR_STATE, "server is stopping");
  auto it = s->residents.find(handle);
  if (it == s->residents.end())
    return sccb::set_error(SCC_ERR_INVALID, "unknown graph handle %llu", (unsigned long long)handle);
  Resident *res = it->second.get();
  std::unique_ptr<Request> r(new Request());
  r->res = res;
  r->labels = labels;
  r->t_submit = Clock::now();
  ++s->st.submitted;
  ++res->pending;
  res->last_use = ++s->lru_clock;
  r->id = s->next_id++;
  *id = r->id;
  Request *rp = r.get();
  s->reqs.emplace(r->id, std::move(r));
  if (!res->uploading && res->dg.dmem) {  // on the device: ready at once, no admission needed
    rp->t_admit = rp->t_submit;
    rp->state = RQ_READY;
    s->cv_solve.notify_one();
  } else {  // evicted: the admission thread uploads it again
    s->admit_q.push_back(rp);
    s->cv_admit.notify_one();
  }
  return SCC_OK;
}

int scc_server_unregister(scc_server *s, uint64_t handle) {
  sccb::clear_error();
  if (!s) return sccb::set_error(SCC_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->residents.find(handle);
  if (it == s->residents.end())
    return sccb::set_error(SCC_ERR_INVALID, "unknown graph handle %llu", (unsigned long long)handle);
  Resident *r = it->second.get();
  if (r->pending || r->uploading)
    return sccb::set_error(SCC_ERR_BUSY, "graph %llu still has %u requests in flight", (unsigned long long)handle,
                           r->pending);
  if (r->dg.dmem) {
    s->evict(r);
    --s->st.evictions;  // a release, not an eviction
  }
  if (r->dg.uploaded) cudaEventDestroy(r->dg.uploaded);
  if (r->dg.featured) cudaEventDestroy(r->dg.featured);
  if (r->released) cudaEventDestroy(r->released);
  s->residents.erase(it);
  return SCC_OK;
}

int scc_server_submit(scc_server *s, const scc_host_csr *g, uint32_t *labels, uint64_t *id) {
  sccb::clear_error();
  if (!s || !g || !labels || !id) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  int rc = check_host_graph(g);
  if (rc) return rc;
  std::unique_ptr<Request> r(new Request());
  r->own.g = *g;
  r->own.bytes = DevGraph::alloc_bytes(g->n, g->m);
  r->labels = labels;
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return sccb::set_error(SCC_ERR_STATE, "server is stopping");
  ++s->st.submitted;
  if (r->own.bytes > s->st.budget_bytes) {
    ++s->st.rejected;
    return sccb::set_error(SCC_ERR_REJECTED, "graph needs %llu bytes, the budget is %llu",
                           (unsigned long long)r->own.bytes, (unsigned long long)s->st.budget_bytes);
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
    DevGraph &d = kv.second->own;
    if (d.dmem) cudaFree(d.dmem);
    if (d.uploaded) cudaEventDestroy(d.uploaded);
    if (d.featured) cudaEventDestroy(d.featured);
  }
  for (auto &kv : s->residents) {
    Resident *r = kv.second.get();
    if (r->dg.dmem) cudaFree(r->dg.dmem);
    if (r->dg.uploaded) cudaEventDestroy(r->dg.uploaded);
    if (r->dg.featured) cudaEventDestroy(r->dg.featured);
    if (r->released) cudaEventDestroy(r->released);
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
