// Persistent Forward-Backward SCC engine for B200 (sm_100a).
//
// One cooperative launch runs the whole reference driver loop
// (scc.cu:217-910: trim-1, pivot, forward/backward reach, trim, update,
// WCC + trim-2 once, repeat) with grid barriers instead of host round trips.
// Each phase is a __device__ member of Eng; the phase-level C ABI launches
// the same code one phase at a time.
//
// Per-vertex state (reference scc.h:48-93 packs it in one byte; here it is
// split so the hot tests hit L2-resident bitmaps, n/8 bytes each):
//   elim   - vertex already assigned to an SCC (reference bit E = 4)
//   fvis   - forward visited (F = 2)          bvis - backward visited (B = 1)
//   fexp   - forward expanded (FExt = 64)      bexp - backward expanded (BExt = 32)
//   tflag  - removed by trim-1 (T = 8)         queued - trim candidate / trim-2 mark
//   label  - u32 SCC label, range - u32 partition id (reference `ranges`).
// Partition ids are exact: a refined partition is identified by the id of its
// pivot, elected as the smallest (priority, id) key among its members, so the
// reference's 3r+k hashing into 2^20 slots (scc_routines.cu:168-176) and its
// collisions and wrap-around do not exist here.
#include <cstdio>

#include "scc_device.cuh"
#include "scc_engine.h"

namespace sccb {

enum : uint32_t {
  C_CHG = 0, C_DEG = 1, C_Q = 2, C_Q2 = 3, C_CNT = 4, C_CNT2 = 5, C_REM = 6,
  // results of a run of CTA-local levels (reach_wl)
  C_LN = 7, C_LSEL = 8, C_LD = 9, C_LMF = 10, C_LEX = 11, C_LREF = 12
};
// CTA-local reach levels: frontiers of at most kLocalMax vertices and
// kLocalEdges edges are expanded by CTA 0 alone with CTA barriers, at most
// kLocalLevels levels per grid barrier
constexpr uint32_t kLocalMax = 2048, kLocalEdges = 4096, kLocalLevels = 4096;
// push levels whose frontier has at most this many edges per vertex test
// targets with try_visit_wide
constexpr uint32_t kWideDegree = 16;
// polls of a partly filled window before an asynchronous step expands it
constexpr uint32_t kAsyncHold = 1;
// frontiers below this many vertices stay in CTA-local levels rather than
// starting an asynchronous phase
constexpr uint32_t kAsyncMin = 32;
// claims an asynchronous step keeps for the warp's next step (the rest go to
// the shared queue)
constexpr uint32_t kAsyncKeep = 32;
// WCC switches from full sweeps to frontier sweeps once fewer than live / this
// many colours change in a sweep
constexpr uint32_t kWccFrontier = 64;
// graphs of at most this many vertices run on one CTA per SM by default
constexpr uint32_t kSmallGraphN = 1u << 21;
// HYBRID / COMBINE / BEST tails are asynchronous reaches on graphs of at most
// this many edges per vertex
constexpr uint32_t kAsyncTailDegree = 12;
enum : uint32_t { ARM_Q = 0, ARM_T = 1, ARM_D = 2, ARM_L = 3, ARM_B = 6, ARM_TA = 7 };

constexpr int kSlotCache = 128;  // per-CTA cache of partition-election slots
constexpr int kSizeCache = 32;   // per-CTA cache of SCC-size counters

template <int BS>
struct Eng {
  const Params &P;
  Ctl *c;
  uint32_t k;  // barrier interval index, identical in every CTA
  uint32_t list_mode, act_count, act_sel;
  // asynchronous reach: items seeded for the pending phase; a_defer: a
  // reach seeds and returns, and the caller runs both directions' phase
  uint32_t a_seeded;
  bool a_defer;
  bool a_trim;  // trims run their worklist asynchronously (the solve, with async reaches on)

  __device__ explicit Eng(const Params &p)
      : P(p), c(p.s.ctl), k(0), list_mode(0), act_count(0), act_sel(0), a_seeded(0), a_defer(false),
        a_trim(false) {}

  // ------------------------------------------------------------ plumbing
  __device__ __forceinline__ uint32_t *cur() { return c->ctr[k % 3]; }
  __device__ __forceinline__ uint32_t *prv() { return c->ctr[(k + 2) % 3]; }
  __device__ __forceinline__ unsigned long long *cur64() { return &c->ctr64[k % 3]; }
  __device__ __forceinline__ unsigned long long *prv64() { return &c->ctr64[(k + 2) % 3]; }
  __device__ __forceinline__ uint32_t rdprv(uint32_t i) { return ldm(prv() + i); }

  __device__ __forceinline__ bool bar(uint32_t where) {
    if (P.o.test_stall_ns && k == 1 && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
      // fault-path test hook: a bounded delay of this CTA's arrival (the
      // others' barrier waits run out first when timeout_ns is shorter)
      const unsigned long long t0 = globaltimer_ns();
      while (globaltimer_ns() - t0 < P.o.test_stall_ns) __nanosleep(1000);
    }
    if (blockIdx.x == 0) {
      if (threadIdx.x < 16) c->ctr[(k + 1) % 3][threadIdx.x] = 0;
      if (threadIdx.x == 16) c->ctr64[(k + 1) % 3] = 0;
    }
    const bool ok = grid_barrier(reinterpret_cast<GridSync *>(&c->gs), (unsigned long long)(k + 1) * gridDim.x,
                                 P.o.timeout_ns, where);
    ++k;
    return ok;
  }
  __device__ __forceinline__ void refresh_mode() {
    list_mode = ldm(&c->list_mode);
    act_count = ldm(&c->act_count);
    act_sel = ldm(&c->act_sel);
  }
  __device__ __forceinline__ uint32_t *err() { return &c->gs.err; }
  __device__ __forceinline__ void fail(uint32_t bits) { atomicOr(&c->gs.err, bits); }
  __device__ __forceinline__ bool is_lead() { return blockIdx.x == 0 && threadIdx.x == 0; }
  // CTA 0 / thread 0 accumulates the time since t0 under profile slot `slot`
  __device__ __forceinline__ void prof(uint32_t slot, unsigned long long t0, uint32_t a = 0, uint32_t b = 0) {
    if (is_lead()) {
      const unsigned long long dt = globaltimer_ns() - t0;
      c->prof_ns[slot] += dt;
      c->prof_cnt[slot] += 1;
      const uint32_t i = c->trace_n;
      if (i < kTrace) {
        c->trace_slot[i] = slot;
        c->trace_a[i] = a;
        c->trace_b[i] = b;
        c->trace_ns[i] = dt;
        c->trace_n = i + 1;
      }
    }
  }

  // Sets bit v of `bm` for every lane with pred; all 32 lanes must call.
  // Lanes whose ids share a bitmap word combine into one atomicOr instead of
  // 32 serialised ones.  aligned: lane i holds id 32*w + i of a single word w
  // (full-mode for_vertices), so one ballot forms the word.
  __device__ __forceinline__ void warp_set_bits(uint32_t *bm, uint32_t v, bool pred, bool aligned) {
    if (aligned) {
      const uint32_t bits = __ballot_sync(kFull, pred);
      if (bits && lane_id() == 0) atomicOr(bm + (v >> 5), bits);
      return;
    }
    const uint32_t word = pred ? (v >> 5) : kNone;
    const uint32_t grp = __match_any_sync(kFull, word);
    if (pred) {
      const uint32_t bits = __reduce_or_sync(grp, 1u << (v & 31u));
      if (lane_id() == (uint32_t)(__ffs(grp) - 1)) atomicOr(bm + word, bits);
    }
  }

  // block-reduced atomicAdd into a global counter
  __device__ __forceinline__ void add_count(uint32_t *dst, uint32_t x) {
    const uint32_t s = block_sum(x);
    if (threadIdx.x == 0 && s) atomicAdd(dst, s);
  }

  // Members of the SCC of pivot p eliminated together: a CTA-local cache
  // (kSizeCache direct-mapped slots) absorbs the adds of its few large
  // components, so a giant SCC costs one global atomic per CTA, not one per
  // warp.  Running totals only grow, so the largest total any add returns
  // is the largest component.
  __device__ __forceinline__ void size_flush(const EngState &s, uint32_t p, uint32_t cnt) {
    const uint32_t tot = atomicAdd(s.sccsize + p, cnt) + cnt;
    if (tot > ldm(&c->largest_fb)) atomicMax(&c->largest_fb, tot);
  }
  __device__ __forceinline__ void size_add(const EngState &s, uint32_t *s_szkey, uint32_t *s_szcnt, uint32_t p, uint32_t cnt) {
    const uint32_t h = p % kSizeCache;
    uint32_t owner = s_szkey[h];
    if (owner == kNone) owner = atomicCAS(&s_szkey[h], kNone, p) == kNone ? p : s_szkey[h];
    if (owner == p) atomicAdd(&s_szcnt[h], cnt);
    else size_flush(s, p, cnt);
  }

  __device__ __forceinline__ uint32_t gtid() const { return blockIdx.x * BS + threadIdx.x; }
  __device__ __forceinline__ uint32_t gstride() const { return gridDim.x * BS; }
  __device__ __forceinline__ uint32_t gwarp() const { return (blockIdx.x * BS + threadIdx.x) >> 5; }
  __device__ __forceinline__ uint32_t nwarps() const { return (gridDim.x * BS) >> 5; }

  // Calls f(v, valid) for every vertex of the current sweep set, all 32
  // lanes of a warp together (valid = false pads the last block), then
  // after() once per iteration with the whole CTA (every CTA runs whole
  // iterations, so after() may __syncthreads).  Full mode covers ids
  // 0 .. nwords*32-1 so that a warp owns exactly one bitmap word.
  template <class F, class H>
  __device__ __forceinline__ void for_vertices(F &&f, H &&after) {
    if (list_mode) {
      const uint32_t *lst = P.s.act[act_sel];
      const uint32_t cnt = act_count;
      const uint32_t lim = (cnt + BS - 1u) / BS * BS;
      for (uint32_t base = blockIdx.x * BS; base < lim; base += gstride()) {
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < cnt;
        f(valid ? ldm(lst + i) : 0u, valid);
        after();
      }
    } else {
      const uint32_t lim = P.s.nwords * 32u;  // a multiple of 1024 >= BS
      const uint32_t n = P.g.n;
      for (uint32_t base = blockIdx.x * BS; base < lim; base += gstride()) {
        const uint32_t v = base + threadIdx.x;
        f(v, v >= 1 && v <= n);
        after();
      }
    }
  }
  template <class F>
  __device__ __forceinline__ void for_vertices(F &&f) {
    for_vertices(f, [] {});
  }

  // for_vertices with a one-deep software pipeline: load(v, valid) issues
  // the loads of the NEXT iteration before f(v, valid, pre) runs on the
  // current one, so their latency overlaps the current vertex's dependent
  // chain.  load() may only read data that f() of the same iteration does
  // not change for other lanes' vertices (bitmap words, offsets, ranges).
  // The same over an explicit list lst[0, cnt): two-deep, the entry two
  // iterations ahead and the per-vertex loads of the next entry are in
  // flight while f runs on the current one.  Whole CTAs iterate together.
  template <class L, class F>
  __device__ __forceinline__ void for_list_pf(const uint32_t *lst, uint32_t cnt, L &&load, F &&f) {
    const uint32_t lim = (cnt + BS - 1u) / BS * BS;
    const uint32_t stride = gstride();
    uint32_t base = blockIdx.x * BS;
    if (base >= lim) return;
    const uint32_t i0 = base + threadIdx.x, i1 = i0 + stride;
    bool val0 = i0 < cnt, val1 = i1 < cnt;
    uint32_t v0 = val0 ? ldm(lst + i0) : 0u;
    uint32_t v1 = val1 ? ldm(lst + i1) : 0u;
    auto pre = load(v0, val0);
    for (; base < lim; base += stride) {
      const uint32_t i2 = base + 2u * stride + threadIdx.x;
      const bool val2 = i2 < cnt;
      const uint32_t v2 = val2 ? ldm(lst + i2) : 0u;
      auto nxt = pre;
      if (base + stride < lim) nxt = load(v1, val1);
      f(v0, val0, pre);
      pre = nxt;
      v0 = v1;
      val0 = val1;
      v1 = v2;
      val1 = val2;
    }
  }

  // The same with two entries per thread, i and i + half (half = ceil(cnt/2)),
  // so f gets two independent vertices whose dependent loads can overlap.
  template <class L, class F>
  __device__ __forceinline__ void for_list_pairs_pf(const uint32_t *lst, uint32_t cnt, L &&load, F &&f) {
    const uint32_t half = (cnt + 1u) / 2u;
    const uint32_t lim = (half + BS - 1u) / BS * BS;
    const uint32_t stride = gstride();
    uint32_t base = blockIdx.x * BS;
    if (base >= lim) return;
    auto id = [&](uint32_t i, bool &va, uint32_t &a, bool &vb, uint32_t &b) {
      va = i < half;
      vb = i + half < cnt;
      a = va ? ldm(lst + i) : 0u;
      b = vb ? ldm(lst + i + half) : 0u;
    };
    const uint32_t i0 = base + threadIdx.x;
    bool a0v, b0v, a1v, b1v;
    uint32_t a0, b0, a1, b1;
    id(i0, a0v, a0, b0v, b0);
    id(i0 + stride, a1v, a1, b1v, b1);
    auto pa = load(a0, a0v);
    auto pb = load(b0, b0v);
    for (; base < lim; base += stride) {
      bool a2v, b2v;
      uint32_t a2, b2;
      id(base + 2u * stride + threadIdx.x, a2v, a2, b2v, b2);
      auto na = pa, nb = pb;
      if (base + stride < lim) {
        na = load(a1, a1v);
        nb = load(b1, b1v);
      }
      f(a0, a0v, pa, b0, b0v, pb);
      pa = na;
      pb = nb;
      a0 = a1, a0v = a1v, b0 = b1, b0v = b1v;
      a1 = a2, a1v = a2v, b1 = b2, b1v = b2v;
    }
  }

  template <class L, class F>
  __device__ __forceinline__ void for_vertices_pf(L &&load, F &&f) {
    if (list_mode) {
      for_list_pf(P.s.act[act_sel], act_count, load, f);
      return;
    }
    const uint32_t lim = P.s.nwords * 32u;
    const uint32_t n = P.g.n;
    uint32_t base = blockIdx.x * BS;
    if (base >= lim) return;
    auto pre = load(base + threadIdx.x, base + threadIdx.x >= 1 && base + threadIdx.x <= n);
    for (; base < lim; base += gstride()) {
      const uint32_t v = base + threadIdx.x;
      const uint32_t nb = base + gstride();
      auto nxt = pre;
      if (nb < lim) {
        const uint32_t nv = nb + threadIdx.x;
        nxt = load(nv, nv >= 1 && nv <= n);
      }
      f(v, v >= 1 && v <= n, pre);
      pre = nxt;
    }
  }

  // Warp-staged worklist append.  Items a warp emits during a sweep collect
  // in its own shared-memory segment and reach the global list kStage at a
  // time with one atomicAdd, so a sweep that emits millions of items does not
  // serialise every warp of the grid on one counter word in L2, and no CTA
  // barrier is involved (warps never wait for each other).
  struct Stage {
    uint32_t n;      // items staged by this warp (identical in all 32 lanes)
    uint32_t which;  // this warp's segment: stage_buf(which), stage_desc(which)
  };
  // Where a warp's segment drains to.  Kept in shared memory, not in the
  // Stage: a sweep feeding two lists would otherwise hold six more
  // registers per thread for values only a flush reads.
  struct StageDesc {
    uint32_t *dst;
    uint32_t *count;
    uint32_t cap;
  };
  static constexpr uint32_t kStage = BS >= 1024 ? 128 : 256;  // 2 segments per warp within 48 KB static
  // which = 0 or 1: two independent segments per warp (a sweep may feed two lists)
  // the staging segments of all warps, 2 * (BS / 32) * kStage >= 8 * BS words
  __device__ __forceinline__ uint32_t *stage_mem() {
    __shared__ uint32_t buf[2 * (BS / 32) * kStage];
    return buf;
  }
  __device__ __forceinline__ uint32_t *stage_buf(uint32_t which = 0) {
    return stage_mem() + (which * (BS / 32) + (threadIdx.x >> 5)) * kStage;
  }
  __device__ __forceinline__ StageDesc *stage_desc(uint32_t which) {
    __shared__ StageDesc desc[2][BS / 32];
    return &desc[which][threadIdx.x >> 5];
  }
  // all 32 lanes of the warp call it together
  __device__ __forceinline__ Stage stage_open(uint32_t which, uint32_t *dst, uint32_t *count, uint32_t cap) {
    if (lane_id() == 0) *stage_desc(which) = StageDesc{dst, count, cap};
    __syncwarp();
    return Stage{0u, which};
  }
  __device__ __forceinline__ void stage_flush(Stage &q) {
    __syncwarp();
    const StageDesc d = *stage_desc(q.which);
    uint32_t base = 0;
    if (lane_id() == 0 && q.n) base = atomicAdd(d.count, q.n);
    base = __shfl_sync(kFull, base, 0);
    const uint32_t *buf = stage_buf(q.which);
    for (uint32_t i = lane_id(); i < q.n; i += 32) {
      const uint32_t pos = base + i;
      if (pos < d.cap) d.dst[pos] = buf[i];
      else atomicOr(err(), kErrQueueOverflow);
    }
    q.n = 0;
    __syncwarp();
  }
  // all 32 lanes of the warp call it together
  __device__ __forceinline__ void stage_put(Stage &q, bool pred, uint32_t v) {
    const uint32_t mask = __ballot_sync(kFull, pred);
    if (!mask) return;
    if (pred) stage_buf(q.which)[q.n + __popc(mask & lanemask_lt())] = v;
    q.n += __popc(mask);
    if (q.n > kStage - 32) stage_flush(q);
  }
  // every id 0 .. nwords*32-1 regardless of the active list
  template <class F>
  __device__ __forceinline__ void for_all_ids(F &&f) {
    const uint32_t lim = P.s.nwords * 32u;
    const uint32_t n = P.g.n;
    for (uint32_t v = gtid(); v < lim; v += gstride()) f(v, v >= 1 && v <= n);
  }
  // grid-stride over [0, cnt), whole CTAs
  template <class F>
  __device__ __forceinline__ void for_items(uint32_t cnt, F &&f) {
    const uint32_t lim = (cnt + BS - 1u) / BS * BS;
    for (uint32_t i = gtid(); i < lim; i += gstride()) f(i, i < cnt);
  }

  // Helpers below take the parameter blocks they read as arguments.
  __device__ __forceinline__ static bool live(const EngState &s, uint32_t v) { return !bit_test(s.elim, v); }

  __device__ __forceinline__ static uint32_t prio(const EngGraph &g, uint32_t rule, uint32_t v) {
    if (rule == 0) return 0u;
    const unsigned long long dout = ldg(g.off + v + 1) - ldg(g.off + v);
    const unsigned long long din = ldg(g.offT + v + 1) - ldg(g.offT + v);
    unsigned long long s = dout * din;
    if (s > 0xfffffffeull) s = 0xfffffffeull;
    return 0xfffffffeu - (uint32_t)s;
  }

  // ====================================================== trim-1 (a5/a6)
  // scc_routines.cu:276-394: v is trimmed when it has no out-neighbour or no
  // in-neighbour that is not itself, not eliminated and (ranged) in its
  // partition.  Trimmed vertices become singleton SCCs (state 28).
  __device__ __forceinline__ static bool live_nbr(const EngState &s, const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                  uint32_t v, uint32_t rv, bool ranged, bool snap) {
    const uint32_t b = ldg(off + v), e = ldg(off + v + 1);
    if (snap) {  // nothing eliminated yet and lists sorted-unique
      const uint32_t d = e - b;
      return d >= 2 || (d == 1 && ldg(adj + b) != v);
    }
    for (uint32_t i = b; i < e; ++i) {
      const uint32_t u = ldg(adj + i);
      if (u == v || !live(s, u)) continue;
      if (ranged && ldm(s.range + u) != rv) continue;
      return true;
    }
    return false;
  }

  // Returns the number of trim iterations.  Iteration 1 sweeps the active
  // set; later iterations only re-check neighbours of vertices trimmed in the
  // previous one (deduplicated through the `queued` bitmap).
  // pick: also elect the first pivot among the survivors of the sweep (only
  // valid when no further trim iteration follows, i.e. max_it == 1).
  // The first trim sweep when nothing is eliminated yet and every list is
  // sorted-unique: only degrees decide (a list of one entry counts unless it
  // is a self-loop).  Each thread takes four consecutive ids with one 16-byte
  // load of each offset array (the fifth offset comes from the next lane;
  // lane 31 loads it), next iteration's loads in flight, so a warp covers
  // four bitmap words per iteration and the sweep streams the offsets with
  // no dependent load: an id whose decision needs the head of a single-entry
  // list (the self-loop test) goes to its warp's shared-memory buffer, which
  // the warp resolves in batches with all head loads in flight together.
  // Eliminated/trimmed words are assembled in registers.  Returns this
  // thread's count of trimmed ids.
  __device__ __noinline__ uint32_t trim_snap_sweep(bool pick, unsigned long long &best) {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    const uint32_t rule = P.o.pivot_rule;
    const uint32_t n = g.n;
    const uint32_t lim = s.nwords * 32u;  // multiple of 1024
    const uint32_t lane = lane_id();
    const bool vec = ((reinterpret_cast<uintptr_t>(g.off) | reinterpret_cast<uintptr_t>(g.offT)) & 15u) == 0;
    const bool vlab = (reinterpret_cast<uintptr_t>(s.label) & 15u) == 0;  // labels stored four at a time
    const uint32_t step = gstride() * 4u;
    struct Quad {
      uint32_t o[4], t[4], o4, t4;
    };
    auto load = [&](uint32_t v0) {
      Quad q;
      if (vec && v0 + 4u <= n + 2u) {  // off / offT hold n+2 entries
        const uint4 a = __ldg(reinterpret_cast<const uint4 *>(g.off + v0));
        const uint4 b = __ldg(reinterpret_cast<const uint4 *>(g.offT + v0));
        q.o[0] = a.x, q.o[1] = a.y, q.o[2] = a.z, q.o[3] = a.w;
        q.t[0] = b.x, q.t[1] = b.y, q.t[2] = b.z, q.t[3] = b.w;
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const bool in = v0 + i <= n + 1u;
          q.o[i] = in ? ldg(g.off + v0 + i) : 0u;
          q.t[i] = in ? ldg(g.offT + v0 + i) : 0u;
        }
      }
      const bool in4 = lane == 31 && v0 + 4u <= n + 1u;
      q.o4 = in4 ? ldg(g.off + v0 + 4u) : 0u;
      q.t4 = in4 ? ldg(g.offT + v0 + 4u) : 0u;
      return q;
    };
    uint32_t ntrim = 0;
    // ids waiting for the self-loop test: this warp's stage segment
    uint32_t *pend = stage_buf(0);
    uint32_t npend = 0;  // warp-uniform
    auto resolve = [&]() {
      __syncwarp();
      for (uint32_t i0 = 0; i0 < npend; i0 += 128u) {
        uint32_t v[4], x[4], y[4];
        bool ok[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint32_t i = i0 + j * 32u + lane;
          ok[j] = i < npend;
          v[j] = ok[j] ? pend[i] : 0u;
        }
        uint32_t ob[4], dout[4], tb[4], din[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          ob[j] = ok[j] ? ldg(g.off + v[j]) : 0u;
          dout[j] = ok[j] ? ldg(g.off + v[j] + 1) - ob[j] : 0u;
          tb[j] = ok[j] ? ldg(g.offT + v[j]) : 0u;
          din[j] = ok[j] ? ldg(g.offT + v[j] + 1) - tb[j] : 0u;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          x[j] = (ok[j] && dout[j] == 1) ? ldg(g.adj + ob[j]) : 0u;
          y[j] = (ok[j] && din[j] == 1) ? ldg(g.adjT + tb[j]) : 0u;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const bool tr = ok[j] && ((dout[j] == 1 && x[j] == v[j]) || (din[j] == 1 && y[j] == v[j]));
          if (tr) {
            s.label[v[j]] = v[j];
            ++ntrim;
          } else if (pick && ok[j]) {
            const unsigned long long key = ((unsigned long long)prio(g, rule, v[j]) << 32) | v[j];
            best = key < best ? key : best;
          }
          warp_set_bits(s.elim, v[j], tr, false);
          warp_set_bits(s.tflag, v[j], tr, false);
        }
      }
      npend = 0;
      __syncwarp();
    };
    uint32_t base = blockIdx.x * BS * 4u;
    const uint32_t wofs = (threadIdx.x >> 5) * 128u + lane * 4u;
    if (base >= lim) return 0;
    Quad cur_q = load(base + wofs);
    for (; base < lim; base += step) {
      const uint32_t v0 = base + wofs;
      // next iteration's offsets are in flight while this one is decided
      Quad nxt = cur_q;
      if (base + step < lim) nxt = load(base + step + wofs);
      const Quad &q = cur_q;
      uint32_t o4 = __shfl_down_sync(kFull, q.o[0], 1), t4 = __shfl_down_sync(kFull, q.t[0], 1);
      if (lane == 31) o4 = q.o4, t4 = q.t4;
      uint32_t bits = 0, amb = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const uint32_t v = v0 + i;
        const uint32_t dout = (i < 3 ? q.o[i + 1] : o4) - q.o[i];
        const uint32_t din = (i < 3 ? q.t[i + 1] : t4) - q.t[i];
        if (v < 1u || v > n) continue;
        if (dout == 0 || din == 0) {
          if (!vlab) s.label[v] = v;
          bits |= 1u << i;
          ++ntrim;
        } else if (dout == 1 || din == 1) {
          amb |= 1u << i;  // decided by the self-loop test
        } else if (pick) {
          const unsigned long long key = ((unsigned long long)prio(g, rule, v) << 32) | v;
          best = key < best ? key : best;
        }
      }
      if (vlab && v0 + 4u <= n + 1u) {
        // one 16-byte store of the four labels: whole sectors written, no
        // partial-sector merges in L2 (an id not trimmed here gets 0, and
        // its label is written when it is eliminated; ambiguous ids are
        // resolved below, after this store)
        const uint4 l = make_uint4((bits & 1u) ? v0 : 0u, (bits & 2u) ? v0 + 1u : 0u, (bits & 4u) ? v0 + 2u : 0u,
                                   (bits & 8u) ? v0 + 3u : 0u);
        *reinterpret_cast<uint4 *>(s.label + v0) = l;
      } else if (vlab) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((bits >> i) & 1u) s.label[v0 + i] = v0 + i;
      }
      // lanes 8j .. 8j+7 hold the 32 ids of word j of this warp's four
      const uint32_t grp = 0xffu << (lane & ~7u);
      const uint32_t word = __reduce_or_sync(grp, bits << (4u * (lane & 7u)));
      if ((lane & 7u) == 0 && word) {
        const uint32_t w = (v0 >> 5);
        atomicOr(s.elim + w, word);
        atomicOr(s.tflag + w, word);
      }
      // append this iteration's undecided ids (at most 128 per warp)
      const uint32_t na = __popc(amb);
      const uint32_t incl = warp_incl_scan(na);
      const uint32_t tot = __shfl_sync(kFull, incl, 31);
      if (npend + tot > kStage) resolve();
      uint32_t at = npend + incl - na;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if ((amb >> i) & 1u) pend[at++] = v0 + i;
      npend += tot;
      cur_q = nxt;
    }
    resolve();
    return ntrim;
  }

  __device__ __noinline__ uint32_t trim(bool ranged, bool snap, uint32_t max_it, bool pick = false) {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    const uint32_t rule = P.o.pivot_rule;
    unsigned long long t0 = globaltimer_ns();
    uint32_t ntrim = 0;
    unsigned long long best = ~0ull;
    if (snap && !ranged && max_it == 1 && !list_mode) {
      ntrim = trim_snap_sweep(pick, best);
      add_count(&c->n_trimmed, ntrim);
      if (pick) {
        best = block_min_u64(best);
        if (threadIdx.x == 0 && best != ~0ull) atomicMin(&c->best, best);
      }
      if (!bar(100)) return 1;
      prof(PR_TRIM_SWEEP, t0, 0);
      return 1;
    }
    Stage tq = stage_open(0, s.qa, cur() + C_Q, s.qcap);
    struct Pre {
      uint32_t ew, a0, a1, b0, b1;
    };
    // a word's elimination bits change only through its own warp in this sweep
    auto load = [&](uint32_t v, bool valid) {
      const uint32_t vv = valid ? v : 0u;
      return Pre{ldm(s.elim + (v >> 5)), ldg(g.off + vv), ldg(g.off + vv + 1), ldg(g.offT + vv),
                 ldg(g.offT + vv + 1)};
    };
    for_vertices_pf(load, [&](uint32_t v, bool valid, const Pre &p) {
      const uint32_t ew = p.ew;
      if (!list_mode && ~ew == 0u) return;  // whole word already eliminated
      const bool lv = valid && !((ew >> (v & 31u)) & 1u);
      const uint32_t a0 = p.a0, a1 = p.a1, b0 = p.b0, b1 = p.b1;
      bool t = false;
      if (lv) {
        if (snap) {  // nothing eliminated yet, lists sorted-unique: degrees decide
          const uint32_t dout = a1 - a0, din = b1 - b0;
          const uint32_t x = dout == 1 ? ldg(g.adj + a0) : 0u;
          const uint32_t y = din == 1 ? ldg(g.adjT + b0) : 0u;
          t = !(dout >= 2 || (dout == 1 && x != v)) || !(din >= 2 || (din == 1 && y != v));
        } else {
          const uint32_t rv = ranged ? ldm(s.range + v) : 0u;
          t = !live_nbr(s, g.off, g.adj, v, rv, ranged, false) || !live_nbr(s, g.offT, g.adjT, v, rv, ranged, false);
        }
        if (t) s.label[v] = v;
        if (pick && !t) {
          const unsigned long long key = ((unsigned long long)prio(g, rule, v) << 32) | v;
          best = key < best ? key : best;
        }
      }
      // neighbours can only lose their last partner if v has edges at all;
      // a single-iteration trim never reads the queue
      const bool q = max_it > 1 && t && (a1 != a0 || b1 != b0);
      warp_set_bits(s.tflag, v, t, !list_mode);
      warp_set_bits(s.elim, v, t, !list_mode);
      stage_put(tq, q, v);
      ntrim += t;
    });
    stage_flush(tq);
    add_count(&c->n_trimmed, ntrim);
    if (pick) {
      best = block_min_u64(best);
      if (threadIdx.x == 0 && best != ~0ull) atomicMin(&c->best, best);
    }
    if (!bar(100)) return 1;
    prof(PR_TRIM_SWEEP, t0, rdprv(C_Q));
    t0 = globaltimer_ns();
    uint32_t it = 1;
    uint32_t nq = rdprv(C_Q);
    if (a_trim && nq > 0 && it < max_it) {
      // the solve's range-aware trims: the worklist runs asynchronously
      ntrim = async_trim(nq, ranged);
      add_count(&c->n_trimmed, ntrim);
      if (!bar(103)) return 2;
      prof(PR_TRIM_WL, t0, 1);
      return 2;
    }
    while (nq > 0 && it < max_it) {
      // candidates: live partition-mates adjacent (either direction) to a vertex just trimmed
      for_items(nq, [&](uint32_t i, bool valid) {
        const uint32_t t = valid ? ldm(s.qa + i) : 0u;
        const uint32_t rt = (valid && ranged) ? ldm(s.range + t) : 0u;
        auto visit = [&](uint32_t, uint32_t u, uint32_t rtag) {
          if (!live(s, u)) return;
          if (ranged && ldm(s.range + u) != rtag) return;
          if (bit_claim(s.queued, u)) queue_push(s.qb, cur() + C_Q2, s.qcap, u, err());
        };
        uint32_t b = valid ? ldg(g.off + t) : 0u, d = valid ? ldg(g.off + t + 1) - b : 0u;
        warp_gather(t, b, d, rt, g.adj, visit);
        b = valid ? ldg(g.offT + t) : 0u;
        d = valid ? ldg(g.offT + t + 1) - b : 0u;
        warp_gather(t, b, d, rt, g.adjT, visit);
      });
      if (!bar(101)) return it;
      const uint32_t nc = rdprv(C_Q2);
      ntrim = 0;
      for_items(nc, [&](uint32_t i, bool valid) {
        bool t = false;
        uint32_t u = 0;
        if (valid) {
          u = ldm(s.qb + i);
          bit_clear(s.queued, u);
          if (live(s, u)) {
            const uint32_t ru = ranged ? ldm(s.range + u) : 0u;
            t = !live_nbr(s, g.off, g.adj, u, ru, ranged, false) || !live_nbr(s, g.offT, g.adjT, u, ru, ranged, false);
            if (t) s.label[u] = u;
          }
        }
        warp_set_bits(s.tflag, u, t, false);
        warp_set_bits(s.elim, u, t, false);
        warp_push(s.qa, cur() + C_Q, s.qcap, u, t, err());
        ntrim += t;
      });
      add_count(&c->n_trimmed, ntrim);
      if (!bar(102)) return it;
      nq = rdprv(C_Q);
      ++it;
    }
    if (it > 1) prof(PR_TRIM_WL, t0, it - 1);
    return it;
  }

  // ===================================================== first pivot (a3)
  // scc.cu:234-253: after the first trim the pivot is the first vertex that
  // is not eliminated (or, with SCC_PIVOT_MAX_DEGREE, the one with the
  // largest in x out degree).  Single partition only.
  __device__ __noinline__ uint32_t pick_first_pivot() {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    const uint32_t rule = P.o.pivot_rule;
    unsigned long long best = ~0ull;
    for_vertices([&](uint32_t v, bool valid) {
      if (valid && live(s, v)) {
        const unsigned long long key = ((unsigned long long)prio(g, rule, v) << 32) | v;
        best = key < best ? key : best;
      }
    });
    best = block_min_u64(best);
    if (threadIdx.x == 0 && best != ~0ull) atomicMin(&c->best, best);
    if (!bar(200)) return 0;
    return commit_first_pivot();
  }
  // c->best holds the elected (priority, id) key; make it the pivot
  __device__ __forceinline__ uint32_t commit_first_pivot() {
    const unsigned long long b = ldm64(&c->best);
    const uint32_t p = b == ~0ull ? 0u : (uint32_t)b;
    // c->best is reset by the lead after the next barrier (everyone has read it by then)
    if (is_lead()) {
      if (p) {
        P.s.rpivot[0] = p;
        P.s.sccsize[p] = 0u;
        P.s.piv[0] = p;
        bit_set(P.s.fvis, p);
        bit_set(P.s.bvis, p);
      }
      c->piv_count = p ? 1u : 0u;
    }
    if (!bar(201)) return 0;
    if (is_lead()) c->best = ~0ull;
    return p;
  }

  // ======================================================== update (a13)
  // scc_routines.cu:147-224: F∩B -> SCC of the partition's pivot; every other
  // live vertex moves to partition (range, F, B); one pivot per non-empty new
  // partition (smallest (priority, id)), which starts visited both ways.
  // Also used for the first election when the graph is segmented (F = B = 0).
  __device__ __noinline__ void update() {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    const uint32_t rule = P.o.pivot_rule;
    __shared__ uint32_t s_key[kSlotCache];
    __shared__ unsigned long long s_val[kSlotCache];
    __shared__ uint32_t s_szkey[kSizeCache], s_szcnt[kSizeCache];
    for (int i = threadIdx.x; i < kSlotCache; i += BS) {
      s_key[i] = kNone;
      s_val[i] = ~0ull;
    }
    for (int i = threadIdx.x; i < kSizeCache; i += BS) {
      s_szkey[i] = kNone;
      s_szcnt[i] = 0u;
    }
    __syncthreads();
    uint32_t nelim = 0, nfound = 0;
    // per-vertex words and the partition id, loaded one iteration ahead (only
    // v's own lane changes v's bits and range during either sweep)
    struct Pre {
      uint32_t ew, fw, bw, r;
    };
    auto load = [&](uint32_t v, bool valid) {
      const uint32_t w = v >> 5;
      return Pre{ldm(s.elim + w), ldm(s.fvis + w), ldm(s.bvis + w), ldm(s.range + (valid ? v : 0u))};
    };
    // A: eliminate F∩B, elect pivots (CTA-local min per key, flushed below).
    // A partition id is its pivot's id (rpivot[r] == r) once pivots have been
    // elected; only the first round of a single partition still runs under
    // id 0, whose pivot is rpivot[0] -- so no per-vertex rpivot load.
    const uint32_t p0 = ldm(s.rpivot);
    for_vertices_pf(load, [&](uint32_t v, bool valid, const Pre &pre) {
      const uint32_t ew = pre.ew, fw = pre.fw, bw = pre.bw;
      if (!list_mode && ~ew == 0u) return;  // whole word already eliminated
      const uint32_t r = pre.r;
      uint32_t key = kNone;
      unsigned long long val = ~0ull;
      bool fb = false;
      uint32_t p = kNone;
      if (valid && !((ew >> (v & 31u)) & 1u)) {
        const bool f = (fw >> (v & 31u)) & 1u, b = (bw >> (v & 31u)) & 1u;
        if (f && b) {
          p = r ? r : p0;
          s.label[v] = p;
          fb = true;
          ++nelim;
          nfound += p == v;  // one SCC per eliminated pivot
        } else {
          key = 3u * r + (f ? 1u : 0u) + (b ? 2u : 0u);
          val = ((unsigned long long)prio(g, rule, v) << 32) | v;
        }
      }
      warp_set_bits(s.elim, v, fb, !list_mode);
      {  // SCC sizes: the warp's members of one component counted together
        const uint32_t pg = __match_any_sync(kFull, p);
        if (fb && lane_id() == (uint32_t)(__ffs(pg) - 1)) size_add(s, s_szkey, s_szcnt, p, __popc(pg));
      }
      const uint32_t grp = __match_any_sync(kFull, key);
      if (key != kNone) {
        const uint32_t hi = (uint32_t)(val >> 32), lo = (uint32_t)val;
        const uint32_t mhi = __reduce_min_sync(grp, hi);
        const uint32_t mlo = __reduce_min_sync(grp, hi == mhi ? lo : kNone);
        if (lane_id() == (uint32_t)(__ffs(grp) - 1)) {
          const unsigned long long m = ((unsigned long long)mhi << 32) | mlo;
          const uint32_t h = key % kSlotCache;
          uint32_t owner = s_key[h];
          if (owner == kNone) owner = atomicCAS(&s_key[h], kNone, key) == kNone ? key : s_key[h];
          if (owner == key) {
            atomicMin(&s_val[h], m);
          } else if (ldm64(s.slot + key) > m) {
            atomicMin(s.slot + key, m);
          }
        }
      }
    });
    __syncthreads();
    for (int i = threadIdx.x; i < kSlotCache; i += BS) {
      const uint32_t key = s_key[i];
      if (key != kNone && ldm64(s.slot + key) > s_val[i]) atomicMin(s.slot + key, s_val[i]);
    }
    for (int i = threadIdx.x; i < kSizeCache; i += BS)
      if (s_szkey[i] != kNone) size_flush(s, s_szkey[i], s_szcnt[i]);
    add_count(&c->n_fbe, nelim);
    add_count(&c->n_fbscc, nfound);
    if (!bar(300)) return;
    // B: new partition id = elected pivot; pivots go to the pivot list
    __shared__ unsigned long long s_hit[kSlotCache];  // (key << 32) | pivot
    for (int i = threadIdx.x; i < kSlotCache; i += BS) s_hit[i] = ~0ull;
    __syncthreads();
    for_vertices_pf(load, [&](uint32_t v, bool valid, const Pre &pre) {
      bool is_piv = false;
      uint32_t key = 0;
      const uint32_t bit = 1u << (v & 31u);
      if (valid && !(pre.ew & bit)) {
        const bool f = pre.fw & bit, b = pre.bw & bit;
        key = 3u * pre.r + (f ? 1u : 0u) + (b ? 2u : 0u);
        const uint32_t h = key % kSlotCache;
        const unsigned long long cached = s_hit[h];
        uint32_t np;
        if ((uint32_t)(cached >> 32) == key) {
          np = (uint32_t)cached;
        } else {
          np = (uint32_t)ldm64(s.slot + key);
          s_hit[h] = ((unsigned long long)key << 32) | np;
        }
        s.range[v] = np;
        is_piv = np == v;
      }
      const uint32_t mask = __ballot_sync(kFull, is_piv);
      if (mask) {
        const uint32_t leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if (lane_id() == leader) base = atomicAdd(cur() + C_Q, __popc(mask));
        base = __shfl_sync(kFull, base, leader);
        if (is_piv) {
          const uint32_t slot_i = base + __popc(mask & lanemask_lt());
          s.piv[slot_i] = v;
          s.pivkey[slot_i] = key;
        }
      }
    });
    if (!bar(301)) return;
    const uint32_t np = rdprv(C_Q);
    // C: release the election slots, clear the visit bitmaps
    for_items(np, [&](uint32_t i, bool valid) {
      if (valid) s.slot[ldm(s.pivkey + i)] = ~0ull;
    });
    for (uint32_t w = gtid(); w < s.nwords; w += gstride()) {
      s.fvis[w] = 0u;
      s.bvis[w] = 0u;
      s.fexp[w] = 0u;
      s.bexp[w] = 0u;
    }
    if (is_lead()) c->piv_count = np;
    if (!bar(302)) return;
    // D: pivots start F and B visited (state 19)
    for_items(np, [&](uint32_t i, bool valid) {
      if (valid) {
        const uint32_t p = ldm(s.piv + i);
        s.rpivot[p] = p;
        s.sccsize[p] = 0u;
        bit_set(s.fvis, p);
        bit_set(s.bvis, p);
      }
    });
    bar(303);
  }

  // scc_routines.cu:10-19 unsetPivots: the pivots of the last election stop
  // being pivots (their visit bits go), used right before WCC.
  __device__ __forceinline__ void unset_pivots() {
    const EngState &s = P.s;
    for (uint32_t w = gtid(); w < s.nwords; w += gstride()) {
      s.fvis[w] = 0u;
      s.bvis[w] = 0u;
      s.fexp[w] = 0u;
      s.bexp[w] = 0u;
    }
    if (is_lead()) c->piv_count = 0;
    bar(400);
  }

  // ======================================================== reach (a8-a11)
  // Visit predicate shared by every arm: u joins the visited set of the
  // current direction when it is live, in the source's partition (unless
  // first step) and not visited yet; exactly one caller wins the claim.
  __device__ __forceinline__ static bool try_visit(const EngState &s, uint32_t *vis, uint32_t u, bool ranged, uint32_t rsrc) {
    const uint32_t w = u >> 5, b = 1u << (u & 31u);
    const uint32_t vw = ldm(vis + w);      // both bitmap words are requested
    const uint32_t ew = ldm(s.elim + w);   // before either is tested
    if ((vw | ew) & b) return false;
    if (ranged && ldm(s.range + u) != rsrc) return false;
    return !(atomicOr(vis + w, b) & b);
  }
  // try_visit that requests u's partition id and (want_deg) u's offsets
  // together with the bitmap words: one round trip before the claim instead
  // of up to three, for levels bound by latency rather than by bytes
  __device__ __forceinline__ static bool try_visit_wide(const EngState &s, const uint32_t *__restrict__ off, uint32_t *vis,
                                                        uint32_t u, bool ranged, uint32_t rsrc, bool want_deg,
                                                        uint32_t &deg) {
    const uint32_t w = u >> 5, b = 1u << (u & 31u);
    const uint32_t vw = ldm(vis + w), ew = ldm(s.elim + w);
    const uint32_t rg = ranged ? ldm(s.range + u) : rsrc;
    const uint32_t o0 = want_deg ? ldg(off + u) : 0u, o1 = want_deg ? ldg(off + u + 1) : 0u;
    deg = o1 - o0;
    if (((vw | ew) & b) || rg != rsrc) return false;
    return !(atomicOr(vis + w, b) & b);
  }

  // Pull test: does adj[b, e) hold a visited partition-mate?  Lists are read
  // four entries at a time (one 16-byte load once aligned) and the four
  // bitmap words are requested together, so a thread keeps several
  // independent L2 requests in flight instead of one dependent chain.
  // wide: eight probes per step on unranged tests (more loads in flight per
  // thread, but up to seven wasted bitmap lines when an early entry hits;
  // callers that keep many candidates in flight pass false)
  __device__ __forceinline__ static bool any_visited(const EngState &s, uint32_t m, const uint32_t *__restrict__ adj, uint32_t b,
                                     uint32_t e, const uint32_t *vis, bool ranged, uint32_t rv, bool wide = true) {
    const uint32_t *rng = s.range;
    auto hit = [&](uint32_t u) {
      return ((ldm(vis + (u >> 5)) >> (u & 31u)) & 1u) && (!ranged || ldm(rng + u) == rv);
    };
    uint32_t i = b;
    // 16-byte loads only when the list base is 16-byte aligned (caller-bound
    // graphs may not be); otherwise the scalar tail loop below does it all
    const bool vec = (reinterpret_cast<uintptr_t>(adj) & 15u) == 0;
    if (vec && i < e && (i & 3u)) {
      // the aligned 16 bytes holding the list head (entries of the previous
      // list masked off) instead of up to three dependent scalar probes
      const uint32_t a = i & ~3u;
      if ((unsigned long long)a + 4ull <= m) {
        const uint4 q = __ldg(reinterpret_cast<const uint4 *>(adj + a));
        const uint32_t u[4] = {q.x, q.y, q.z, q.w};
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = (a + j >= i && a + j < e) ? ldm(vis + (u[j] >> 5)) : 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (((w[j] >> (u[j] & 31u)) & 1u) && (!ranged || ldm(rng + u[j]) == rv)) return true;
        i = a + 4u;
      } else {
        while (i < e && (i & 3u)) {
          if (hit(ldg(adj + i))) return true;
          ++i;
        }
      }
    }
    if (!ranged && wide) {  // eight probes in flight per step
      for (; vec && i + 8 <= e; i += 8) {
        const uint4 q = __ldg(reinterpret_cast<const uint4 *>(adj + i));
        const uint4 r = __ldg(reinterpret_cast<const uint4 *>(adj + i + 4));
        const uint32_t w0 = ldm(vis + (q.x >> 5)), w1 = ldm(vis + (q.y >> 5));
        const uint32_t w2 = ldm(vis + (q.z >> 5)), w3 = ldm(vis + (q.w >> 5));
        const uint32_t w4 = ldm(vis + (r.x >> 5)), w5 = ldm(vis + (r.y >> 5));
        const uint32_t w6 = ldm(vis + (r.z >> 5)), w7 = ldm(vis + (r.w >> 5));
        const uint32_t h = ((w0 >> (q.x & 31u)) | (w1 >> (q.y & 31u)) | (w2 >> (q.z & 31u)) | (w3 >> (q.w & 31u)) |
                            (w4 >> (r.x & 31u)) | (w5 >> (r.y & 31u)) | (w6 >> (r.z & 31u)) | (w7 >> (r.w & 31u))) &
                           1u;
        if (h) return true;
      }
    }
    for (; vec && i + 4 <= e; i += 4) {
      const uint4 q = __ldg(reinterpret_cast<const uint4 *>(adj + i));
      const uint32_t w0 = ldm(vis + (q.x >> 5)), w1 = ldm(vis + (q.y >> 5));
      const uint32_t w2 = ldm(vis + (q.z >> 5)), w3 = ldm(vis + (q.w >> 5));
      const bool h0 = (w0 >> (q.x & 31u)) & 1u, h1 = (w1 >> (q.y & 31u)) & 1u;
      const bool h2 = (w2 >> (q.z & 31u)) & 1u, h3 = (w3 >> (q.w & 31u)) & 1u;
      if (!ranged) {
        if (h0 | h1 | h2 | h3) return true;
      } else {
        if ((h0 && ldm(rng + q.x) == rv) || (h1 && ldm(rng + q.y) == rv) || (h2 && ldm(rng + q.z) == rv) ||
            (h3 && ldm(rng + q.w) == rv))
          return true;
      }
    }
    for (; i < e; ++i)
      if (hit(ldg(adj + i))) return true;
    return false;
  }

  // QUADRATIC (reach_q.cu:12-79,160-231): every sweep expands each visited,
  // not yet expanded vertex, one thread per vertex.
  __device__ __noinline__ uint32_t reach_q(const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj, uint32_t *vis,
                              uint32_t *exp, bool ranged) {
    const EngState &s = P.s;
    const uint32_t heavy = P.o.heavy_degree;
    uint32_t depth = 0;
    for (;;) {
      const unsigned long long ts = globaltimer_ns();
      uint32_t chg = 0;
      auto visit = [&](uint32_t, uint32_t u, uint32_t rsrc) { chg += try_visit(s, vis, u, ranged, rsrc); };
      for_vertices([&](uint32_t v, bool valid) {
        // No warp-level "skip this word" shortcut here: visit bits change
        // under other warps during the sweep, so such a test would not be
        // warp-uniform.  The lists of this sweep's frontier vertices are
        // walked by the whole warp (warp_gather); a list longer than
        // heavy_degree goes to the grid (one hub's list would otherwise keep
        // a single thread busy for the whole sweep).
        const bool fr = valid && live(s, v) && bit_test(vis, v) && !bit_test(exp, v);
        warp_set_bits(exp, v, fr, !list_mode);
        uint32_t b = 0, d = 0, rv = 0;
        if (fr) {
          rv = ranged ? ldm(s.range + v) : 0u;
          b = ldg(off + v);
          d = ldg(off + v + 1) - b;
          if (d > heavy) {
            heavy_push(s, v, b, d, rv);
            d = 0;
          }
        }
        warp_gather(v, b, d, rv, adj, visit);
      });
      add_count(cur() + C_CHG, chg);
      if (!bar(500)) return depth;
      const unsigned long long h = ldm64(prv64());
      if ((uint32_t)(h >> 32) != 0) {
        if (is_lead()) atomicAdd(cur() + C_CHG, rdprv(C_CHG));
        chg = 0;
        heavy_expand(s, adj, h, visit);
        add_count(cur() + C_CHG, chg);
        if (!bar(501)) return depth;
      }
      prof(PR_Q, ts, rdprv(C_CHG));
      ++depth;
      if (rdprv(C_CHG) == 0) break;
      if (depth >= P.o.max_iters) {
        fail(kErrIterCap);
        break;
      }
    }
    return depth;
  }

  // Edges of lists longer than heavy_degree, collected during a push sweep
  // and expanded afterwards by the whole grid in 256-edge chunks.
  __device__ __forceinline__ void heavy_push(const EngState &s, uint32_t v, uint32_t beg, uint32_t deg, uint32_t tag) {
    const unsigned long long old = atomicAdd(cur64(), (1ull << 32) | deg);
    const uint32_t idx = (uint32_t)(old >> 32);
    if (idx >= s.hcap) {
      fail(kErrQueueOverflow);
      return;
    }
    s.hv[idx] = v;
    s.hbeg[idx] = beg;
    s.hdeg[idx] = deg;
    s.htag[idx] = tag;
    s.hbase[idx] = (uint32_t)old;
  }

  // heavy_expand for whole-warp visitors: visit(src, dst, tag, valid) on all
  // lanes at every step (valid = false past the end).
  template <class Visit>
  __device__ __forceinline__ void heavy_expand_all(const EngState &s, const uint32_t *__restrict__ adj, unsigned long long h,
                                   Visit &&visit) {
    const uint32_t cnt = (uint32_t)(h >> 32), tot = (uint32_t)h;
    if (cnt == 0 || cnt > s.hcap) return;  // overflow already flagged by heavy_push
    const uint32_t lane = lane_id();
    for (uint32_t chunk = gwarp(); (unsigned long long)chunk * 256ull < tot; chunk += nwarps()) {
      const uint32_t e0 = chunk * 256u;
      uint32_t j = 0;
      if (lane == 0) {  // largest j with hbase[j] <= e0
        uint32_t lo = 0, hi = cnt - 1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (ldm(s.hbase + mid) <= e0) lo = mid;
          else hi = mid - 1;
        }
        j = lo;
      }
      j = __shfl_sync(kFull, j, 0);
      for (uint32_t sft = 0; sft < 256u; sft += 32u) {
        if (e0 + sft >= tot) break;
        const uint32_t e = e0 + sft + lane;
        const bool valid = e < tot;
        uint32_t src = 0, dst = 0, tag = 0;
        if (valid) {
          uint32_t jj = j;
          while (jj + 1 < cnt && ldm(s.hbase + jj + 1) <= e) ++jj;
          dst = ldg(adj + ldm(s.hbeg + jj) + (e - ldm(s.hbase + jj)));
          src = ldm(s.hv + jj);
          tag = ldm(s.htag + jj);
        }
        visit(src, dst, tag, valid);
      }
    }
  }

  template <class Visit>
  __device__ __forceinline__ void heavy_expand(const EngState &s, const uint32_t *__restrict__ adj, unsigned long long h,
                               Visit &&visit) {
    const uint32_t cnt = (uint32_t)(h >> 32), tot = (uint32_t)h;
    if (cnt == 0 || cnt > s.hcap) return;  // overflow already flagged by heavy_push
    const uint32_t lane = lane_id();
    for (uint32_t chunk = gwarp(); (unsigned long long)chunk * 256ull < tot; chunk += nwarps()) {
      const uint32_t e0 = chunk * 256u;
      uint32_t j = 0;
      if (lane == 0) {  // largest j with hbase[j] <= e0
        uint32_t lo = 0, hi = cnt - 1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (ldm(s.hbase + mid) <= e0) lo = mid;
          else hi = mid - 1;
        }
        j = lo;
      }
      j = __shfl_sync(kFull, j, 0);
      for (uint32_t sft = 0; sft < 256u; sft += 32u) {
        const uint32_t e = e0 + sft + lane;
        if (e0 + sft >= tot) break;
        if (e < tot) {
          uint32_t jj = j;
          while (jj + 1 < cnt && ldm(s.hbase + jj + 1) <= e) ++jj;
          const uint32_t dst = ldg(adj + ldm(s.hbeg + jj) + (e - ldm(s.hbase + jj)));
          visit(ldm(s.hv + jj), dst, ldm(s.htag + jj));
        }
      }
    }
  }

  // Push levels run by CTA 0 alone while the frontier stays small (high-
  // diameter graphs spend hundreds of levels on a few dozen vertices each,
  // where a grid barrier per level costs more than the level).  Same visit
  // rule as the grid levels; the next frontier goes to the other queue
  // through a shared-memory counter.  Results land in the counters C_L*.
  // The frontier's edges are checked first: too many and nothing is done
  // (C_LREF = 1), the grid expands that level instead.
  // CTA-wide exclusive scan of x (every thread calls); the total goes to `tot`.
  __device__ __forceinline__ static uint32_t block_excl_scan(uint32_t x, uint32_t &tot) {
    __shared__ uint32_t s_w[BS / 32 + 1];
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_scan(x);
    if (lane == 31) s_w[w] = incl;
    __syncthreads();
    if (w == 0) {
      const uint32_t t = lane < BS / 32 ? s_w[lane] : 0u;
      const uint32_t ti = warp_incl_scan(t);
      if (lane < BS / 32) s_w[lane] = ti - t;
      if (lane == 31) s_w[BS / 32] = ti;
    }
    __syncthreads();
    tot = s_w[BS / 32];
    const uint32_t r = s_w[w] + incl - x;
    __syncthreads();
    return r;
  }

  // Levels of a small frontier expanded by this CTA alone (CTA 0, between
  // two grid barriers), CTA barriers between levels.  A level's edges are
  // spread over all threads of the CTA, whatever the lists' lengths (a
  // pivot's list of thousands of edges takes a few steps of the CTA, not
  // thousands / 32 steps of one warp): the frontier is taken BS sources at a
  // time, their degrees scanned into a shared-memory table, and every thread
  // then takes edges e, e + BS, ... of the chunk, four per step, finding each
  // edge's source by binary search in the table.  The bitmap words, the
  // partition id and the offsets of the four targets are requested together,
  // so a step costs three dependent round trips (list entry, tests, claim).
  // Results for the level driver go to cur()[C_L*]; C_LREF = 1 when the
  // frontier's edges exceed kLocalEdges (nothing done).
  __device__ __noinline__ void local_levels(const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj, uint32_t *vis,
                               bool ranged, const uint32_t *in, uint32_t nin, uint32_t sel, uint32_t max_levels,
                               uint32_t stop_at) {
    const EngState &s = P.s;
    __shared__ uint32_t s_cnt, s_deg;
    // source table of the current chunk, in the staging segments (no stage
    // is open in this CTA between the grid barriers around this call)
    uint32_t *const s_base = stage_mem();  // adjacency index of a chunk edge = s_base[src] + edge
    uint32_t *const s_ex = s_base + BS;    // first chunk edge of each source
    uint32_t *const s_rv = s_base + 2 * BS;
    uint32_t d = 0;
    for (uint32_t i = threadIdx.x; i < nin; i += BS) {
      const uint32_t v = ldm(in + i);
      d += ldg(off + v + 1) - ldg(off + v);
    }
    d = block_sum(d);
    if (threadIdx.x == 0) s_deg = d;
    __syncthreads();
    uint32_t lmf = s_deg;
    __syncthreads();
    if (lmf > kLocalEdges) {
      if (threadIdx.x == 0) cur()[C_LREF] = 1u;
      return;
    }
    uint32_t lnin = nin, ld = 0, lsel = sel, lex = 0;
    const uint32_t *lin = in;
    const uint32_t qcap = s.qcap;
    while (lnin > 0 && ld < max_levels) {
      uint32_t *lout = lsel ? s.qb : s.qa;
      if (threadIdx.x == 0) {
        s_cnt = 0;
        s_deg = 0;
      }
      // (the scan's barriers order these writes before any use)
      uint32_t degsum = 0;
      for (uint32_t base = 0; base < lnin; base += BS) {
        const uint32_t i = base + threadIdx.x;
        uint32_t v = 0, b = 0, dd = 0, rv = 0;
        if (i < lnin) {
          v = ldm(lin + i);
          b = ldg(off + v);
          dd = ldg(off + v + 1) - b;
          rv = ranged ? ldm(s.range + v) : 0u;
        }
        uint32_t tot;
        const uint32_t ex = block_excl_scan(dd, tot);
        s_base[threadIdx.x] = b - ex;
        s_ex[threadIdx.x] = ex;
        s_rv[threadIdx.x] = rv;
        __syncthreads();
        const uint32_t nsrc = lnin - base < (uint32_t)BS ? lnin - base : (uint32_t)BS;
        for (uint32_t e0 = threadIdx.x; e0 < tot; e0 += 4u * BS) {
          uint32_t u[4], r[4];
          bool ok[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t e = e0 + (uint32_t)j * BS;
            ok[j] = e < tot;
            // largest source index whose first edge is <= e (sources without
            // edges share their successor's first edge and are skipped)
            uint32_t lo = 0, hi = nsrc;
            while (hi - lo > 1u) {
              const uint32_t mid = (lo + hi) >> 1;
              if (s_ex[mid] <= e) lo = mid;
              else hi = mid;
            }
            // u32 sum first: s_base holds list start - first chunk edge, modulo 2^32
            u[j] = ok[j] ? ldg(adj + (s_base[lo] + e)) : 0u;
            r[j] = s_rv[lo];
          }
          uint32_t vw[4], ew[4], rg[4], o0[4], o1[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t w = u[j] >> 5;
            vw[j] = ok[j] ? ldm(vis + w) : ~0u;
            ew[j] = ok[j] ? ldm(s.elim + w) : ~0u;
            rg[j] = ok[j] && ranged ? ldm(s.range + u[j]) : 0u;
            o0[j] = ok[j] ? ldg(off + u[j]) : 0u;
            o1[j] = ok[j] ? ldg(off + u[j] + 1) : 0u;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t bit = 1u << (u[j] & 31u);
            const bool cand = !((vw[j] | ew[j]) & bit) && (!ranged || rg[j] == r[j]);
            if (cand && !(atomicOr(vis + (u[j] >> 5), bit) & bit)) {
              const uint32_t pos = atomicAdd(&s_cnt, 1u);
              if (pos < qcap) lout[pos] = u[j];
              else fail(kErrQueueOverflow);
              degsum += o1[j] - o0[j];
            }
          }
        }
        __syncthreads();  // the table is rewritten by the next chunk
      }
      degsum = __reduce_add_sync(kFull, degsum);
      if (lane_id() == 0 && degsum) atomicAdd(&s_deg, degsum);
      __syncthreads();
      lnin = s_cnt;
      lmf = s_deg;
      lex += lmf;
      ++ld;
      lin = lout;
      lsel ^= 1u;
      __syncthreads();
      if (lnin > kLocalMax || lmf > kLocalEdges || lnin >= stop_at) break;
    }
    if (threadIdx.x == 0) {
      uint32_t *o = cur();
      o[C_LN] = lnin;
      o[C_LSEL] = lsel;
      o[C_LD] = ld;
      o[C_LMF] = lmf;
      o[C_LEX] = lex;
    }
  }

  // One pull sweep: every candidate (the vertices of `lst[0, lcnt)`, or
  // every id when lst is null) that is live and not yet visited looks for a
  // visited partition-mate among its reverse neighbours (poff / padj).  Found
  // vertices are marked visited and appended to `out` (counter cur()[C_Q]);
  // candidates not found go to `rem_out` (cur()[C_REM]); the found vertices'
  // reverse degrees are summed into cur()[C_DEG].  Runs as its own function
  // so the level driver's state does not take registers from the sweep.
  template <bool ranged>
  __device__ __noinline__ void pull_sweep(const uint32_t *__restrict__ poff, const uint32_t *__restrict__ padj,
                                          uint32_t *vis, const uint32_t *lst, uint32_t lcnt, uint32_t *out,
                                          uint32_t *rem_out, bool head_only) {
    const EngState &s = P.s;
    uint32_t degsum = 0;
    Stage pq = stage_open(0, out, cur() + C_Q, s.qcap);
    Stage rq = stage_open(1, rem_out, cur() + C_REM, s.qcap);
    struct Pre {
      uint32_t vw, ew, pb, pe, rv;
    };
    // Only v's own lane sets v's visit bit during a pull sweep, so the
    // prefetched word is current for the bit this lane tests.  The
    // frontier's edge count (for the direction heuristics) is taken from
    // the reverse lists already loaded: in-degree stands in for
    // out-degree, saving a random read of the other offsets per vertex.
    auto load = [&](uint32_t v, bool valid) {
      const uint32_t w = v >> 5, vv = valid ? v : 0u;
      return Pre{ldm(vis + w), ldm(s.elim + w), ldg(poff + vv), ldg(poff + vv + 1),
                 ranged ? ldm(s.range + vv) : 0u};
    };
    // Every lane's test starts with the aligned 16 bytes holding its list
    // head; only entries of the list itself are probed (those 16 bytes
    // also hold entries of the neighbouring lists, and these sweeps pay
    // per distinct cache line their scattered loads touch).
    const bool vec = (reinterpret_cast<uintptr_t>(padj) & 15u) == 0;
    const uint32_t m = P.g.m;
    auto head = [&](const Pre &p, bool cand, uint4 &q) {
      const uint32_t a = p.pb & ~3u;  // a <= pb < pe <= m: m - a does not wrap
      const bool h = vec && cand && p.pe > p.pb && m - a >= 4u;
      q = h ? __ldg(reinterpret_cast<const uint4 *>(padj + a)) : make_uint4(0u, 0u, 0u, 0u);
      return h;
    };
    auto probe_head = [&](const Pre &p, const uint4 &q, bool h, uint32_t (&w)[4]) {
      const uint32_t a = p.pb & ~3u;
      const uint32_t u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) w[j] = (h && a + j >= p.pb && a + j < p.pe) ? ldm(vis + (u[j] >> 5)) : 0u;
    };
    auto head_hit = [&](const Pre &p, const uint4 &q, const uint32_t (&w)[4]) {
      const uint32_t a = p.pb & ~3u;
      const uint32_t u[4] = {q.x, q.y, q.z, q.w};
      bool hit = false;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (a + j >= p.pb && a + j < p.pe && ((w[j] >> (u[j] & 31u)) & 1u) && (!ranged || ldm(s.range + u[j]) == p.rv))
          hit = true;
      return hit;
    };
    // rest of the list after the head: not in a heads-only sweep (unless
    // the head could not be read, e.g. unaligned adjacency)
    auto rest = [&](const Pre &p, bool cand, bool h) {
      if (!cand || (head_only && h)) return false;
      return any_visited(s, m, padj, h ? (p.pb & ~3u) + 4u : p.pb, p.pe, vis, ranged, p.rv, false);
    };
    if (lst) {
      // two vertices per thread: both heads' loads, then both heads'
      // probes, are issued together
      for_list_pairs_pf(lst, lcnt, load,
                        [&](uint32_t va, bool vla, const Pre &pa, uint32_t vb, bool vlb, const Pre &pb) {
                          const bool ca = vla && !(((pa.vw | pa.ew) >> (va & 31u)) & 1u);
                          const bool cb = vlb && !(((pb.vw | pb.ew) >> (vb & 31u)) & 1u);
                          uint4 qa, qb;
                          const bool ha = head(pa, ca, qa), hb = head(pb, cb, qb);
                          uint32_t wa[4], wb[4];
                          probe_head(pa, qa, ha, wa);
                          probe_head(pb, qb, hb, wb);
                          bool fa = ha && head_hit(pa, qa, wa);
                          bool fb = hb && head_hit(pb, qb, wb);
                          if (!fa) fa = rest(pa, ca, ha);
                          if (!fb) fb = rest(pb, cb, hb);
                          if (fa) degsum += pa.pe - pa.pb;
                          if (fb) degsum += pb.pe - pb.pb;
                          warp_set_bits(vis, va, fa, false);
                          warp_set_bits(vis, vb, fb, false);
                          stage_put(pq, fa, va);
                          stage_put(pq, fb, vb);
                          stage_put(rq, ca && !fa, va);
                          stage_put(rq, cb && !fb, vb);
                        });
    } else {
      // every id; a warp covers one bitmap word and skips words without a
      // live unvisited vertex
      for_vertices_pf(load, [&](uint32_t v, bool valid, const Pre &p) {
        if ((~p.vw & ~p.ew) == 0u) return;
        const bool cand = valid && !(((p.vw | p.ew) >> (v & 31u)) & 1u);
        uint4 q;
        uint32_t w[4];
        const bool h = head(p, cand, q);
        probe_head(p, q, h, w);
        bool found = h && head_hit(p, q, w);
        if (!found) found = rest(p, cand, h);
        if (found) degsum += p.pe - p.pb;
        warp_set_bits(vis, v, found, true);
        stage_put(pq, found, v);
        stage_put(rq, cand && !found, v);
      });
    }
    stage_flush(pq);
    stage_flush(rq);
    add_count(cur() + C_DEG, degsum);
  }

  // One push level of the LINEAR / TOPO / BEST arms: the frontier in[0, nin)
  // expands its lists warp-wide; newly reached vertices are appended to
  // `out` through warp-staged segments (one global atomic per 224 items).
  // Lists longer than `split` go to the grid-wide heavy list, expanded after
  // a barrier in 256-edge chunks.  Returns false if a barrier failed; qoff
  // receives the items the first interval appended (the heavy interval's
  // count is in prv()[C_Q]); C_DEG sums the reached vertices' out-degrees
  // when count_deg.
  __device__ __noinline__ bool push_level(const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                          uint32_t *vis, bool ranged, bool count_deg, const uint32_t *in,
                                          uint32_t nin, uint32_t *out, uint32_t split, uint32_t &qoff, bool wide) {
    const EngState &s = P.s;
    uint32_t degsum = 0;
    qoff = 0;
    // frontiers of short lists are latency-bound: their targets' tests and
    // offsets are requested in one round trip (wide; for long lists the
    // extra loads of targets already visited cost more than they save)
    auto claim = [&](uint32_t u, uint32_t rsrc, bool valid) {
      if (wide) {
        uint32_t dg = 0;
        const bool claimed = valid && try_visit_wide(s, off, vis, u, ranged, rsrc, count_deg, dg);
        if (claimed) degsum += dg;
        return claimed;
      }
      const bool claimed = valid && try_visit(s, vis, u, ranged, rsrc);
      if (claimed && count_deg) degsum += ldg(off + u + 1) - ldg(off + u);
      return claimed;
    };
    {
      Stage fq = stage_open(0, out, cur() + C_Q, s.qcap);
      auto visit_all = [&](uint32_t, uint32_t u, uint32_t rsrc, bool valid) { stage_put(fq, claim(u, rsrc, valid), u); };
      for_items(nin, [&](uint32_t i, bool valid) {
        uint32_t v = 0, b = 0, d = 0, rv = 0;
        if (valid) {
          v = ldm(in + i);
          b = ldg(off + v);
          d = ldg(off + v + 1) - b;
          rv = ranged ? ldm(s.range + v) : 0u;
          if (d > split) {
            heavy_push(s, v, b, d, rv);
            d = 0;
          }
        }
        warp_gather_all(v, b, d, rv, adj, visit_all);
      });
      stage_flush(fq);
    }
    add_count(cur() + C_DEG, degsum);
    if (!bar(700)) return false;
    const unsigned long long h = ldm64(prv64());
    if ((uint32_t)(h >> 32) != 0) {
      const unsigned long long th = globaltimer_ns();
      qoff = rdprv(C_Q);
      if (is_lead()) atomicAdd(cur() + C_DEG, rdprv(C_DEG));
      degsum = 0;
      Stage hq = stage_open(0, out + qoff, cur() + C_Q, s.qcap - qoff);
      heavy_expand_all(s, adj, h, [&](uint32_t, uint32_t u, uint32_t rsrc, bool valid) {
        stage_put(hq, claim(u, rsrc, valid), u);
      });
      stage_flush(hq);
      add_count(cur() + C_DEG, degsum);
      if (!bar(701)) return false;
      prof(PR_HEAVY, th, (uint32_t)(h >> 32), (uint32_t)h);
    }
    return true;
  }

  // One level of the DATA arm (reach_d.cu): a thread per frontier item walks
  // its list alone.
  __device__ __noinline__ void data_level(const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                          uint32_t *vis, bool ranged, const uint32_t *in, uint32_t nin,
                                          uint32_t *out) {
    const EngState &s = P.s;
    uint32_t *cnt = cur() + C_Q;
    for (uint32_t i = gtid(); i < nin; i += gstride()) {
      const uint32_t v = ldm(in + i);
      const uint32_t rv = ranged ? ldm(s.range + v) : 0u;
      const uint32_t b = ldg(off + v), e = ldg(off + v + 1);
      for (uint32_t j = b; j < e; ++j) {
        const uint32_t u = ldg(adj + j);
        if (try_visit(s, vis, u, ranged, rv)) queue_push(out, cnt, s.qcap, u, err());
      }
    }
  }

  // Asynchronous tail of worklist reaches (no levels).  A deep, thin reach
  // (a grid's thousands of levels of a few thousand vertices) is bound by
  // per-level latency -- a grid barrier plus the dependent loads of one
  // expansion -- not by bytes.  Reachability does not need levels: the
  // frontier is copied into the queue aq (async_seed; in the solve the
  // forward and the backward reach both seed it, items tagged with their
  // direction in bit 31, and their asynchronous parts run as one phase, so
  // a round costs the deeper of the two reaches, not their sum).  Every
  // warp takes the next 32 slots (one atomicAdd on aq_head) whenever it has
  // nothing else to do, expands the vertices of its slots as they are
  // filled (the 32 lists walked as one concatenation, 128 edges per round
  // of loads) and claims new vertices exactly once through the visited
  // bitmap.  Up to kAsyncKeep of a step's claims stay with the warp for its
  // next step; the rest are published at aq_pos.  aq_td holds the vertices
  // created (high half: seeds and claims) and expanded (low half); a warp
  // adds its counts to it before it publishes and when it runs out of
  // work, so the halves can only meet when no expansion is in flight and
  // none can start, which ends the phase.  A consumed slot is reset to
  // kNone, so aq is all ones again when the phase ends.  Filled slots never
  // wait long behind unfilled ones of the same window (at most kAsyncHold
  // polls).  Waits are bounded: no progress for timeout_ns sets
  // kErrBarrierTimeout.  async_loop holds this machinery; async_run and
  // async_trim supply the expansion step.
  // Ends (or, mid-step, drains) an asynchronous step: the k claims staged
  // in stb are added to this warp's count of created vertices and `done` to
  // its count of expanded ones; at the end of a step (keep) up to
  // kAsyncKeep - nl claims stay with this warp in loc for its next step, and
  // the rest are published to the queue.  The warp's counts reach aq_td
  // (created << 32 | expanded) in one atomic before anything is published
  // and whenever the warp runs out of work (async_flush), never otherwise:
  // while a warp holds unflushed counts it has expanded vertices whose
  // expansion the global count lacks, so the global counts cannot meet
  // before that warp's work is done (all 32 lanes call).
  __device__ __forceinline__ void async_commit(const uint32_t *stb, uint32_t k, uint32_t done, uint32_t *loc,
                                               uint32_t &nl, bool keep, unsigned long long &acc) {
    __syncwarp();
    const uint32_t lane = lane_id();
    acc += ((unsigned long long)k << 32) | done;
    const uint32_t kept = keep ? (k < kAsyncKeep - nl ? k : kAsyncKeep - nl) : 0u;
    for (uint32_t i = lane; i < kept; i += 32u) loc[nl + i] = stb[i];
    const uint32_t npub = k - kept;
    if (npub) {
      uint32_t pos = 0;
      if (lane == 0) {
        atomicAdd(&c->aq_td, acc);
        __threadfence();  // the creation count is visible before any published item
        pos = atomicAdd(&c->aq_pos, npub);
      }
      acc = 0;
      pos = __shfl_sync(kFull, pos, 0);
      const uint32_t cap = 2u * P.s.qcap;
      for (uint32_t i = lane; i < npub; i += 32u) {
        if (pos + i < cap) P.s.aq[pos + i] = stb[kept + i];
        else fail(kErrQueueOverflow);
      }
    }
    nl += kept;
    __syncwarp();
  }
  __device__ __forceinline__ void async_flush(unsigned long long &acc) {
    if (acc && lane_id() == 0) atomicAdd(&c->aq_td, acc);
    acc = 0;
  }

  // Appends the frontier in[0, nin) of direction dir to the asynchronous
  // queue at slot `at` (every CTA calls it with the same arguments; the
  // items are read after a later grid barrier).
  __device__ __forceinline__ void async_seed(const uint32_t *in, uint32_t nin, uint32_t at, uint32_t dir) {
    const uint32_t cap = 2u * P.s.qcap;
    for_items(nin, [&](uint32_t i, bool valid) {
      if (valid && at + i < cap) P.s.aq[at + i] = ldm(in + i) | (dir << 31);
    });
    if (is_lead() && at + nin > cap) fail(kErrQueueOverflow);
  }

  // Expands the ntot items seeded in aq (bit 31: 0 = forward, 1 =
  // backward) and everything they reach, both directions at once.
  // The loop of an asynchronous phase: windows of the shared queue, claims
  // kept for the warp's next step, the warp's counts, termination (see
  // async_run).  step(v, have, hmask, stb, loc, nl, acc) expands the lanes'
  // items and ends with async_commit.  Returns this warp's step count
  // (lane 0).
  template <class Step>
  __device__ __forceinline__ uint32_t async_loop(Step &&step) {
    const EngState &s = P.s;
    uint32_t *aq = s.aq;
    const uint32_t qcap = 2u * s.qcap;
    const uint32_t lane = lane_id();
    uint32_t *const stb = stage_buf(0);  // this warp's claims of the current step
    uint32_t *const loc = stage_buf(1);  // claims this warp keeps for its next step
    uint32_t nl = 0;                     // kept claims (warp-uniform)
    unsigned long long acc = 0;          // this warp's unflushed counts (created << 32 | expanded)
    uint32_t steps = 0;                  // warp steps (lane 0 counts them)
    bool over = false;
    uint32_t slot = 0;
    bool pend = false;  // this lane's window slot is still to be expanded
    unsigned long long idle0 = 0;
    uint32_t nap = 32, idle = 0, hold = 0;
    while (!over) {
      if (!__any_sync(kFull, pend) && nl == 0) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&c->aq_head, 32u);
        base = __shfl_sync(kFull, base, 0);
        if (base >= qcap) {  // every slot is taken: nothing more can come this warp's way
          async_flush(acc);
          break;
        }
        slot = base + lane;
        pend = slot < qcap;
      }
      const uint32_t wv = pend ? ldm(aq + slot) : kNone;
      const bool rdy = pend && wv != kNone;
      const uint32_t rmask = __ballot_sync(kFull, rdy);
      // a partly filled window with nothing kept is polled once more before
      // it is expanded: while the reach is wide its other slots fill within
      // nanoseconds, and a step then expands up to 32 vertices, not two
      if (nl == 0 && rmask && rmask != __ballot_sync(kFull, pend) && hold < kAsyncHold) {
        ++hold;
        __nanosleep(32);
        continue;
      }
      // lanes without a filled slot take kept claims (from the top)
      const uint32_t freem = ~rmask;
      const uint32_t take = nl < (uint32_t)__popc(freem) ? nl : (uint32_t)__popc(freem);
      const uint32_t rank = __popc(freem & lanemask_lt());
      const bool fromloc = !rdy && rank < take;
      const uint32_t v = rdy ? wv : fromloc ? loc[nl - 1u - rank] : kNone;
      const bool have = rdy || fromloc;
      const uint32_t hmask = __ballot_sync(kFull, have);
      if (hmask) {
        __syncwarp();  // kept claims read before the slots are reused below
        nl -= take;
        idle0 = 0;
        nap = 32;
        idle = 0;
        hold = 0;
        ++steps;
        if (rdy) aq[slot] = kNone;  // consumed: the queue is all ones again after the phase
        pend = pend && !rdy;
        step(v, have, hmask, stb, loc, nl, acc);
        continue;
      }
      async_flush(acc);  // out of work: this warp's counts go out first
      // nothing to expand: finished when every created vertex is expanded.
      // Checked on every eighth empty poll only: thousands of idle warps
      // reading aq_td would queue ahead of the steps' atomics on it in its
      // L2 slice.  Lane 0 decides for the warp, so the warp leaves as a
      // whole.
      uint32_t fin = 0;
      if (lane == 0 && (++idle & 7u) == 0) {
        const unsigned long long td = ld_acquire64(&c->aq_td);
        fin = (uint32_t)(td >> 32) == (uint32_t)td || ldm(&c->gs.err) != 0;
        if (!fin) {
          const unsigned long long now = globaltimer_ns();
          if (idle0 == 0) idle0 = now;
          if (now - idle0 > P.o.timeout_ns) {
            atomicOr(&c->gs.err, kErrBarrierTimeout);
            atomicExch(&c->gs.err_where, 712u);
            fin = 1;
          }
        }
      }
      if (__shfl_sync(kFull, fin, 0)) over = true;
      else {
        __nanosleep(nap);
        if (nap < 256u) nap <<= 1;
      }
    }
    return steps;
  }

  __device__ __noinline__ void async_run(uint32_t ntot, bool ranged) {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    if (is_lead()) {
      c->aq_head = 0;
      c->aq_pos = ntot;
      c->aq_td = (unsigned long long)ntot << 32;
    }
    if (!bar(710)) return;
    const uint32_t lane = lane_id();
    auto reach_step = [&](uint32_t v, bool have, uint32_t hmask, uint32_t *stb, uint32_t *loc, uint32_t &nl,
                          unsigned long long &acc) {
        uint32_t b = 0, d = 0, rv = 0;
        const uint32_t dir = have ? v >> 31 : 0u, x = v & 0x7fffffffu;
        if (have) {
          const uint32_t *off = dir ? g.offT : g.off;
          b = ldg(off + x);
          d = ldg(off + x + 1) - b;
          rv = ranged ? ldm(s.range + x) : 0u;
        }
        // the 32 lists walked as one concatenation, four 32-edge rounds
        // at a time with each round's loads issued together; claimed
        // vertices wait in this warp's staging segment
        const uint32_t incl = warp_incl_scan(d);
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        const uint32_t excl = incl - d;
        uint32_t nst = 0;  // staged claims (warp-uniform)
        for (uint32_t e0 = 0; e0 < total; e0 += 128u) {
          uint32_t u[4], rs[4], dr[4];
          bool val[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t e = e0 + 32u * r + lane;
            uint32_t lo = 0;  // owner: largest lane whose slice starts at or before e
#pragma unroll
            for (uint32_t sft = 16; sft >= 1; sft >>= 1) {
              const uint32_t cand = lo + sft;
              const uint32_t ex = __shfl_sync(kFull, excl, cand & 31u);
              if (cand < 32 && ex <= e) lo = cand;
            }
            const uint32_t o_beg = __shfl_sync(kFull, b, lo), o_ex = __shfl_sync(kFull, excl, lo);
            rs[r] = __shfl_sync(kFull, rv, lo);
            dr[r] = __shfl_sync(kFull, dir, lo);
            val[r] = e < total;
            u[r] = val[r] ? ldg((dr[r] ? g.adjT : g.adj) + o_beg + (e - o_ex)) : 0u;
          }
          uint32_t vw[4], ew[4], rg[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            vw[r] = val[r] ? ldm((dr[r] ? s.bvis : s.fvis) + (u[r] >> 5)) : ~0u;
            ew[r] = val[r] ? ldm(s.elim + (u[r] >> 5)) : ~0u;
            rg[r] = val[r] && ranged ? ldm(s.range + u[r]) : rs[r];
          }
          bool cl[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t bit = 1u << (u[r] & 31u);
            cl[r] = !((vw[r] | ew[r]) & bit) && rg[r] == rs[r] &&
                    !(atomicOr((dr[r] ? s.bvis : s.fvis) + (u[r] >> 5), bit) & bit);
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t m = __ballot_sync(kFull, cl[r]);
            if (cl[r]) stb[nst + __popc(m & lanemask_lt())] = u[r] | (dr[r] << 31);
            nst += __popc(m);
          }
          if (nst > kStage - 128u) {  // room for the next four rounds
            async_commit(stb, nst, 0u, loc, nl, false, acc);
            nst = 0;
          }
        }
        async_commit(stb, nst, (uint32_t)__popc(hmask), loc, nl, true, acc);
    };
    const uint32_t steps = async_loop(reach_step);
    add_count(cur() + C_CHG, lane == 0 ? steps : 0u);
    if (!bar(711)) return;
    if (is_lead()) c->phase_ret2 = rdprv(C_CHG);
  }

  // Asynchronous trim-1 worklist: the vertices trimmed by the sweep, in
  // s.qa[0, nq), seed the queue; expanding a trimmed vertex t examines its
  // live partition-mate neighbours (out- and in-lists) and trims each one
  // left without a live partition-mate in- or out-neighbour, claiming it
  // exactly once through its elim bit and appending it.  Same fixpoint as
  // the synchronous iterations (a vertex's last relevant neighbour to go is
  // expanded after its elim bit is set, and that expansion examines the
  // vertex), without a grid barrier per iteration.  Returns the trimmed
  // count of this thread.
  __device__ __noinline__ uint32_t async_trim(uint32_t nq, bool ranged) {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    async_seed(s.qa, nq, 0u, 0u);
    if (is_lead()) {
      c->aq_head = 0;
      c->aq_pos = nq;
      c->aq_td = (unsigned long long)nq << 32;
    }
    if (!bar(720)) return 0;
    const uint32_t lane = lane_id();
    uint32_t ntrim = 0;
    auto trim_step = [&](uint32_t t, bool have, uint32_t hmask, uint32_t *stb, uint32_t *loc, uint32_t &nl,
                         unsigned long long &acc) {
      const uint32_t rt = have && ranged ? ldm(s.range + t) : 0u;
      uint32_t nst = 0;
      for (uint32_t pass = 0; pass < 2; ++pass) {  // out-lists, then in-lists
        const uint32_t *off = pass ? g.offT : g.off, *adj = pass ? g.adjT : g.adj;
        uint32_t b = 0, d = 0;
        if (have) {
          b = ldg(off + t);
          d = ldg(off + t + 1) - b;
        }
        const uint32_t incl = warp_incl_scan(d);
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        const uint32_t excl = incl - d;
        for (uint32_t e0 = 0; e0 < total; e0 += 32u) {
          const uint32_t e = e0 + lane;
          uint32_t lo = 0;
#pragma unroll
          for (uint32_t sft = 16; sft >= 1; sft >>= 1) {
            const uint32_t cand = lo + sft;
            const uint32_t ex = __shfl_sync(kFull, excl, cand & 31u);
            if (cand < 32 && ex <= e) lo = cand;
          }
          const uint32_t o_beg = __shfl_sync(kFull, b, lo), o_ex = __shfl_sync(kFull, excl, lo);
          const uint32_t rs = __shfl_sync(kFull, rt, lo);
          const bool val = e < total;
          const uint32_t u = val ? ldg(adj + o_beg + (e - o_ex)) : 0u;
          const uint32_t ew = val ? ldm(s.elim + (u >> 5)) : ~0u;
          const uint32_t ru = val && ranged ? ldm(s.range + u) : rs;
          const uint32_t bit = 1u << (u & 31u);
          bool tr = false;
          if (val && !(ew & bit) && ru == rs &&
              !(live_nbr(s, g.off, g.adj, u, ru, ranged, false) && live_nbr(s, g.offT, g.adjT, u, ru, ranged, false))) {
            tr = !(atomicOr(s.elim + (u >> 5), bit) & bit);
            if (tr) {
              atomicOr(s.tflag + (u >> 5), bit);
              s.label[u] = u;
              ++ntrim;
            }
          }
          const uint32_t m = __ballot_sync(kFull, tr);
          if (tr) stb[nst + __popc(m & lanemask_lt())] = u;
          nst += __popc(m);
          if (nst > kStage - 32u) {
            async_commit(stb, nst, 0u, loc, nl, false, acc);
            nst = 0;
          }
        }
      }
      async_commit(stb, nst, (uint32_t)__popc(hmask), loc, nl, true, acc);
    };
    const uint32_t steps = async_loop(trim_step);
    (void)steps;
    bar(721);
    return ntrim;
  }

  // Worklist reach: DATA / LINEAR / TOPO / BEST.  Levels are synchronous:
  // level k expands the vertices first reached in level k-1 (the pivots at
  // k = 0) and appends each vertex it reaches, exactly once, to the next
  // worklist, so the n-slot worklists cannot overflow (reference
  // worklistc.h:79-81 drops items instead).  DATA expands one item per
  // thread (reach_d.cu); LINEAR gathers a level's edges warp-wide and splits
  // heavy lists across the grid (reach_l.cu).  TOPO / BEST add the bottom-up
  // topology sweep (reach_t.cu sweeps every vertex each level; reach_b.cu
  // switches direction): when the frontier's edges exceed the unexplored
  // edges / alpha, a level becomes a pull sweep -- every live unvisited
  // vertex scans its reverse list for a visited partition-mate -- until fewer
  // than live / beta vertices are reached per sweep.
  __device__ uint32_t reach_wl(const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj,
                               const uint32_t *__restrict__ poff, const uint32_t *__restrict__ padj, uint32_t *vis,
                               bool ranged, bool balanced, bool allow_pull, uint32_t dir, uint32_t async_from = kNone) {
    const EngState &s = P.s;
    const long long alpha = P.o.pull_alpha > 0 ? P.o.pull_alpha : 14;
    const long long beta = P.o.pull_beta > 0 ? P.o.pull_beta : 24;
    const unsigned long long mtot = P.g.m;
    const uint32_t *in = s.piv;
    uint32_t nin = ldm(&c->piv_count);
    uint32_t depth = 0, sel = 0;
    unsigned long long explored = 0, mf = 0;
    bool pull = false;
    // unreached candidates of the last pull sweep (aux / pivkey are free during reach)
    const uint32_t *rem_in = nullptr;
    uint32_t rem_n = 0, rem_sel = 0;
    bool rem_valid = false;
    // the last pull sweep tested list heads only: the next level must be a
    // full pull sweep over the remaining list, even with an empty frontier
    bool partial = false;
    // thin, deep reaches continue asynchronously (the frontier's edges are
    // known only where pulls are allowed)
    const uint32_t async_after = async_from != kNone ? async_from : P.o.async_depth > 0 ? (uint32_t)P.o.async_depth : kNone;
    const bool thin = (unsigned long long)P.g.m <= (unsigned long long)P.g.n * kAsyncTailDegree;
    while (nin > 0 || partial) {
      const unsigned long long ts = globaltimer_ns();
      // (on graphs that are not thin, a frontier of a few vertices -- the
      // end of a power-law reach -- finishes or grows in CTA-local levels
      // first: an asynchronous phase's seeding and barriers cost more; thin
      // graphs' deep reaches go asynchronous at once)
      const bool may_async = allow_pull && !pull && !partial && depth >= async_after;
      if (may_async && (nin >= kAsyncMin || thin) && mf <= (unsigned long long)nin * 8ull) {
        // the frontier goes to the asynchronous queue; with a_defer the
        // other direction's reach runs first and both finish together
        async_seed(in, nin, a_seeded, dir);
        a_seeded += nin;
        ++depth;
        if (!a_defer) async_finish(ranged);
        break;
      }
      // a small frontier goes to CTA 0; if it refuses (too many edges), the
      // grid expands this level as usual and the next level tries again
      if (!pull && !partial && nin <= kLocalMax) {
        const uint32_t room = P.o.max_iters > depth ? P.o.max_iters - depth : 0u;
        uint32_t lroom = room < kLocalLevels ? room : kLocalLevels;
        // a reach that may turn asynchronous stops its local levels there
        if (allow_pull && depth < async_after && async_after - depth < lroom) lroom = async_after - depth;
        if (blockIdx.x == 0)
          local_levels(off, adj, vis, ranged, in, nin, sel, lroom, may_async && !thin ? kAsyncMin : kNone);
        if (!bar(704)) return depth;
        if (!rdprv(C_LREF) && rdprv(C_LD) > 0) {
          const uint32_t ld = rdprv(C_LD);
          depth += ld;
          nin = rdprv(C_LN);
          mf = rdprv(C_LMF);
          explored += rdprv(C_LEX);
          sel = rdprv(C_LSEL);
          in = sel ? s.qa : s.qb;  // the queue the last local level filled
          rem_valid = false;
          prof(PR_WL, ts, ld, nin);
          if (depth >= P.o.max_iters) {
            fail(kErrIterCap);
            break;
          }
          continue;
        }
      }
      if (partial) {
        pull = true;
      } else if (allow_pull) {
        const unsigned long long unexplored = mtot > explored ? mtot - explored : 0ull;
        if (!pull && depth > 0 && (long long)mf * alpha > (long long)unexplored) pull = true;
        else if (pull && (long long)nin * beta < (long long)ldm(&c->n_live)) pull = false;
      }
      uint32_t *out = sel ? s.qb : s.qa;
      uint32_t qoff = 0;  // items already appended to `out` in an earlier interval of this level
      uint32_t slot = PR_WL;
      if (pull) {
        slot = PR_PULL;
        if (is_lead()) atomicAdd(&c->pull_sweeps, 1u);
        // Vertices a pull sweep examines but does not reach are kept in a
        // list, and the next pull sweep of this reach examines only them.
        uint32_t *rem_out = rem_sel ? s.pivkey : s.aux;
        const uint32_t *lst = rem_valid ? rem_in : list_mode ? s.act[act_sel] : nullptr;
        const uint32_t lcnt = rem_valid ? rem_n : list_mode ? act_count : 0u;
        // The first pull sweep after push levels covers every live vertex
        // and most of them find a visited neighbour in their list head, so
        // when the sweep set is large it tests heads only: a vertex whose
        // head holds none goes to the remaining list unexamined beyond it,
        // and the next sweep (forced to be a full pull sweep over that list)
        // walks the rest.  Warps then no longer wait, iteration after
        // iteration, for the few lanes walking long lists.
        const uint32_t span = lst ? lcnt : P.g.n;
        const bool head_only = (reinterpret_cast<uintptr_t>(padj) & 15u) == 0 && !rem_valid &&
                               span >= 8u * gstride();
        if (ranged) pull_sweep<true>(poff, padj, vis, lst, lcnt, out, rem_out, head_only);
        else pull_sweep<false>(poff, padj, vis, lst, lcnt, out, rem_out, head_only);
        if (!bar(703)) return depth;
        rem_in = rem_out;
        rem_n = rdprv(C_REM);
        rem_valid = true;
        rem_sel ^= 1u;
        partial = head_only;
      } else if (balanced) {
        rem_valid = false;
        // with a small frontier, lists longer than a chunk go to the whole grid
        // (one warp would otherwise walk thousands of edges while the rest wait)
        // (at most nwarps lists qualify, so the heavy-list counter sees few atomics);
        // mf (the frontier's edges) is known only where pulls are allowed
        const uint32_t heavy = P.o.heavy_degree;
        const unsigned long long per_warp = mf / nwarps();
        uint32_t split = heavy;
        if (allow_pull && per_warp < heavy) split = per_warp < 256ull ? 256u : (uint32_t)per_warp;
        const bool wide = !allow_pull || mf <= (unsigned long long)nin * kWideDegree;
        if (!push_level(off, adj, vis, ranged, allow_pull, in, nin, out, split, qoff, wide)) return depth;
      } else {
        rem_valid = false;
        data_level(off, adj, vis, ranged, in, nin, out);
        if (!bar(702)) return depth;
      }
      ++depth;
      nin = qoff + rdprv(C_Q);
      mf = rdprv(C_DEG);
      explored += mf;
      prof(slot, ts, nin, (uint32_t)mf);
      in = out;
      sel ^= 1u;
      if (depth >= P.o.max_iters) {
        fail(kErrIterCap);
        break;
      }
    }
    return depth;
  }

  // Runs the asynchronous phase for whatever reaches seeded it.
  __device__ void async_finish(bool ranged) {
    if (a_seeded == 0) return;
    const unsigned long long ts = globaltimer_ns();
    async_run(a_seeded, ranged);
    prof(PR_ASYNC, ts, (uint32_t)(ldm64(&c->aq_td) >> 32), ldm(&c->phase_ret2));  // vertices expanded, warp steps
    a_seeded = 0;
  }

  __device__ uint32_t reach(uint32_t dir, uint32_t arm, bool ranged) {
    const EngGraph &g = P.g;
    const EngState &s = P.s;
    const uint32_t *off = dir ? g.offT : g.off, *adj = dir ? g.adjT : g.adj;
    const uint32_t *poff = dir ? g.off : g.offT, *padj = dir ? g.adj : g.adjT;
    uint32_t *vis = dir ? s.bvis : s.fvis, *exp = dir ? s.bexp : s.fexp;
    switch (arm) {
      case ARM_Q: return reach_q(off, adj, vis, exp, ranged);
      case ARM_D: return reach_wl(off, adj, poff, padj, vis, ranged, false, false, dir);
      case ARM_L: return reach_wl(off, adj, poff, padj, vis, ranged, true, false, dir);
      case ARM_B: return reach_wl(off, adj, poff, padj, vis, ranged, true, true, dir);
      case ARM_TA: return reach_wl(off, adj, poff, padj, vis, ranged, true, true, dir, 0u);
      default: return reach_wl(off, adj, poff, padj, vis, ranged, true, P.o.pull_alpha >= 0, dir);
    }
  }

  // ========================================================== trim-2 (a7)
  // scc_routines.cu:397-523: v whose only live partition-mate out-neighbour
  // u has v as its only live partition-mate out-neighbour (or the same with
  // in-neighbours) forms the 2-vertex SCC {v, u}; the smaller id is its
  // representative (states 20 / 4).  Detection reads a snapshot (no
  // eliminations until every vertex has been examined), so the result does
  // not depend on thread order.
  __device__ __forceinline__ static uint32_t single_live(const EngState &s, const uint32_t *__restrict__ off,
                                         const uint32_t *__restrict__ adj, uint32_t v, uint32_t rv) {
    const uint32_t b = ldg(off + v), e = ldg(off + v + 1);
    uint32_t found = kNone, n = 0;
    for (uint32_t i = b; i < e; ++i) {
      const uint32_t u = ldg(adj + i);
      if (u == v || !live(s, u) || ldm(s.range + u) != rv) continue;
      if (++n > 1) return kNone;
      found = u;
    }
    return found;
  }
  __device__ __forceinline__ static bool only_to(const EngState &s, const uint32_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                 uint32_t u, uint32_t v, uint32_t rv) {
    const uint32_t b = ldg(off + u), e = ldg(off + u + 1);
    uint32_t n = 0;
    for (uint32_t i = b; i < e; ++i) {
      const uint32_t w = ldg(adj + i);
      if (w == u || !live(s, w) || ldm(s.range + w) != rv) continue;
      if (w != v) return false;
      ++n;
    }
    return n == 1;
  }
  __device__ __noinline__ uint32_t trim2() {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    for_vertices([&](uint32_t v, bool valid) {
      if (!valid || !live(s, v)) return;
      const uint32_t rv = ldm(s.range + v);
      uint32_t u = single_live(s, g.off, g.adj, v, rv);
      bool pair = u != kNone && only_to(s, g.off, g.adj, u, v, rv);
      if (!pair) {
        u = single_live(s, g.offT, g.adjT, v, rv);
        pair = u != kNone && only_to(s, g.offT, g.adjT, u, v, rv);
      }
      if (pair) {
        s.aux[v] = u;
        bit_set(s.queued, v);
      }
    });
    if (!bar(800)) return 0;
    uint32_t cnt = 0;
    for_vertices([&](uint32_t v, bool valid) {
      if (!valid || !bit_test(s.queued, v)) return;
      const uint32_t u = ldm(s.aux + v);
      s.label[v] = u < v ? u : v;
      bit_set(s.elim, v);
      bit_clear(s.queued, v);
      ++cnt;
    });
    add_count(&c->n_trim2, cnt);
    add_count(cur() + C_CNT, cnt);
    if (!bar(801)) return 0;
    return rdprv(C_CNT);
  }

  // ============================================================= WCC (a15)
  // wcc.cu:7-52,79-144: colour = smallest id reachable through out-edges
  // inside the partition (min-label propagation plus pointer jumping, to a
  // fixpoint); each colour becomes a partition whose pivot is the colour's
  // root.  The colour is constant on an SCC, so no SCC is split.
  // wcc.cu:7-226: colour = smallest id reachable inside the partition along
  // out-edges, with one pointer jump per sweep; SCC members share a colour.
  // Labels only decrease and always name a vertex reachable from the one
  // they label, so updates may land in any order (atomicMin) and the fixpoint
  // is the same.  Lists are walked warp-wide, lists longer than heavy_degree
  // by the whole grid.
  // Appends the ids of every set bit of bm to out (counter cur()[C_Q]): a
  // lane per bitmap word, one atomicAdd per warp-step.
  __device__ __forceinline__ void bitmap_list(const uint32_t *bm, uint32_t *out) {
    const EngState &s = P.s;
    const uint32_t lane = lane_id();
    for (uint32_t w0 = gwarp() * 32u; w0 < s.nwords; w0 += nwarps() * 32u) {
      const uint32_t w = w0 + lane;
      const uint32_t bits = w < s.nwords ? ldm(bm + w) : 0u;
      const uint32_t cnt = __popc(bits);
      const uint32_t incl = warp_incl_scan(cnt);
      uint32_t base = 0;
      if (lane == 31 && incl) base = atomicAdd(cur() + C_Q, incl);
      base = __shfl_sync(kFull, base, 31);
      uint32_t pos = base + incl - cnt;
      for (uint32_t x = bits; x; x &= x - 1u) {
        if (pos < s.qcap) out[pos] = w * 32u + (uint32_t)(__ffs(x) - 1);
        else fail(kErrQueueOverflow);
        ++pos;
      }
    }
  }

  // Frontier sweep of the WCC colouring: every vertex of cl[0, nc) (its
  // colour fell in the last sweep; bit set in cbm) offers its colour to its
  // live partition-mate in-neighbours; each one whose colour falls is
  // claimed once in nbm and appended to out.  cbm's bits of cl are cleared
  // on the way, so cbm is empty afterwards.
  __device__ __noinline__ void wcc_push(const uint32_t *cl, uint32_t nc, uint32_t *cbm, uint32_t *nbm, uint32_t *out) {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    uint32_t *lab = s.aux;
    Stage oq = stage_open(0, out, cur() + C_Q, s.qcap);
    for_items(nc, [&](uint32_t i, bool valid) {
      uint32_t v = 0, b = 0, d = 0, rv = 0, lv = kNone;
      if (valid) {
        v = ldm(cl + i);
        bit_clear(cbm, v);
        b = ldg(g.offT + v);
        d = ldg(g.offT + v + 1) - b;
        rv = ldm(s.range + v);
        lv = ldm(lab + v);
      }
      warp_gather_all(lv, b, d, rv, g.adjT, [&](uint32_t l, uint32_t w, uint32_t rsrc, bool ok) {
        bool claimed = false;
        if (ok) {
          const uint32_t ww = w >> 5, bit = 1u << (w & 31u);
          const uint32_t ew = ldm(s.elim + ww), rw = ldm(s.range + w), lw = ldm(lab + w);
          if (!(ew & bit) && rw == rsrc && l < lw && atomicMin(lab + w, l) > l) claimed = bit_claim(nbm, w);
        }
        stage_put(oq, claimed, w);
      });
    });
    stage_flush(oq);
  }

  // ============================================================ WCC (a15)
  // wcc.cu:7-144: colour of a live vertex = the smallest id it reaches
  // through out-edges between live partition-mates.  Full sweeps (every
  // live vertex takes its out-neighbours' smallest colour and jumps to its
  // colour's colour) while many colours change; they record the vertices
  // whose colour fell in a bitmap (fexp / bexp alternately: both are empty
  // from unset_pivots until the next reach).  Once fewer than live/64
  // colours changed in a sweep, those vertices form a list and later sweeps
  // push colours from the changed vertices to their in-neighbours only
  // (wcc_push): the tail of long, thin chains then costs a few items per
  // sweep instead of a sweep over every live vertex.  Both modes reach the
  // same fixpoint: after a full sweep, only a vertex whose colour fell
  // during it can still lower an in-neighbour's colour, and every such
  // vertex is in the list.
  __device__ __noinline__ uint32_t wcc() {
    const EngState &s = P.s;
    const EngGraph &g = P.g;
    const uint32_t heavy = P.o.heavy_degree;
    uint32_t *lab = s.aux;
    uint32_t *const bm[2] = {s.fexp, s.bexp};
    for (uint32_t w = gtid(); w < s.nwords; w += gstride()) {
      s.fexp[w] = 0u;
      s.bexp[w] = 0u;
    }
    for_vertices([&](uint32_t v, bool valid) {
      if (valid && live(s, v)) lab[v] = v;
    });
    if (!bar(900)) return 0;
    const uint32_t nlive = ldm(&c->n_live);
    uint32_t it = 0;
    bool front = false;
    uint32_t nc = 0, cb = 0;  // frontier length, bitmap holding its members
    uint32_t *cl = s.qa, *cn = s.qb;
    for (;;) {
      const unsigned long long tw = globaltimer_ns();
      if (front) {
        wcc_push(cl, nc, bm[cb], bm[cb ^ 1u], cn);
        if (!bar(905)) return it;
        nc = rdprv(C_Q);
        uint32_t *t = cl;
        cl = cn;
        cn = t;
        cb ^= 1u;
        ++it;
        prof(PR_WCC_IT, tw, nc, 1u);
        if (nc == 0) break;
        if (it >= P.o.max_iters) {
          fail(kErrIterCap);
          break;
        }
        continue;
      }
      uint32_t chg = 0;
      uint32_t *const mk = bm[it & 1u];
      // the other bitmap (marks of the sweep before) is cleared for the next
      for (uint32_t w = gtid(); w < s.nwords; w += gstride()) bm[(it + 1u) & 1u][w] = 0u;
      auto lower = [&](uint32_t v, uint32_t x) {
        if (atomicMin(lab + v, x) > x) {
          ++chg;
          bit_set(mk, v);
        }
      };
      // called from divergent code (heavy chunks): no warp collectives
      auto relax = [&](uint32_t src, uint32_t u, uint32_t rsrc) {
        if (!live(s, u) || ldm(s.range + u) != rsrc) return;
        const uint32_t x = ldm(lab + u);
        if (x < ldm(lab + src)) lower(src, x);
      };
      // The next vertex's state, offsets and colour are loaded one
      // iteration ahead; the warp's lists are walked 128 edges per round
      // with each round's loads (list entry; bitmap word, partition and
      // colour of the target) issued together.  Colours only decrease and
      // every colour a vertex ever holds is one it reaches, so a stale
      // colour read here costs at most a redundant atomicMin (and a sweep
      // with no change read only current colours).
      struct Pre {
        uint32_t ew, rv, b, e, l;
      };
      auto load = [&](uint32_t v, bool valid) {
        const uint32_t vv = valid ? v : 0u;
        return Pre{ldm(s.elim + (vv >> 5)), ldm(s.range + vv), ldg(g.off + vv), ldg(g.off + vv + 1), ldm(lab + vv)};
      };
      for_vertices_pf(load, [&](uint32_t v, bool valid, const Pre &p) {
        const bool lv = valid && !((p.ew >> (v & 31u)) & 1u);
        uint32_t b = lv ? p.b : 0u, d = lv ? p.e - p.b : 0u;
        if (d > heavy) {
          heavy_push(s, v, b, d, p.rv);
          d = 0;
        }
        // pointer jump, issued with the first round's loads
        const uint32_t jl = lv ? ldm(lab + p.l) : kNone;
        const uint32_t lane = lane_id();
        const uint32_t incl = warp_incl_scan(d);
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        const uint32_t excl = incl - d;
        for (uint32_t e0 = 0; e0 < total; e0 += 128u) {
          uint32_t u[4], src[4], rs[4], sl[4];
          bool val[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t e = e0 + 32u * r + lane;
            uint32_t lo = 0;
#pragma unroll
            for (uint32_t sft = 16; sft >= 1; sft >>= 1) {
              const uint32_t cand = lo + sft;
              const uint32_t ex = __shfl_sync(kFull, excl, cand & 31u);
              if (cand < 32 && ex <= e) lo = cand;
            }
            const uint32_t o_beg = __shfl_sync(kFull, b, lo), o_ex = __shfl_sync(kFull, excl, lo);
            src[r] = __shfl_sync(kFull, v, lo);
            rs[r] = __shfl_sync(kFull, p.rv, lo);
            sl[r] = __shfl_sync(kFull, p.l, lo);
            val[r] = e < total;
            u[r] = val[r] ? ldg(g.adj + o_beg + (e - o_ex)) : 0u;
          }
          uint32_t ew[4], rg[4], lu[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            ew[r] = val[r] ? ldm(s.elim + (u[r] >> 5)) : ~0u;
            rg[r] = val[r] ? ldm(s.range + u[r]) : 0u;
            lu[r] = val[r] ? ldm(lab + u[r]) : kNone;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const bool ok = val[r] && !((ew[r] >> (u[r] & 31u)) & 1u) && rg[r] == rs[r] && lu[r] < sl[r];
            if (ok) lower(src[r], lu[r]);
          }
        }
        if (lv && jl < p.l) lower(v, jl);
      });
      add_count(cur() + C_CHG, chg);
      if (!bar(901)) return it;
      const unsigned long long h = ldm64(prv64());
      if ((uint32_t)(h >> 32) != 0) {
        if (is_lead()) atomicAdd(cur() + C_CHG, rdprv(C_CHG));
        chg = 0;
        heavy_expand(s, g.adj, h, relax);
        add_count(cur() + C_CHG, chg);
        if (!bar(904)) return it;
      }
      ++it;
      const uint32_t nchg = rdprv(C_CHG);
      prof(PR_WCC_IT, tw, nchg, list_mode ? act_count : P.g.n);
      if (nchg == 0) break;
      if (it >= P.o.max_iters) {
        fail(kErrIterCap);
        break;
      }
      if ((unsigned long long)nchg * kWccFrontier < nlive) {
        // the marked vertices become the frontier list (mk = bm[(it - 1) & 1])
        bitmap_list(mk, cl);
        if (!bar(906)) return it;
        nc = rdprv(C_Q);
        cb = (it - 1u) & 1u;
        front = true;
      }
    }
    // roots become pivots of fresh partitions; members join their root's
    for_vertices([&](uint32_t v, bool valid) {
      bool root = false;
      if (valid && live(s, v)) {
        const uint32_t r = ldm(lab + v);
        s.range[v] = r;
        root = r == v;
        if (root) {
          s.rpivot[v] = v;
          s.sccsize[v] = 0u;
        }
      }
      warp_push(s.piv, cur() + C_Q, s.qcap, v, root, err());
    });
    if (!bar(902)) return it;
    const uint32_t np = rdprv(C_Q);
    for_items(np, [&](uint32_t i, bool valid) {
      if (valid) {
        const uint32_t p = ldm(s.piv + i);
        bit_set(s.fvis, p);
        bit_set(s.bvis, p);
      }
    });
    if (is_lead()) c->piv_count = np;
    bar(903);
    return it;
  }

  // ============================================= active-list compaction
  __device__ __noinline__ void compact() {
    const EngState &s = P.s;
    uint32_t *dst = s.act[act_sel ^ 1u];
    if (!list_mode) {
      // one bitmap word per lane (ids 0 and > n are marked eliminated at
      // init): a warp covers 1024 ids per step, scans its live counts and
      // appends them with one atomicAdd; then word by word, the lanes whose
      // bit is set write that word's ids side by side (coalesced stores)
      const uint32_t lane = lane_id();
      for (uint32_t w0 = gwarp() * 32u; w0 < s.nwords; w0 += nwarps() * 32u) {
        const uint32_t w = w0 + lane;
        const uint32_t live = w < s.nwords ? ~ldm(s.elim + w) : 0u;
        const uint32_t cnt = __popc(live);
        const uint32_t incl = warp_incl_scan(cnt);
        uint32_t base = 0;
        if (lane == 31 && incl) base = atomicAdd(cur() + C_Q, incl);
        base = __shfl_sync(kFull, base, 31);
        const uint32_t pos = base + incl - cnt;
        for (uint32_t j = 0; j < 32u; ++j) {
          const uint32_t lj = __shfl_sync(kFull, live, j);
          if (lj == 0u) continue;
          const uint32_t pj = __shfl_sync(kFull, pos, j);
          if ((lj >> lane) & 1u) {
            const uint32_t at = pj + __popc(lj & lanemask_lt());
            if (at < s.qcap) dst[at] = (w0 + j) * 32u + lane;
            else fail(kErrQueueOverflow);
          }
        }
      }
    } else {
      Stage aq = stage_open(0, dst, cur() + C_Q, s.qcap);
      for_vertices_pf([&](uint32_t v, bool) { return ldm(s.elim + (v >> 5)); },
                      [&](uint32_t v, bool valid, uint32_t ew) {
                        stage_put(aq, valid && !((ew >> (v & 31u)) & 1u), v);
                      });
      stage_flush(aq);
    }
    if (!bar(1000)) return;
    if (is_lead()) {
      c->act_count = rdprv(C_Q);
      c->act_sel = act_sel ^ 1u;
      c->list_mode = 1;
    }
    if (!bar(1001)) return;
    refresh_mode();
  }

  // compacts when fewer than span * den / num vertices are live
  __device__ __forceinline__ void maybe_compact(uint32_t num = 4, uint32_t den = 1) {
    const uint32_t nlive = ldm(&c->n_live);
    const uint32_t span = list_mode ? act_count : P.g.n;
    if (nlive > 0 && (unsigned long long)nlive * num < (unsigned long long)span * den) compact();
  }

  __device__ __forceinline__ void sync_live() {
    // n_live = n - trimmed - trim2 - F∩B; every CTA computes the same value
    if (is_lead()) {
      const uint32_t gone = ldm(&c->n_trimmed) + ldm(&c->n_trim2) + ldm(&c->n_fbe);
      c->n_live = P.g.n - gone;
    }
  }

  // ================================================== finalize labels
  __device__ __noinline__ void finalize() {
    const EngState &s = P.s;
    list_mode = 0;
    if (P.o.pivot_rule != 0) {  // representatives are pivots: canonicalise to min id
      for_all_ids([&](uint32_t v, bool valid) {
        if (valid) s.aux[v] = kNone;
      });
      if (!bar(1100)) return;
      for_all_ids([&](uint32_t v, bool valid) {
        const uint32_t l = valid ? ldm(s.label + v) : kNone;
        const uint32_t grp = __match_any_sync(kFull, l);
        if (valid) {
          const uint32_t mn = __reduce_min_sync(grp, v);
          if (lane_id() == (uint32_t)(__ffs(grp) - 1) && l != 0) atomicMin(s.aux + l, mn);
        }
      });
      if (!bar(1101)) return;
      for_all_ids([&](uint32_t v, bool valid) {
        if (valid) {
          const uint32_t l = ldm(s.label + v);
          if (l != 0) s.label[v] = ldm(s.aux + l);
        }
      });
      if (!bar(1102)) return;
    }
    // No counting sweep: every SCC was counted when its representative was
    // assigned (trim-1: one per vertex, trim-2: one per pair, F∩B: one per
    // eliminated pivot).  phase_ret = vertices still without a component.
    if (is_lead()) {
      c->nscc = ldm(&c->n_trimmed) + ldm(&c->n_trim2) / 2 + ldm(&c->n_fbscc);
      c->phase_ret = ldm(&c->n_live);
      s.label[0] = 0;
    }
  }

  // ================================================= the driver (a3)
  __device__ __forceinline__ void timed(unsigned long long &acc, unsigned long long t0) {
    if (is_lead()) acc += globaltimer_ns() - t0;
  }

  __device__ __forceinline__ uint32_t arm_for(bool below) const {
    // graphs of more than kAsyncTailDegree edges per vertex keep QUADRATIC
    // tails: theirs are few and short, and a sweep over the survivors costs
    // less than an asynchronous reach's seeding and two barriers
    const bool thin = (unsigned long long)P.g.m <= (unsigned long long)P.g.n * kAsyncTailDegree;
    const uint32_t tail = P.o.async_depth < 0 || !thin ? ARM_Q : ARM_TA;
    switch (P.o.alg) {
      case 0: return ARM_Q;
      case 1: return ARM_T;
      case 2: return ARM_D;
      case 3: return ARM_L;
      // past the switch point the reference sweeps (QUADRATIC); here the
      // tails are asynchronous worklist reaches from all partitions' pivots
      // at once unless async reaches are off (async_depth < 0)
      case 4: return below ? ARM_T : tail;  // HYBRID: reach_t below n/100, reach_q above
      case 5: return below ? ARM_L : tail;  // COMBINE
      case 6: return below ? ARM_B : tail;  // BEST
      default: return ARM_T;
    }
  }

  __device__ void solve() {
    const EngOpts &o = P.o;
    // asynchronous trim worklists on thin graphs, whose trims cascade over
    // many iterations (elsewhere a trim's worklist is an iteration or two,
    // cheaper than an asynchronous phase's seeding and barriers)
    a_trim = o.async_depth >= 0 && (unsigned long long)P.g.m <= (unsigned long long)P.g.n * kAsyncTailDegree;
    const bool single = P.s.nseg <= 1;
    refresh_mode();
    unsigned long long t0 = globaltimer_ns();
    // true while the live set and the partitions equal those of the last
    // trim fixpoint: another trim pass then provably removes nothing
    bool trim_fresh = false;
    // with one degree sweep and a single partition the first pivot is elected
    // inside that sweep (its survivors are exactly the live vertices)
    const uint32_t tf_cap = o.trim_first_depth > 0 ? (uint32_t)o.trim_first_depth : o.max_iters;
    const bool fused_pick = o.trim_first && single && tf_cap == 1;
    if (o.trim_first) {
      const uint32_t it = trim(false, P.g.sorted_unique != 0, tf_cap, fused_pick);
      if (is_lead()) c->trim_iters += it;
      sync_live();
      if (!bar(1)) return;
      // The first round's trim would run on the same live set and partition;
      // what it could still remove, later partition-aware trims remove.
      trim_fresh = true;
      // power-law graphs lose most vertices to the first trim: sweep the
      // survivors' list from the first round on
      const unsigned long long tc = globaltimer_ns();
      maybe_compact(5, 4);
      prof(PR_COMPACT, tc);
    }
    timed(c->ns_trim, t0);
    t0 = globaltimer_ns();
    if (fused_pick) {
      commit_first_pivot();
      prof(PR_PIVOT, t0);
    } else if (single) {
      pick_first_pivot();
      prof(PR_PIVOT, t0);
    } else {
      update();
      sync_live();
      if (!bar(2)) return;
    }
    timed(c->ns_update, t0);
    uint32_t step = 0;
    bool wcc_done = false;  // CTA-uniform: every CTA takes the WCC branch in the same round
    while (ldm(&c->piv_count) > 0) {
      if (ldm(&c->gs.err)) return;
      ++step;
      if (step > o.max_iters) {
        fail(kErrIterCap);
        return;
      }
      const uint32_t nel = ldm(&c->n_fbe) + ldm(&c->n_trim2);
      const uint32_t arm = arm_for(nel < o.switch_thr);
      // In the first round every partition is a whole segment (one graph of a
      // batch, or the graph) and no edge leaves a segment, so the reach and
      // trim of that round need no partition test.
      const bool ranged = step != 1;
      // reaches that turn asynchronous leave their frontiers in the queue,
      // and the two directions' asynchronous parts run as one phase
      a_defer = true;
      t0 = globaltimer_ns();
      const uint32_t fd = reach(0, arm, ranged);
      timed(c->ns_fwd, t0);
      t0 = globaltimer_ns();
      const uint32_t bd = reach(1, arm, ranged);
      a_defer = false;
      async_finish(ranged);
      timed(c->ns_bwd, t0);
      t0 = globaltimer_ns();
      uint32_t ti = 0;
      // The reference trims here every round (scc.cu:717-722).  In the first
      // round of a single partition right after the global trim-1 fixpoint,
      // reach changed only visit bits, so that trim cannot remove anything.
      if (o.trim_depth >= 0 && !(step == 1 && single && trim_fresh)) {
        const uint32_t cap = o.trim_depth == 0 ? o.max_iters : (uint32_t)o.trim_depth;
        ti = trim(ranged, false, cap);
      }
      sync_live();
      if (!bar(3)) return;
      timed(c->ns_trim, t0);
      t0 = globaltimer_ns();
      update();
      sync_live();
      if (!bar(4)) return;
      timed(c->ns_update, t0);
      prof(PR_UPDATE, t0);
      if (is_lead()) {
        c->steps = step;
        c->fwd_depth += fd;
        c->bwd_depth += bd;
        c->trim_iters += ti;
      }
      // shrink the sweep set first, so WCC and the next round cover only live vertices
      t0 = globaltimer_ns();
      maybe_compact();
      if (!bar(6)) return;
      prof(PR_COMPACT, t0);
      if (o.wcc && !wcc_done) {
        const uint32_t nel2 = ldm(&c->n_fbe) + ldm(&c->n_trim2);
        if (nel2 >= o.switch_thr) {
          t0 = globaltimer_ns();
          wcc_done = true;
          if (is_lead()) {
            c->wcc_done = 1;
            c->wcc_step = step;
          }
          if (ldm(&c->n_live) > 0) {
            unset_pivots();
            if (o.trim2) {
              trim2();
              sync_live();
              if (!bar(5)) return;
            }
            const uint32_t wi = wcc();
            if (is_lead()) c->wcc_iters += wi;
          }
          timed(c->ns_wcc, t0);
          prof(PR_WCC, t0);
        }
      }
      if (!bar(7)) return;
    }
    t0 = globaltimer_ns();
    finalize();
    prof(PR_FINAL, t0);
  }
};

// ------------------------------------------------------------------ kernels
// MINB: resident CTAs per SM the register allocation is sized for (the
// 1024/BS variant caps registers at 64, the 768/BS one at 80).
// __grid_constant__: Eng keeps a reference to the parameter block, which then
// stays in the constant bank instead of being copied to local memory.
template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) scc_persistent(const __grid_constant__ Params p, uint32_t phase,
                                                            uint32_t a0, uint32_t a1, uint32_t a2) {
  Eng<BS> e(p);
  Ctl *c = p.s.ctl;
  e.refresh_mode();
  switch (phase) {
    case PH_SOLVE: e.solve(); break;
    case PH_TRIM1: {
      const bool snap = p.g.sorted_unique && ldm(&c->n_live) == p.g.n;
      const uint32_t it = e.trim(false, snap, p.o.max_iters);
      e.sync_live();
      if (e.is_lead()) c->phase_ret = it;
      // as in the solve: later sweeps cover the survivors' list when few survive
      if (e.bar(1)) e.maybe_compact(5, 4);
      break;
    }
    case PH_TRIM: {
      const uint32_t it = e.trim(true, false, p.o.max_iters);
      e.sync_live();
      if (e.is_lead()) c->phase_ret = it;
      break;
    }
    case PH_TRIM2: {
      const uint32_t r = e.trim2();
      e.sync_live();
      if (e.is_lead()) c->phase_ret = r;
      break;
    }
    case PH_SELECT:
      if (p.s.nseg <= 1) {
        e.pick_first_pivot();
      } else {
        e.update();
        e.sync_live();
      }
      break;
    case PH_REACH: {
      const uint32_t d = e.reach(a0, a1, a2 != 0);
      if (e.is_lead()) c->phase_ret = d;
      break;
    }
    case PH_UPDATE:
      e.update();
      e.sync_live();
      break;
    case PH_UNSET: e.unset_pivots(); break;
    case PH_WCC: {
      const uint32_t it = e.wcc();
      if (e.is_lead()) c->phase_ret = it;
      break;
    }
    case PH_FINALIZE: e.finalize(); break;
    default: break;
  }
}

// per-solve reset: partitions (segment index or 0), bitmaps.  Labels need no
// reset: every vertex gets one when it is eliminated, and a solve ends only
// when all are (n_live == 0).
__global__ void scc_init_kernel(Params p) {
  const uint32_t n = p.g.n;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  if (blockIdx.x == 0) {  // the control block starts at zero (barrier arrivals included)
    uint32_t *w = reinterpret_cast<uint32_t *>(p.s.ctl);
    for (uint32_t i = threadIdx.x; i < sizeof(Ctl) / 4; i += blockDim.x) w[i] = 0u;
    __syncthreads();
  }
  for (uint32_t v = tid; v <= n; v += stride) {
    uint32_t r = 0;
    if (p.s.nseg > 1 && v >= 1) {
      uint32_t lo = 0, hi = p.s.nseg - 1;  // largest s with seg[s] <= v
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (p.s.seg[mid] <= v) lo = mid;
        else hi = mid - 1;
      }
      r = lo;
    }
    p.s.range[v] = r;
  }
  for (uint32_t w = tid; w < p.s.nwords; w += stride) {
    uint32_t e = 0;
    const uint32_t lo = w * 32u;
    for (uint32_t b = 0; b < 32; ++b) {
      const uint32_t v = lo + b;
      if (v == 0 || v > n) e |= 1u << b;
    }
    p.s.elim[w] = e;
    p.s.fvis[w] = 0;
    p.s.bvis[w] = 0;
    p.s.fexp[w] = 0;
    p.s.bexp[w] = 0;
    p.s.tflag[w] = 0;
    p.s.queued[w] = 0;
  }
  if (tid == 0) {
    p.s.ctl->best = ~0ull;
    p.s.ctl->n_live = n;
  }
}

__global__ void scc_states_kernel(Params p, uint8_t *out) {
  const uint32_t n = p.g.n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x) {
    if (v == 0) {
      out[0] = 0;
      continue;
    }
    auto bit = [&](const uint32_t *bm) { return (bm[v >> 5] >> (v & 31u)) & 1u; };
    const bool e = v <= n && bit(p.s.elim) && v != 0;
    uint8_t st = 0;
    if (bit(p.s.bvis)) st |= 1;
    if (bit(p.s.fvis)) st |= 2;
    if (e) st |= 4;
    if (bit(p.s.tflag)) st |= 8;
    if (e && p.s.label[v] == v) st |= 16;
    if (!e && (st & 3) == 3 && p.s.rpivot[p.s.range[v]] == v) st |= 16;  // live pivot (state 19)
    out[v] = st;
  }
}

// CSR sanity for caller-provided device graphs: offsets start at 0, never
// decrease and end at m; every neighbour id lies in 1..n.  Offsets are
// checked in a first launch so the second only reads inside adj[0, m).
__global__ void scc_check_offsets_kernel(const uint32_t *off, uint32_t n, uint32_t m, uint32_t *bad) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x + 1; v <= n; v += gridDim.x * blockDim.x) {
    const uint32_t a = off[v], b = off[v + 1];
    if (a > b || b > m || (v == 1 && a != 0) || (v == n && b != m)) atomicOr(bad, 1u);
  }
}
__global__ void scc_check_edges_kernel(const uint32_t *adj, uint32_t n, uint32_t m, uint32_t *bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const uint32_t u = adj[i];
    if (u < 1 || u > n) atomicOr(bad, 2u);
  }
}

// Segment sanity for packed graphs: every edge stays inside its source's
// segment (seg: nseg+1 first ids, seg[nseg] = n+1).  A thread per vertex.
__global__ void scc_check_segments_kernel(const uint32_t *off, const uint32_t *adj, uint32_t n, const uint32_t *seg,
                                          uint32_t nseg, uint32_t *bad) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x + 1; v <= n; v += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nseg - 1;  // largest s with seg[s] <= v
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (seg[mid] <= v) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t first = seg[lo], past = seg[lo + 1];
    for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
      const uint32_t u = adj[e];
      if (u < first || u >= past) {
        atomicOr(bad, 4u);
        break;
      }
    }
  }
}

cudaError_t check_segments(const uint32_t *off, const uint32_t *adj, uint32_t n, const uint32_t *seg, uint32_t nseg,
                           uint32_t *d_bad, uint32_t *h_bad, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d_bad, 0, 4, st);
  if (e != cudaSuccess) return e;
  if (n && nseg) scc_check_segments_kernel<<<148 * 8, 256, 0, st>>>(off, adj, n, seg, nseg, d_bad);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_bad, d_bad, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

cudaError_t check_device_csr(const uint32_t *off, const uint32_t *adj, uint32_t n, uint32_t m, uint32_t *d_bad,
                             uint32_t *h_bad, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d_bad, 0, 4, st);
  if (e != cudaSuccess) return e;
  if (n) scc_check_offsets_kernel<<<148 * 4, 256, 0, st>>>(off, n, m, d_bad);
  e = cudaMemcpyAsync(h_bad, d_bad, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess || *h_bad) return e;
  if (m) scc_check_edges_kernel<<<148 * 8, 256, 0, st>>>(adj, n, m, d_bad);
  e = cudaMemcpyAsync(h_bad, d_bad, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

__global__ void scc_ranges_kernel(Params p, uint32_t *out) {
  const uint32_t n = p.g.n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x) {
    const bool e = v == 0 || ((p.s.elim[v >> 5] >> (v & 31u)) & 1u);
    out[v] = e ? 0u : p.s.range[v];
  }
}

template <int BS, int MINB>
static cudaError_t coop_launch(const Params &p, uint32_t phase, uint32_t a0, uint32_t a1, uint32_t a2,
                               uint32_t grid_blocks, cudaStream_t stream, uint32_t *grid_used) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scc_persistent<BS, MINB>, BS, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  uint32_t maxg = (uint32_t)(sms * per_sm);
  // default grid: every co-resident CTA, except for small graphs, which get
  // one CTA per SM (their phases are barrier-bound, and a grid barrier
  // costs less with fewer arrivals)
  uint32_t g = maxg;
  if (grid_blocks) g = grid_blocks < maxg ? grid_blocks : maxg;
  else if (p.g.n <= kSmallGraphN && (uint32_t)sms < maxg) g = (uint32_t)sms;
  if (grid_used) *grid_used = g;
  Params pp = p;
  void *args[] = {&pp, &phase, &a0, &a1, &a2};
  return cudaLaunchCooperativeKernel((const void *)scc_persistent<BS, MINB>, dim3(g), dim3(BS), args, 0, stream);
}

template <int BS>
static cudaError_t coop_launch_occ(const Params &p, uint32_t phase, uint32_t a0, uint32_t a1, uint32_t a2,
                                   uint32_t grid_blocks, cudaStream_t stream, uint32_t *grid_used, int occupancy) {
  constexpr int kHi = 1024 / BS;
  constexpr int kLo = 768 / BS > 0 ? 768 / BS : 1;
  if (occupancy == 3) return coop_launch<BS, kLo>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used);
  if constexpr (BS == 256) {  // tighter register budgets, 256-thread CTAs only
    if (occupancy == 5) return coop_launch<BS, 5>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used);
    if (occupancy == 6) return coop_launch<BS, 6>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used);
  }
  return coop_launch<BS, kHi>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used);
}

cudaError_t launch_phase(const Params &p, uint32_t phase, uint32_t a0, uint32_t a1, uint32_t a2, int block_size,
                         uint32_t grid_blocks, cudaStream_t stream, uint32_t *grid_used, int occupancy) {
  // default register budget for 256-thread blocks: 80 registers (three CTAs
  // per SM) on graphs of more than kAsyncTailDegree edges per vertex, whose
  // solve is dominated by list sweeps that spill at 64; thin graphs keep
  // four CTAs per SM (more warps for their latency-bound phases)
  if (occupancy == 0 && block_size == 256 &&
      (unsigned long long)p.g.m > (unsigned long long)p.g.n * kAsyncTailDegree)
    occupancy = 3;
  switch (block_size) {
    case 128: return coop_launch_occ<128>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used, occupancy);
    case 512: return coop_launch_occ<512>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used, occupancy);
    case 1024: return coop_launch_occ<1024>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used, occupancy);
    default: return coop_launch_occ<256>(p, phase, a0, a1, a2, grid_blocks, stream, grid_used, occupancy);
  }
}

cudaError_t launch_init(const Params &p, cudaStream_t stream) {
  const uint32_t work = p.g.n + 1 > p.s.nwords ? p.g.n + 1 : p.s.nwords;
  uint32_t blocks = (work + 255) / 256;
  if (blocks > 148u * 16u) blocks = 148u * 16u;
  if (blocks == 0) blocks = 1;
  scc_init_kernel<<<blocks, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_states(const Params &p, uint8_t *d_states, cudaStream_t stream) {
  uint32_t blocks = (p.g.n + 256) / 256;
  if (blocks > 148u * 16u) blocks = 148u * 16u;
  scc_states_kernel<<<blocks, 256, 0, stream>>>(p, d_states);
  return cudaGetLastError();
}

cudaError_t launch_ranges(const Params &p, uint32_t *d_ranges, cudaStream_t stream) {
  uint32_t blocks = (p.g.n + 256) / 256;
  if (blocks > 148u * 16u) blocks = 148u * 16u;
  scc_ranges_kernel<<<blocks, 256, 0, stream>>>(p, d_ranges);
  return cudaGetLastError();
}

}  // namespace sccb
