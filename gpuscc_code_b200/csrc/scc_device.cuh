// Device-side building blocks of the persistent SCC kernels (sm_100a).
//
// Everything the persistent kernel shares between CTAs goes through L2:
// mutable arrays are read with ld.global.cg (__ldcg) so a stale L1 line can
// never be observed after a grid barrier; the CSR arrays are immutable for
// the whole launch and use the read-only path.
#pragma once

#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

namespace sccb {

namespace cg = cooperative_groups;

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kNone = 0xffffffffu;

// error bits written to Ctl::err (host maps any of them to SCC_ERR_TIMEOUT)
constexpr uint32_t kErrBarrierTimeout = 1u;
constexpr uint32_t kErrIterCap = 2u;
constexpr uint32_t kErrQueueOverflow = 4u;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// mutable data (written by other CTAs during this launch)
__device__ __forceinline__ uint32_t ldm(const uint32_t *p) { return __ldcg(p); }
__device__ __forceinline__ unsigned long long ldm64(const unsigned long long *p) { return __ldcg(p); }
// immutable CSR data
__device__ __forceinline__ uint32_t ldg(const uint32_t *p) { return __ldg(p); }

// ------------------------------------------------------------ bitmaps
__device__ __forceinline__ bool bit_test(const uint32_t *bm, uint32_t v) {
  return (ldm(bm + (v >> 5)) >> (v & 31u)) & 1u;
}
// returns true if this call flipped the bit from 0 to 1 (exactly-once)
__device__ __forceinline__ bool bit_claim(uint32_t *bm, uint32_t v) {
  const uint32_t b = 1u << (v & 31u);
  uint32_t *w = bm + (v >> 5);
  if (ldm(w) & b) return false;
  return !(atomicOr(w, b) & b);
}
__device__ __forceinline__ void bit_set(uint32_t *bm, uint32_t v) { atomicOr(bm + (v >> 5), 1u << (v & 31u)); }
__device__ __forceinline__ void bit_clear(uint32_t *bm, uint32_t v) {
  atomicAnd(bm + (v >> 5), ~(1u << (v & 31u)));
}

// ------------------------------------------------------ grid barrier
// Counting barrier for a cooperative (co-resident) grid.  `arrived` only
// grows during a launch (the host clears it before every launch): barrier
// number k of the launch is passed once it reaches (k+1) * gridDim.x, so
// the last CTA to arrive has nothing to reset and the others leave as soon
// as its arrival is visible.  The wait is bounded by `timeout_ns` of
// %globaltimer; on expiry the CTA records kErrBarrierTimeout and leaves the
// barrier, and every later barrier returns false at once so the whole grid
// drains and the kernel exits.
struct GridSync {
  unsigned long long arrived;
  uint32_t err;
  uint32_t err_where;
};

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier(GridSync *gs, unsigned long long target, uint64_t timeout_ns,
                                             uint32_t where) {
  __shared__ uint32_t s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    if (ld_acquire(&gs->err) != 0) {
      ok = 0;
    } else {
      __threadfence();  // this CTA's writes (ordered before thread 0 by the CTA barrier) go first
      atomicAdd(&gs->arrived, 1ull);
      if (ld_acquire64(&gs->arrived) < target) {
        const uint64_t t0 = globaltimer_ns();
        uint32_t spins = 0;
        while (ld_acquire64(&gs->arrived) < target) {
          __nanosleep(32);
          if ((++spins & 63u) == 0) {
            if (ld_acquire(&gs->err) != 0) { ok = 0; break; }
            if (globaltimer_ns() - t0 > timeout_ns) {
              atomicOr(&gs->err, kErrBarrierTimeout);
              atomicExch(&gs->err_where, where);
              ok = 0;
              break;
            }
          }
        }
      }
      __threadfence();
      if (ok && ld_acquire(&gs->err) != 0) ok = 0;
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// --------------------------------------------------- warp primitives
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  return x;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t x) { return __reduce_add_sync(kFull, x); }

// Warp-aggregated append to a global queue.  Callable from divergent code:
// the lanes that arrive together share one atomicAdd.  Returns false (and
// drops the item) only if the queue is full, which callers rule out by
// construction (every push is guarded by an exactly-once claim).
__device__ __forceinline__ void queue_push(uint32_t *q, uint32_t *count, uint32_t cap, uint32_t item,
                                           uint32_t *err) {
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, g.size());
  base = g.shfl(base, 0) + g.thread_rank();
  if (base < cap) q[base] = item;
  else atomicOr(err, kErrQueueOverflow);
}

// Full-warp push of the lanes with pred set (all 32 lanes must call).
__device__ __forceinline__ void warp_push(uint32_t *q, uint32_t *count, uint32_t cap, uint32_t item,
                                          bool pred, uint32_t *err) {
  const uint32_t mask = __ballot_sync(kFull, pred);
  if (mask == 0) return;
  const uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(kFull, base, leader);
  if (pred) {
    const uint32_t slot = base + __popc(mask & lanemask_lt());
    if (slot < cap) q[slot] = item;
    else atomicOr(err, kErrQueueOverflow);
  }
}

// Warp-gather expansion: every lane owns an adjacency slice
// adj[beg, beg+deg) of source `src` (deg may be 0).  The warp walks the
// concatenation of the 32 slices 32 edges at a time, so consecutive lanes
// read consecutive adjacency words whenever the slices are adjacent (they are
// in vertex-order sweeps).  `visit(src, dst, tag)` runs once per edge with
// the owning lane's `tag`.  All 32 lanes must call.
template <class Visit>
__device__ __forceinline__ void warp_gather(uint32_t src, uint32_t beg, uint32_t deg, uint32_t tag,
                                            const uint32_t *__restrict__ adj, Visit &&visit) {
  const uint32_t lane = lane_id();
  const uint32_t incl = warp_incl_scan(deg);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  const uint32_t excl = incl - deg;
  for (uint32_t b = 0; b < total; b += 32) {
    const uint32_t e = b + lane;
    // owner = largest lane j with excl_j <= e
    uint32_t lo = 0;
#pragma unroll
    for (uint32_t s = 16; s >= 1; s >>= 1) {
      const uint32_t cand = lo + s;
      const uint32_t ex = __shfl_sync(kFull, excl, cand & 31u);
      if (cand < 32 && ex <= e) lo = cand;
    }
    const uint32_t o_src = __shfl_sync(kFull, src, lo);
    const uint32_t o_beg = __shfl_sync(kFull, beg, lo);
    const uint32_t o_ex = __shfl_sync(kFull, excl, lo);
    const uint32_t o_tag = __shfl_sync(kFull, tag, lo);
    if (e < total) {
      const uint32_t dst = ldg(adj + o_beg + (e - o_ex));
      visit(o_src, dst, o_tag);
    }
  }
}

// warp_gather for visitors that need the whole warp (e.g. warp-staged
// appends): every lane calls visit(src, dst, tag, valid) at every step, with
// valid = false (and dst = 0) past the end of the concatenated slices.
template <class Visit>
__device__ __forceinline__ void warp_gather_all(uint32_t src, uint32_t beg, uint32_t deg, uint32_t tag,
                                                const uint32_t *__restrict__ adj, Visit &&visit) {
  const uint32_t lane = lane_id();
  const uint32_t incl = warp_incl_scan(deg);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  const uint32_t excl = incl - deg;
  for (uint32_t b = 0; b < total; b += 32) {
    const uint32_t e = b + lane;
    uint32_t lo = 0;
#pragma unroll
    for (uint32_t s = 16; s >= 1; s >>= 1) {
      const uint32_t cand = lo + s;
      const uint32_t ex = __shfl_sync(kFull, excl, cand & 31u);
      if (cand < 32 && ex <= e) lo = cand;
    }
    const uint32_t o_src = __shfl_sync(kFull, src, lo);
    const uint32_t o_beg = __shfl_sync(kFull, beg, lo);
    const uint32_t o_ex = __shfl_sync(kFull, excl, lo);
    const uint32_t o_tag = __shfl_sync(kFull, tag, lo);
    const bool valid = e < total;
    const uint32_t dst = valid ? ldg(adj + o_beg + (e - o_ex)) : 0u;
    visit(o_src, dst, o_tag, valid);
  }
}

// u64 min over a CTA, result valid in thread 0.
__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long x) {
  __shared__ unsigned long long s_min[32];
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const unsigned long long y = __shfl_down_sync(kFull, x, o);
    x = y < x ? y : x;
  }
  const uint32_t w = threadIdx.x >> 5;
  __syncthreads();
  if (lane_id() == 0) s_min[w] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    const uint32_t nw = blockDim.x >> 5;
    x = threadIdx.x < nw ? s_min[threadIdx.x] : ~0ull;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      const unsigned long long y = __shfl_down_sync(kFull, x, o);
      x = y < x ? y : x;
    }
  }
  return x;
}

// u32 sum over a CTA, result valid in thread 0.
__device__ __forceinline__ uint32_t block_sum(uint32_t x) {
  __shared__ uint32_t s_sum[32];
  x = __reduce_add_sync(kFull, x);
  const uint32_t w = threadIdx.x >> 5;
  __syncthreads();
  if (lane_id() == 0) s_sum[w] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    const uint32_t nw = blockDim.x >> 5;
    x = threadIdx.x < nw ? s_sum[threadIdx.x] : 0u;
    x = __reduce_add_sync(kFull, x);
  }
  return x;
}

}  // namespace sccb
