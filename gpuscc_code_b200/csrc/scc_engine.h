// Host/device view of the persistent SCC engine: kernel parameters, the
// device control block and the launch entry points used by the C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sccb {

struct GridSyncH {
  unsigned long long arrived;  // barrier arrivals of the current launch (cleared before each launch)
  uint32_t err, err_where;
};

// Device control block.  One per context, cleared by scc_phase_begin / the
// solve launch.  ctr[] is triple-buffered per barrier interval: counters
// written between barriers i and i+1 live in ctr[i % 3]; CTA 0 zeroes
// ctr[(i+1) % 3] before arriving at barrier i+1 (that slot was last read
// during interval i-1).
struct Ctl {
  GridSyncH gs;
  uint32_t ctr[3][16];
  unsigned long long ctr64[3];
  unsigned long long best;      // first-pivot selection (prio << 32 | id)
  uint32_t n_live;              // vertices not yet assigned to an SCC
  uint32_t n_trimmed;           // removed by trim-1
  uint32_t n_trim2;             // removed by trim-2
  uint32_t n_fbe;               // removed as F∩B
  uint32_t n_fbscc;             // SCCs found as F∩B (their pivots)
  uint32_t nscc;
  uint32_t piv_count;           // pivots chosen by the last selection
  uint32_t list_mode;           // 0: sweeps cover 0..n; 1: sweeps cover the active list
  uint32_t act_count;           // active list length
  uint32_t act_sel;             // which active list buffer is current
  uint32_t steps, fwd_depth, bwd_depth, trim_iters, wcc_iters, wcc_step, pull_sweeps;
  uint32_t wcc_done;
  uint32_t phase_ret, phase_ret2;
  uint32_t trim_first_done;
  uint32_t largest_fb;          // largest SCC found as F∩B (members counted per pivot)
  unsigned long long ns_trim, ns_fwd, ns_bwd, ns_update, ns_wcc;
  // finer device timers (globaltimer, CTA 0) and counts, indexed by Prof
  unsigned long long prof_ns[16];
  uint32_t prof_cnt[16];
  // per-sweep trace (first kTrace events of a launch): slot, two counters, ns
  uint32_t trace_n, trace_pad;
  uint32_t trace_slot[128], trace_a[128], trace_b[128];
  unsigned long long trace_ns[128];
  // asynchronous reach: next slot to take; next slot to fill; vertices
  // created << 32 | vertices expanded (each in its own 128-byte line)
  uint32_t aq_head, aq_pad0[31];
  uint32_t aq_pos, aq_pad2[31];
  unsigned long long aq_td, aq_pad1[15];
};
constexpr uint32_t kTrace = 128;

enum Prof : uint32_t {
  PR_TRIM_SWEEP = 0,  // first sweep of a trim
  PR_TRIM_WL = 1,     // worklist iterations of a trim
  PR_PUSH = 2,        // push sweeps (TOPO/BEST)
  PR_PULL = 3,        // pull sweeps
  PR_HEAVY = 4,       // grid-split heavy lists
  PR_WL = 5,          // DATA/LINEAR levels
  PR_Q = 6,           // QUADRATIC sweeps
  PR_UPDATE = 7,
  PR_WCC = 8,
  PR_TRIM2 = 9,
  PR_COMPACT = 10,
  PR_FINAL = 11,
  PR_PIVOT = 12,
  PR_ASYNC = 13,     // asynchronous reach tails
  PR_WCC_IT = 14,    // one WCC relaxation sweep
  PR_COUNT = 16
};

struct EngGraph {
  uint32_t n, m;
  uint32_t sorted_unique;
  uint32_t pad;
  const uint32_t *off, *adj, *offT, *adjT;
};

struct EngState {
  uint32_t *label;   // n+1: 0 = unresolved, else SCC label
  uint32_t *range;   // n+1: partition id (the pivot id of the partition after the first selection)
  uint32_t *rpivot;  // n+1: pivot of partition id
  uint32_t *aux;     // n+1: WCC colours / trim-2 partners / canonical ids
  uint32_t *sccsize; // n+1: F∩B members counted per pivot (zeroed when the pivot is elected)
  uint32_t *elim, *fvis, *bvis, *fexp, *bexp, *tflag, *queued;  // bitmaps, nwords each
  uint32_t *qa, *qb;       // queues, qcap each
  uint32_t *act[2];        // active lists, qcap each
  uint32_t *piv, *pivkey;  // pivot list, qcap each
  unsigned long long *slot;  // 3(n+1): partition-refinement pivot election, all ones between uses
  uint32_t *aq;              // 2 qcap: asynchronous reach queue (bit 31: direction), all ones between uses
  uint32_t *hv, *hbeg, *hdeg, *htag, *hbase;  // heavy adjacency list split across the grid
  const uint32_t *seg;       // nseg+1 segment first ids (device) or null
  uint32_t *out_labels;      // optional destination of the final labels (device)
  Ctl *ctl;
  uint32_t nwords;  // bitmap words (covers ids 0..nwords*32-1; ids 0 and > n carry the elim bit)
  uint32_t qcap;    // n+1
  uint32_t hcap;    // heavy list capacity
  uint32_t nseg;
};

struct EngOpts {
  uint32_t alg, wcc, trim2, trim_first, pivot_rule;
  uint32_t switch_thr;  // eliminated-vertex count at which HYBRID/COMBINE/BEST switch and WCC runs
  int32_t trim_depth;
  int32_t pull_alpha, pull_beta;
  uint32_t warp_degree, heavy_degree, max_iters;
  unsigned long long timeout_ns;
  int32_t trim_first_depth;
  int32_t async_depth;  // levels before a thin reach turns asynchronous; < 0: never
  unsigned long long test_stall_ns;  // fault-path test hook: last CTA stalls before barrier interval 1 ends
};

struct Params {
  EngGraph g;
  EngState s;
  EngOpts o;
};

// Bitmap words swept for an n-vertex graph: ids 0..n rounded up to a whole
// number of 1024-thread blocks (32 words), so every CTA of a full-id sweep
// runs the same number of iterations (it may synchronise inside them).
// Allocations add kBitmapSlack words.
constexpr uint32_t bitmap_words(uint32_t n) {
  return (uint32_t)((((uint64_t)n + 1 + 31) / 32 + 31) / 32 * 32);
}
constexpr uint32_t kBitmapSlack = 4;

enum Phase : uint32_t {
  PH_SOLVE = 0,
  PH_TRIM1 = 1,
  PH_TRIM = 2,
  PH_TRIM2 = 3,
  PH_SELECT = 4,
  PH_REACH = 5,
  PH_UPDATE = 6,
  PH_UNSET = 7,
  PH_WCC = 8,
  PH_FINALIZE = 9,
  PH_STATES = 10,
};

// Launch helpers (implemented in scc_engine.cu).
// Cooperative launch of the persistent kernel for `phase`; occupancy selects
// the register budget (4: four 256-thread CTAs per SM, 64 registers; 3:
// three CTAs, 80 registers).
cudaError_t launch_phase(const Params &p, uint32_t phase, uint32_t a0, uint32_t a1, uint32_t a2,
                         int block_size, uint32_t grid_blocks, cudaStream_t stream,
                         uint32_t *grid_used, int occupancy);
// Per-solve reset of the per-vertex state (plain launch).
cudaError_t launch_init(const Params &p, cudaStream_t stream);
// states export in the reference bit encoding.
cudaError_t launch_states(const Params &p, uint8_t *d_states, cudaStream_t stream);
cudaError_t launch_ranges(const Params &p, uint32_t *d_ranges, cudaStream_t stream);

// Validates a device CSR (offsets monotone from 0 to m, ids in 1..n); *h_bad
// is nonzero on a violation.  d_bad: 4 bytes of device scratch.
cudaError_t check_device_csr(const uint32_t *off, const uint32_t *adj, uint32_t n, uint32_t m, uint32_t *d_bad,
                             uint32_t *h_bad, cudaStream_t st);
// Checks that no edge leaves its source's segment (seg: device, nseg+1
// first ids); *h_bad is nonzero on a violation.
cudaError_t check_segments(const uint32_t *off, const uint32_t *adj, uint32_t n, const uint32_t *seg, uint32_t nseg,
                           uint32_t *d_bad, uint32_t *h_bad, cudaStream_t st);

}  // namespace sccb
namespace sccg {
struct BatchGraph;
}
namespace sccb {

// Device build of a batch of independent graphs packed with global 1-based
// ids (graph g owns a contiguous id range); arrays are cudaMalloc'ed.
cudaError_t gen_batch_device(const sccg::BatchGraph *plan, uint32_t count, cudaStream_t st, uint32_t **d_off,
                             uint32_t **d_adj, uint32_t **d_offT, uint32_t **d_adjT, uint32_t *n_out,
                             uint32_t *m_out);

// Device R-MAT build (scc_gen_device.cu); output arrays are cudaMalloc'ed.
cudaError_t gen_rmat_device(uint32_t scale, uint64_t samples, uint32_t a_ppm, uint32_t b_ppm, uint32_t c_ppm,
                            uint64_t seed, int permute, cudaStream_t st, uint32_t **d_off, uint32_t **d_adj,
                            uint32_t **d_offT, uint32_t **d_adjT, uint32_t *m_out);

}  // namespace sccb
