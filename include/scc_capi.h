/*
 * scc_capi.h — C ABI of the B200 strongly-connected-components engine.
 *
 * The reference (chenxuhao/gpuscc_code) exposes its hot path as C++ host
 * functions with C++ linkage (overloads on bool* / Worklist2*, alg_opt by
 * value, errors abort the process).  Every entry point below replaces one of
 * them with a plain C symbol: plain pointers and sizes, an int status
 * (0 = SCC_OK, negative = error, text from scc_last_error()), no exit().
 *
 * Graph conventions follow the reference exactly (load.cpp:125-197):
 *   vertex ids are 1..n, slot 0 is unused;
 *   nodes[n+2]: out-edges of v are edges[nodes[v] .. nodes[v+1]), nodes[1] = 0;
 *   nodesT/edgesT: the transpose (in-edges), same layout;
 *   edges hold 1-based vertex ids.
 * Labels: labels[v] (v = 1..n) is the smallest vertex id of v's strongly
 * connected component; labels[0] = 0.
 *
 * Thread safety: one context per host thread (each context owns one CUDA
 * stream); different contexts may be used concurrently.
 */
#ifndef GPUSCC_B200_SCC_CAPI_H
#define GPUSCC_B200_SCC_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SCC_OK 0
#define SCC_ERR_INVALID (-1)   /* bad argument */
#define SCC_ERR_IO (-2)        /* file missing / unparsable */
#define SCC_ERR_NOMEM (-3)     /* host or device allocation failed */
#define SCC_ERR_CUDA (-4)      /* CUDA runtime error */
#define SCC_ERR_TIMEOUT (-5)   /* a device-side bounded wait or iteration cap ran out */
#define SCC_ERR_NODEVICE (-6)  /* no CUDA device */
#define SCC_ERR_STATE (-7)     /* call out of order (e.g. phase before scc_phase_begin) */
#define SCC_ERR_CAPACITY (-8)  /* graph exceeds the 32-bit id / offset range or a fixed limit */
#define SCC_ERR_BUSY (-9)      /* server: request not finished yet */
#define SCC_ERR_REJECTED (-10) /* server: admission refused (does not fit in device memory) */

/* Message of the last error raised on this host thread ("" if none). */
const char *scc_last_error(void);
/* Library version string. */
const char *scc_version(void);

/* -------------------------------------------------------------- options */
/* Reachability strategies; values equal the reference enum reach_strategy
 * (scc.h:7-16) so the -a flag maps one to one. */
enum scc_alg {
  SCC_ALG_QUADRATIC = 0, /* -a q: topology sweep, one thread per vertex     (reach_q.cu) */
  SCC_ALG_TOPO = 1,      /* -a t: topology sweep, warp-gather load balance  (reach_t.cu) */
  SCC_ALG_DATA = 2,      /* -a d: data-driven worklist, thread per item     (reach_d.cu) */
  SCC_ALG_LINEAR = 3,    /* -a l: data-driven worklist, degree-binned gather (reach_l.cu) */
  SCC_ALG_HYBRID = 4,    /* -a h: TOPO until switch point, then QUADRATIC  (scc.cu:493-563) */
  SCC_ALG_COMBINE = 5,   /* -a c: LINEAR until switch point, then QUADRATIC (scc.cu:565-638) */
  SCC_ALG_BEST = 6       /* -a b: TOPO with pull sweeps until switch, then QUADRATIC (scc.cu:641-703) */
};

enum scc_pivot_rule {
  SCC_PIVOT_MIN_ID = 0,    /* smallest active id of the partition (reference: first id, scc.cu:235-245) */
  SCC_PIVOT_MAX_DEGREE = 1 /* largest in-degree x out-degree, ties to the smaller id */
};

typedef struct scc_opts {
  int32_t alg;             /* enum scc_alg (reference default TOPO, scc.cu:80) */
  int32_t wcc;             /* 1: WCC colouring once after the first big elimination (-DWCC, scc_w) */
  int32_t trim2;           /* 1: trim-2 once together with WCC (-DTRIM_2, scc_2_w) */
  int32_t trim_first;      /* 1: global trim-1 fixpoint before the first pivot (TRIM_FIRST, scc.cu:38) */
  int32_t block_size;      /* threads per block of the persistent kernels (0 = 256); -b */
  int32_t warp_size;       /* accepted for -w compatibility, not used (alg_opt.warp_size is never read) */
  int32_t pivot_rule;      /* enum scc_pivot_rule */
  int32_t switch_permille; /* hybrid/combine/best/WCC switch: eliminated >= n*permille/1000 (reference 10 = n/100) */
  int32_t trim_depth;      /* per-round range-aware trim-1: 0 = to fixpoint, k > 0 = at most k iterations, -1 = off */
  int32_t pull_alpha;      /* TOPO/BEST push->pull switch: frontier edges > unexplored edges / alpha (0 = 14) */
  int32_t pull_beta;       /* pull->push switch: newly reached < active / beta (0 = 24) */
  uint32_t warp_degree;    /* adjacency length from which a list is expanded by a whole warp (0 = 32) */
  uint32_t heavy_degree;   /* adjacency length from which a list is split across the grid (0 = 4096) */
  uint32_t max_iters;      /* cap on sweeps of any one fixpoint/reach loop and on FB rounds (0 = 1<<20) */
  uint32_t grid_blocks;    /* persistent grid size (0 = every co-resident block; one block per SM for
                              graphs of at most 2^21 vertices) */
  uint32_t timeout_ms;     /* bound on any device-side wait inside the persistent kernel (0 = 10000) */
  int32_t trim_first_depth;/* global trim-1 before the first pivot: 0 = to its fixpoint (reference trim1),
                              k > 0 = at most k iterations; later partition-aware trims remove the rest */
  int32_t occupancy;       /* register budget of the persistent kernel: 4 = four 256-thread CTAs per SM
                              (64 registers), 3 = three (80 registers); 0 = engine default (256-thread
                              blocks: 3 on graphs of more than 12 edges per vertex, else 4) */
  int32_t async_depth;     /* TOPO / BEST / HYBRID reaches: after this many synchronous levels, a frontier of
                              at most 8 edges per vertex is expanded asynchronously (every warp takes queued
                              vertices as they are appended, no level barriers; for deep, thin reaches such as
                              grids), and on graphs of at most 12 edges per vertex the HYBRID / COMBINE /
                              BEST tails past the switch point are asynchronous reaches instead of QUADRATIC
                              sweeps; 0 = 4, -1 = never (the reference's synchronous levels and QUADRATIC
                              tails).  Labels do not depend on it. */
  /* Fault-path test hooks (0 = off; labels are never affected while off).
   * test_stall_us: the last CTA of the grid waits this long (a bounded
   *   %globaltimer spin) before its second grid-barrier arrival, so that the
   *   other CTAs' bounded barrier waits (timeout_ms) run out: the solve then
   *   returns SCC_ERR_TIMEOUT and the context stays usable.
   * test_queue_cap: caps every worklist's usable length (entries) below its
   *   allocation, so that a push past it reports SCC_ERR_TIMEOUT (queue
   *   overflow) instead of the reference's silent drop (worklistc.h:79-81). */
  uint32_t test_stall_us;
  uint32_t test_queue_cap;
} scc_opts;

/* Reference defaults: alg TOPO, wcc 0, trim2 0, trim_first 1, block 256, pivot MIN_ID, switch 10;
 * engine default trim_first_depth 1 (one degree sweep; the labels do not depend on it). */
void scc_opts_default(scc_opts *opts);

/* ----------------------------------------------------------- host graph */
typedef struct scc_host_csr {
  uint32_t n;          /* countOfNodes */
  uint32_t m;          /* stored (deduplicated) edges = nodes[n+1] */
  uint32_t nnz_header; /* countOfEdges as load() reports it (header nnz; + extra for symmetric) */
  int32_t symmetric;   /* 1: nodesT == nodes, edgesT == edges (MatrixMarket "symmetric") */
  int32_t sorted_unique; /* 1: every adjacency list is strictly increasing (load() guarantees it) */
  int32_t owned;       /* 1: arrays were allocated by this library (scc_host_csr_free frees them) */
  uint32_t *nodes;     /* n+2 */
  uint32_t *edges;     /* m (+1 slack) */
  uint32_t *nodesT;    /* n+2 */
  uint32_t *edgesT;    /* m (+1 slack) */
} scc_host_csr;

/* load.h:5 / load.cpp:18 `bool load(char*, bool header, unsigned* countOfNodes,
 * unsigned* countOfEdges, unsigned** nodes, unsigned** edges, unsigned** nodesT,
 * unsigned** edgesT, unsigned*, unsigned*)`.  Same text / MatrixMarket format:
 * first line checked for "pattern" / "symmetric", '%' comment lines skipped,
 * header "m n nnz" for *.mtx (m must equal n) else "n nnz", each edge line is
 * "dst src [w]" giving the edge src->dst, symmetric files add both directions,
 * duplicates merged, neighbours sorted, self-loops kept.  `header` is accepted
 * and ignored exactly like the reference.  Parses with sort+unique instead of
 * std::set.  Returns SCC_ERR_IO instead of exit(1). */
int scc_load(const char *path, int header, scc_host_csr *out);
void scc_host_csr_free(scc_host_csr *csr);
/* Binary CSR cache (no counterpart in the reference, whose text parse
 * dominates its run time on large graphs): scc_save writes the CSR and
 * transpose as they are; scc_load recognises such a file by its first bytes
 * and reads it without parsing.  Large text files are parsed by all host
 * threads (same result as the serial reader, load.cpp semantics). */
int scc_save(const char *path, const scc_host_csr *csr);
/* Build a host CSR (+transpose) from an edge list of 1-based (src, dst) pairs:
 * duplicates merged, lists sorted, self-loops kept unless drop_self_loops. */
int scc_csr_from_edges(uint32_t n, uint64_t n_edges, const uint32_t *src, const uint32_t *dst,
                       int drop_self_loops, scc_host_csr *out);

/* tarjan.h:5 / tarjan.cpp:72 `TR_Decomposition(CSize, RSize, Fc, Fr)`: the CPU
 * decomposition behind the apps' -t flag (sequential, one host thread).
 * labels: optional (n+1) output, canonical min-id labels.  secs: wall time. */
int scc_tarjan(const scc_host_csr *csr, uint32_t *labels, uint32_t *nscc, double *secs);

/* --------------------------------------------------------- synthetic graphs
 * Deterministic generators (counter-based hashing: identical output for the
 * same arguments on any machine and on the device).  All produce deduplicated
 * sorted CSR + transpose with self-loops removed. */
/* R-MAT, n = 2^scale, `samples` edge draws, (a,b,c,d) given in parts per
 * million, vertex ids permuted by a seeded bijection when permute != 0. */
int scc_gen_rmat(uint32_t scale, uint64_t samples, uint32_t a_ppm, uint32_t b_ppm, uint32_t c_ppm,
                 uint64_t seed, int permute, scc_host_csr *out);
/* Erdos-Renyi style: `samples` uniform directed draws over n vertices. */
int scc_gen_er(uint32_t n, uint64_t samples, uint64_t seed, scc_host_csr *out);
/* side x side grid, each undirected grid edge oriented by a coin flip,
 * bidir_ppm of them made bidirectional, plus floor(grid_edges*longrange_ppm/1e6)
 * uniform random directed long-range edges. */
int scc_gen_grid(uint32_t side, uint32_t bidir_ppm, uint32_t longrange_ppm, uint64_t seed,
                 scc_host_csr *out);

/* `count` independent graphs packed into one CSR (the batched workload):
 * graph g is Erdos-Renyi or R-MAT (0.57, 0.19, 0.19, 0.05) with equal
 * probability, n log-uniform in [n_lo, n_hi], average out-degree uniform in
 * [deg_lo, deg_hi] (given in thousandths), self-loops dropped, duplicates
 * merged; graph g owns the global ids seg_first[g] .. seg_first[g+1]-1
 * (seg_first: count+1 entries, seg_first[0] = 1). */
int scc_gen_batch(uint32_t count, uint32_t n_lo, uint32_t n_hi, uint32_t deg_lo_milli, uint32_t deg_hi_milli,
                  uint64_t seed, scc_host_csr *out, uint32_t *seg_first);

/* ---------------------------------------------------------- device graph */
typedef struct scc_dev_csr {
  uint32_t n, m;
  int32_t sorted_unique;
  const uint32_t *nodes, *edges, *nodesT, *edgesT; /* device pointers, reference layout */
} scc_dev_csr;

/* Same R-MAT graph as scc_gen_rmat, generated, sorted and laid out on the
 * device of `ctx` (the 2^26-vertex / 2^30-sample graph does not fit a host
 * std::sort budget).  The arrays are owned by ctx and bound as its graph. */
typedef struct scc_ctx scc_ctx;
int scc_gen_rmat_device(scc_ctx *ctx, uint32_t scale, uint64_t samples, uint32_t a_ppm,
                        uint32_t b_ppm, uint32_t c_ppm, uint64_t seed, int permute,
                        scc_dev_csr *out);

/* Same batch as scc_gen_batch, built on the device of `ctx`, bound as its
 * graph with the segment table installed (seg_first: host, count+1). */
int scc_gen_batch_device(scc_ctx *ctx, uint32_t count, uint32_t n_lo, uint32_t n_hi, uint32_t deg_lo_milli,
                         uint32_t deg_hi_milli, uint64_t seed, scc_dev_csr *out, uint32_t *seg_first);

/* --------------------------------------------------------------- context */
int scc_ctx_create(int device, const scc_opts *opts, scc_ctx **out);
int scc_ctx_destroy(scc_ctx *ctx);
int scc_ctx_set_opts(scc_ctx *ctx, const scc_opts *opts);
int scc_ctx_get_opts(const scc_ctx *ctx, scc_opts *opts);
/* cudaStream_t the context launches on. */
void *scc_ctx_stream(scc_ctx *ctx);
/* Copy a host graph into context-owned device buffers (grown on demand). */
int scc_ctx_upload(scc_ctx *ctx, const scc_host_csr *csr);
/* Use a caller-owned device graph (borrowed; must outlive its use). */
int scc_ctx_bind_device(scc_ctx *ctx, const scc_dev_csr *csr);
/* Copy the bound graph back to the host (for the apps' -t and for tests). */
int scc_ctx_download(scc_ctx *ctx, scc_host_csr *out);
/* Same, into caller-owned host arrays (nodes/nodesT: n+2, edges/edgesT: m),
 * e.g. pinned buffers for later uploads. */
int scc_ctx_download_into(scc_ctx *ctx, uint32_t *nodes, uint32_t *edges, uint32_t *nodesT, uint32_t *edgesT);
/* Independent graphs packed in one CSR (batching): segment s owns vertices
 * seg_first[s] .. seg_first[s+1]-1 (1-based, seg_first[0] = 1,
 * seg_first[nseg] = n+1; no edge may cross segments).  nseg = 0 clears. */
int scc_ctx_set_segments(scc_ctx *ctx, uint32_t nseg, const uint32_t *seg_first);

typedef struct scc_stats {
  uint32_t steps;          /* FB rounds (scc.cu:998 "steps") */
  uint32_t fwd_depth;      /* sum of forward reach sweeps (scc.cu:999) */
  uint32_t bwd_depth;      /* sum of backward reach sweeps (scc.cu:1000) */
  uint32_t trim_iters;     /* sum of trim iterations (scc.cu:1001) */
  uint32_t wcc_iters;      /* WCC propagation sweeps */
  uint32_t wcc_step;       /* round in which WCC ran (0 = never) */
  uint32_t n_trimmed;      /* vertices removed by trim-1 */
  uint32_t n_trim2;        /* vertices removed by trim-2 */
  uint32_t n_fb_elim;      /* vertices eliminated as F∩B or trim-2 (reference countElimmed) */
  uint32_t nscc;           /* number of SCCs */
  uint32_t largest_scc;    /* vertices in the largest SCC (tarjan.cpp:155 biggestSCC); 0 only for n = 0 */
  uint32_t pull_sweeps;    /* reach sweeps done in pull (bottom-up) direction */
  uint32_t grid_blocks;    /* persistent grid actually launched */
  uint32_t block_size;
  uint32_t kernel_launches;/* kernels this call launched */
  uint32_t reserved;
  double ms_total;         /* device time of the solve (CUDA events) */
  double ms_trim;          /* device time by phase (globaltimer inside the persistent kernel) */
  double ms_fwd;
  double ms_bwd;
  double ms_update;
  double ms_wcc;
} scc_stats;

/* scc.cu:150 computeSCC(countOfNodes, countOfEdges, nodes, edges, nodesT,
 * edgesT, alg_opt): the whole decomposition on the bound graph in one
 * persistent cooperative launch.  labels: host (n+1) or NULL; nscc: count
 * (reference output "count of SCC"); stats: optional. */
int scc_solve(scc_ctx *ctx, uint32_t *labels, uint32_t *nscc, scc_stats *stats);
/* Same, labels left in device memory (d_labels: device (n+1) or NULL). */
int scc_solve_device(scc_ctx *ctx, uint32_t *d_labels, uint32_t *nscc, scc_stats *stats);
/* Captures the enqueue sequence of scc_solve_enqueue (control reset, state
 * init, the persistent cooperative launch) into a CUDA graph owned by the
 * context, so repeated solves of the bound graph (e.g. a packed batch) are
 * one graph launch each.  scc_solve_replay launches it and collects the
 * result like scc_solve_collect.  Re-capture after binding another graph. */
int scc_solve_capture(scc_ctx *ctx, uint32_t *d_labels);
int scc_solve_replay(scc_ctx *ctx, uint32_t *nscc, scc_stats *stats);
/* Batching (no counterpart in the reference, which solves one graph per run).
 * scc_batch_pack: independent graphs (reference layout each) into one CSR
 * with disjoint id ranges -- graph g owns ids seg_first[g] .. seg_first[g+1]-1
 * (seg_first: count+1 entries); out is owned by the library
 * (scc_host_csr_free).  scc_batch_solve: pack, upload, solve all graphs in
 * one persistent launch with one partition per graph, and return each
 * graph's labels in its own ids (labels[g]: host n_g+1, or NULL) and SCC
 * count (nscc[g], or NULL). */
int scc_batch_pack(uint32_t count, const scc_host_csr *graphs, scc_host_csr *out, uint32_t *seg_first);
int scc_batch_solve(scc_ctx *ctx, uint32_t count, const scc_host_csr *graphs, uint32_t *const *labels,
                    uint32_t *nscc);
/* Copy the labels of the last solve that wrote the context's own label
 * buffer (d_labels = NULL) to the host: labels (n+1). */
int scc_read_labels(scc_ctx *ctx, uint32_t *labels);
/* No counterpart in the reference (it cudaMallocs everything per call).
 * The whole decomposition for callers that cannot allocate device memory:
 * plugins whose host framework owns the whole device-memory budget and
 * forbids side allocations, and latency-critical loops that must not hit the
 * allocator's implicit synchronisation.  Needs no context: all scratch
 * lives in one static device array (about 5 MB per GPU, held until the
 * process exits), so graphs are limited to 65536 vertices and 4194304 edges
 * (SCC_ERR_CAPACITY beyond).  g: device CSR in the reference layout;
 * d_labels: device (n+1) output or NULL; stream: cudaStream_t or NULL.
 * Options are validated as for scc_ctx_create.  Returns once the solve has
 * finished (it waits for `stream` to read the result back).
 * Calls that overlap on the GPU share the array and race; serialise them.
 * The first call on each device does a one-time set-up for that device
 * (it looks up the array's device address).  cudaDeviceReset invalidates
 * that set-up: after resetting a device, do not call this entry point on
 * that device again in the same process. */
int scc_solve_noalloc(const scc_dev_csr *g, const scc_opts *opts, uint32_t *d_labels, uint32_t *nscc,
                      void *stream);
/* Enqueue the solve on the context stream without synchronising (capturable
 * in a CUDA graph).  Results: scc_solve_collect after the stream drained. */
int scc_solve_enqueue(scc_ctx *ctx, uint32_t *d_labels);
int scc_solve_collect(scc_ctx *ctx, uint32_t *nscc, scc_stats *stats);

/* Device-side phase timers of the last solve or phase call (the reference's
 * STOPWATCH accumulators, timing.h:14, taken inside the persistent kernel
 * with %globaltimer): ms[i] / counts[i] for i < 16 in the order trim first
 * sweep, trim worklist iterations, push sweeps, pull sweeps, heavy lists,
 * worklist levels, quadratic sweeps, update, WCC, trim-2, compaction,
 * finalize, first pivot, (3 reserved). */
int scc_get_profile(scc_ctx *ctx, double *ms, uint32_t *counts);
/* The first (up to) 128 timed events of the last call, in order: slot (as
 * above), two event counters (reach sweeps: vertices reached and their
 * edge count; trim: vertices removed; heavy: lists and edges) and ms.
 * Arrays hold 128 entries; *n receives the number filled. */
int scc_get_trace(scc_ctx *ctx, uint32_t *n, uint32_t *slot, uint32_t *a, uint32_t *b, double *ms);

/* -------------------------------------------------------- phase level API
 * Each call runs one phase of the reference driver on the context's device
 * state (one persistent launch iterating to its device-side fixpoint) and
 * returns the reference wrapper's return value through the out pointer. */
/* Reset per-vertex state: nothing eliminated, one partition per segment. */
int scc_phase_begin(scc_ctx *ctx);
/* scc_routines.h:47 trim1: global trim-1 to a fixpoint. */
int scc_trim1(scc_ctx *ctx, uint32_t *iterations);
/* scc_routines.h:41 trim: partition-aware trim-1 to a fixpoint. */
int scc_trim(scc_ctx *ctx, uint32_t *iterations);
/* scc_routines.h:50 trim2: one pass of 2-vertex sink/source SCC removal. */
int scc_trim2(scc_ctx *ctx, uint32_t *removed);
/* scc.cu:234-253: pick a pivot for every partition without one (first pivot). */
int scc_select_pivots(scc_ctx *ctx, uint32_t *n_pivots);
/* reach_{q,t,d,l}.h fwd_reach[1]_* / bwd_reach[1]_*: dir 0 = forward (out-edges),
 * 1 = backward (in-edges); variant = SCC_ALG_QUADRATIC/TOPO/DATA/LINEAR/BEST;
 * first_step != 0 ignores partitions (the *1 variants). depth = sweeps. */
int scc_reach(scc_ctx *ctx, int dir, int variant, int first_step, uint32_t *depth);
/* scc_routines.h:33 update: F∩B -> SCC, refine partitions, pick pivots.
 * has_pivot: 1 if another round is needed. */
int scc_update(scc_ctx *ctx, int32_t *has_pivot);
/* scc.cu:42-51 countElimmed: vertices eliminated but not trimmed. */
int scc_count_elimmed(scc_ctx *ctx, uint32_t *n_elimmed);
/* scc_routines.h:8 unsetPivots: drop the pivots chosen by the last update. */
int scc_unset_pivots(scc_ctx *ctx);
/* wcc.h:23 update_wcc: WCC colouring within partitions, one pivot per colour. */
int scc_update_wcc(scc_ctx *ctx, uint32_t *depth, int32_t *has_pivot);
/* Per-vertex state in the reference bit encoding (scc.h:48-93): 1 = B visited,
 * 2 = F visited, 4 = eliminated, 8 = trimmed, 16 = SCC representative.
 * states: host (n+1). */
int scc_get_states(scc_ctx *ctx, uint8_t *states);
/* Partition id of every active vertex (0 for eliminated ones): host (n+1). */
int scc_get_ranges(scc_ctx *ctx, uint32_t *ranges);
/* Finish: canonical labels for all vertices (host n+1) and the SCC count.
 * Fails with SCC_ERR_STATE while active vertices remain. */
int scc_get_labels(scc_ctx *ctx, uint32_t *labels, uint32_t *nscc);

/* ------------------------------------------------------ strategy network
 * No counterpart in the reference (its strategy is fixed by -a).  A 3-layer
 * fp32 MLP, 16 -> 64 -> 64 -> 8 with ReLU, whose three softmax heads pick,
 * per graph, options that never change the labels:
 *   head 0 (2 classes): pivot_rule  {MIN_ID, MAX_DEGREE}
 *   head 1 (2 classes): trim_depth  {0 = to fixpoint, 1 = one iteration}
 *   head 2 (4 classes): reach arm / switch point
 *                       {h at 10 permille, h at 100, h at 1000, c at 10}
 * Choice (0,0,0) is the plain hybrid (-a h, reference switch n/100). */
#define SCC_FEATURES 16
#define SCC_MLP_HEADS 3
#define SCC_MLP_OUTPUTS 8
/* Statistics of the bound graph, computed on the device (see the feature
 * list in scc_features.h): feat receives 16 floats. */
int scc_graph_features(scc_ctx *ctx, float *feat);
typedef struct scc_mlp scc_mlp;
/* Parameters He-uniform from seed, biases 0, normalisation mean 0 / scale 1. */
int scc_mlp_create(int device, uint64_t seed, scc_mlp **out);
int scc_mlp_destroy(scc_mlp *m);
/* Number of floats in the flat parameter vector: W1[16][64], b1[64],
 * W2[64][64], b2[64], W3[64][8], b3[8] (row = input unit). */
uint32_t scc_mlp_param_count(void);
/* get != 0: copy the parameters to buf; else load them from buf (and reset
 * the optimiser state). */
int scc_mlp_params(scc_mlp *m, float *buf, int get);
/* Input normalisation applied inside the forward pass: x' = (x - mean) * scale
 * (16 floats each); get != 0 reads it back. */
int scc_mlp_norm(scc_mlp *m, float *mean, float *scale, int get);
/* logits: B x 8 (head 0 in [0,2), head 1 in [2,4), head 2 in [4,8)). */
int scc_mlp_forward(scc_mlp *m, const float *x, uint32_t B, float *logits);
/* Mean over the B samples of the summed per-head cross-entropy (y: B x 3
 * class indices) and its gradient w.r.t. the flat parameters (either
 * output may be NULL). */
int scc_mlp_loss_grad(scc_mlp *m, const float *x, const int32_t *y, uint32_t B, float *loss, float *grad);
/* Adam (beta 0.9/0.999, eps 1e-8) over seeded shuffled minibatches, all on
 * the device; final_loss = loss of the last minibatch. */
int scc_mlp_train(scc_mlp *m, const float *x, const int32_t *y, uint32_t B, uint32_t epochs, uint32_t batch,
                  float lr, uint64_t seed, float *final_loss);
/* Arg-max class of each head: choice B x 3. */
int scc_mlp_predict(scc_mlp *m, const float *x, uint32_t B, int32_t *choice);
/* Writes the options a choice stands for into opts (other fields kept). */
int scc_mlp_apply(const int32_t *choice, scc_opts *opts);

/* ---------------------------------------------------------------- server
 * No counterpart in the reference.  A request loop on one device: graphs
 * are admitted while their CSR fits in the memory budget (FIFO), uploaded
 * on a copy stream while earlier work runs (or registered once and kept
 * resident), and solved in batches of the requests that are ready when the
 * device frees up (one segmented persistent launch per batch; a graph alone
 * is bound in place).
 * With a strategy network loaded, each request's options come from it and
 * only requests with the same options share a batch.  A batch runs as many
 * rounds and levels as its deepest graph, so thin graphs (at most four edges
 * per vertex, e.g. grids) share batches only with other thin graphs. */
typedef struct scc_server scc_server;
typedef struct scc_server_cfg {
  int32_t device;
  int32_t batching;            /* 0: one graph per launch, in arrival order */
  uint32_t max_batch_graphs;   /* 0 = 256 */
  uint32_t max_batch_vertices; /* capacity of the packed batch CSR (0 = 1<<24) */
  uint32_t max_batch_edges;    /* (0 = 1<<27) */
  uint32_t solo_vertices;      /* graphs with more vertices are solved alone: one such graph
                                  already fills the device, and a batch runs as many rounds as
                                  its slowest graph (0 = 1<<18) */
  uint64_t mem_budget;         /* device bytes for resident request graphs (0 = half the free memory) */
  scc_opts opts;               /* options of the plain method (and the base the network edits) */
} scc_server_cfg;
typedef struct scc_request_info {
  uint32_t nscc;
  uint32_t batch_graphs;       /* requests solved in the same launch */
  int32_t choice[3];           /* options picked (all 0 without a network) */
  int32_t status;              /* SCC_OK or the solve's error code */
  double queue_ms;             /* submit -> upload started (waiting for memory) */
  double latency_ms;           /* submit -> labels on the host */
  double solve_ms;             /* device time of the batch's solve */
} scc_request_info;
typedef struct scc_server_stats {
  uint64_t submitted, completed, rejected, batches, graphs_batched;
  uint64_t resident_bytes, peak_resident_bytes, budget_bytes;
  uint64_t registered;  /* graphs registered (scc_server_register) */
  uint64_t evictions;   /* resident device copies dropped to make room (least recently used first) */
  uint64_t reuploads;   /* requests of a resident graph that found it evicted and uploaded it again */
} scc_server_stats;
void scc_server_cfg_default(scc_server_cfg *cfg);
int scc_server_start(const scc_server_cfg *cfg, scc_server **out);
/* Load a strategy network (flat parameters and normalisation as in
 * scc_mlp_params / scc_mlp_norm); NULL params unloads it. */
int scc_server_set_model(scc_server *s, const float *params, const float *mean, const float *scale);
/* Queue a graph.  g's arrays and labels (host, n+1) must stay valid until
 * the request completes.  SCC_ERR_REJECTED if the graph alone exceeds the
 * memory budget. */
int scc_server_submit(scc_server *s, const scc_host_csr *g, uint32_t *labels, uint64_t *id);
/* Resident graphs: upload g once and keep its CSR on the device under
 * *handle (returns when the upload is done; g's host arrays must stay valid
 * until scc_server_unregister).  When an upload needs room, resident graphs
 * with no request in flight are evicted, least recently used first; a later
 * request of an evicted graph uploads it again from those host arrays.
 * SCC_ERR_REJECTED if g alone exceeds the budget. */
int scc_server_register(scc_server *s, const scc_host_csr *g, uint64_t *handle);
/* Queue a solve of a resident graph (no upload while it stays resident);
 * labels: host (n+1), valid until the request completes. */
int scc_server_submit_resident(scc_server *s, uint64_t handle, uint32_t *labels, uint64_t *id);
/* Drop a resident graph (SCC_ERR_BUSY while requests naming it are in flight). */
int scc_server_unregister(scc_server *s, uint64_t handle);
/* SCC_ERR_BUSY while the request runs; otherwise its info, and the request
 * is retired.  A failed solve returns its error code (info->status). */
int scc_server_poll(scc_server *s, uint64_t id, scc_request_info *info);
/* Like poll but blocks up to timeout_ms (0 = no limit). */
int scc_server_wait(scc_server *s, uint64_t id, uint32_t timeout_ms, scc_request_info *info);
int scc_server_get_stats(scc_server *s, scc_server_stats *st);
/* Finishes the queued requests, then stops. */
int scc_server_stop(scc_server *s);

#ifdef __cplusplus
}
#endif
#endif /* GPUSCC_B200_SCC_CAPI_H */
