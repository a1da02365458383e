// TEST / BENCH INFRASTRUCTURE — never linked into the product.
//
// Exposes the reference's own GPU decomposition (scc.cu computeSCC, a
// file-static function, with its reach / trim / WCC kernels) through one
// C symbol so that bench.py can time "the plain GPU FB" of the reference on
// the same device and graph.  Built by oracle/Makefile from the reference
// sources where they lie, with -DWCC -DTRIM_2 (the scc_2_w build), into
// oracle/_ref/libscc_ref_gpu.so; the reference's main() is renamed away.
#define main scc_reference_main
#include "scc.cu"
#undef main

// alg: the reference's reach_strategy value (scc.h:7-16); returns the SCC
// count and the reference's own timer (seconds, scc.cu:217 -> 1011).
extern "C" int ref_gpu_scc(unsigned n, unsigned m, unsigned *nodes, unsigned *edges, unsigned *nodesT,
                           unsigned *edgesT, int alg, int block_size, unsigned *nscc, float *secs) {
  alg_opt opt;
  opt.alg = (reach_strategy)alg;  // defaults as in scc.cu:80-86
  opt.warp_size = 32;
  opt.block_size = block_size;
  opt.trim_strat = 0;
  opt.trim_switch_limit = 20;
  opt.trim_both = true;
  opt.lin_cull_strat = 1;
  pair<unsigned, float> r = computeSCC(n, m, nodes, edges, nodesT, edgesT, opt);
  *nscc = r.first;
  *secs = r.second;
  return 0;
}
