// scc / scc_w / scc_2_w: the reference apps' command line (scc.cu:57-148)
// on top of the C ABI.  One source, three binaries: SCC_APP_WCC adds the
// WCC colouring pass (reference -DWCC), SCC_APP_TRIM2 adds trim-2
// (-DTRIM_2).  Flags: -t (CPU Tarjan too), -a q|t|d|l|h|c|b|a, -f graph,
// -w N (accepted, unused), -b N (threads per block), -h (header, unused).
// Extra: -o file writes "vertex label" lines (label = min id of the SCC);
// -v dir writes the reference's VERIFY files (scc.cu:920-995) from the labels:
// trivial.txt (ids of one-vertex SCCs), scc_dist.txt ("size count" lines) and
// parallel_scc.txt (each SCC's members on one line, SCCs by smallest id).
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "scc_capi.h"

static int compute(scc_ctx *ctx, const scc_opts &base, int alg, uint32_t n, std::vector<uint32_t> *labels) {
  scc_opts o = base;
  o.alg = alg;
  if (scc_ctx_set_opts(ctx, &o) != SCC_OK) {
    std::fprintf(stderr, "error: %s\n", scc_last_error());
    return 1;
  }
  std::printf("computing SCC in parallel - alg: %d...\n", alg);
  uint32_t nscc = 0;
  scc_stats st;
  if (labels) labels->assign((size_t)n + 1, 0);
  if (scc_solve(ctx, labels ? labels->data() : nullptr, &nscc, &st) != SCC_OK) {
    std::fprintf(stderr, "error: %s\n", scc_last_error());
    return 1;
  }
  std::printf("FB done!\n\n");
  const double steps = st.steps ? st.steps : 1;
  std::printf("    ->steps: %u\n", st.steps);
  std::printf("    ->sum of fwdDepths: %u and avg fwd depth: %.1f\n", st.fwd_depth, st.fwd_depth / steps);
  std::printf("    ->sum of bwdDepths: %u and avg bwd depth: %.1f\n", st.bwd_depth, st.bwd_depth / steps);
  std::printf("    ->sum of trimIterations: %u and avg of trimIterations: %.1f\n", st.trim_iters,
              st.trim_iters / steps);
  std::printf("    ->time spent by fwd_reach: %f\n", st.ms_fwd / 1000.0);
  std::printf("    ->time spent by bwd_reach: %f\n", st.ms_bwd / 1000.0);
  std::printf("    ->time spent by trimming:  %f\n", st.ms_trim / 1000.0);
  std::printf("    ->time spent by updating:  %f\n", (st.ms_update + st.ms_wcc) / 1000.0);
  std::printf("    ->count of SCC: %u\n", nscc);
  std::printf("    ->time: %f\n", st.ms_total / 1000.0);
  return 0;
}

static int write_verify(const char *dir, uint32_t n, const std::vector<uint32_t> &labels) {
  // members grouped by label (counting sort keeps them in id order)
  std::vector<uint32_t> size((size_t)n + 2, 0), start((size_t)n + 2, 0), members(n);
  for (uint32_t v = 1; v <= n; ++v) ++size[labels[v]];
  for (uint32_t r = 1; r <= n; ++r) start[r + 1] = start[r] + size[r];
  {
    std::vector<uint32_t> fill(start);
    for (uint32_t v = 1; v <= n; ++v) members[fill[labels[v]]++] = v;
  }
  const std::string d(dir);
  FILE *ft = std::fopen((d + "/trivial.txt").c_str(), "w");
  FILE *fd = std::fopen((d + "/scc_dist.txt").c_str(), "w");
  FILE *fs = std::fopen((d + "/parallel_scc.txt").c_str(), "w");
  if (!ft || !fd || !fs) {
    std::fprintf(stderr, "error: cannot write the verify files in %s\n", dir);
    if (ft) std::fclose(ft);
    if (fd) std::fclose(fd);
    if (fs) std::fclose(fs);
    return 1;
  }
  std::vector<uint32_t> dist((size_t)n + 1, 0);
  uint32_t trivial = 0, nontrivial = 0;
  for (uint32_t r = 1; r <= n; ++r) {
    if (!size[r]) continue;
    ++dist[size[r]];
    if (size[r] == 1) {
      ++trivial;
      std::fprintf(ft, "%u\n", r);
    } else {
      ++nontrivial;
    }
    for (uint32_t i = start[r]; i < start[r] + size[r]; ++i) std::fprintf(fs, "%u ", members[i]);
    std::fprintf(fs, "\n");
  }
  for (uint32_t k = 1; k <= n; ++k)
    if (dist[k]) std::fprintf(fd, "%u %u\n", k, dist[k]);
  std::fclose(ft);
  std::fclose(fd);
  std::fclose(fs);
  std::printf("    ->trivial SCCs: %u, non-trivial SCCs: %u\n", trivial, nontrivial);
  return 0;
}

int main(int argc, char **argv) {
  scc_opts opts;
  scc_opts_default(&opts);
#ifdef SCC_APP_WCC
  opts.wcc = 1;
#endif
#ifdef SCC_APP_TRIM2
  opts.trim2 = 1;
#endif
  bool tarjan = false, all = false;
  const char *file = nullptr, *out_file = nullptr;
  int alg = SCC_ALG_TOPO;  // scc.cu:80
  int c;
  const char *verify_dir = nullptr;
  while ((c = getopt(argc, argv, "htf:a:w:b:o:v:")) != -1) {
    switch (c) {
      case 'h': break;  // "header": accepted and unused, as in load.cpp
      case 't': tarjan = true; break;
      case 'f': file = optarg; break;
      case 'a':
        switch (optarg[0]) {
          case 'q': alg = SCC_ALG_QUADRATIC; break;
          case 't': alg = SCC_ALG_TOPO; break;
          case 'd': alg = SCC_ALG_DATA; break;
          case 'l': alg = SCC_ALG_LINEAR; break;
          case 'h': alg = SCC_ALG_HYBRID; break;
          case 'c': alg = SCC_ALG_COMBINE; break;
          case 'b': alg = SCC_ALG_BEST; break;
          case 'a': all = true; break;
        }
        break;
      case 'w': opts.warp_size = (int)std::strtoul(optarg, nullptr, 0); break;
      case 'b': opts.block_size = (int)std::strtoul(optarg, nullptr, 0); break;
      case 'o': out_file = optarg; break;
      case 'v': verify_dir = optarg; break;
    }
  }
  if (!file) {
    std::fprintf(stderr, "usage: %s [-t] [-a q/t/d/l/h/c/b/a] [-b block] [-o labels.txt] [-v verify_dir] -f graph\n", argv[0]);
    return 1;
  }
  std::printf("loading graph...\n");
  scc_host_csr g;
  if (scc_load(file, 0, &g) != SCC_OK) {
    std::fprintf(stderr, "error: %s\n", scc_last_error());
    return 1;
  }
  std::printf("    ->nodes: %u\n", g.n);
  std::printf("    ->edges: %u\n", g.nnz_header);
  if (tarjan) {
    std::printf("tarjan decomposition...\n");
    uint32_t nscc = 0;
    double secs = 0;
    if (scc_tarjan(&g, nullptr, &nscc, &secs) != SCC_OK) {
      std::fprintf(stderr, "error: %s\n", scc_last_error());
      return 1;
    }
    std::printf("    ->count of SCC: %u\n", nscc);
    std::printf("    ->time: %f\n", secs);
  }
  scc_ctx *ctx = nullptr;
  if (scc_ctx_create(0, &opts, &ctx) != SCC_OK || scc_ctx_upload(ctx, &g) != SCC_OK) {
    std::fprintf(stderr, "error: %s\n", scc_last_error());
    return 1;
  }
  int rc = 0;
  std::vector<uint32_t> labels;
  if (all) {
    for (int a = SCC_ALG_QUADRATIC; a <= SCC_ALG_BEST && rc == 0; ++a)
      rc = compute(ctx, opts, a, g.n, (out_file || verify_dir) ? &labels : nullptr);
  } else {
    rc = compute(ctx, opts, alg, g.n, (out_file || verify_dir) ? &labels : nullptr);
  }
  if (rc == 0 && verify_dir) rc = write_verify(verify_dir, g.n, labels);
  if (rc == 0 && out_file) {
    FILE *f = std::fopen(out_file, "w");
    if (!f) {
      std::fprintf(stderr, "error: cannot write %s\n", out_file);
      rc = 1;
    } else {
      for (uint32_t v = 1; v <= g.n; ++v) std::fprintf(f, "%u %u\n", v, labels[v]);
      std::fclose(f);
    }
  }
  scc_ctx_destroy(ctx);
  scc_host_csr_free(&g);
  return rc;
}
