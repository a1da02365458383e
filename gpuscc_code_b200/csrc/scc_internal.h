// Library-internal helpers shared by the host translation units.
#pragma once

#include <cstdint>

#include "scc_capi.h"

namespace sccb {

// Records a printf-style message as this thread's last error; returns code.
int set_error(int code, const char *fmt, ...);
void clear_error();
// Validates engine options (every solve entry point accepts the same set).
int check_opts(const scc_opts *o);
// Binding and segment table without the device checks, for graphs this
// library packed or validated itself (the request server).
int ctx_bind_unchecked(scc_ctx *c, const scc_dev_csr *g);
int ctx_set_segments_unchecked(scc_ctx *c, uint32_t nseg, const uint32_t *seg_first);

// 1-based pairs -> reference-layout CSR + transpose (sorted, deduplicated).
int build_csr(uint32_t n, uint64_t ne, const uint32_t *src, const uint32_t *dst, bool drop_self, scc_host_csr *out);

}  // namespace sccb
#include <vector>

#include "scc_gen.h"
namespace sccb {

// Per-graph parameters of a batch (deterministic in the arguments): type
// ER / R-MAT 50/50, n log-uniform in [n_lo, n_hi], average out-degree
// uniform in [deg_lo, deg_hi] (milli-units), per-graph seed.
int plan_batch(uint32_t count, uint32_t n_lo, uint32_t n_hi, uint32_t deg_lo_milli, uint32_t deg_hi_milli,
               uint64_t seed, std::vector<sccg::BatchGraph> *plan);

}  // namespace sccb
