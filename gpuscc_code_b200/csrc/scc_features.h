// Graph statistics fed to the strategy network (16 floats per graph).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "scc_engine.h"

namespace sccb {

constexpr int kFeatures = 16;

// Device scratch that graph_features needs for an n-vertex graph.
size_t features_scratch_bytes(uint32_t n);
// Computes the features of the device graph g on stream st (synchronises it).
// f[0] log2 n, f[1] log2(m+1), f[2] mean out-degree, f[3] log2(1+var), f[4]
// log2(1+max out-degree), f[5] log2(1+max in-degree), f[6..8] fraction with
// out-, in-, or either degree 0 (the first trim-1 sweep's yield), f[9..10]
// fraction with out-/in-degree 1, f[11] fraction with both degrees <= 2,
// f[12] sampled reciprocity, f[13..15] log2(1+|BFS level k|)/log2(n+1) for
// k = 1..3 from the vertex of largest total degree.
cudaError_t graph_features(const EngGraph &g, void *scratch, size_t scratch_bytes, float *feat, cudaStream_t st);
// The same in two halves: launch enqueues the kernels and the copy of the
// accumulators (features_acc_bytes of them) to host_acc (page-locked) on st
// without waiting; finish forms the features from host_acc once st has
// passed that point.  scratch may be released (stream-ordered) right after.
size_t features_acc_bytes();
cudaError_t graph_features_launch(const EngGraph &g, void *scratch, size_t scratch_bytes, void *host_acc,
                                  cudaStream_t st);
void graph_features_finish(uint32_t n, uint32_t m, const void *host_acc, float *feat);
void features_from_counts(uint32_t n, uint32_t m, unsigned long long sum_out, double sumsq_out, uint32_t max_out,
                          uint32_t max_in, uint32_t z_out, uint32_t z_in, uint32_t z_any, uint32_t one_out,
                          uint32_t one_in, uint32_t low, uint32_t recip, uint32_t recip_n, const uint32_t lvl[4],
                          float *f);

}  // namespace sccb
