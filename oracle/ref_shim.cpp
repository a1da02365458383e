// C-linkage shim over the reference's own host code (load.cpp, tarjan.cpp,
// timing.cpp compiled unmodified from the reference tree by oracle/Makefile
// into oracle/_ref/).  TEST INFRASTRUCTURE ONLY: used by tests/ and by
// bench.py's reference / cpu_baseline legs, never by the product.
#include <cstdlib>
#include <string>
#include <utility>

#include "load.h"
#include "tarjan.h"

extern "C" int ref_tarjan(unsigned m, unsigned n, unsigned *edges, unsigned *nodes, unsigned *count, float *secs) {
  std::pair<unsigned, float> r = TR_Decomposition(m, n, edges, nodes);
  *count = r.first;
  *secs = r.second;
  return 0;
}

extern "C" int ref_load(const char *file, unsigned *n, unsigned *nnz, unsigned **nodes, unsigned **edges,
                        unsigned **nodesT, unsigned **edgesT) {
  std::string f(file);
  return load(&f[0], false, n, nnz, nodes, edges, nodesT, edgesT, nullptr, nullptr) ? 0 : 1;
}

extern "C" void ref_free(void *p) { std::free(p); }
