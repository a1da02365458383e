// Library-internal helpers shared by the host translation units.
#pragma once

#include <cstdint>

#include "scc_capi.h"

namespace sccb {

// Records a printf-style message as this thread's last error; returns code.
int set_error(int code, const char *fmt, ...);
void clear_error();

// 1-based pairs -> reference-layout CSR + transpose (sorted, deduplicated).
int build_csr(uint32_t n, uint64_t ne, const uint32_t *src, const uint32_t *dst, bool drop_self, scc_host_csr *out);

}  // namespace sccb
