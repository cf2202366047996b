// Host helpers shared by the single-channel driver (dns_api.cu) and the
// batched engine (batch_api.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/dns_embed.h"

namespace dns {

// NVTX range around one ABI call, so that a profiler's timeline (nsys, ncu
// --nvtx) groups the kernels of a step, a batch run or a file operation; a
// no-op when no tool is attached
struct Range {
  explicit Range(const char *name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range &) = delete;
  Range &operator=(const Range &) = delete;
};

// wall-plane flags [nyf][nxf] of the pattern in p (-1 solid, -2 slip)
std::vector<int8_t> wall_flags(const dns_params &p, const dns_geometry &g);
// running statistics rows acc[nz_profile][kStatRow] (kernels.h) -> out[DNS_NSTAT][nz_profile]
void stats_from_acc(const dns_geometry &g, const double *acc, double *out, long *nsamples);
// record msg for dns_last_error() and return code
int fail_with(int code, const std::string &msg);

}  // namespace dns
