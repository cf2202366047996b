// Allocation-free flow-rate reduction (dns_flow_sums_static).
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured, hosts that hand this library a fixed memory budget and
// forbid device allocation after start-up, or allocator-managed embeddings
// where an extra cudaMalloc would fragment or overrun the pool.  For them this
// file offers the constant-flow-rate reduction (the reference's encalc2
// momentum / mass sums and the force they set) over a state the caller already
// holds on the device, using for its per-block partial sums a fixed scratch
// array compiled into the library instead of an allocation.
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/dns_embed.h"
#include "kernels.h"

using namespace dns;

// 262144 partial pairs = 4 MiB: enough for the reduction grid of the
// 384 x 192 x 115 channel (about 169k blocks); every GPU that loads the
// library holds this array until the process exits.
static constexpr long kStaticPairs = 262144;
static __device__ __align__(256) double g_flow_scratch[2 * kStaticPairs];

namespace {

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int static_fail(int code, const std::string &m) {
  dns::set_last_error(m);  // reported by dns_last_error()
  return code;
}

// Device address of the scratch array on the current device.  The array's
// host-side name is only a stand-in, so the address is looked up once per
// device with that device current.
int scratch_address(double **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return static_fail(DNS_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return static_fail(DNS_EINVAL, "device ordinal beyond the scratch table");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_flow_scratch);
    if (e != cudaSuccess || !p)
      return static_fail(DNS_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return DNS_OK;
}

}  // namespace

extern "C" int dns_flow_sums_static(const dns_params *p, const double *fc, const double *ff, double *out4,
                                    void *cuda_stream) {
  if (!p || !fc || !ff || !out4) return static_fail(DNS_EINVAL, "null argument");
  dns_geometry g;
  int rc = dns_geometry_of(p, &g);
  if (rc) return static_fail(rc, "invalid parameters");
  const Dims d{g.nx, g.ny, g.nzc, g.nxf, g.nyf, g.zdf, p->zds, g.gr, g.nzs};
  const LaunchShape s = make_shape(d);
  const long need = flow_sums_pairs(d, s);
  if (need > kStaticPairs)
    return static_fail(DNS_EINVAL, "domain needs " + std::to_string(need) + " reduction slots; the static scratch holds " +
                                       std::to_string(kStaticPairs));
  cudaError_t e = cudaSetDevice(p->device);
  if (e != cudaSuccess) return static_fail(DNS_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  double *scratch = nullptr;
  if ((rc = scratch_address(&scratch))) return rc;
  const StepParams sp{g.omega_c, g.omega_f, p->ub, p->force_const, p->forcing == DNS_FORCING_CFR ? 1 : 0};
  // every partial slot read by the finalize step is written by this call's
  // reduction blocks first, so nothing in the scratch needs clearing
  launch_flow_sums_scratch(fc, ff, reinterpret_cast<DevState *>(out4), scratch, d, s, sp,
                           static_cast<cudaStream_t>(cuda_stream));
  e = cudaGetLastError();
  if (e != cudaSuccess) return static_fail(DNS_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  return DNS_OK;
}
