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

int static_fail(int code, const std::string &m) {
  dns::set_last_error(m);  // reported by dns_last_error()
  return code;
}

// Device address of the scratch array on the current device.  The array's
// host-side name is only a stand-in, so the address is asked of the runtime
// with the device current, on every call: the lookup allocates nothing, and a
// context the caller recreated (cudaDeviceReset) gets the array's new address
// instead of a stale one.  The first lookup on a device may load the library's
// device code, which is why the first call must precede any stream capture.
int scratch_address(double **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_flow_scratch);
  if (e != cudaSuccess || !p)
    return static_fail(DNS_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = static_cast<double *>(p);
  return DNS_OK;
}

// Makes p->device current for the call and puts the caller's device back.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int dev) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int dns_flow_sums_static(const dns_params *p, const double *fc, const double *ff, double *out4,
                                    void *cuda_stream) {
  if (!p || !fc || !ff || !out4) return static_fail(DNS_EINVAL, "null argument");
  if (p->precision != DNS_FP64)
    return static_fail(DNS_EINVAL, "dns_flow_sums_static reads FP64 populations: params.precision must be DNS_FP64");
  dns_geometry g;
  const int rc = dns_geometry_of(p, &g);
  if (rc) return rc;  // dns_geometry_of has recorded which parameter is wrong
  const Dims d{g.nx, g.ny, g.nzc, g.nxf, g.nyf, g.zdf, p->zds, g.gr, g.nzs};
  const LaunchShape s = make_shape(d);
  const long need = flow_sums_pairs(d, s);
  if (need > kStaticPairs)
    return static_fail(DNS_EINVAL, "domain needs " + std::to_string(need) + " reduction slots; the static scratch holds " +
                                       std::to_string(kStaticPairs));
  DeviceScope scope(p->device);
  if (scope.err != cudaSuccess)
    return static_fail(DNS_ECUDA, std::string("selecting the device: ") + cudaGetErrorString(scope.err));
  double *scratch = nullptr;
  if (const int e = scratch_address(&scratch)) return e;
  const StepParams sp{g.omega_c, g.omega_f, p->ub, p->force_const, p->forcing == DNS_FORCING_CFR ? 1 : 0};
  // every partial slot read by the finalize step is written by this call's
  // reduction blocks first, so nothing in the scratch needs clearing
  launch_flow_sums_scratch(fc, ff, reinterpret_cast<DevState *>(out4), scratch, d, s, sp,
                           static_cast<cudaStream_t>(cuda_stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return static_fail(DNS_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  return DNS_OK;
}
