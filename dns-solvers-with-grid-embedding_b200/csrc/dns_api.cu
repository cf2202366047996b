// Host driver and C ABI of the grid-embedded channel solver (include/dns_embed.h).
//
// Replaces the reference main program's set-up, file I/O and step loop
// (DNS-solver-with-grid-embedding/src/dns-q-mgrd-all-patterns-xyc.c) for one
// GPU-resident domain.  All device memory is allocated in dns_create; a coarse
// step issues the kernels of kernels_f64.cu on the handle's stream.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/dns_embed.h"
#include "host.h"
#include "kernels.h"

using namespace dns;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

#define CUDA_TRY(expr)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (expr);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(DNS_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));           \
  } while (0)

constexpr int kLogCap = 1024;
constexpr int kXferChunks = 8;  // x runs per level transfer (state import / export)
constexpr int kProfSteps = 256;  // steps per chunk while profiling (bounds the event pool)

// CUDA-event timing of every launch (dns_set_profiling)
struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // pairs
  std::vector<int> cls;
  size_t used = 0;
  double ms[DNS_NKERNEL] = {0};
  long cnt[DNS_NKERNEL] = {0};
};

}  // namespace

struct dns_handle {
  dns_params p{};
  dns_geometry g{};
  Dims d{};
  LaunchShape shape{};
  PartialLayout pl{};
  StepParams sp{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  double *fc[2] = {nullptr, nullptr};  // coarse SoA, [cur] holds S
  double *ff[2] = {nullptr, nullptr};  // fine SoA (both blocks)
  double *hist = nullptr;              // [3 slots][2 walls][23][ny][nx]
  int hn = 0, hp = 1, hpp = 2;         // ring slots of levels n, p, pp
  int8_t *wflag = nullptr;             // [nyf][nxf]
  double *partials = nullptr;
  DevState *state = nullptr;
  DevLog *dlog = nullptr;              // kLogCap rows
  DevLog *hlog = nullptr;              // pinned mirror
  double *stats_acc = nullptr;         // [nz_profile][kStatRow] running statistics
  double *iface_mac = nullptr;         // FP64: interface rho, u [2][4][nyf][nxf]; FP32: corner data
  void *tke_ws = nullptr;              // statistics / budget work space (allocated on first use)
  size_t tke_ws_bytes = 0;
  double *tke_wall = nullptr;          // planar fields of the two wall planes [2][4][nyf][nxf]
  long tke_wall_gen = -1;              // wall_gen they were made from
  unsigned int *fin_counter = nullptr; // finalize's block counter
  cudaStream_t aux = nullptr;          // fine substeps and injection (lowest priority)
  cudaEvent_t ev_start = nullptr, ev_inj = nullptr, ev_fine[4] = {}, ev_if[4] = {};
  cudaEvent_t ev_xfer[kXferChunks] = {};  // one per x run of a level transfer
  bool xfer_ok = false;                // the runs overlap on the two streams
  int cur_c = 0, cur_f = 0;
  long ss = 0;                         // coarse steps since load / seed
  int tm = 0;                          // time origin of the log stamps (TSTR or restart counter)
  long sample_every = 0;
  // Wall-plane populations (the step never reads or writes them; files carry
  // them): wall_dev [2 walls][GR xdv][GR ydv][19] on the device is the primary
  // copy, which the AoS transfers fill and read without a host pass;
  // wall_lo / wall_hi mirror it on the host for the field files, refreshed
  // when stale
  double *wall_dev = nullptr;
  std::vector<double> wall_lo, wall_hi;
  bool wall_host_stale = false;
  long wall_gen = 0;                     // bumped whenever the wall planes change
  double *stage = nullptr;               // FP32 form: one level in reference AoS doubles (allocated on first use)
  Profiler prof;
};

static bool d_gr_ok(const dns_handle *h) { return h->d.gr <= 4; }

// Bracket one launch with events when profiling; returns the pair index or -1.
static int prof_begin(dns_handle *h, int cls) {
  Profiler &P = h->prof;
  if (!P.on) return -1;
  if (P.used * 2 + 2 > P.ev.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    P.ev.push_back(a);
    P.ev.push_back(b);
    P.cls.push_back(0);
  }
  const int q = (int)P.used++;
  P.cls[q] = cls;
  cudaEventRecord(P.ev[2 * q], h->stream);
  return q;
}
static void prof_end(dns_handle *h, int q) {
  if (q >= 0) cudaEventRecord(h->prof.ev[2 * q + 1], h->stream);
}
// after a stream synchronize: fold the recorded pairs into the totals
static void prof_collect(dns_handle *h) {
  Profiler &P = h->prof;
  for (size_t q = 0; q < P.used; q++) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, P.ev[2 * q], P.ev[2 * q + 1]) == cudaSuccess) {
      P.ms[P.cls[q]] += t;
      P.cnt[P.cls[q]] += 1;
    }
  }
  P.used = 0;
}
#define PROFILED(h, cls, launch)      \
  do {                                \
    const int pq_ = prof_begin(h, cls); \
    launch;                           \
    prof_end(h, pq_);                 \
  } while (0)

// ---------------------------------------------------------------- parameters
extern "C" int dns_params_default(dns_params *p) {
  if (!p) return fail(DNS_EINVAL, "null params");
  std::memset(p, 0, sizeof(*p));
  // reference src/definitions.h:34-119
  p->Rebs = 7200.0;
  p->ub = 0.0866034;
  p->zdv = 220;
  p->ydv = 256;
  p->xdv = 512;
  p->TSTR = 400;
  p->TEND = 800;
  p->CFL = 0.1;
  p->gratio = 4;
  p->zds = 10;
  p->gyplussize = 56;
  p->wyplussize = 8;
  p->gxplussize = 4;
  p->wxplussize = 4;
  p->pattern = DNS_PATTERN_RSLIP;
  p->XDIM = 1;
  p->YDIM = 1;
  p->ITER = -1;
  p->forcing = DNS_FORCING_CFR;
  p->force_const = 0.0;
  p->precision = DNS_FP64;
  p->device = 0;
  p->xdu = 512;
  p->ydu = 256;
  p->zdu = 221;
  p->fltr = 0;
  return DNS_OK;
}

extern "C" int dns_params_from_definitions(const char *path, dns_params *p) {
  if (!path || !p) return fail(DNS_EINVAL, "null argument");
  FILE *fp = std::fopen(path, "r");
  if (!fp) return fail(DNS_EIO, std::string("cannot open ") + path);
  dns_params_default(p);
  p->pattern = DNS_PATTERN_NONE;
  char line[1024];
  while (std::fgets(line, sizeof line, fp)) {
    const char *s = line;
    while (*s == ' ' || *s == '\t') s++;
    if (std::strncmp(s, "#define", 7) != 0) continue;  // commented-out switches start with //
    s += 7;
    char name[128] = {0}, val[256] = {0};
    if (std::sscanf(s, "%127s %255s", name, val) < 1) continue;
    const std::string n(name);
    auto num = [&](double &dst) { if (val[0]) dst = std::strtod(val, nullptr); };
    auto inum = [&](int &dst) { if (val[0]) dst = (int)std::strtol(val, nullptr, 10); };
    if (n == "Rebs") num(p->Rebs);
    else if (n == "ub") num(p->ub);
    else if (n == "zdv") inum(p->zdv);
    else if (n == "ydv") inum(p->ydv);
    else if (n == "xdv") inum(p->xdv);
    else if (n == "TSTR") inum(p->TSTR);
    else if (n == "TEND") inum(p->TEND);
    else if (n == "CFL") num(p->CFL);
    else if (n == "gratio") inum(p->gratio);
    else if (n == "zds") inum(p->zds);
    else if (n == "gyplussize") inum(p->gyplussize);
    else if (n == "wyplussize") inum(p->wyplussize);
    else if (n == "gxplussize") inum(p->gxplussize);
    else if (n == "wxplussize") inum(p->wxplussize);
    else if (n == "XDIM") inum(p->XDIM);
    else if (n == "xdu") inum(p->xdu);
    else if (n == "ydu") inum(p->ydu);
    else if (n == "zdu") inum(p->zdu);
    else if (n == "YDIM") inum(p->YDIM);
    else if (n == "ITER") p->ITER = val[0] ? std::strtol(val, nullptr, 10) : 1;
    else if (n == "RSLIP") p->pattern = DNS_PATTERN_RSLIP;
    else if (n == "PSLIP") p->pattern = DNS_PATTERN_PSLIP;
    else if (n == "SSLIP") p->pattern = DNS_PATTERN_SSLIP;
    else if (n == "FLTR") p->fltr = 1;
  }
  std::fclose(fp);
  return DNS_OK;
}

extern "C" int dns_geometry_of(const dns_params *p, dns_geometry *g) {
  if (!p || !g) return fail(DNS_EINVAL, "null argument");
  if (p->gratio < 2 || p->gratio > 4) return fail(DNS_EINVAL, "gratio must be 2, 3 or 4");
  if (p->xdv < 4 || p->ydv < 4) return fail(DNS_EINVAL, "xdv and ydv must be >= 4");
  if (p->zdv < 5) return fail(DNS_EINVAL, "zdv (coarse wall-normal nodes) must be >= 5");
  if (p->zds < p->gratio + 2 || p->zds < 4)
    return fail(DNS_EINVAL, "zds must be >= max(4, gratio + 2) (transfer planes inside the fine block)");
  if (p->pattern < DNS_PATTERN_NONE || p->pattern > DNS_PATTERN_SSLIP) return fail(DNS_EINVAL, "bad pattern");
  if (p->Rebs <= 0 || p->ub <= 0 || p->CFL <= 0) return fail(DNS_EINVAL, "Rebs, ub and CFL must be positive");
  if (p->precision != DNS_FP64 && p->precision != DNS_FP32) return fail(DNS_EINVAL, "precision must be DNS_FP64 or DNS_FP32");
  if (p->precision == DNS_FP32 && p->zds > 32) return fail(DNS_EINVAL, "the FP32 form supports zds <= 32");
  if (p->fltr != 0 && p->fltr != 1) return fail(DNS_EINVAL, "fltr must be 0 or 1");
  if (p->fltr && (p->gratio != 4 || p->zds < 7))
    return fail(DNS_EINVAL,
                "the filtered transfer (FLTR) needs gratio 4 (the reference's 5-plane stencil array) and zds >= 7");
  // the kernels index one population array with 32-bit offsets: every
  // population array (coarse nzc x ny x nx, fine 2 zds x nyf x nxf) must hold
  // fewer than 2^31 nodes (a bound HBM reaches first: 2^31 nodes are 326 GB of
  // FP64 populations per lattice)
  if ((long long)p->gratio * p->xdv > (1LL << 20) || (long long)p->gratio * p->ydv > (1LL << 20) ||
      (long long)p->zdv * p->ydv * p->xdv >= (1LL << 31) ||
      2LL * p->zds * p->gratio * p->ydv * p->gratio * p->xdv >= (1LL << 31))
    return fail(DNS_EINVAL, "grid too large: a population array must hold fewer than 2^31 nodes");
  std::memset(g, 0, sizeof(*g));
  const int GR = p->gratio;
  g->gr = GR;
  g->nx = p->xdv;
  g->ny = p->ydv;
  g->nzc = p->zdv;
  g->nxf = GR * p->xdv;
  g->nyf = GR * p->ydv;
  g->zdf = p->zds + 1;
  // dns-q-mgrd-all-patterns-xyc.c:155
  g->nzs = 2 * g->zdf + GR * (g->nzc - 4) + GR - 1;
  g->nz_profile = 2 * g->zdf + g->nzc - 4;
  // :439-451, evaluated in the same order
  double utime = ((double)(0.5 * (g->nzs - 2.) / p->CFL)) / ((double)(GR));
  g->utime = (int)utime;
  double tauf = (3. / p->Rebs) * p->ub * (g->nzs - 2.) + 0.5;
  double tauc = (1. / ((double)GR)) * (3. / p->Rebs) * p->ub * (g->nzs - 2.) + 0.5;
  g->omega_f = 1. / tauf;
  g->omega_c = 1. / tauc;
  g->updates_per_step = (long long)p->xdv * p->ydv * p->zdv +
                        2LL * GR * ((long long)GR * p->xdv) * ((long long)GR * p->ydv) * p->zds;
  Dims d{g->nx, g->ny, g->nzc, g->nxf, g->nyf, g->zdf, p->zds, GR, g->nzs};
  LaunchShape s = make_shape(d);
  PartialLayout pl = partial_layout(d, s);
  const long long nc = 19LL * g->nzc * g->ny * g->nx, nf = 19LL * 2 * p->zds * g->nyf * g->nxf;
  const long long esz = p->precision == DNS_FP32 ? 4 : 8;  // bytes per stored population
  const long long mac = esz == 4 ? 2LL * 23 * g->ny * g->nx * 4 : 8LL * g->nyf * g->nxf;  // elements of esz
  g->device_bytes = esz * (2 * nc + 2 * nf + 3LL * 2 * 23 * g->ny * g->nx + mac) +
                    8 * (pl.total + (long long)kStatRow * g->nz_profile + 2LL * 19 * g->nyf * g->nxf) +
                    (long long)g->nyf * g->nxf + (long long)kLogCap * sizeof(DevLog) + sizeof(DevState);
  return DNS_OK;
}

// wall flags: solid_init.c:46-69, slip_ridges_init.c:35-66, slip_posts_init.c:45-117,
// slip_spanwise_init.c:34-66 (global index; writes past the span are dropped)
std::vector<int8_t> dns::wall_flags(const dns_params &p, const dns_geometry &g) {
  std::vector<int8_t> sx(g.nxf, -1), sy(g.nyf, -1), w((size_t)g.nyf * g.nxf, -1);
  const bool ys = p.pattern == DNS_PATTERN_RSLIP || p.pattern == DNS_PATTERN_PSLIP;
  const bool xs = p.pattern == DNS_PATTERN_SSLIP || p.pattern == DNS_PATTERN_PSLIP;
  if (ys)
    for (int j = p.wyplussize / 2; j < g.nyf; j += p.gyplussize + p.wyplussize)
      for (int a = 0; a < p.gyplussize && j + a < g.nyf; a++) sy[j + a] = -2;
  if (xs)
    for (int i = p.wxplussize / 2; i < g.nxf; i += p.gxplussize + p.wxplussize)
      for (int a = 0; a < p.gxplussize && i + a < g.nxf; a++) sx[i + a] = -2;
  for (int j = 0; j < g.nyf; j++)
    for (int i = 0; i < g.nxf; i++) {
      int8_t f = -1;
      if (p.pattern == DNS_PATTERN_RSLIP) f = sy[j];
      else if (p.pattern == DNS_PATTERN_SSLIP) f = sx[i];
      else if (p.pattern == DNS_PATTERN_PSLIP) f = (sx[i] == -2 || sy[j] == -2) ? -2 : -1;
      w[(size_t)j * g.nxf + i] = f;
    }
  return w;
}

// ---------------------------------------------------------------- lifecycle
extern "C" void dns_destroy(dns_handle *h) {
  if (!h) return;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int q = 0; q < 2; q++) {
    cudaFree(h->fc[q]);
    cudaFree(h->ff[q]);
  }
  cudaFree(h->hist);
  cudaFree(h->wflag);
  cudaFree(h->partials);
  cudaFree(h->state);
  cudaFree(h->dlog);
  cudaFree(h->stats_acc);
  cudaFree(h->iface_mac);
  cudaFree(h->tke_ws);
  cudaFree(h->tke_wall);
  cudaFree(h->wall_dev);
  cudaFree(h->stage);
  cudaFree(h->fin_counter);
  if (h->hlog) cudaFreeHost(h->hlog);
  for (cudaEvent_t e : h->prof.ev) cudaEventDestroy(e);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  if (h->aux) cudaStreamDestroy(h->aux);
  cudaEvent_t *evs[] = {&h->ev_start, &h->ev_inj, &h->ev_fine[0], &h->ev_fine[1], &h->ev_fine[2],
                        &h->ev_fine[3], &h->ev_if[0], &h->ev_if[1], &h->ev_if[2], &h->ev_if[3]};
  for (cudaEvent_t *e : evs)
    if (*e) cudaEventDestroy(*e);
  for (cudaEvent_t e : h->ev_xfer)
    if (e) cudaEventDestroy(e);
  delete h;
}

extern "C" int dns_create(const dns_params *p, dns_handle **out) {
  if (!p || !out) return fail(DNS_EINVAL, "null argument");
  *out = nullptr;
  dns_geometry g;
  int rc = dns_geometry_of(p, &g);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(DNS_ECUDA, "no CUDA device");
  if (p->device < 0 || p->device >= ndev) return fail(DNS_EINVAL, "device ordinal out of range");
  size_t freeb = 0, totalb = 0;
  CUDA_TRY(cudaSetDevice(p->device));
  CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  if ((long long)freeb < g.device_bytes) return fail(DNS_ENOMEM, "not enough free device memory for this channel");
  dns_handle *h = new dns_handle();
  h->p = *p;
  h->g = g;
  h->d = Dims{g.nx, g.ny, g.nzc, g.nxf, g.nyf, g.zdf, p->zds, g.gr, g.nzs};
  h->shape = make_shape(h->d);
  h->pl = partial_layout(h->d, h->shape);
  h->sp = StepParams{g.omega_c, g.omega_f, p->ub, p->force_const, p->forcing == DNS_FORCING_CFR ? 1 : 0, 0.0};
  // the FP32 form's mass partials sum deviations from w: add the weight sum once
  if (p->precision == DNS_FP32) h->sp.den_offset = encalc2_weight_sum(h->d);
  const size_t esz = p->precision == DNS_FP32 ? 4 : 8;
  h->tm = p->TSTR;
  const size_t nc = 19ull * g.nzc * g.ny * g.nx, nf = 19ull * 2 * p->zds * g.nyf * g.nxf;
  auto alloc = [&](void **ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
      dns_destroy(h);
      return fail(DNS_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return DNS_OK;
  };
  for (int q = 0; q < 2; q++) {
    if ((rc = alloc((void **)&h->fc[q], nc * esz))) return rc;
    if ((rc = alloc((void **)&h->ff[q], nf * esz))) return rc;
  }
  if ((rc = alloc((void **)&h->hist, 3ull * 2 * 23 * g.ny * g.nx * esz))) return rc;
  if ((rc = alloc((void **)&h->wflag, (size_t)g.nyf * g.nxf))) return rc;
  if ((rc = alloc((void **)&h->partials, (size_t)h->pl.total * 8))) return rc;
  if ((rc = alloc((void **)&h->state, sizeof(DevState)))) return rc;
  if ((rc = alloc((void **)&h->dlog, kLogCap * sizeof(DevLog)))) return rc;
  if ((rc = alloc((void **)&h->stats_acc, (size_t)g.nz_profile * kStatRow * 8))) return rc;
  // FP64: interface rho, u at fine nodes; FP32: corner values and derivatives (float4)
  const size_t mac_bytes = esz == 4 ? 2ull * 23 * g.ny * g.nx * 16 : 8ull * g.nyf * g.nxf * esz;
  if ((rc = alloc((void **)&h->iface_mac, mac_bytes))) return rc;
  if ((rc = alloc((void **)&h->fin_counter, 256))) return rc;
  cudaMemset(h->fin_counter, 0, 256);
  if ((rc = alloc((void **)&h->wall_dev, 2ull * g.nxf * g.nyf * 19 * 8))) return rc;
  cudaMemset(h->wall_dev, 0, 2ull * g.nxf * g.nyf * 19 * 8);
  if (cudaMallocHost((void **)&h->hlog, kLogCap * sizeof(DevLog)) != cudaSuccess) {
    dns_destroy(h);
    return fail(DNS_ENOMEM, "cudaMallocHost failed");
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    dns_destroy(h);
    return fail(DNS_ECUDA, "cudaStreamCreate failed");
  }
  h->own_stream = true;
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  bool ev_ok = cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, prio_low) == cudaSuccess;
  cudaEvent_t *evs[] = {&h->ev_start, &h->ev_inj, &h->ev_fine[0], &h->ev_fine[1], &h->ev_fine[2],
                        &h->ev_fine[3], &h->ev_if[0], &h->ev_if[1], &h->ev_if[2], &h->ev_if[3]};
  for (cudaEvent_t *e : evs) ev_ok = ev_ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
  h->xfer_ok = ev_ok;
  for (cudaEvent_t &e : h->ev_xfer)
    h->xfer_ok = h->xfer_ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
  if (!ev_ok) {
    dns_destroy(h);
    return fail(DNS_ECUDA, "stream / event creation failed");
  }
  std::vector<int8_t> wf = wall_flags(*p, g);
  cudaMemcpy(h->wflag, wf.data(), wf.size(), cudaMemcpyHostToDevice);
  cudaMemset(h->partials, 0, (size_t)h->pl.total * 8);
  cudaMemset(h->stats_acc, 0, (size_t)g.nz_profile * kStatRow * 8);
  cudaMemset(h->state, 0, sizeof(DevState));
  h->wall_lo.assign((size_t)g.nxf * g.nyf * 19, 0.0);
  h->wall_hi.assign((size_t)g.nxf * g.nyf * 19, 0.0);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    dns_destroy(h);
    return fail(DNS_ECUDA, cudaGetErrorString(e));
  }
  *out = h;
  return DNS_OK;
}

extern "C" int dns_set_stream(dns_handle *h, void *cuda_stream) {
  if (!h) return fail(DNS_EINVAL, "null handle");
  CUDA_TRY(cudaSetDevice(h->p.device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (cuda_stream) {
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)cuda_stream;
    h->own_stream = false;
  } else if (!h->own_stream) {
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return DNS_OK;
}

extern "C" int dns_get_geometry(const dns_handle *h, dns_geometry *g) {
  if (!h || !g) return fail(DNS_EINVAL, "null argument");
  *g = h->g;
  return DNS_OK;
}

// ---------------------------------------------------------------- state transfer
// device SoA <-> reference AoS of one level, staged through the idle ping-pong buffer
static bool is_f32(const dns_handle *h) { return h->p.precision == DNS_FP32; }
static float *F(double *p) { return reinterpret_cast<float *>(p); }

// the host mirror of the wall planes, brought up to date from the device
static int sync_wall_host(dns_handle *h) {
  if (!h->wall_host_stale) return DNS_OK;
  const size_t n = h->wall_lo.size();
  CUDA_TRY(cudaMemcpyAsync(h->wall_lo.data(), h->wall_dev, n * 8, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaMemcpyAsync(h->wall_hi.data(), h->wall_dev + n, n * 8, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->wall_host_stale = false;
  return DNS_OK;
}

static size_t level_doubles(const dns_geometry &g, int level) {
  return level == 0 ? 19ull * g.nzc * g.ny * g.nx : 19ull * g.zdf * g.nyf * g.nxf;
}

// Device staging for one level in reference AoS doubles: the idle ping-pong
// buffer of the FP64 form (it holds as many doubles as a level with its wall
// plane: zds planes stored per block, zdf = zds + 1 in a level, and two blocks);
// for the FP32 form a buffer kept by the handle after its first use.
static int staging(dns_handle *h, int level, double **out) {
  if (!is_f32(h)) {
    *out = level == 0 ? h->fc[1 - h->cur_c] : h->ff[1 - h->cur_f];
    return DNS_OK;
  }
  if (!h->stage) {
    const size_t n = std::max(level_doubles(h->g, 0), level_doubles(h->g, 1));
    if (cudaMalloc(&h->stage, n * 8) != cudaSuccess) return fail(DNS_ENOMEM, "AoS staging buffer");
  }
  *out = h->stage;
  return DNS_OK;
}

// One level of the post-stream state: device SoA (FP64, or FP32 deviations)
// <-> reference AoS doubles on the host, through the device staging buffer:
// the transpose and the wall plane (from / into wall_dev) are device kernels,
// the host sees one copy of the whole level and one synchronisation.
// A level moves in kXferChunks runs of x indices (contiguous on the AoS side):
// the transpose of one run overlaps the host copy of another, the copies on
// the second stream back to back.
static void transpose_level(dns_handle *h, int level, double *stage, bool to_aos, int i0, int i1, cudaStream_t st) {
  const dns_geometry &g = h->g;
  const int zds = h->p.zds;
  const bool f32 = is_f32(h);
  if (level == 0) {
    if (to_aos) {
      if (f32) launch_dev_to_aos_f32(F(h->fc[h->cur_c]), stage, g.nx, g.ny, g.nzc, 0, g.nzc, g.nzc, 0, st, i0, i1);
      else launch_soa_to_aos(h->fc[h->cur_c], stage, g.nx, g.ny, g.nzc, 0, g.nzc, g.nzc, 0, st, i0, i1);
    } else {
      if (f32) launch_aos_to_dev_f32(stage, F(h->fc[h->cur_c]), g.nx, g.ny, g.nzc, 0, g.nzc, g.nzc, 0, st, i0, i1);
      else launch_aos_to_soa(stage, h->fc[h->cur_c], g.nx, g.ny, g.nzc, 0, g.nzc, g.nzc, 0, st, i0, i1);
    }
    return;
  }
  // lower block: device planes 0..zds-1 are k = 1..zdf-1; upper: zds.. are k = 0..zdf-2
  const int p0 = level == 1 ? 0 : zds, k0 = level == 1 ? 1 : 0;
  if (to_aos) {
    if (f32) launch_dev_to_aos_f32(F(h->ff[h->cur_f]), stage, g.nxf, g.nyf, 2 * zds, p0, zds, g.zdf, k0, st, i0, i1);
    else launch_soa_to_aos(h->ff[h->cur_f], stage, g.nxf, g.nyf, 2 * zds, p0, zds, g.zdf, k0, st, i0, i1);
  } else {
    if (f32) launch_aos_to_dev_f32(stage, F(h->ff[h->cur_f]), g.nxf, g.nyf, 2 * zds, p0, zds, g.zdf, k0, st, i0, i1);
    else launch_aos_to_soa(stage, h->ff[h->cur_f], g.nxf, g.nyf, 2 * zds, p0, zds, g.zdf, k0, st, i0, i1);
  }
}

static int export_level(dns_handle *h, int level, double *out) {
  const dns_geometry &g = h->g;
  double *stage = nullptr;
  int rc = staging(h, level, &stage);
  if (rc) return rc;
  const int nxl = level == 0 ? g.nx : g.nxf;
  const size_t col = level_doubles(g, level) / (size_t)nxl;  // AoS doubles per x index
  if (level > 0)
    launch_wall_plane(stage, h->wall_dev + (size_t)(level - 1) * g.nxf * g.nyf * 19, (long long)g.nxf * g.nyf,
                      g.zdf, level == 1 ? 0 : g.zdf - 1, true, h->stream);
  const int C = h->xfer_ok ? kXferChunks : 1;
  cudaStream_t cs = C > 1 ? h->aux : h->stream;
  for (int c = 0; c < C; c++) {
    const int i0 = (int)((long long)nxl * c / C), i1 = (int)((long long)nxl * (c + 1) / C);
    if (i1 <= i0) continue;
    transpose_level(h, level, stage, true, i0, i1, h->stream);
    if (C > 1) {
      CUDA_TRY(cudaEventRecord(h->ev_xfer[c], h->stream));
      CUDA_TRY(cudaStreamWaitEvent(cs, h->ev_xfer[c], 0));
    }
    CUDA_TRY(cudaMemcpyAsync(out + (size_t)i0 * col, stage + (size_t)i0 * col, (size_t)(i1 - i0) * col * 8,
                             cudaMemcpyDeviceToHost, cs));
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(cs));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DNS_OK;
}

static int import_level(dns_handle *h, int level, const double *in) {
  const dns_geometry &g = h->g;
  double *stage = nullptr;
  int rc = staging(h, level, &stage);
  if (rc) return rc;
  const int nxl = level == 0 ? g.nx : g.nxf;
  const size_t col = level_doubles(g, level) / (size_t)nxl;
  const int C = h->xfer_ok ? kXferChunks : 1;
  cudaStream_t cs = C > 1 ? h->aux : h->stream;
  if (C > 1) {  // the copies follow whatever the handle's stream has queued
    CUDA_TRY(cudaEventRecord(h->ev_start, h->stream));
    CUDA_TRY(cudaStreamWaitEvent(cs, h->ev_start, 0));
  }
  for (int c = 0; c < C; c++) {
    const int i0 = (int)((long long)nxl * c / C), i1 = (int)((long long)nxl * (c + 1) / C);
    if (i1 <= i0) continue;
    CUDA_TRY(cudaMemcpyAsync(stage + (size_t)i0 * col, in + (size_t)i0 * col, (size_t)(i1 - i0) * col * 8,
                             cudaMemcpyHostToDevice, cs));
    if (C > 1) {
      CUDA_TRY(cudaEventRecord(h->ev_xfer[c], cs));
      CUDA_TRY(cudaStreamWaitEvent(h->stream, h->ev_xfer[c], 0));
    }
    transpose_level(h, level, stage, false, i0, i1, h->stream);
  }
  if (level > 0) {
    launch_wall_plane(stage, h->wall_dev + (size_t)(level - 1) * g.nxf * g.nyf * 19, (long long)g.nxf * g.nyf,
                      g.zdf, level == 1 ? 0 : g.zdf - 1, false, h->stream);
    h->wall_host_stale = true;
    h->wall_gen++;
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DNS_OK;
}

// history: device [slot][wall][23][ny][nx] <-> file order [level][wall][nx][ny][23]
static int export_history(dns_handle *h, double *out) {
  const dns_geometry &g = h->g;
  const size_t plane = (size_t)g.ny * g.nx, per = 2 * 23 * plane;
  std::vector<double> tmp(3 * per);
  if (is_f32(h)) {
    // float [drho, u, fneq] -> reference [rho, u, fneq]
    std::vector<float> t32(3 * per);
    CUDA_TRY(cudaMemcpyAsync(t32.data(), h->hist, 3 * per * 4, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (size_t q = 0; q < t32.size(); q++) tmp[q] = t32[q];
    for (size_t sl = 0; sl < 6; sl++)
      for (size_t q = 0; q < plane; q++) tmp[sl * 23 * plane + q] += 1.0;
  } else {
    CUDA_TRY(cudaMemcpyAsync(tmp.data(), h->hist, 3 * per * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  const int slots[3] = {h->hn, h->hp, h->hpp};
  for (int l = 0; l < 3; l++)
    for (int w = 0; w < 2; w++)
      for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
          for (int b = 0; b < 23; b++)
            out[((((size_t)l * 2 + w) * g.nx + i) * g.ny + j) * 23 + b] =
                tmp[(((size_t)slots[l] * 2 + w) * 23 + b) * plane + (size_t)j * g.nx + i];
  return DNS_OK;
}

static int import_history(dns_handle *h, const double *in) {
  const dns_geometry &g = h->g;
  const size_t plane = (size_t)g.ny * g.nx, per = 2 * 23 * plane;
  std::vector<double> tmp(3 * per);
  for (int l = 0; l < 3; l++)
    for (int w = 0; w < 2; w++)
      for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
          for (int b = 0; b < 23; b++)
            tmp[(((size_t)l * 2 + w) * 23 + b) * plane + (size_t)j * g.nx + i] =
                in[((((size_t)l * 2 + w) * g.nx + i) * g.ny + j) * 23 + b];
  if (is_f32(h)) {
    std::vector<float> t32(3 * per);
    for (size_t sl = 0; sl < 6; sl++)
      for (size_t q = 0; q < plane; q++) tmp[sl * 23 * plane + q] -= 1.0;
    for (size_t q = 0; q < t32.size(); q++) t32[q] = (float)tmp[q];
    CUDA_TRY(cudaMemcpyAsync(h->hist, t32.data(), 3 * per * 4, cudaMemcpyHostToDevice, h->stream));
  } else {
    CUDA_TRY(cudaMemcpyAsync(h->hist, tmp.data(), 3 * per * 8, cudaMemcpyHostToDevice, h->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->hn = 0;
  h->hp = 1;
  h->hpp = 2;
  return DNS_OK;
}

// encalc2 of the stored state -> device scalars (force for the next step)
static int refresh_flow(dns_handle *h, double force_file) {
  DevState st{force_file, 0., 0., 0.};
  CUDA_TRY(cudaMemcpyAsync(h->state, &st, sizeof st, cudaMemcpyHostToDevice, h->stream));
  if (is_f32(h))
    launch_flow_sums_f32(F(h->fc[h->cur_c]), F(h->ff[h->cur_f]), h->state, h->partials, h->pl, h->d, h->shape, h->sp,
                         h->stream);
  else
    launch_flow_sums_f64(h->fc[h->cur_c], h->ff[h->cur_f], h->state, h->partials, h->pl, h->d, h->shape, h->sp,
                         h->stream);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DNS_OK;
}

extern "C" int dns_export_state(dns_handle *h, int level, double *aos_out) {
  if (!h || !aos_out || level < 0 || level > 2) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  return export_level(h, level, aos_out);
}

extern "C" int dns_import_state(dns_handle *h, int level, const double *aos_in) {
  if (!h || !aos_in || level < 0 || level > 2) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  int rc = import_level(h, level, aos_in);
  if (rc) return rc;
  return refresh_flow(h, h->p.force_const);
}

extern "C" int dns_export_history(dns_handle *h, double *out) {
  if (!h || !out) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  return export_history(h, out);
}

extern "C" int dns_import_history(dns_handle *h, const double *in) {
  if (!h || !in) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  return import_history(h, in);
}

extern "C" int dns_get_force(dns_handle *h, double *force) {
  if (!h || !force) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  DevState st;
  CUDA_TRY(cudaMemcpyAsync(&st, h->state, sizeof st, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  *force = st.force;
  return DNS_OK;
}

extern "C" int dns_init_seeded(dns_handle *h, uint64_t seed, double uc, double amp) {
  Range range("dns_init_seeded");
  if (!h) return fail(DNS_EINVAL, "null handle");
  CUDA_TRY(cudaSetDevice(h->p.device));
  h->cur_c = 0;
  h->cur_f = 0;
  h->hn = 0;
  h->hp = 1;
  h->hpp = 2;
  if (is_f32(h))
    launch_seed_f32(F(h->fc[0]), F(h->ff[0]), F(h->hist), h->d, seed, uc, amp, h->stream);
  else
    launch_seed_f64(h->fc[0], h->ff[0], h->hist, h->d, seed, uc, amp, h->stream);
  CUDA_TRY(cudaGetLastError());
  std::fill(h->wall_lo.begin(), h->wall_lo.end(), 0.0);
  std::fill(h->wall_hi.begin(), h->wall_hi.end(), 0.0);
  CUDA_TRY(cudaMemsetAsync(h->wall_dev, 0, 2 * h->wall_lo.size() * 8, h->stream));
  h->wall_host_stale = false;
  h->wall_gen++;
  h->ss = 0;
  h->tm = h->p.TSTR;
  return refresh_flow(h, h->p.forcing == DNS_FORCING_CFR ? 0.0 : h->p.force_const);
}

// ---------------------------------------------------------------- restart files
static int read_file(const std::string &fn, double *dst, size_t n, size_t skip = 0) {
  FILE *fp = std::fopen(fn.c_str(), "rb");
  if (!fp) return fail(DNS_EIO, "cannot open " + fn);
  if (skip && std::fseek(fp, (long)(skip * 8), SEEK_SET) != 0) {
    std::fclose(fp);
    return fail(DNS_EIO, "seek failed in " + fn);
  }
  size_t got = std::fread(dst, 8, n, fp);
  std::fclose(fp);
  if (got != n) return fail(DNS_EIO, "short read in " + fn);
  return DNS_OK;
}

static std::string cname(const char *dir, const char *base, int cntr) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%s.%.4d", base, cntr);
  return std::string(dir) + "/" + buf;
}

// A restart file shorter than its format for this grid is truncated (or was
// written for a smaller grid).  The reference's MPI-IO reads (main
// :1003-1163) would return short counts unchecked and run on from stale
// memory; this load refuses.  A longer file is read like the reference reads
// it, from the front (its writer opens without truncating, so a file that
// replaced a larger one keeps the old tail).
static int check_size(const std::string &fn, size_t n_doubles) {
  FILE *fp = std::fopen(fn.c_str(), "rb");
  if (!fp) return fail(DNS_EIO, "cannot open " + fn);
  long sz = -1;
  if (std::fseek(fp, 0, SEEK_END) == 0) sz = std::ftell(fp);
  std::fclose(fp);
  if (sz < 0) return fail(DNS_EIO, "cannot size " + fn);
  if ((size_t)sz < n_doubles * 8)
    return fail(DNS_EIO, fn + " is truncated: " + std::to_string(sz) + " bytes, this grid's file has " +
                             std::to_string(n_doubles * 8));
  return DNS_OK;
}

extern "C" int dns_load_restart(dns_handle *h, const char *dir, int cntr) {
  Range range("dns_load_restart");
  if (!h || !dir) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  const dns_geometry &g = h->g;
  int rc;
  // every file is sized before anything is imported, so a failed load leaves
  // the state as it was
  {
    const size_t nc = 19ull * g.nzc * g.ny * g.nx, nf = 19ull * g.zdf * g.nyf * g.nxf;
    const size_t nh = 3ull * g.nx * g.ny * 23;
    const struct { const char *base; size_t n; } files[6] = {
        {"lbf-c", 2 * nc}, {"lbf-slf", 2 * nf}, {"lbf-suf", 2 * nf}, {"force", 1}, {"lbf-lin", nh}, {"lbf-uin", nh}};
    for (const auto &f : files)
      if ((rc = check_size(cname(dir, f.base, cntr), f.n))) return rc;
  }
  std::vector<double> buf(19ull * std::max((size_t)g.nzc * g.ny * g.nx, (size_t)g.zdf * g.nyf * g.nxf));
  // lbf-c: [ftemp | f]; the post-stream state is the first half (:1006-1016)
  if ((rc = read_file(cname(dir, "lbf-c", cntr), buf.data(), 19ull * g.nzc * g.ny * g.nx))) return rc;
  if ((rc = import_level(h, 0, buf.data()))) return rc;
  if ((rc = read_file(cname(dir, "lbf-slf", cntr), buf.data(), 19ull * g.zdf * g.nyf * g.nxf))) return rc;
  if ((rc = import_level(h, 1, buf.data()))) return rc;
  if ((rc = read_file(cname(dir, "lbf-suf", cntr), buf.data(), 19ull * g.zdf * g.nyf * g.nxf))) return rc;
  if ((rc = import_level(h, 2, buf.data()))) return rc;
  double force = 0.;
  if ((rc = read_file(cname(dir, "force", cntr), &force, 1))) return rc;
  const size_t per = (size_t)g.nx * g.ny * 23;
  std::vector<double> hist(3 * 2 * per), one(3 * per);
  const char *hn[2] = {"lbf-lin", "lbf-uin"};
  for (int w = 0; w < 2; w++) {
    if ((rc = read_file(cname(dir, hn[w], cntr), one.data(), 3 * per))) return rc;
    for (int l = 0; l < 3; l++) std::memcpy(hist.data() + ((size_t)l * 2 + w) * per, one.data() + l * per, per * 8);
  }
  if ((rc = import_history(h, hist.data()))) return rc;
  h->ss = 0;
  h->tm = cntr;
  if ((rc = refresh_flow(h, h->p.forcing == DNS_FORCING_CFR ? force : h->p.force_const))) return rc;
  if (h->p.forcing == DNS_FORCING_CFR) {
    // The reference recomputes the force with encalc2 at the top of its loop;
    // a restart it (or this solver) wrote holds that same value, up to the
    // association of the domain sum.  When the file agrees to rounding, keep
    // the file's bits so a resumed run continues exactly.
    DevState st;
    CUDA_TRY(cudaMemcpyAsync(&st, h->state, sizeof st, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (std::fabs(st.force - force) <= 1e-13 * h->p.ub) {
      st.force = force;
      CUDA_TRY(cudaMemcpyAsync(h->state, &st, sizeof st, cudaMemcpyHostToDevice, h->stream));
      CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
  }
  return DNS_OK;
}

static int write_file(const std::string &fn, const double *a, size_t n, int copies) {
  FILE *fp = std::fopen(fn.c_str(), "wb");
  if (!fp) return fail(DNS_EIO, "cannot create " + fn);
  bool ok = true;
  for (int c = 0; c < copies; c++) ok = ok && std::fwrite(a, 8, n, fp) == n;
  ok = (std::fclose(fp) == 0) && ok;
  return ok ? DNS_OK : fail(DNS_EIO, "short write in " + fn);
}

extern "C" int dns_write_restart(dns_handle *h, const char *dir, int cntr) {
  Range range("dns_write_restart");
  if (!h || !dir) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  const dns_geometry &g = h->g;
  std::vector<double> buf(19ull * std::max((size_t)g.nzc * g.ny * g.nx, (size_t)g.zdf * g.nyf * g.nxf));
  int rc;
  // [ftemp | f]: the second half is the reference's scratch lattice, which its
  // step overwrites before reading; the post-stream state fills both halves
  const char *names[3] = {"lbf-c", "lbf-slf", "lbf-suf"};
  for (int lv = 0; lv < 3; lv++) {
    if ((rc = export_level(h, lv, buf.data()))) return rc;
    const size_t n = lv == 0 ? 19ull * g.nzc * g.ny * g.nx : 19ull * g.zdf * g.nyf * g.nxf;
    if ((rc = write_file(cname(dir, names[lv], cntr), buf.data(), n, 2))) return rc;
  }
  double force;
  if ((rc = dns_get_force(h, &force))) return rc;
  if ((rc = write_file(cname(dir, "force", cntr), &force, 1, 1))) return rc;
  const size_t per = (size_t)g.nx * g.ny * 23;
  std::vector<double> hist(3 * 2 * per), one(3 * per);
  if ((rc = export_history(h, hist.data()))) return rc;
  const char *hn[2] = {"lbf-lin", "lbf-uin"};
  for (int w = 0; w < 2; w++) {
    for (int l = 0; l < 3; l++) std::memcpy(one.data() + l * per, hist.data() + ((size_t)l * 2 + w) * per, per * 8);
    if ((rc = write_file(cname(dir, hn[w], cntr), one.data(), 3 * per, 1))) return rc;
  }
  return DNS_OK;
}

// ---------------------------------------------------------------- field output
// vel_print's moments of a wall plane held on the host (n nodes): vel[n][3], den[n]
static void wall_plane_fields(const std::vector<double> &wall, size_t n, double *vel, double *den) {
  static const double EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0};
  static const double EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
  static const double EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  for (size_t c = 0; c < n; c++) {
    const double *f = wall.data() + c * 19;
    double ux = 0., uy = 0., uz = 0., dens = 0.;
    for (int a = 0; a < 19; a++) {
      ux += EX[a] * f[a];
      uy += EY[a] * f[a];
      uz += EZ[a] * f[a];
      dens += f[a];
    }
    if (dens > 0.) {
      ux /= dens;
      uy /= dens;
      uz /= dens;
    } else {
      ux = uy = uz = dens = 0.;
    }
    vel[c * 3] = ux;
    vel[c * 3 + 1] = uy;
    vel[c * 3 + 2] = uz;
    den[c] = dens;
  }
}

// vel_print.c:15-275 (called by main at :1342): per level, u = (sum E f) / rho
// and rho = sum f of the post-stream state, summed in population order, zero
// where rho <= 0; vel-* (nx, ny, nz, 3) and den-* (nx, ny, nz), C order,
// native doubles.  The moments are formed on the device (4 of the 19 values per
// node cross to the host); the wall planes, kept on the host, are done here.
extern "C" int dns_write_fields(dns_handle *h, const char *dir, int cntr) {
  Range range("dns_write_fields");
  if (!h || !dir) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  if (const int r = sync_wall_host(h)) return r;
  const dns_geometry &g = h->g;
  const int zds = h->p.zds;
  const size_t nmax = std::max((size_t)g.nx * g.ny * g.nzc, (size_t)g.nxf * g.nyf * g.zdf);
  double *dvel = nullptr, *dden = nullptr;
  if (cudaMalloc(&dvel, nmax * 3 * 8) != cudaSuccess) return fail(DNS_ENOMEM, "field staging");
  if (cudaMalloc(&dden, nmax * 8) != cudaSuccess) {
    cudaFree(dvel);
    return fail(DNS_ENOMEM, "field staging");
  }
  std::vector<double> vel(nmax * 3), den(nmax);
  const char *names[3] = {"c", "slf", "suf"};
  int rc = DNS_OK;
  for (int lv = 0; lv < 3 && rc == DNS_OK; lv++) {
    const int nx = lv == 0 ? g.nx : g.nxf, ny = lv == 0 ? g.ny : g.nyf, nz = lv == 0 ? g.nzc : g.zdf;
    const size_t n = (size_t)nx * ny * nz;
    const int P = lv == 0 ? g.nzc : 2 * zds, p0 = lv == 2 ? zds : 0, np = lv == 0 ? g.nzc : zds;
    const int k0 = lv == 1 ? 1 : 0;
    if (is_f32(h))
      launch_fields_f32(F(lv == 0 ? h->fc[h->cur_c] : h->ff[h->cur_f]), dvel, dden, nx, ny, P, p0, np, nz, k0,
                        h->stream);
    else
      launch_fields_f64(lv == 0 ? h->fc[h->cur_c] : h->ff[h->cur_f], dvel, dden, nx, ny, P, p0, np, nz, k0,
                        h->stream);
    cudaError_t e = cudaMemcpyAsync(vel.data(), dvel, n * 3 * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(den.data(), dden, n * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      rc = fail(DNS_ECUDA, cudaGetErrorString(e));
      break;
    }
    if (lv > 0) {
      const size_t npl = (size_t)nx * ny;
      std::vector<double> wv(npl * 3), wd(npl);
      wall_plane_fields(lv == 1 ? h->wall_lo : h->wall_hi, npl, wv.data(), wd.data());
      const int kw = lv == 1 ? 0 : g.zdf - 1;
      for (size_t c = 0; c < npl; c++) {
        const size_t o = c * nz + kw;
        std::memcpy(&vel[o * 3], &wv[c * 3], 3 * 8);
        den[o] = wd[c];
      }
    }
    char base[16];
    std::snprintf(base, sizeof base, "vel-%s", names[lv]);
    rc = write_file(cname(dir, base, cntr), vel.data(), n * 3, 1);
    if (rc == DNS_OK) {
      std::snprintf(base, sizeof base, "den-%s", names[lv]);
      rc = write_file(cname(dir, base, cntr), den.data(), n, 1);
    }
  }
  cudaFree(dvel);
  cudaFree(dden);
  return rc;
}

// ---------------------------------------------------------------- statistics / budget
static size_t level_nodes(const dns_geometry &g, int lv) {
  return lv == 0 ? (size_t)g.nx * g.ny * g.nzc : (size_t)g.nxf * g.nyf * g.zdf;
}

// The fields of the current state as planar device arrays q[l] = [4][nz][ny][nx]
// (u, v, w, den / 3; the moments vel_print writes), the wall planes from the
// host copies.
static int fields_planar(dns_handle *h, double *const q[3]) {
  const dns_geometry &g = h->g;
  const int zds = h->p.zds;
  if (const int r = sync_wall_host(h)) return r;
  for (int lv = 0; lv < 3; lv++) {
    const int nx = lv == 0 ? g.nx : g.nxf, ny = lv == 0 ? g.ny : g.nyf, nz = lv == 0 ? g.nzc : g.zdf;
    const int P = lv == 0 ? g.nzc : 2 * zds, p0 = lv == 2 ? zds : 0, np = lv == 0 ? g.nzc : zds;
    const int k0 = lv == 1 ? 1 : 0;
    if (is_f32(h))
      launch_fields_planar_f32(F(lv == 0 ? h->fc[h->cur_c] : h->ff[h->cur_f]), q[lv], nx, ny, P, p0, np, nz, k0,
                               h->stream);
    else
      launch_fields_planar_f64(lv == 0 ? h->fc[h->cur_c] : h->ff[h->cur_f], q[lv], nx, ny, P, p0, np, nz, k0,
                               h->stream);
    CUDA_TRY(cudaGetLastError());
  }
  // wall planes: lower k = 0, upper k = zdf - 1, [c][j][i] per plane; made on
  // the host from the wall populations when those change, kept on the device
  const size_t npl = (size_t)g.nxf * g.nyf, lvl = level_nodes(g, 1);
  if (h->tke_wall_gen != h->wall_gen) {
    if (!h->tke_wall && cudaMalloc(&h->tke_wall, 2 * 4 * npl * 8) != cudaSuccess)
      return fail(DNS_ENOMEM, "wall-plane fields for the budget");
    std::vector<double> wv(npl * 3), wd(npl), planes(2 * 4 * npl);
    for (int lv = 1; lv < 3; lv++) {
      wall_plane_fields(lv == 1 ? h->wall_lo : h->wall_hi, npl, wv.data(), wd.data());
      double *o = planes.data() + (size_t)(lv - 1) * 4 * npl;
      for (int i = 0; i < g.nxf; i++)
        for (int j = 0; j < g.nyf; j++) {
          const size_t c = (size_t)i * g.nyf + j, t = (size_t)j * g.nxf + i;
          o[t] = wv[c * 3];
          o[npl + t] = wv[c * 3 + 1];
          o[2 * npl + t] = wv[c * 3 + 2];
          o[3 * npl + t] = (1. / 3.) * wd[c];
        }
    }
    CUDA_TRY(cudaMemcpyAsync(h->tke_wall, planes.data(), planes.size() * 8, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));  // planes goes out of scope
    h->tke_wall_gen = h->wall_gen;
  }
  for (int lv = 1; lv < 3; lv++) {
    const int kw = lv == 1 ? 0 : g.zdf - 1;
    for (int c = 0; c < 4; c++)
      CUDA_TRY(cudaMemcpyAsync(q[lv] + c * lvl + (size_t)kw * npl, h->tke_wall + ((size_t)(lv - 1) * 4 + c) * npl,
                               npl * 8, cudaMemcpyDeviceToDevice, h->stream));
  }
  return DNS_OK;
}

extern "C" int dns_tke_budget(dns_handle *h, double *prof, double *ufl, double *vfl) {
  Range range("dns_tke_budget");
  if (!h || !prof) return fail(DNS_EINVAL, "bad argument");
  int rc = tke_validate(h->p);
  if (rc) return rc;
  CUDA_TRY(cudaSetDevice(h->p.device));
  const dns_geometry &g = h->g;
  size_t tot = 0;
  for (int l = 0; l < 3; l++) tot += level_nodes(g, l) * 4;
  // planar fields and the budget's work space stay allocated for later calls
  const size_t need = tot * 8 + tke_workspace_bytes(g);
  if (h->tke_ws_bytes < need) {
    cudaFree(h->tke_ws);
    h->tke_ws = nullptr;
    h->tke_ws_bytes = 0;
    if (cudaMalloc(&h->tke_ws, need) != cudaSuccess) return fail(DNS_ENOMEM, "field buffers for the budget");
    h->tke_ws_bytes = need;
  }
  double *q[3], *o = static_cast<double *>(h->tke_ws);
  for (int l = 0; l < 3; l++) {
    q[l] = o;
    o += level_nodes(g, l) * 4;
  }
  rc = fields_planar(h, q);
  if (rc == DNS_OK) {
    const double *cq[3] = {q[0], q[1], q[2]};
    rc = tke_budget_planar(h->p, g, cq, prof, ufl, vfl, h->stream, o);
  }
  return rc;
}

// reading.c:14-226: vel-* / den-* of the three levels (the first xdv (or
// GR xdv) x-planes; the reference reads its x-halo planes from the same files)
extern "C" int dns_tke_budget_files(const dns_params *p, const char *dir, int cntr, double *prof, double *ufl,
                                    double *vfl) {
  Range range("dns_tke_budget_files");
  if (!p || !dir || !prof) return fail(DNS_EINVAL, "bad argument");
  dns_geometry g;
  int rc = dns_geometry_of(p, &g);
  if (rc) return rc;
  if ((rc = tke_validate(*p))) return rc;
  CUDA_TRY(cudaSetDevice(p->device));
  size_t tot = 0;
  for (int l = 0; l < 3; l++) tot += level_nodes(g, l) * 4;
  std::vector<double> host(tot);
  const char *names[3] = {"c", "slf", "suf"};
  double *hv[3], *hd[3], *o = host.data();
  for (int l = 0; l < 3 && rc == DNS_OK; l++) {
    hv[l] = o;
    hd[l] = o + level_nodes(g, l) * 3;
    o += level_nodes(g, l) * 4;
    char base[16];
    std::snprintf(base, sizeof base, "vel-%s", names[l]);
    rc = read_file(cname(dir, base, cntr), hv[l], level_nodes(g, l) * 3);
    if (rc == DNS_OK) {
      std::snprintf(base, sizeof base, "den-%s", names[l]);
      rc = read_file(cname(dir, base, cntr), hd[l], level_nodes(g, l));
    }
  }
  if (rc) return rc;
  cudaStream_t st;
  CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  double *buf = nullptr;
  if (cudaMalloc(&buf, tot * 8) != cudaSuccess) {
    cudaStreamDestroy(st);
    return fail(DNS_ENOMEM, "field buffers for the budget");
  }
  cudaError_t e = cudaMemcpyAsync(buf, host.data(), tot * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    const double *cv[3], *cd[3];
    for (int l = 0; l < 3; l++) {
      cv[l] = buf + (hv[l] - host.data());
      cd[l] = buf + (hd[l] - host.data());
    }
    rc = tke_budget_device(*p, g, cv, cd, prof, ufl, vfl, st);
  } else {
    rc = fail(DNS_ECUDA, cudaGetErrorString(e));
  }
  cudaStreamSynchronize(st);
  cudaFree(buf);
  cudaStreamDestroy(st);
  return rc;
}

extern "C" int dns_write_tke_budget(const dns_params *p, const char *dir, int cntr, const double *prof,
                                    const double *ufl, const double *vfl) {
  if (!p || !dir || !prof) return fail(DNS_EINVAL, "bad argument");
  dns_geometry g;
  int rc = dns_geometry_of(p, &g);
  if (rc) return rc;
  const size_t NZ = g.nz_profile;
  // budget2D.c:1553 / :1583 / :1590: name.RANK.TTTT, rank 000
  const char *names[3] = {"turb-fld-2d", "vort-fluc-2d", "KE-Budget-2d"};
  const int rows[3] = {19, 3, 30};
  const double *src = prof;
  for (int f = 0; f < 3 && rc == DNS_OK; f++) {
    char base[32];
    std::snprintf(base, sizeof base, "%s.000", names[f]);
    rc = write_file(cname(dir, base, cntr), src, rows[f] * NZ, 1);
    src += rows[f] * NZ;
  }
  const size_t npl = (size_t)g.nxf * g.nyf;
  if (rc == DNS_OK && ufl) rc = write_file(cname(dir, "ufl4", cntr), ufl, npl, 1);
  if (rc == DNS_OK && vfl) rc = write_file(cname(dir, "vfl4", cntr), vfl, npl, 1);
  return rc;
}

// ---------------------------------------------------------------- stepping
// Precision dispatch for one launch of each kernel.  Buffers are addressed by
// ping-pong index; history slots by ring index.
static size_t hslot_elems(const dns_handle *h) { return 2ull * 23 * h->d.ny * h->d.nx; }

static void L_coarse(dns_handle *h, int src, int dst, bool sample, cudaStream_t st) {
  if (is_f32(h))
    launch_coarse_f32(F(h->fc[src]), F(h->fc[dst]), h->d, h->shape, h->g.omega_c, h->state, h->partials, h->pl,
                      sample, st);
  else
    launch_coarse_f64(h->fc[src], h->fc[dst], h->d, h->shape, h->g.omega_c, h->state, h->partials, h->pl, sample,
                      st);
}
static void L_extract(dns_handle *h, int cbuf, int slot, cudaStream_t st) {
  if (is_f32(h))
    launch_extract_f32(F(h->fc[cbuf]), F(h->hist) + slot * hslot_elems(h), h->d, h->shape, st);
  else
    launch_extract_f64(h->fc[cbuf], h->hist + slot * hslot_elems(h), h->d, h->shape, st);
}
static void L_fine(dns_handle *h, int src, int dst, bool first, bool last, bool stats, cudaStream_t st) {
  if (is_f32(h))
    launch_fine_f32(F(h->ff[src]), F(h->ff[dst]), h->wflag, h->d, h->shape, h->g.omega_f, h->state, h->partials,
                    h->pl, first, last, stats, st);
  else
    launch_fine_f64(h->ff[src], h->ff[dst], h->wflag, h->d, h->shape, h->g.omega_f, h->state, h->partials, h->pl,
                    first, last, stats, st);
}
static void L_iface(dns_handle *h, int fbuf, int it, cudaStream_t st) {
  const size_t hs = hslot_elems(h);
  if (is_f32(h)) {
    float *H = F(h->hist);
    launch_interface_f32(H + h->hn * hs, H + h->hp * hs, H + h->hpp * hs, F(h->iface_mac), F(h->ff[fbuf]), h->d, it,
                         h->g.omega_c, h->g.omega_f, st);
  } else {
    launch_interface_f64(h->hist + h->hn * hs, h->hist + h->hp * hs, h->hist + h->hpp * hs, h->iface_mac,
                         h->ff[fbuf], h->d, h->shape, it, h->g.omega_c, h->g.omega_f, st);
  }
}
static void L_inject(dns_handle *h, int fbuf, int cbuf, cudaStream_t st) {
  if (is_f32(h))
    launch_inject_f32(F(h->ff[fbuf]), F(h->fc[cbuf]), h->d, h->shape, h->g.omega_c, h->g.omega_f, h->partials, h->pl,
                      h->p.fltr != 0, st);
  else
    launch_inject_f64(h->ff[fbuf], h->fc[cbuf], h->d, h->shape, h->g.omega_c, h->g.omega_f, h->partials, h->pl,
                      h->p.fltr != 0, st);
}
static void rotate_history(dns_handle *h) {
  // the new level n takes the slot of pp (xcomputations.c:548-556)
  const int t = h->hpp;
  h->hpp = h->hp;
  h->hp = h->hn;
  h->hn = t;
}

// ---------------------------------------------------------------- mode -i start
// dns-q-mgrd-all-patterns-xyc.c:978-997: init (every node the rest equilibrium,
// before the wall flags exist), initializer (uniform grid -> coarse and both
// fine blocks), inter_init (interface history from the coarse state).  The
// uniform state is the first half of lbf.cntr, [xdu][ydu][zdu + 2][19]; the
// second half (the uniform solver's scratch lattice) is not needed.  Each level
// is interpolated on the device into reference AoS order and then imported like
// a restart level.  The history is the extraction of the coarse planes k = 1
// and zdc - 2 (inter_init.c:150-226) on all three levels: the reference copies
// only 19 of every 23 fields into levels p and pp (inter_init.c:237-248) and
// writes the upper plane's density and velocity into the lower history
// (inter_init.c:202-205); neither slip is reproduced.
extern "C" int dns_load_uniform(dns_handle *h, const char *dir, int cntr) {
  Range range("dns_load_uniform");
  if (!h || !dir) return fail(DNS_EINVAL, "bad argument");
  const dns_params &p = h->p;
  if (p.xdu < 1 || p.ydu < 1 || p.zdu < 1) return fail(DNS_EINVAL, "xdu, ydu and zdu must be positive");
  CUDA_TRY(cudaSetDevice(p.device));
  const dns_geometry &g = h->g;
  const int zd = p.zdu + 2;
  const size_t nuni = 19ull * p.xdu * p.ydu * zd;
  const std::string fn = cname(dir, "lbf", cntr);
  {
    FILE *fp = std::fopen(fn.c_str(), "rb");
    if (!fp) return fail(DNS_EIO, "cannot open " + fn);
    const bool ok = std::fseek(fp, 0, SEEK_END) == 0 && std::ftell(fp) >= (long)(nuni * 8);
    std::fclose(fp);
    if (!ok) return fail(DNS_EIO, fn + " is shorter than one (xdu, ydu, zdu + 2, 19) lattice");
  }
  std::vector<double> host(nuni);
  int rc = read_file(fn, host.data(), nuni);
  if (rc) return rc;
  const size_t nlev = std::max(19ull * g.nx * g.ny * g.nzc, 19ull * g.nxf * g.nyf * g.zdf);
  double *uni = nullptr, *lev = nullptr;
  int *bad = nullptr;
  auto release = [&]() {
    cudaFree(uni);
    cudaFree(lev);
    cudaFree(bad);
  };
  if (cudaMalloc(&uni, nuni * 8) != cudaSuccess || cudaMalloc(&lev, nlev * 8) != cudaSuccess ||
      cudaMalloc(&bad, sizeof(int)) != cudaSuccess) {
    release();
    return fail(DNS_ENOMEM, "uniform-grid staging");
  }
  cudaError_t e = cudaMemcpyAsync(uni, host.data(), nuni * 8, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    release();
    return fail(DNS_ECUDA, cudaGetErrorString(e));
  }
  host.clear();
  host.shrink_to_fit();
  // initializer.c:43-45 and main :443-444, the uniform grid's relaxation rate
  const double dxf = 2. / ((double)(g.nzs - 2.));
  const double dxc = g.gr * dxf;
  const double dxr = 2. / ((double)(zd - 2.));
  const double omega_u = 1. / ((3. / p.Rebs) * p.ub * (zd - 2.) + 0.5);
  std::vector<double> aos(nlev);
  for (int level = 0; level < 3 && rc == DNS_OK; level++) {
    UniformMap m;
    m.level = level;
    m.nxl = level == 0 ? g.nx : g.nxf;
    m.nyl = level == 0 ? g.ny : g.nyf;
    m.nzl = level == 0 ? g.nzc : g.zdf;
    m.xu = p.xdu;
    m.yu = p.ydu;
    m.zd = zd;
    m.gr = g.gr;
    m.zdf = g.zdf;
    m.zdc = g.nzc;
    m.dxf = dxf;
    m.dxc = dxc;
    m.dxr = dxr;
    m.fac = level == 0 ? (dxr / dxc) * (omega_u / g.omega_c) : (dxr / dxf) * (omega_u / g.omega_f);
    const size_t n = 19ull * m.nxl * m.nyl * m.nzl;
    launch_uniform_interp_f64(uni, m, lev, bad, h->stream);
    int flag = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(aos.data(), lev, n * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(DNS_ECUDA, cudaGetErrorString(e));
    else if (flag) rc = fail(DNS_EINVAL, "the uniform grid (xdu, ydu, zdu) does not cover the embedded grid");
    else rc = import_level(h, level, aos.data());
  }
  release();
  if (rc) return rc;
  // inter_init: level n from the new coarse state, then p = pp = n
  h->hn = 0;
  h->hp = 1;
  h->hpp = 2;
  L_extract(h, h->cur_c, 0, h->stream);
  CUDA_TRY(cudaGetLastError());
  const size_t hbytes = hslot_elems(h) * (is_f32(h) ? 4 : 8);
  char *hist = reinterpret_cast<char *>(h->hist);
  CUDA_TRY(cudaMemcpyAsync(hist + hbytes, hist, hbytes, cudaMemcpyDeviceToDevice, h->stream));
  CUDA_TRY(cudaMemcpyAsync(hist + 2 * hbytes, hist, hbytes, cudaMemcpyDeviceToDevice, h->stream));
  h->ss = 0;
  h->tm = cntr;
  return refresh_flow(h, p.forcing == DNS_FORCING_CFR ? 0.0 : p.force_const);
}

// One coarse step on two streams.  The interface transfer of substep s
// writes only the interface planes of the buffer whose other planes the fine
// kernel of substep s writes, so the two run concurrently; the coarse kernel
// and the extraction run beside the first fine substep.
//   main:  coarse, extract, iface(1), [wait fine(s-1)] iface(s) ..., [wait inject] finalize
//   aux:   [wait start] fine(1), [wait iface(s-1)] fine(s) ..., inject
// (Measured on B200 with per-kernel device timestamps: the FP64 interface
// transfer is bound by FP64 issue; moved with the extraction to a stream of
// the greatest priority it ran beside the fine kernels but slowed them by as
// much as it hid, 711 against 705 us per step, so it stays in order here.)
// Schedule (compile-time): 0 one stream in order, 1 this schedule.
#ifndef DNS_SCHED
#define DNS_SCHED 1
#endif
static void issue_step_overlapped(dns_handle *h, DevLog *log_row, bool sample) {
  const Dims &d = h->d;
  cudaStream_t S = h->stream, T = h->aux;
  const int nc = 1 - h->cur_c;
  cudaEventRecord(h->ev_start, S);
  cudaStreamWaitEvent(T, h->ev_start, 0);
  L_coarse(h, h->cur_c, nc, sample, S);
  rotate_history(h);
  L_extract(h, nc, h->hn, S);
  int cur = h->cur_f;
  for (int it = 1; it <= d.gr; it++) {
    const int nf = 1 - cur;
    if (it > 1) cudaStreamWaitEvent(T, h->ev_if[it - 2], 0);
    L_fine(h, cur, nf, it == 1, it == d.gr, sample && it == 1, T);
    cudaEventRecord(h->ev_fine[it - 1], T);
    if (it > 1) cudaStreamWaitEvent(S, h->ev_fine[it - 2], 0);
    L_iface(h, nf, it, S);
    cudaEventRecord(h->ev_if[it - 1], S);
    cur = nf;
  }
  L_inject(h, cur, nc, T);
  cudaEventRecord(h->ev_inj, T);
  cudaStreamWaitEvent(S, h->ev_inj, 0);
  launch_finalize(h->state, log_row, h->partials, h->fin_counter, h->pl, d, h->shape, h->sp, S);
  if (sample) launch_stats_finalize(h->stats_acc, h->partials, h->pl, d, h->shape, S);
  h->cur_f = cur;
  h->cur_c = nc;
}

// The same step in stream order on one stream (used while profiling, so that
// every launch can be bracketed by its own pair of events).
static void issue_step(dns_handle *h, DevLog *log_row, bool sample) {
  if (DNS_SCHED > 0 && !h->prof.on && d_gr_ok(h)) {
    issue_step_overlapped(h, log_row, sample);
    return;
  }
  const Dims &d = h->d;
  const int nc = 1 - h->cur_c;
  PROFILED(h, 0, L_coarse(h, h->cur_c, nc, sample, h->stream));
  rotate_history(h);
  PROFILED(h, 1, L_extract(h, nc, h->hn, h->stream));
  for (int it = 1; it <= d.gr; it++) {
    const int nf = 1 - h->cur_f;
    PROFILED(h, 2, L_fine(h, h->cur_f, nf, it == 1, it == d.gr, sample && it == 1, h->stream));
    PROFILED(h, 3, L_iface(h, nf, it, h->stream));
    h->cur_f = nf;
  }
  PROFILED(h, 4, L_inject(h, h->cur_f, nc, h->stream));
  PROFILED(h, 5, launch_finalize(h->state, log_row, h->partials, h->fin_counter, h->pl, d, h->shape, h->sp, h->stream));
  if (sample) PROFILED(h, 6, launch_stats_finalize(h->stats_acc, h->partials, h->pl, d, h->shape, h->stream));
  h->cur_c = nc;
}

extern "C" int dns_step(dns_handle *h, long ncoarse, dns_step_log *log) {
  Range range("dns_step");
  if (!h || ncoarse < 0) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  const double dt = h->g.gr * 1. / ((double)(0.5 * (h->g.nzs - 2.) / h->p.CFL));
  long done = 0;
  int status = DNS_OK;
  while (done < ncoarse) {
    const long n = std::min<long>(h->prof.on ? kProfSteps : kLogCap, ncoarse - done);
    const long ss0 = h->ss;
    for (long q = 0; q < n; q++) {
      const bool sample = h->sample_every > 0 && (h->ss % h->sample_every) == 0;
      issue_step(h, h->dlog + q, sample);
      h->ss++;
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(h->hlog, h->dlog, n * sizeof(DevLog), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    prof_collect(h);
    for (long q = 0; q < n; q++) {
      const DevLog &r = h->hlog[q];
      if (log) {
        dns_step_log &o = log[done + q];
        o.time = (double)h->tm + dt * (double)(ss0 + q);
        o.force = r.force;
        o.momentum = r.momentum;
        o.denst = r.denst;
        o.flowrate = r.flowrate;
        o.stup = r.stup;
        o.stdown = r.stdown;
        o.stress = r.stress;
        o.pgrad = r.pgrad;
      }
      // wshearstr.c:139-143 aborts on NaN only; an infinite stress is logged and the run goes on
      if (status == DNS_OK && std::isnan(r.stress)) {
        status = fail(DNS_ENAN, "NaN wall shear stress at step " + std::to_string(ss0 + q));
      }
    }
    done += n;
    if (status != DNS_OK) break;
  }
  return status;
}

// ---------------------------------------------------------------- statistics
extern "C" int dns_set_sampling(dns_handle *h, long every) {
  if (!h || every < 0) return fail(DNS_EINVAL, "bad argument");
  h->sample_every = every;
  return DNS_OK;
}

extern "C" int dns_stats_reset(dns_handle *h) {
  if (!h) return fail(DNS_EINVAL, "null handle");
  CUDA_TRY(cudaSetDevice(h->p.device));
  CUDA_TRY(cudaMemsetAsync(h->stats_acc, 0, (size_t)h->g.nz_profile * kStatRow * 8, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DNS_OK;
}

// z/H of the composite profile points (statistics.c:319-329)
static void profile_z(const dns_geometry &g, std::vector<double> &z) {
  const int NZ = g.nz_profile, zdf = g.zdf, zdc = g.nzc, GR = g.gr;
  z.assign(NZ, 0.0);
  for (int k = 1; k < zdf; k++) z[k] = k - 0.5;
  for (int k = 2; k < zdc - 2; k++) z[zdf - 2 + k] = GR * (k - 1) + (zdf - 1 - 0.5);
  for (int k = 0; k < zdf - 1; k++) z[zdf + zdc - 4 + k] = k + GR * (zdc - 3) + zdf - 1. - 0.5;
  z[2 * zdf + zdc - 5] = 2 * zdf + GR * (zdc - 4) + GR - 3;
  for (int k = 0; k < NZ; k++) z[k] /= ((double)(g.nzs - 2.));
}

void dns::stats_from_acc(const dns_geometry &g, const double *acc, double *out, long *nsamples) {
  const int NZ = g.nz_profile;
  std::vector<double> z;
  profile_z(g, z);
  long ns = 0;
  for (int p = 0; p < NZ; p++) ns = std::max(ns, (long)acc[(size_t)p * kStatRow + 15]);
  if (nsamples) *nsamples = ns;
  std::memset(out, 0, sizeof(double) * DNS_NSTAT * NZ);
  for (int p = 0; p < NZ; p++) {
    const double *a = acc + (size_t)p * kStatRow;
    out[0 * NZ + p] = z[p];
    const double S = a[15], N = a[14];
    if (S <= 0 || N <= 0) continue;
    // plane means: the first sample's plus the mean offset; per-sample
    // moments: their time means (statistics.c with time_stat.c's averaging);
    // about the time-and-plane mean: the mean per-sample variance plus the
    // variance of the plane means over the samples
    const double du = a[0] / S, dv = a[1] / S, dw = a[2] / S;
    out[1 * NZ + p] = a[16] + du;
    out[2 * NZ + p] = a[17] + dv;
    out[3 * NZ + p] = a[18] + dw;
    out[4 * NZ + p] = a[19] + a[3] / S;
    for (int c = 0; c < 5; c++) out[(5 + c) * NZ + p] = a[9 + c] / S;
    out[10 * NZ + p] = a[9] / S + (a[4] / S - du * du);
    out[11 * NZ + p] = a[10] / S + (a[5] / S - dv * dv);
    out[12 * NZ + p] = a[11] / S + (a[6] / S - dw * dw);
    out[13 * NZ + p] = a[12] / S + (a[7] / S - du * dw);
  }
}

extern "C" int dns_stats(dns_handle *h, double *out, long *nsamples) {
  if (!h || !out) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  std::vector<double> acc((size_t)h->g.nz_profile * kStatRow);
  CUDA_TRY(cudaMemcpyAsync(acc.data(), h->stats_acc, acc.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  dns::stats_from_acc(h->g, acc.data(), out, nsamples);
  return DNS_OK;
}

// instantaneous plane statistics exactly as statistics.c:48-300 (two passes over
// the exported state, same summation order)
extern "C" int dns_plane_stats(dns_handle *h, double *out) {
  Range range("dns_plane_stats");
  if (!h || !out) return fail(DNS_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(h->p.device));
  const dns_geometry &g = h->g;
  const int zdf = g.zdf, zdc = g.nzc, NZ = g.nz_profile;
  std::vector<double> lv[3];
  lv[0].resize(19ull * g.nzc * g.ny * g.nx);
  lv[1].resize(19ull * g.zdf * g.nyf * g.nxf);
  lv[2].resize(19ull * g.zdf * g.nyf * g.nxf);
  int rc;
  for (int l = 0; l < 3; l++)
    if ((rc = export_level(h, l, lv[l].data()))) return rc;
  static const int EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0};
  static const int EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
  static const int EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  double *U = out, *V = out + NZ, *W = out + 2 * NZ, *UT = out + 3 * NZ, *VT = out + 4 * NZ, *WT = out + 5 * NZ,
         *RE = out + 6 * NZ, *DA = out + 7 * NZ, *DT = out + 8 * NZ;
  std::memset(out, 0, sizeof(double) * 9 * NZ);
  struct Seg { int lvl, k0, k1, off, ex, ey, nz, d0, d1; } segs[3] = {
      {1, 1, zdf, 0, g.nxf, g.nyf, zdf, 0, zdf},
      {0, 2, zdc - 2, zdf - 2, g.nx, g.ny, zdc, zdf, zdf + zdc - 4},
      {2, 0, zdf - 1, zdf + zdc - 4, g.nxf, g.nyf, zdf, zdf + zdc - 4, 2 * zdf + zdc - 4}};
  for (int pass = 0; pass < 2; pass++)
    for (const Seg &sg : segs) {
      const double *a = lv[sg.lvl].data();
      for (int i = 0; i < sg.ex; i++)
        for (int j = 0; j < sg.ey; j++)
          for (int k = sg.k0; k < sg.k1; k++) {
            const double *f = a + (((size_t)i * sg.ey + j) * sg.nz + k) * 19;
            double u = 0., v = 0., w = 0., dens = 0.;
            for (int q = 0; q < 19; q++) {
              dens += f[q];
              u += (double)EX[q] * f[q];
              v += (double)EY[q] * f[q];
              w += (double)EZ[q] * f[q];
            }
            const int p = sg.off + k;
            if (pass == 0) {
              U[p] += (u / dens);
              V[p] += (v / dens);
              W[p] += (w / dens);
              DA[p] += dens;
            } else {
              const double uf = (u / dens) - U[p], vf = (v / dens) - V[p], wf = (w / dens) - W[p],
                           df = dens - DA[p];
              UT[p] += uf * uf;
              VT[p] += vf * vf;
              WT[p] += wf * wf;
              RE[p] += uf * wf;
              DT[p] += df * df;
            }
          }
      const double norm = (double)(sg.ex * sg.ey * 1 * 1);
      for (int p = sg.d0; p < sg.d1; p++) {
        if (pass == 0) {
          U[p] /= norm; V[p] /= norm; W[p] /= norm; DA[p] /= norm;
        } else {
          UT[p] /= norm; VT[p] /= norm; WT[p] /= norm; RE[p] /= norm; DT[p] /= norm;
        }
      }
    }
  for (int p = 0; p < NZ; p++) {
    UT[p] = std::sqrt(UT[p]);
    VT[p] = std::sqrt(VT[p]);
    WT[p] = std::sqrt(WT[p]);
    DT[p] = std::sqrt(DT[p]);
  }
  return DNS_OK;
}

// ---------------------------------------------------------------- measurement
extern "C" int dns_set_profiling(dns_handle *h, int on) {
  if (!h) return fail(DNS_EINVAL, "null handle");
  CUDA_TRY(cudaSetDevice(h->p.device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  prof_collect(h);
  h->prof.on = on != 0;
  if (h->prof.on)
    for (int c = 0; c < DNS_NKERNEL; c++) {
      h->prof.ms[c] = 0.;
      h->prof.cnt[c] = 0;
    }
  return DNS_OK;
}

extern "C" int dns_kernel_times(dns_handle *h, double *ms, long *launches) {
  if (!h) return fail(DNS_EINVAL, "null handle");
  for (int c = 0; c < DNS_NKERNEL; c++) {
    if (ms) ms[c] = h->prof.ms[c];
    if (launches) launches[c] = h->prof.cnt[c];
  }
  return DNS_OK;
}

// ---------------------------------------------------------------- errors
extern "C" const char *dns_error_string(int code) {
  switch (code) {
    case DNS_OK: return "ok";
    case DNS_EINVAL: return "invalid argument";
    case DNS_ENOMEM: return "out of memory";
    case DNS_EIO: return "i/o error";
    case DNS_ENAN: return "non-finite wall shear stress";
    case DNS_ETIMEOUT: return "wait timed out";
    case DNS_ECUDA: return "CUDA error";
    default: return "unknown error";
  }
}

extern "C" const char *dns_last_error(void) { return g_last_error.c_str(); }

void dns::set_last_error(const std::string &msg) { g_last_error = msg; }

int dns::fail_with(int code, const std::string &msg) { return fail(code, msg); }
