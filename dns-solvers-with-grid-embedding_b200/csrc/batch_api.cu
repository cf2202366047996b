// Host side of the batched FP32 engine: the dns_batch_* C ABI
// (include/dns_embed.h).  Owns the instances' device memory (one
// stream-ordered allocation each), the device-resident mix tables the
// persistent kernels walk, the captured step-group graphs and the tile-shape
// tuning table.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/dns_embed.h"
#include "batch.h"
#include "host.h"
#include "kernels.h"

using namespace dns;
using namespace dns::batch;

namespace {

#define BTRY(expr)                                                                            \
  do {                                                                                        \
    cudaError_t e_ = (expr);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail_with(DNS_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));        \
  } while (0)

constexpr int kGroup = kLogRows / 2;  // steps per graph replay: two groups fit the log ring
constexpr int kNumEvents = 10;

struct Record {
  dns_params p{};
  dns_geometry g{};
  dns_tile tile{};
  Inst inst{};
  void *chunk = nullptr;
  long long bytes = 0;
  int status = DNS_OK;
  bool live = false;
  long long steps_done = 0, remaining = 0;
  std::vector<DevLog> log;  // rows of the steps taken
};

using ShapeKey = std::tuple<int, int, int, int, int>;
ShapeKey key_of(const dns_params &p) { return ShapeKey{p.xdv, p.ydv, p.zdv, p.zds, p.gratio}; }

// threads along a row for n four-node groups: the widest power of two up to
// 128 that divides n, else the widest that does not exceed it
int pick_width(int n) {
  for (int w = 128; w >= 8; w >>= 1)
    if (n % w == 0) return w;
  for (int w = 128; w >= 8; w >>= 1)
    if (n >= w) return w;
  return 8;
}

bool width_ok(int w) { return w == 8 || w == 16 || w == 32 || w == 64 || w == 128; }
bool tile_ok(const dns_tile &t) {
  return width_ok(t.cw) && width_ok(t.fw) && t.cjb >= 1 && t.cjb <= 64 && t.fjb >= 1 && t.fjb <= 64;
}

// Row iterations per work item (each iteration: 128 / W rows of 4 W nodes).
// Coarse 4 (2048 nodes an item on a 256-node row); fine 2: the tuner's choice
// for c2 (1.8% faster than 4: 4096 fine items fill 6.9 waves of the 592
// resident blocks where 2048 fill 3.5, so less of the last wave idles) and
// within noise of 4 on mixed batches.
#ifndef DNS_DEFAULT_CJB
#define DNS_DEFAULT_CJB 4
#endif
#ifndef DNS_DEFAULT_FJB
#define DNS_DEFAULT_FJB 2
#endif
dns_tile default_tile(const dns_geometry &g) {
  dns_tile t;
  t.cw = pick_width(g.nx / 4);
  t.cjb = DNS_DEFAULT_CJB;
  t.fw = pick_width(g.nxf / 4);
  t.fjb = DNS_DEFAULT_FJB;
  return t;
}

int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// FP32 geometry of p (the batch stores deviations in float whatever p asks).
// The stream-collide kernels move four consecutive nodes along x with 16-byte
// memory operations, so every row must start on a 16-byte boundary: xdv a
// multiple of 4.
int geometry32(const dns_params *p, dns_params &q, dns_geometry &g) {
  q = *p;
  q.precision = DNS_FP32;
  const int rc = dns_geometry_of(&q, &g);
  if (rc) return rc;
  if (q.xdv % 4 != 0) return fail_with(DNS_EINVAL, "the batched engine needs xdv a multiple of 4");
  return DNS_OK;
}

void shape_inst(Inst &I, const dns_params &p, const dns_geometry &g, const dns_tile &t) {
  std::memset(&I, 0, sizeof I);
  I.nx = g.nx;
  I.ny = g.ny;
  I.nzc = g.nzc;
  I.nxf = g.nxf;
  I.nyf = g.nyf;
  I.zdf = g.zdf;
  I.zds = p.zds;
  I.gr = g.gr;
  I.cw = t.cw;
  I.cjb = t.cjb;
  I.cgx = cdiv(g.nx, 4LL * t.cw);
  I.cgy = cdiv(g.ny, (long long)(128 / t.cw) * t.cjb);
  I.fw = t.fw;
  I.fjb = t.fjb;
  I.fgx = cdiv(g.nxf, 4LL * t.fw);
  I.fgy = cdiv(g.nyf, (long long)(128 / t.fw) * t.fjb);
  I.igx = cdiv(g.nx, kCornerTX);
  I.igy = cdiv(g.ny, kCornerTY);
  I.egx = cdiv(g.nx, 128);
  I.nzp = g.nz_profile;
}

struct Layout {
  size_t fc[2], ff[2], hist, corner, wflag, part, stats, total;
  long long pc, pf, pi, pw, psc, psf, pl2, npart;
};

size_t take(size_t &off, size_t bytes) {
  const size_t o = off;
  off += (bytes + 255) & ~(size_t)255;
  return o;
}

Layout layout_of(const Inst &I) {
  Layout L{};
  size_t off = 0;
  const size_t nc = 19ull * I.nzc * I.ny * I.nx * 4, nf = 19ull * 2 * I.zds * I.nyf * I.nxf * 4;
  L.fc[0] = take(off, nc);
  L.fc[1] = take(off, nc);
  L.ff[0] = take(off, nf);
  L.ff[1] = take(off, nf);
  L.hist = take(off, 3ull * 2 * 23 * I.ny * I.nx * 4);
  L.corner = take(off, (size_t)I.gr * 2 * 23 * I.ny * I.nx * 16);
  L.wflag = take(off, (size_t)I.nyf * I.nxf);
  const long long cb = (long long)I.nzc * I.cgy * I.cgx, fb = 2LL * I.zds * I.fgy * I.fgx,
                  ib = 2LL * I.ny * I.egx;
  long long o = 0;
  L.pc = o; o += cb * 2;
  L.pf = o; o += fb * 2;
  L.pi = o; o += ib * 2;
  L.pw = o; o += fb * 2;
  L.psc = o; o += cb * kStatPart;
  L.psf = o; o += fb * kStatPart;
  L.pl2 = o; o += (long long)kFinChunks * 18;
  L.npart = o;
  L.part = take(off, (size_t)o * 8);
  L.stats = take(off, (size_t)I.nzp * kStatRow * 8);
  L.total = off;
  return L;
}

}  // namespace

struct dns_batch {
  int device = 0;
  int gr = 0;
  cudaStream_t s = nullptr, aux = nullptr;
  cudaEvent_t ev[kNumEvents] = {};
  cudaEvent_t done[2] = {};
  Mix *dmix = nullptr;
  std::unique_ptr<Mix> hmix;
  Dyn *ddyn = nullptr;
  DevState *dstate = nullptr;
  DevLog *dlog = nullptr;
  unsigned int *dcount = nullptr;         // finalize counters, one per slot
  Dyn *hdyn[2] = {nullptr, nullptr};      // pinned snapshots
  DevLog *hlog[2] = {nullptr, nullptr};
  Grids grids{};
  // [with statistics phases][kGroup steps, 1 step]; the statistics launches
  // are left out while no resident instance samples
  cudaGraphExec_t gexec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  std::vector<Record> recs;  // by id
  std::vector<int> free_slots;
  std::map<ShapeKey, dns_tile> tuned;
  bool dirty = true;
};

static void release(dns_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->s) cudaStreamSynchronize(b->s);
  for (Record &r : b->recs)
    if (r.chunk) cudaFreeAsync(r.chunk, b->s);
  if (b->s) cudaStreamSynchronize(b->s);
  for (auto &row : b->gexec)
    for (cudaGraphExec_t &g : row)
      if (g) cudaGraphExecDestroy(g);
  cudaFree(b->dmix);
  cudaFree(b->ddyn);
  cudaFree(b->dstate);
  cudaFree(b->dlog);
  cudaFree(b->dcount);
  for (int q = 0; q < 2; q++) {
    if (b->hdyn[q]) cudaFreeHost(b->hdyn[q]);
    if (b->hlog[q]) cudaFreeHost(b->hlog[q]);
    if (b->done[q]) cudaEventDestroy(b->done[q]);
  }
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->aux) cudaStreamDestroy(b->aux);
  if (b->s) cudaStreamDestroy(b->s);
  delete b;
}

extern "C" void dns_batch_destroy(dns_batch *b) { release(b); }

extern "C" int dns_batch_create(int device, dns_batch **out) {
  if (!out) return fail_with(DNS_EINVAL, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail_with(DNS_ECUDA, "no CUDA device");
  if (device < 0 || device >= ndev) return fail_with(DNS_EINVAL, "device ordinal out of range");
  BTRY(cudaSetDevice(device));
  dns_batch *b = new dns_batch();
  b->device = device;
  b->hmix.reset(new Mix());
  std::memset(b->hmix.get(), 0, sizeof(Mix));
  bool ok = cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking) == cudaSuccess;
  for (cudaEvent_t &e : b->ev) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
  for (cudaEvent_t &e : b->done) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaMalloc(&b->dmix, sizeof(Mix)) == cudaSuccess &&
       cudaMalloc(&b->ddyn, sizeof(Dyn) * kMaxInst) == cudaSuccess &&
       cudaMalloc(&b->dstate, sizeof(DevState) * kMaxInst) == cudaSuccess &&
       cudaMalloc(&b->dlog, sizeof(DevLog) * kMaxInst * kLogRows) == cudaSuccess &&
       cudaMalloc(&b->dcount, sizeof(unsigned int) * kMaxInst) == cudaSuccess;
  for (int q = 0; q < 2; q++)
    ok = ok && cudaMallocHost(&b->hdyn[q], sizeof(Dyn) * kMaxInst) == cudaSuccess &&
         cudaMallocHost(&b->hlog[q], sizeof(DevLog) * kMaxInst * kLogRows) == cudaSuccess;
  if (!ok) {
    release(b);
    return fail_with(DNS_ENOMEM, "batch creation failed (streams, events or tables)");
  }
  cudaMemset(b->dmix, 0, sizeof(Mix));
  cudaMemset(b->ddyn, 0, sizeof(Dyn) * kMaxInst);
  cudaMemset(b->dstate, 0, sizeof(DevState) * kMaxInst);
  cudaMemset(b->dlog, 0, sizeof(DevLog) * kMaxInst * kLogRows);
  cudaMemset(b->dcount, 0, sizeof(unsigned int) * kMaxInst);
  // keep freed instance memory in the stream-ordered pool for the next admission
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  for (int q = kMaxInst - 1; q >= 0; q--) b->free_slots.push_back(q);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    release(b);
    return fail_with(DNS_ECUDA, cudaGetErrorString(e));
  }
  *out = b;
  return DNS_OK;
}

extern "C" int dns_batch_footprint(const dns_params *p, long long *bytes) {
  if (!p || !bytes) return fail_with(DNS_EINVAL, "null argument");
  dns_params q;
  dns_geometry g;
  int rc = geometry32(p, q, g);
  if (rc) return rc;
  Inst I;
  shape_inst(I, q, g, default_tile(g));
  *bytes = (long long)layout_of(I).total;
  return DNS_OK;
}

extern "C" int dns_batch_tile_for(const dns_batch *b, const dns_params *p, dns_tile *t) {
  if (!p || !t) return fail_with(DNS_EINVAL, "null argument");
  dns_params q;
  dns_geometry g;
  int rc = geometry32(p, q, g);
  if (rc) return rc;
  if (b) {
    auto it = b->tuned.find(key_of(q));
    if (it != b->tuned.end()) {
      *t = it->second;
      return DNS_OK;
    }
  }
  *t = default_tile(g);
  return DNS_OK;
}

extern "C" int dns_batch_set_tile(dns_batch *b, const dns_params *shape, const dns_tile *t) {
  if (!b || !shape || !t) return fail_with(DNS_EINVAL, "null argument");
  if (!tile_ok(*t)) return fail_with(DNS_EINVAL, "tile widths must be 8, 16, 32, 64 or 128, row iterations 1..64");
  b->tuned[key_of(*shape)] = *t;
  return DNS_OK;
}

// encalc2 of the state in buffers (cc, cf) -> the instance's force for its
// next step, as the single-channel refresh after a seed or an import
static int refresh_flow(dns_batch *b, const Inst &I, const dns_params &q, const dns_geometry &g, int slot, int cc,
                        int cf) {
  const Dims d{g.nx, g.ny, g.nzc, g.nxf, g.nyf, g.zdf, q.zds, g.gr, g.nzs};
  const DevState st0{I.cfr ? 0.0 : q.force_const, 0., 0., 0.};
  BTRY(cudaMemcpyAsync(b->dstate + slot, &st0, sizeof st0, cudaMemcpyHostToDevice, b->s));
  const LaunchShape shp = make_shape(d);
  double *scratch = nullptr;
  if (cudaMallocAsync(&scratch, (size_t)flow_sums_pairs(d, shp) * 2 * 8, b->s) != cudaSuccess)
    return fail_with(DNS_ENOMEM, "flow-sum scratch");
  PartialLayout pl{};
  const StepParams sp{g.omega_c, g.omega_f, q.ub, q.force_const, I.cfr, I.den_offset};
  launch_flow_sums_f32(I.fc[cc], I.ff[cf], b->dstate + slot, scratch, pl, d, shp, sp, b->s);
  BTRY(cudaFreeAsync(scratch, b->s));
  return DNS_OK;
}

extern "C" int dns_batch_add(dns_batch *b, const dns_params *p, const dns_tile *tile, uint64_t seed, double uc,
                             double amp, long long steps, long long sample_every, int *id) {
  if (!b || !p || !id || steps < 0 || sample_every < 0) return fail_with(DNS_EINVAL, "bad argument");
  dns_params q;
  dns_geometry g;
  int rc = geometry32(p, q, g);
  if (rc) return rc;
  if (b->gr != 0 && g.gr != b->gr) return fail_with(DNS_EINVAL, "every instance of a batch must have the same gratio");
  if (b->free_slots.empty()) return fail_with(DNS_ENOMEM, "batch is full");
  dns_tile t;
  if (tile) t = *tile;
  else dns_batch_tile_for(b, &q, &t);
  if (!tile_ok(t)) return fail_with(DNS_EINVAL, "bad tile shape");
  BTRY(cudaSetDevice(b->device));
  if (b->gr == 0) {
    if (query_grids(g.gr, &b->grids)) return fail_with(DNS_ECUDA, "occupancy query failed");
    b->gr = g.gr;
  }
  Record r;
  r.p = q;
  r.g = g;
  r.tile = t;
  Inst &I = r.inst;
  shape_inst(I, q, g, t);
  int counts[PH_NPHASE];
  tile_counts(I, counts);
  for (int c : counts)
    if (c <= 0) return fail_with(DNS_EINVAL, "instance too small for the batched kernels");
  const Layout L = layout_of(I);
  size_t freeb = 0, totalb = 0;
  BTRY(cudaMemGetInfo(&freeb, &totalb));
  cudaError_t e = cudaMallocAsync(&r.chunk, L.total, b->s);
  if (e != cudaSuccess) return fail_with(DNS_ENOMEM, std::string("instance allocation: ") + cudaGetErrorString(e));
  r.bytes = (long long)L.total;
  char *base = static_cast<char *>(r.chunk);
  for (int k = 0; k < 2; k++) {
    I.fc[k] = reinterpret_cast<float *>(base + L.fc[k]);
    I.ff[k] = reinterpret_cast<float *>(base + L.ff[k]);
  }
  I.hist = reinterpret_cast<float *>(base + L.hist);
  I.corner = reinterpret_cast<float4 *>(base + L.corner);
  I.wflag = reinterpret_cast<int8_t *>(base + L.wflag);
  I.part = reinterpret_cast<double *>(base + L.part);
  I.pc = L.pc;
  I.pf = L.pf;
  I.pi = L.pi;
  I.pw = L.pw;
  I.psc = L.psc;
  I.psf = L.psf;
  I.pl2 = L.pl2;
  I.stats = reinterpret_cast<double *>(base + L.stats);
  I.sample_every = sample_every;
  I.om_c = (float)g.omega_c;
  I.om_f = (float)g.omega_f;
  I.fac_if = (float)(g.omega_c / ((double)g.gr * g.omega_f));
  I.fac_inj = (float)(g.gr * (g.omega_f / g.omega_c));
  const Dims d{g.nx, g.ny, g.nzc, g.nxf, g.nyf, g.zdf, q.zds, g.gr, g.nzs};
  // encalc2.c:109-129, wshearstr.c:67-132 (the single-channel finalize's constants)
  I.g3 = (double)g.gr * g.gr * g.gr;
  I.norm = (double)((double)g.nxf * (double)g.nyf * (g.nzs - 2.));
  I.norm2 = (double)g.nxf * (double)g.nyf;
  I.mu = (1. / 6.) * (2. / g.omega_f - 1);
  I.ub = q.ub;
  I.gconst = q.force_const;
  I.pgrad_scale = (g.nzs - 2.) / (2. * g.gr);
  I.flow_scale = (double)((long)g.nyf * (g.nzs - 2));
  I.cfr = q.forcing == DNS_FORCING_CFR ? 1 : 0;
  I.fltr = q.fltr;
  I.den_offset = encalc2_weight_sum(d);
  const int slot = b->free_slots.back();
  I.slot = slot;
  std::vector<int8_t> wf = wall_flags(q, g);
  BTRY(cudaMemcpyAsync(I.wflag, wf.data(), wf.size(), cudaMemcpyHostToDevice, b->s));
  BTRY(cudaMemsetAsync(I.part, 0, (size_t)L.npart * 8, b->s));
  BTRY(cudaMemsetAsync(I.stats, 0, (size_t)I.nzp * kStatRow * 8, b->s));
  launch_seed_f32(I.fc[0], I.ff[0], I.hist, d, seed, uc, amp, b->s);
  // encalc2 of the seeded state -> force of the first step (as dns_init_seeded)
  if ((rc = refresh_flow(b, I, q, g, slot, 0, 0))) {
    cudaFreeAsync(r.chunk, b->s);
    return rc;
  }
  const Dyn dy0{0, 0, 0, 1, 2, 0, 0, steps};
  BTRY(cudaMemcpyAsync(b->ddyn + slot, &dy0, sizeof dy0, cudaMemcpyHostToDevice, b->s));
  e = cudaStreamSynchronize(b->s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFreeAsync(r.chunk, b->s);
    cudaStreamSynchronize(b->s);
    return fail_with(DNS_ECUDA, std::string("instance set-up: ") + cudaGetErrorString(e));
  }
  b->free_slots.pop_back();
  r.live = true;
  r.remaining = steps;
  b->recs.push_back(std::move(r));
  b->dirty = true;
  *id = (int)b->recs.size() - 1;
  return DNS_OK;
}

static Record *record_of(dns_batch *b, int id) {
  if (!b || id < 0 || id >= (int)b->recs.size() || !b->recs[id].live) return nullptr;
  return &b->recs[id];
}

extern "C" int dns_batch_remove(dns_batch *b, int id) {
  Record *r = record_of(b, id);
  if (!r) return fail_with(DNS_EINVAL, "no such instance");
  BTRY(cudaSetDevice(b->device));
  BTRY(cudaStreamSynchronize(b->s));
  BTRY(cudaFreeAsync(r->chunk, b->s));
  r->chunk = nullptr;
  r->live = false;
  b->free_slots.push_back(r->inst.slot);
  b->dirty = true;
  return DNS_OK;
}

// rewrite the device tables from the live instances (ids in increasing order)
static int upload_mix(dns_batch *b) {
  Mix &M = *b->hmix;
  int n = 0;
  for (int ph = 0; ph < PH_NPHASE; ph++) M.start[ph][0] = 0;
  for (const Record &r : b->recs) {
    if (!r.live) continue;
    M.inst[n] = r.inst;
    int c[PH_NPHASE];
    tile_counts(r.inst, c);
    for (int ph = 0; ph < PH_NPHASE; ph++) {
      const long long next = (long long)M.start[ph][n] + c[ph];
      if (next > 0x7fffffffLL) return fail_with(DNS_EINVAL, "batch work table exceeds 2^31 items");
      M.start[ph][n + 1] = (int)next;
    }
    n++;
  }
  M.n = n;
  BTRY(cudaMemcpyAsync(b->dmix, &M, offsetof(Mix, inst) + sizeof(Inst) * (size_t)n, cudaMemcpyHostToDevice, b->s));
  b->dirty = false;
  return DNS_OK;
}

static int capture(dns_batch *b, int steps, bool stats, cudaGraphExec_t *out) {
  cudaGraph_t graph = nullptr;
  BTRY(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
  for (int q = 0; q < steps; q++)
    launch_step(b->dmix, b->ddyn, b->dstate, b->dlog, b->dcount, b->gr, b->grids, b->s, b->aux, b->ev, stats);
  cudaError_t e = cudaStreamEndCapture(b->s, &graph);
  if (e != cudaSuccess) return fail_with(DNS_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail_with(DNS_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return DNS_OK;
}

// fold one snapshot (dyn + log ring after a group) into the host records
static int absorb(dns_batch *b, int q) {
  const Dyn *D = b->hdyn[q];
  const DevLog *Lg = b->hlog[q];
  for (Record &r : b->recs) {
    if (!r.live) continue;
    const int slot = r.inst.slot;
    const long long upto = D[slot].step;
    for (long long st = r.steps_done; st < upto; st++) {
      const DevLog &row = Lg[(size_t)slot * kLogRows + (size_t)(st % kLogRows)];
      r.log.push_back(row);
      if (r.status == DNS_OK && !std::isfinite(row.stress)) {
        r.status = DNS_ENAN;
        // stop the instance: only its budget field is written
        const long long zero = 0;
        BTRY(cudaMemcpyAsync(reinterpret_cast<char *>(b->ddyn + slot) + offsetof(Dyn, remaining), &zero,
                             sizeof zero, cudaMemcpyHostToDevice, b->s));
        BTRY(cudaStreamSynchronize(b->s));
      }
    }
    r.steps_done = upto;
    r.remaining = r.status == DNS_OK ? D[slot].remaining : 0;
  }
  return DNS_OK;
}

extern "C" int dns_batch_run(dns_batch *b, long long nsteps, int *active) {
  Range range("dns_batch_run");
  if (!b || nsteps < 0) return fail_with(DNS_EINVAL, "bad argument");
  BTRY(cudaSetDevice(b->device));
  int rc;
  int live = 0, maxslot = -1;
  bool sampling = false;
  for (const Record &r : b->recs)
    if (r.live) {
      live++;
      maxslot = std::max(maxslot, r.inst.slot);
      sampling = sampling || r.inst.sample_every > 0;
    }
  if (live > 0 && nsteps > 0) {
    if (b->dirty && (rc = upload_mix(b))) return rc;
    cudaGraphExec_t *gx = b->gexec[sampling ? 1 : 0];
    if (!gx[0] && (rc = capture(b, kGroup, sampling, &gx[0]))) return rc;
    if (!gx[1] && (rc = capture(b, 1, sampling, &gx[1]))) return rc;
    const size_t logbytes = sizeof(DevLog) * kLogRows * (size_t)(maxslot + 1);
    long long left = nsteps;
    int k = 0;
    while (left > 0) {
      const int n = left >= kGroup ? kGroup : (int)left;
      if (n == kGroup) {
        BTRY(cudaGraphLaunch(gx[0], b->s));
      } else {
        for (int q = 0; q < n; q++) BTRY(cudaGraphLaunch(gx[1], b->s));
      }
      BTRY(cudaMemcpyAsync(b->hdyn[k & 1], b->ddyn, sizeof(Dyn) * (size_t)(maxslot + 1), cudaMemcpyDeviceToHost, b->s));
      BTRY(cudaMemcpyAsync(b->hlog[k & 1], b->dlog, logbytes, cudaMemcpyDeviceToHost, b->s));
      BTRY(cudaEventRecord(b->done[k & 1], b->s));
      if (k > 0) {
        BTRY(cudaEventSynchronize(b->done[(k - 1) & 1]));
        if ((rc = absorb(b, (k - 1) & 1))) return rc;
      }
      left -= n;
      k++;
    }
    BTRY(cudaEventSynchronize(b->done[(k - 1) & 1]));
    if ((rc = absorb(b, (k - 1) & 1))) return rc;
    BTRY(cudaGetLastError());
  }
  if (active) {
    int a = 0;
    for (const Record &r : b->recs)
      if (r.live && r.remaining > 0) a++;
    *active = a;
  }
  return DNS_OK;
}

extern "C" int dns_batch_info_of(dns_batch *b, int id, dns_batch_info *out) {
  Record *r = record_of(b, id);
  if (!r || !out) return fail_with(DNS_EINVAL, "no such instance");
  BTRY(cudaSetDevice(b->device));
  DevState st;
  BTRY(cudaMemcpyAsync(&st, b->dstate + r->inst.slot, sizeof st, cudaMemcpyDeviceToHost, b->s));
  BTRY(cudaStreamSynchronize(b->s));
  std::memset(out, 0, sizeof *out);
  out->steps_done = r->steps_done;
  out->remaining = r->remaining;
  out->status = r->status;
  out->slot = r->inst.slot;
  out->force = st.force;
  if (!r->log.empty()) {
    out->flowrate = r->log.back().flowrate;
    out->stress = r->log.back().stress;
  }
  out->device_bytes = r->bytes;
  out->updates_per_step = r->g.updates_per_step;
  out->tile = r->tile;
  return DNS_OK;
}

extern "C" int dns_batch_stats_reset(dns_batch *b, int id) {
  Record *r = record_of(b, id);
  if (!r) return fail_with(DNS_EINVAL, "no such instance");
  BTRY(cudaSetDevice(b->device));
  // ordered on the batch's stream, between step groups
  BTRY(cudaMemsetAsync(r->inst.stats, 0, (size_t)r->inst.nzp * kStatRow * 8, b->s));
  return DNS_OK;
}

extern "C" int dns_batch_stats(dns_batch *b, int id, double *out, long *nsamples) {
  Record *r = record_of(b, id);
  if (!r || !out) return fail_with(DNS_EINVAL, "no such instance");
  BTRY(cudaSetDevice(b->device));
  std::vector<double> acc((size_t)r->g.nz_profile * kStatRow);
  BTRY(cudaMemcpyAsync(acc.data(), r->inst.stats, acc.size() * 8, cudaMemcpyDeviceToHost, b->s));
  BTRY(cudaStreamSynchronize(b->s));
  stats_from_acc(r->g, acc.data(), out, nsamples);
  return DNS_OK;
}

extern "C" int dns_batch_export_state(dns_batch *b, int id, int level, double *aos_out) {
  Record *r = record_of(b, id);
  if (!r || !aos_out || level < 0 || level > 2) return fail_with(DNS_EINVAL, "bad argument");
  BTRY(cudaSetDevice(b->device));
  Dyn D;
  BTRY(cudaMemcpyAsync(&D, b->ddyn + r->inst.slot, sizeof D, cudaMemcpyDeviceToHost, b->s));
  BTRY(cudaStreamSynchronize(b->s));
  const dns_geometry &g = r->g;
  const Inst &I = r->inst;
  const size_t n = level == 0 ? 19ull * g.nzc * g.ny * g.nx : 19ull * g.zdf * g.nyf * g.nxf;
  double *stage = nullptr;
  BTRY(cudaMallocAsync(&stage, n * 8, b->s));
  BTRY(cudaMemsetAsync(stage, 0, n * 8, b->s));  // wall planes: no populations are kept there
  if (level == 0)
    launch_dev_to_aos_f32(I.fc[D.cc], stage, g.nx, g.ny, g.nzc, 0, g.nzc, g.nzc, 0, b->s);
  else if (level == 1)
    launch_dev_to_aos_f32(I.ff[D.cf], stage, g.nxf, g.nyf, 2 * I.zds, 0, I.zds, g.zdf, 1, b->s);
  else
    launch_dev_to_aos_f32(I.ff[D.cf], stage, g.nxf, g.nyf, 2 * I.zds, I.zds, I.zds, g.zdf, 0, b->s);
  cudaError_t e = cudaMemcpyAsync(aos_out, stage, n * 8, cudaMemcpyDeviceToHost, b->s);
  cudaFreeAsync(stage, b->s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->s);
  if (e != cudaSuccess) return fail_with(DNS_ECUDA, cudaGetErrorString(e));
  return DNS_OK;
}

extern "C" int dns_batch_import_state(dns_batch *b, int id, int level, const double *aos_in) {
  Record *r = record_of(b, id);
  if (!r || !aos_in || level < 0 || level > 2) return fail_with(DNS_EINVAL, "bad argument");
  BTRY(cudaSetDevice(b->device));
  Dyn D;
  BTRY(cudaMemcpyAsync(&D, b->ddyn + r->inst.slot, sizeof D, cudaMemcpyDeviceToHost, b->s));
  BTRY(cudaStreamSynchronize(b->s));
  const dns_geometry &g = r->g;
  const Inst &I = r->inst;
  const size_t n = level == 0 ? 19ull * g.nzc * g.ny * g.nx : 19ull * g.zdf * g.nyf * g.nxf;
  double *stage = nullptr;
  BTRY(cudaMallocAsync(&stage, n * 8, b->s));
  cudaError_t e = cudaMemcpyAsync(stage, aos_in, n * 8, cudaMemcpyHostToDevice, b->s);
  if (e == cudaSuccess) {
    if (level == 0)
      launch_aos_to_dev_f32(stage, I.fc[D.cc], g.nx, g.ny, g.nzc, 0, g.nzc, g.nzc, 0, b->s);
    else if (level == 1)
      launch_aos_to_dev_f32(stage, I.ff[D.cf], g.nxf, g.nyf, 2 * I.zds, 0, I.zds, g.zdf, 1, b->s);
    else
      launch_aos_to_dev_f32(stage, I.ff[D.cf], g.nxf, g.nyf, 2 * I.zds, I.zds, I.zds, g.zdf, 0, b->s);
  }
  cudaFreeAsync(stage, b->s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->s);
  if (e != cudaSuccess) return fail_with(DNS_ECUDA, cudaGetErrorString(e));
  int rc = refresh_flow(b, I, r->p, g, I.slot, D.cc, D.cf);
  if (rc) return rc;
  BTRY(cudaStreamSynchronize(b->s));
  BTRY(cudaGetLastError());
  return DNS_OK;
}

extern "C" int dns_batch_log(dns_batch *b, int id, long long first, long long n, dns_step_log *rows) {
  Record *r = record_of(b, id);
  if (!r || !rows || first < 0 || n < 0 || first + n > (long long)r->log.size())
    return fail_with(DNS_EINVAL, "bad argument");
  const double dt = r->g.gr * 1. / ((double)(0.5 * (r->g.nzs - 2.) / r->p.CFL));
  for (long long q = 0; q < n; q++) {
    const DevLog &x = r->log[first + q];
    dns_step_log &o = rows[q];
    o.time = (double)r->p.TSTR + dt * (double)(first + q);
    o.force = x.force;
    o.momentum = x.momentum;
    o.denst = x.denst;
    o.flowrate = x.flowrate;
    o.stup = x.stup;
    o.stdown = x.stdown;
    o.stress = x.stress;
    o.pgrad = x.pgrad;
  }
  return DNS_OK;
}

// ---------------------------------------------------------------- autotuner
// Coordinate search over the tile shape on a throw-away instance of the
// shape: the fine tile first (the fine kernels carry most of the traffic),
// then the coarse tile; each candidate is timed
// over `steps` steps with CUDA events after two warm-up steps.
// Copies of a shape that the tuner times together: enough for about 32 M node
// updates a step (the load of a full batch), at most 64 and 8 GB.  A lone
// small channel leaves most of the GPU idle and would favour narrow tiles
// that lose in a full batch.
static int tune_copies(const dns_geometry &g, size_t bytes_each) {
  const double per = (double)g.updates_per_step;
  int c = (int)((32e6 + per - 1.) / per);
  if (c > 64) c = 64;
  if (bytes_each > 0 && (double)c * (double)bytes_each > 8e9) c = (int)(8e9 / (double)bytes_each);
  return c < 1 ? 1 : c;
}

static int time_tile(int device, const dns_params &p, const dns_tile &t, int steps, int copies, double *ms) {
  dns_batch *sb = nullptr;
  int rc = dns_batch_create(device, &sb);
  if (rc) return rc;
  int id = -1;
  for (int c = 0; c < copies && !rc; c++) rc = dns_batch_add(sb, &p, &t, 1 + c, 0.05, 0.005, steps + 2, 0, &id);
  if (!rc) rc = dns_batch_run(sb, 2, nullptr);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!rc) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, sb->s);
    rc = dns_batch_run(sb, steps, nullptr);
    cudaEventRecord(e1, sb->s);
    cudaEventSynchronize(e1);
    float t_ms = 0.f;
    cudaEventElapsedTime(&t_ms, e0, e1);
    *ms = (double)t_ms / steps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  dns_batch_destroy(sb);
  return rc;
}

extern "C" int dns_batch_autotune(dns_batch *b, const dns_params *shape, int steps, dns_tile *best, double *ms) {
  if (!b || !shape || steps < 1) return fail_with(DNS_EINVAL, "bad argument");
  dns_params q;
  dns_geometry g;
  int rc = geometry32(shape, q, g);
  if (rc) return rc;
  dns_tile cur;
  dns_batch_tile_for(b, &q, &cur);
  Inst I0;
  shape_inst(I0, q, g, cur);
  const int copies = tune_copies(g, layout_of(I0).total);
  double cur_ms = 0.;
  if ((rc = time_tile(b->device, q, cur, steps, copies, &cur_ms))) return rc;
  auto consider = [&](const dns_tile &t) -> int {
    if (!tile_ok(t)) return DNS_OK;
    double m = 0.;
    int r2 = time_tile(b->device, q, t, steps, copies, &m);
    if (r2) return r2;
    if (m < 0.99 * cur_ms) {  // a candidate must beat the current best by 1%
      cur_ms = m;
      cur = t;
    }
    return DNS_OK;
  };
  const int widths[5] = {8, 16, 32, 64, 128}, iters[4] = {1, 2, 4, 8};
  dns_tile base = cur;
  for (int w : widths)
    for (int j : iters) {
      dns_tile t = base;
      t.fw = w;
      t.fjb = j;
      if (t.fw == base.fw && t.fjb == base.fjb) continue;
      if ((rc = consider(t))) return rc;
    }
  base = cur;
  for (int w : widths)
    for (int j : iters) {
      dns_tile t = base;
      t.cw = w;
      t.cjb = j;
      if (t.cw == base.cw && t.cjb == base.cjb) continue;
      if ((rc = consider(t))) return rc;
    }
  b->tuned[key_of(q)] = cur;
  if (best) *best = cur;
  if (ms) *ms = cur_ms;
  return DNS_OK;
}

extern "C" int dns_batch_stream(dns_batch *b, void **stream) {
  if (!b || !stream) return fail_with(DNS_EINVAL, "null argument");
  *stream = (void *)b->s;
  return DNS_OK;
}
