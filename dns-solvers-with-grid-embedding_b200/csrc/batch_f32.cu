// Persistent kernels of the batched FP32 engine (see batch.h).  The node
// arithmetic is f32_core.cuh's, shared with the single-channel form; what is
// new here is the work decomposition: each kernel walks a table of work items
// across all resident instances, and each instance's reductions land in its
// own partial arrays in an order fixed by its own tiling, so an instance's
// trajectory does not depend on which other instances share the batch.
#include "batch.h"
#include "f32_core.cuh"
#include "quad_f32.cuh"
#include "kernels.h"
#include "lattice.cuh"

namespace dns {
namespace batch {

namespace {

using namespace f32;

static_assert(CTX == kCornerTX, "host and device interface tiles");

// advance s to the instance owning item w (items are walked in increasing order)
__device__ __forceinline__ int owner(const int *__restrict__ st, int n, int w, int s) {
  while (s < n && __ldg(st + s + 1) <= w) s++;
  return s;
}

__device__ __forceinline__ int log2i(int v) { return 31 - __clz(v); }

// the item this block would take after leaving instance s's range: the
// smallest w' >= end with w' = w (mod stride), minus one stride (the loop adds it)
__device__ __forceinline__ int past(int w, int end, int stride) {
  return w >= end ? w - stride : w + ((end - w + stride - 1) / stride) * stride - stride;
}

__device__ __forceinline__ bool sampling(const Inst &I, const Dyn &D) {
  return D.remaining > 0 && I.sample_every > 0 && D.step % I.sample_every == 0;
}

__device__ __forceinline__ void stat_acc(const float (&f)[19], PlaneStat &sacc) {
  const Mac32 m = macro_f32(f);
  sacc.add(m.u0, m.u1, m.u2, 1.0 + (double)m.drho);
}

// ------------------------------------------------------------------ statistics
// Sums of the state at the start of the step (the state the single-channel
// form samples inside its coarse kernel and first fine substep), four nodes
// per thread on the tiles of the stream-collide kernels.
__global__ void __launch_bounds__(kThreads) b_stats(const Mix *__restrict__ M, const Dyn *__restrict__ dyn) {
  const int n = M->n;
  const int *st = M->start[PH_STATS];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (!sampling(I, D)) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    int local = w - st[s];
    const int ncs = (I.nzc - 4) * I.cgy * I.cgx;
    const bool coarse = local < ncs;
    if (!coarse) local -= ncs;
    const int W = coarse ? I.cw : I.fw, jb = coarse ? I.cjb : I.fjb;
    const int gx = coarse ? I.cgx : I.fgx, gy = coarse ? I.cgy : I.fgy;
    const int nx = coarse ? I.nx : I.nxf, ny = coarse ? I.ny : I.nyf;
    const int z = local / (gx * gy), rem = local - z * gx * gy, by = rem / gx, bx = rem - by * gx;
    const int p = coarse ? z + 2 : z;  // coarse plane k, or fine device plane
    const int lw = log2i(W), tx = threadIdx.x & (W - 1), ty = threadIdx.x >> lw, R = kThreads >> lw;
    const float *src = coarse ? I.fc[D.cc] : I.ff[D.cf];
    const size_t pstride = coarse ? (size_t)I.nzc * I.ny * I.nx : (size_t)2 * I.zds * I.nyf * I.nxf;
    PlaneStat sacc;
    sacc.init();
    for (int r = 0; r < jb; r++) {
      const int j = (by * jb + r) * R + ty;
      const QuadPos P = quad_pos(tx, W, bx * 4 * W, nx, j < ny);
      if (!P.ok) continue;  // no shuffles below
      float q[19][4];
      quad_load(src, ((size_t)p * ny + j) * nx + P.x0, pstride, true, q);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float f[19];
#pragma unroll
        for (int a = 0; a < 19; a++) f[a] = q[a][c];
        stat_acc(f, sacc);
      }
    }
    const size_t blk = ((size_t)p * gy + by) * gx + bx;
    block_reduce_stat(sacc, I.part + (coarse ? I.psc : I.psf) + blk * kStatPart);
  }
}

// per composite-profile plane: sum the plane's block partials (fixed order) and
// add the sample into the instance's running-statistics row (kernels.h layout,
// the single-channel form's)
__global__ void __launch_bounds__(kThreads) b_sfinal(const Mix *__restrict__ M, const Dyn *__restrict__ dyn) {
  const int n = M->n;
  const int *st = M->start[PH_SFINAL];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (!sampling(I, D)) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    const int idx = w - st[s];
    const int zdf = I.zdf, nzc = I.nzc;
    const double *src = nullptr;
    long nb = 0;
    const long bc = (long)I.cgx * I.cgy, bf = (long)I.fgx * I.fgy;
    if (idx >= 1 && idx <= zdf - 1) {  // lower fine k = idx (device plane idx - 1)
      src = I.part + I.psf + (size_t)(idx - 1) * bf * kStatPart; nb = bf;
    } else if (idx >= zdf && idx <= zdf + nzc - 5) {  // coarse k = idx - zdf + 2
      src = I.part + I.psc + (size_t)(idx - zdf + 2) * bc * kStatPart; nb = bc;
    } else if (idx >= zdf + nzc - 4 && idx <= 2 * zdf + nzc - 6) {  // upper fine k
      const int k = idx - (zdf + nzc - 4);
      src = I.part + I.psf + (size_t)(I.zds + k) * bf * kStatPart; nb = bf;
    }
    if (!src) continue;
    stat_plane_finalize(src, nb, I.stats + (size_t)idx * kStatRow);  // block-uniform; ends with a barrier
  }
}

// ------------------------------------------------------------------ coarse
// Every coarse plane in one launch (xcomputations.c:49-86 collision,
// :135-204, 353-420 streaming), four nodes per thread.  Pushes into planes 0
// and zdc-1 are dropped (the fine-to-coarse injection rewrites them): planes
// 2..zdc-3 push everything and their flow-rate partials are the nodes'
// post-collision moments; the four planes 0, 1, zdc-2, zdc-1 drop their
// pushes past plane 1 / zdc-2 and sum what they keep.
#ifndef DNS_F32_QUAD_MINB
#define DNS_F32_QUAD_MINB 4
#endif
__global__ void __launch_bounds__(kThreads, DNS_F32_QUAD_MINB)
    b_coarse(const Mix *__restrict__ M, const Dyn *__restrict__ dyn, const DevState *__restrict__ state) {
  const int n = M->n;
  const int *st = M->start[PH_COARSE];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (D.remaining <= 0) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    const int local = w - st[s];
    const int gxy = I.cgx * I.cgy;
    const int k = local / gxy, rem = local - k * gxy, by = rem / I.cgx, bx = rem - by * I.cgx;
    const int nx = I.nx, ny = I.ny, nzc = I.nzc;
    const int lw = log2i(I.cw), tx = threadIdx.x & (I.cw - 1), ty = threadIdx.x >> lw, R = kThreads >> lw;
    const size_t pstride = (size_t)nzc * ny * nx;
    const float *src = I.fc[D.cc];
    float *dst = I.fc[D.cc ^ 1];
    const float om = I.om_c, G = (float)state[I.slot].force;
    const float one[3] = {1.f, 1.f, 1.f};
    const int plane = ny * nx;
    double acc[2] = {0., 0.};
    for (int r = 0; r < I.cjb; r++) {
      const int jr = (by * I.cjb + r) * R + ty;
      const bool row_ok = jr < ny;
      const int j = row_ok ? jr : 0;
      const QuadPos P = quad_pos(tx, I.cw, bx * 4 * I.cw, nx, row_ok);
      const long long rowoff = ((long long)k * ny + j) * nx;
      float q[19][4];
      quad_load(src, (size_t)(rowoff + P.x0), pstride, P.ok, q);
      Mac32 m[4];
      quad_collide(q, om, G, m);
      const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
      if (k >= 2 && k <= nzc - 3) {
        if (P.ok)
#pragma unroll
          for (int c = 0; c < 4; c++) {
            acc[0] += (double)(m[c].rho * m[c].u0 + m[c].rho * G);
            acc[1] += (double)m[c].drho;
          }
        quad_push<0, 0, false>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, one, acc);
      } else if (k == 0) {
        quad_push<-2, 0, true>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, one, acc);
      } else if (k == 1) {
        quad_push<-1, 0, true>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, one, acc);
      } else if (k == nzc - 2) {
        quad_push<1, 0, true>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, one, acc);
      } else {
        quad_push<2, 0, true>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, one, acc);
      }
    }
    const size_t blk = ((size_t)k * I.cgy + by) * I.cgx + bx;
    block_reduce32<2>(acc, I.part + I.pc + blk * 2);
  }
}

// ------------------------------------------------------------------ fine
// Both fine blocks' planes in one launch per substep (xfcomputations.c:43-214,
// 599-712 collision with force G/GR; :215-442, 724-897 streaming), four nodes
// per thread.  Work item plane order: the two wall-adjacent planes (lower
// k = 1, upper k = zdf-2), then the four interface-adjacent planes (lower
// zdf-2, zdf-1, upper 0, 1), then the bulk planes k = 2..zdf-3 of both
// blocks: the slower items are taken first, so the launch ends on bulk items.
// Interface-adjacent planes drop the pushes that land on or past the
// interface plane (it belongs to the concurrently running coarse-to-fine
// transfer); wall-adjacent planes send their five wall-bound populations
// through the bounce-back / specular rule.  MODE bits as the single-channel
// form: 1 flow-rate partials (last substep), 2 wall-shear sums (first).
__device__ __forceinline__ int fine_plane(int q, int zds) {
  if (q == 0) return 0;
  if (q == 1) return 2 * zds - 1;
  if (q < 6) return zds - 2 + (q - 2);
  const int b = q - 6;
  return b < zds - 3 ? b + 1 : zds + 2 + (b - (zds - 3));
}

// One work item (plane tile) of substep sub; `local`: the item's index within
// its instance.  Block-uniform; ends with the block reductions' barriers.
template <int MODE>
__device__ __forceinline__ void fine_item(const Inst &I, const Dyn &D, int local, const DevState *__restrict__ state,
                                          int sub) {
  {
    const int gxy = I.fgx * I.fgy;
    const int qp = local / gxy, rem = local - qp * gxy, by = rem / I.fgx, bx = rem - by * I.fgx;
    const int zds = I.zds, zdf = I.zdf, gr = I.gr, nx = I.nxf, ny = I.nyf;
    const int p = fine_plane(qp, zds);
    const bool upper = p >= zds;
    const int k = upper ? p - zds : p + 1;
    const int lw = log2i(I.fw), tx = threadIdx.x & (I.fw - 1), ty = threadIdx.x >> lw, R = kThreads >> lw;
    const size_t pstride = (size_t)2 * zds * ny * nx;
    const float *src = I.ff[D.cf ^ ((sub - 1) & 1)];
    float *dst = I.ff[D.cf ^ (sub & 1)];
    const float om = I.om_f, Gf = (float)((1. / (double)gr) * state[I.slot].force);
    const bool wall_sum_plane =
        upper ? (k == zdf - 2 || k == zdf - 3 || k == zdf - 4) : (k == 1 || k == 2 || k == 3);
    const bool wall_rho_plane = upper ? (k == zdf - 4) : (k == 1);
    // plane class: 0 bulk, 1 lower wall-adjacent, 2 upper wall-adjacent,
    // 3..6 interface-adjacent with ZSKIP 1, 2, -1, -2
    const int cls = (!upper && k == 1) ? 1
                    : (upper && k == zdf - 2) ? 2
                    : (!upper && k == zdf - 2) ? 3
                    : (!upper && k == zdf - 1) ? 4
                    : (upper && k == 1) ? 5
                    : (upper && k == 0) ? 6 : 0;
    float wz[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int kd = k + c - 1;  // destination planes k - 1, k, k + 1 (encalc2.c:33-53, 86-107)
      wz[c] = !upper ? ((kd >= 1 && kd < zdf - gr) ? 1.f : 0.f)
                     : ((kd >= gr && kd < zdf - 1) ? (kd == gr ? 0.5f : 1.f) : 0.f);
    }
    const bool wuni = wz[0] == wz[1] && wz[1] == wz[2];
    const int plane = ny * nx;
    double acc[2] = {0., 0.}, wacc[2] = {0., 0.};
    for (int r = 0; r < I.fjb; r++) {
      const int jr = (by * I.fjb + r) * R + ty;
      const bool row_ok = jr < ny;
      const int j = row_ok ? jr : 0;
      const QuadPos P = quad_pos(tx, I.fw, bx * 4 * I.fw, nx, row_ok);
      const long long rowoff = ((long long)p * ny + j) * nx;
      float q[19][4];
      quad_load(src, (size_t)(rowoff + P.x0), pstride, P.ok, q);
      Mac32 m[4];
      quad_collide(q, om, Gf, m);
      if (P.ok) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
          if ((MODE & 2) && wall_sum_plane) wacc[0] += (double)m[c].u0;
          if ((MODE & 2) && wall_rho_plane) wacc[1] += 1.0 + (double)m[c].drho;
        }
      }
      const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
      switch (cls) {
        case 0:
          if ((MODE & 1) && wuni) {
            // every push lands on a plane of the same weight: the partials are
            // the nodes' post-collision moments (collision keeps mass and
            // momentum, the force adds rho G to sum e_x f)
            if (P.ok)
#pragma unroll
              for (int c = 0; c < 4; c++) {
                acc[0] += (double)(wz[1] * (m[c].rho * m[c].u0 + m[c].rho * Gf));
                acc[1] += (double)(wz[1] * m[c].drho);
              }
            quad_push<0, 0, false>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          } else {
            quad_push<0, 0, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          }
          break;
        case 1:
          quad_push<0, -1, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          quad_wall<false, (MODE & 1) != 0>(q, dst, pstride, rowoff, j, nx, ny, I.wflag, P, wz[1], acc);
          break;
        case 2:
          quad_push<0, 1, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          quad_wall<true, (MODE & 1) != 0>(q, dst, pstride, rowoff, j, nx, ny, I.wflag, P, wz[1], acc);
          break;
        case 3:
          quad_push<1, 0, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          break;
        case 4:
          quad_push<2, 0, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          break;
        case 5:
          quad_push<-1, 0, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          break;
        default:
          quad_push<-2, 0, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
          break;
      }
    }
    const size_t blk = ((size_t)p * I.fgy + by) * I.fgx + bx;
    if (MODE & 1) block_reduce32<2>(acc, I.part + I.pf + blk * 2);
    if ((MODE & 2) && wall_sum_plane) block_reduce32<2>(wacc, I.part + I.pw + blk * 2);
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, DNS_F32_QUAD_MINB)
    b_fine(const Mix *__restrict__ M, const Dyn *__restrict__ dyn, const DevState *__restrict__ state, int sub) {
  const int n = M->n;
  const int *st = M->start[PH_FINE];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (D.remaining <= 0) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    fine_item<MODE>(I, D, w - st[s], state, sub);
  }
}

// ------------------------------------------------------------------ interface
// the item's parameters, built in shared memory by thread 0 (not registers)
__device__ __forceinline__ void iface_params_of(IfParams32 &P, const Inst &I, const Dyn &D, int sub, const TimeW &tw) {
  const size_t hs = (size_t)2 * 23 * I.ny * I.nx;
  // ring after this step's rotation: n in the old pp slot, p in old n, pp in old p
  P.hn = I.hist + (size_t)D.hpp * hs;
  P.hp = I.hist + (size_t)D.hn * hs;
  P.hpp = I.hist + (size_t)D.hp * hs;
  P.corner = I.corner + (size_t)(sub - 1) * 2 * 23 * I.ny * I.nx;  // substep sub's corner data
  P.fdst = I.ff[D.cf ^ (sub & 1)];
  P.nx = I.nx;
  P.ny = I.ny;
  P.nxf = I.nxf;
  P.nyf = I.nyf;
  P.zds = I.zds;
  P.an = tw.an;
  P.ap = tw.ap;
  P.app = tw.app;
  P.fac = I.fac_if;
}

// Interface corner data of every substep of the step, with the extraction of
// the new interface history level folded in.  One item: tile (tx, ty) of
// CTX x kCornerTY coarse interface nodes, wall w, field group G.  The level-n values
// of the tile and its two-node halo are formed from the coarse state just
// streamed (xcomputations.c:558-625: [drho, u, f - feq] at k = 1 / zdc - 2) and
// the tile's own nodes are written to the history (the slot that becomes
// level n); levels p and pp come from the history.  Then, for every substep
// t = 1..GR, the Hermite-in-time value (tinterpolate_hrmt.c), the fourth-order
// derivatives (derivative.c) and the corner float4s of substep t's array.
// Every substep's interface depends only on the three history levels, so the
// whole step's corner data is made right after the coarse kernel.  Every
// field of the item's group goes through each barrier phase together: per
// substep the time combination, the y derivatives and the x derivatives with
// the store, the derivative phases four-wide in shared memory.
struct CornerTimes {
  int gr;
  TimeW w[4];  // substeps 1..gr
};
constexpr int kCQX = CTX + 4, kCQY = kCornerTY + 4;
// work items per (tile, wall) of b_icorner_all: field groups (each also forms
// the level-n moments of its tile and halo)
#ifndef DNS_ALL_CORNER_GROUPS
#define DNS_ALL_CORNER_GROUPS 3
#endif
constexpr int kAllCornerGroups = DNS_ALL_CORNER_GROUPS;
static_assert(kAllCornerGroups >= 1 && kAllCornerGroups <= 8, "field groups of b_icorner_all");
__host__ __device__ constexpr int all_corner_field(int g) { return 23 * g / kAllCornerGroups; }
constexpr int kCornerFieldsMax = (23 + kAllCornerGroups - 1) / kAllCornerGroups;
// threads per block of b_icorner_all: the halo's population loads of one item
// are spread over more threads, so that more of them are in flight at once
#ifndef DNS_CORNER_THREADS
#define DNS_CORNER_THREADS 256
#endif
constexpr int kCornerThreads = DNS_CORNER_THREADS;
constexpr int kCNVP = (kCQX * kCQY + kCornerThreads - 1) / kCornerThreads;
static_assert(kCQX % 4 == 0 && CTX % 4 == 0, "four-wide shared-memory rows");
struct __align__(16) CornerAllSmem {
  float N[kCornerFieldsMax][kCQY][kCQX];  // level n of the group's fields, tile and halo
  float V[kCornerFieldsMax][kCQY][kCQX];  // substep t's values
  float DY[kCornerFieldsMax][kCornerTY][kCQX];  // their y derivatives on the tile's rows
};

__device__ __forceinline__ float4 ld4s(const float *p) { return *reinterpret_cast<const float4 *>(p); }

template <int G>
__device__ __forceinline__ void corner_all_tile32(CornerAllSmem &C, const Inst &I, const Dyn &D, int tx, int ty,
                                                  int w, const CornerTimes &ct) {
  constexpr int F0 = all_corner_field(G), F1 = all_corner_field(G + 1), NF = F1 - F0;
  static_assert(NF <= kCornerFieldsMax, "group size");
  // four-wide groups: y derivatives over the halo's columns, x derivatives over the tile's
  constexpr int kDY = NF * kCornerTY * (kCQX / 4), kDX = NF * kCornerTY * (CTX / 4);
  const float c2o3 = 2.f / 3.f, c1o12 = 1.f / 12.f;
  const int nx = I.nx, ny = I.ny, i0 = tx * CTX, j0 = ty * kCornerTY;
  const size_t plane = (size_t)ny * nx, hs = (size_t)2 * 23 * plane;
  const int k = w == 0 ? 1 : I.nzc - 2;
  const size_t pstride = (size_t)I.nzc * plane;
  const float *fc = I.fc[D.cc ^ 1] + (size_t)k * plane;  // the coarse state just streamed
  // ring after this step's rotation: level n in the old pp slot, p in old n, pp in old p
  float *hn = I.hist + (size_t)D.hpp * hs + ((size_t)w * 23 + F0) * plane;
  const float *hp = I.hist + (size_t)D.hn * hs + ((size_t)w * 23 + F0) * plane;
  const float *hpp = I.hist + (size_t)D.hp * hs + ((size_t)w * 23 + F0) * plane;
  const int t0 = threadIdx.x;
#pragma unroll
  for (int s = 0; s < kCNVP; s++) {
    const int q = t0 + s * kCornerThreads;
    if (q >= kCQX * kCQY) continue;
    const int off = wrapf(j0 - 2 + q / kCQX, ny) * nx + wrapf(i0 - 2 + q % kCQX, nx);
    float d[19];
    load19f(fc, (size_t)off, pstride, d);
    const Mac32 m = macro_f32(d);
    const int qi = q % kCQX - 2, qj = q / kCQX - 2;
    const bool own = qi >= 0 && qi < CTX && qj >= 0 && qj < kCornerTY && i0 + qi < nx && j0 + qj < ny;
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const int fg = F0 + f;
      const float v = fg == 0 ? m.drho
                      : fg == 1 ? m.u0
                      : fg == 2 ? m.u1
                      : fg == 3 ? m.u2 : d[fg - 4] - deq_f32(fg - 4, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
      C.N[f][q / kCQX][q % kCQX] = v;
      if (own) hn[(size_t)f * plane + off] = v;
    }
  }
  for (int t = 0; t < ct.gr; t++) {
    const TimeW tw = ct.w[t];
    // Hermite-in-time values of every field of the group on the tile and halo
    // (each thread combines the level-n values it wrote itself); levels p and
    // pp are read only where their weights are not zero (not in the last
    // substep, which is level n alone)
    const bool lv = tw.ap != 0.f || tw.app != 0.f;
#pragma unroll
    for (int s = 0; s < kCNVP; s++) {
      const int q = t0 + s * kCornerThreads;
      if (q >= kCQX * kCQY) continue;
      float a[NF], b[NF];
      if (lv) {
        const int o = wrapf(j0 - 2 + q / kCQX, ny) * nx + wrapf(i0 - 2 + q % kCQX, nx);
#pragma unroll
        for (int f = 0; f < NF; f++) {
          a[f] = __ldg(hp + (size_t)f * plane + o);
          b[f] = __ldg(hpp + (size_t)f * plane + o);
        }
      } else {
#pragma unroll
        for (int f = 0; f < NF; f++) a[f] = b[f] = 0.f;
      }
#pragma unroll
      for (int f = 0; f < NF; f++)
        C.V[f][q / kCQX][q % kCQX] = tw.an * C.N[f][q / kCQX][q % kCQX] + tw.ap * a[f] + tw.app * b[f];
    }
    __syncthreads();
#pragma unroll 2
    for (int s = 0; s < (kDY + kCornerThreads - 1) / kCornerThreads; s++) {
      const int e = t0 + s * kCornerThreads;
      if (e < kDY) {
        const int f = e / (kCornerTY * (kCQX / 4)), r = (e / (kCQX / 4)) % kCornerTY, c = 4 * (e % (kCQX / 4));
        const float4 v0 = ld4s(&C.V[f][r][c]), v1 = ld4s(&C.V[f][r + 1][c]), v3 = ld4s(&C.V[f][r + 3][c]),
                     v4 = ld4s(&C.V[f][r + 4][c]);
        *reinterpret_cast<float4 *>(&C.DY[f][r][c]) =
            make_float4(c2o3 * (v3.x - v1.x) - c1o12 * (v4.x - v0.x), c2o3 * (v3.y - v1.y) - c1o12 * (v4.y - v0.y),
                        c2o3 * (v3.z - v1.z) - c1o12 * (v4.z - v0.z), c2o3 * (v3.w - v1.w) - c1o12 * (v4.w - v0.w));
      }
    }
    __syncthreads();
    float4 *out = I.corner + (size_t)t * hs + ((size_t)w * 23 + F0) * plane;
#pragma unroll 2
    for (int s = 0; s < (kDX + kCornerThreads - 1) / kCornerThreads; s++) {
      const int e = t0 + s * kCornerThreads;
      if (e < kDX) {
        const int f = e / (kCornerTY * (CTX / 4)), r = (e / (CTX / 4)) % kCornerTY, c0 = 4 * (e % (CTX / 4));
        const float4 xa = ld4s(&C.V[f][r + 2][c0]), xb = ld4s(&C.V[f][r + 2][c0 + 4]);
        const float4 ya = ld4s(&C.DY[f][r][c0]), yb = ld4s(&C.DY[f][r][c0 + 4]);
        const float x[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
        const float y[8] = {ya.x, ya.y, ya.z, ya.w, yb.x, yb.y, yb.z, yb.w};
        if (j0 + r < ny) {
          float4 *o = out + (size_t)f * plane + (size_t)(j0 + r) * nx + i0 + c0;
#pragma unroll
          for (int n = 0; n < 4; n++)
            if (i0 + c0 + n < nx)
              o[n] = make_float4(x[n + 2], c2o3 * (x[n + 3] - x[n + 1]) - c1o12 * (x[n + 4] - x[n]), y[n + 2],
                                 c2o3 * (y[n + 3] - y[n + 1]) - c1o12 * (y[n + 4] - y[n]));
        }
      }
    }
    __syncthreads();  // V and DY are rewritten for the next substep or item
  }
}

// resident blocks of b_icorner_all per SM: 4 caps it at 64 registers (no
// spills), 592 blocks for c2's 768 items where 80 registers gave 444
#ifndef DNS_CORNER_MINB
#define DNS_CORNER_MINB 4
#endif
__global__ void __launch_bounds__(kCornerThreads, DNS_CORNER_MINB) b_icorner_all(const Mix *__restrict__ M, const Dyn *__restrict__ dyn,
                                                          CornerTimes ct) {
  __shared__ CornerAllSmem C;
  const int n = M->n;
  const int *st = M->start[PH_ICORNER];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (D.remaining <= 0) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    int local = w - st[s];
    const int tx = local % I.igx;
    local /= I.igx;
    const int ty = local % I.igy;
    local /= I.igy;
    const int wall = local / kAllCornerGroups, g = local - wall * kAllCornerGroups;
    // block-uniform; each ends with a barrier
    switch (g) {
#define DNS_CORNER_GROUP(G) \
  case G:                   \
    if (G < kAllCornerGroups) corner_all_tile32<(G < kAllCornerGroups ? G : 0)>(C, I, D, tx, ty, wall, ct); \
    break;
      DNS_CORNER_GROUP(0) DNS_CORNER_GROUP(1) DNS_CORNER_GROUP(2) DNS_CORNER_GROUP(3)
      DNS_CORNER_GROUP(4) DNS_CORNER_GROUP(5) DNS_CORNER_GROUP(6) DNS_CORNER_GROUP(7)
#undef DNS_CORNER_GROUP
    }
  }
}

// One work item (tile, wall, population group) of substep sub's interface
// evaluation.  Block-uniform; ends with a barrier.
template <int GR>
__device__ __forceinline__ void eval_item(IfEvalSmem<GR> &S, IfParams32 &P, const Inst &I, const Dyn &D, int local,
                                          int sub, const TimeW &tw) {
  const int gx = (I.nx + IfTile<GR>::TX - 1) / IfTile<GR>::TX, gy = (I.ny + IfTile<GR>::TY - 1) / IfTile<GR>::TY;
  const int tx = local % gx;
  local /= gx;
  const int ty = local % gy;
  local /= gy;
  const int wall = local / kEvalPopGroups, g = local - wall * kEvalPopGroups;
  if (threadIdx.x == 0) iface_params_of(P, I, D, sub, tw);
  __syncthreads();
  iface_eval_tile32<GR>(S, P, tx, ty, wall, 19 * g / kEvalPopGroups, 19 * (g + 1) / kEvalPopGroups);
}

#ifndef DNS_EVAL_MINB
#define DNS_EVAL_MINB 5
#endif
template <int GR>
__global__ void __launch_bounds__(kThreads, DNS_EVAL_MINB) b_ieval(const Mix *__restrict__ M, const Dyn *__restrict__ dyn, int sub,
                                                    TimeW tw) {
  __shared__ IfEvalSmem<GR> S;
  __shared__ IfParams32 P;
  const int n = M->n;
  const int *st = M->start[PH_IEVAL];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (D.remaining <= 0) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    eval_item<GR>(S, P, I, D, w - st[s], sub, tw);
  }
}

// ------------------------------------------------------------------ injection
__global__ void __launch_bounds__(kThreads) b_inject(const Mix *__restrict__ M, const Dyn *__restrict__ dyn) {
  const int n = M->n;
  const int *st = M->start[PH_INJECT];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    const Dyn D = dyn[I.slot];
    if (D.remaining <= 0) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    const int local = w - st[s];
    const int row = local / I.egx, bx = local - row * I.egx;
    const int wall = row / I.ny, jc = row - wall * I.ny;
    const int ic = bx * kThreads + threadIdx.x;
    const int gr = I.gr, zdf = I.zdf, zds = I.zds, nx = I.nx, ny = I.ny, nzc = I.nzc;
    double acc[2] = {0., 0.};
    if (I.fltr && ic < nx) {
      float fo[19];
      filtered_node_f32(I.ff[D.cf ^ (gr & 1)], I.nxf, I.nyf, zds, zdf, gr, wall, ic, jc, I.fac_inj, fo);
      const int kc = wall == 0 ? 0 : nzc - 1;
      const size_t cstride = (size_t)nzc * ny * nx;
      float *cdst = I.fc[D.cc ^ 1];
      float mom = 0.f, den = 0.f;
#pragma unroll
      for (int a = 0; a < 19; a++) {
        cdst[(size_t)a * cstride + ((size_t)kc * ny + jc) * nx + ic] = fo[a];
        den += fo[a];
        if (ex_of(a) > 0) mom += fo[a];
        if (ex_of(a) < 0) mom -= fo[a];
      }
      acc[0] = mom;
      acc[1] = den;
    } else if (ic < nx) {
      const int ps = wall == 0 ? (zdf - 1 - gr) - 1 : zds + gr;
      const size_t fstride = (size_t)2 * zds * I.nyf * I.nxf;
      float f[19];
      load19f(I.ff[D.cf ^ (gr & 1)], ((size_t)ps * I.nyf + (size_t)jc * gr) * I.nxf + (size_t)ic * gr, fstride, f);
      const Mac32 m = macro_f32(f);
      const int kc = wall == 0 ? 0 : nzc - 1;
      const size_t cstride = (size_t)nzc * ny * nx;
      float *cdst = I.fc[D.cc ^ 1];
      float mom = 0.f, den = 0.f;
#pragma unroll
      for (int a = 0; a < 19; a++) {
        const float deq = deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
        const float fn = deq + I.fac_inj * (f[a] - deq);
        cdst[(size_t)a * cstride + ((size_t)kc * ny + jc) * nx + ic] = fn;
        den += fn;
        if (ex_of(a) > 0) mom += fn;
        if (ex_of(a) < 0) mom -= fn;
      }
      acc[0] = mom;
      acc[1] = den;
    }
    block_reduce32<2>(acc, I.part + I.pi + (size_t)local * 2);
  }
}

// ------------------------------------------------------------------ finalize
// Per instance, kFinChunks blocks each reduce a fixed chunk of every partial
// region (fixed order) into the instance's level-2 row; the last of them to
// finish sums the rows in chunk order and writes the log row, the encalc2
// values and force of the next step, then advances the step's parity,
// history ring and counters.  Deterministic, one launch, no waiting.
constexpr int kFinComp = 18;

__global__ void __launch_bounds__(kThreads) b_final(const Mix *__restrict__ M, Dyn *__restrict__ dyn,
                                                   DevState *__restrict__ state, DevLog *__restrict__ log,
                                                   unsigned int *__restrict__ count) {
  __shared__ double sh[kFinComp][kThreads / 32 > kFinChunks ? kThreads / 32 : kFinChunks];
  __shared__ bool last;
  const int n = M->n;
  const int *st = M->start[PH_FINAL];
  const int total = st[n];
  int s = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    s = owner(st, n, w, s);
    const Inst &I = M->inst[s];
    Dyn D = dyn[I.slot];
    if (D.remaining <= 0) {
      w = past(w, st[s + 1], gridDim.x);
      continue;
    }
    const int c = w - st[s];
    // the nine partial regions (coarse, fine, injection, six wall planes) as
    // one run of (U, D) pairs; chunk c takes a fixed slice of it, so that a
    // thread's loads are issued together whatever region they fall in
    const int zds = I.zds, zdf = I.zdf;
    const long nc = (long)I.nzc * I.cgy * I.cgx, nf = (long)2 * I.zds * I.fgy * I.fgx;
    const long ni = (long)2 * I.ny * I.egx, wn = (long)I.fgy * I.fgx;
    const int planes[6] = {0, 1, 2, zds + zdf - 2, zds + zdf - 3, zds + zdf - 4};
    long long base[9];
    long cnt[9];
    base[0] = I.pc, cnt[0] = nc;
    base[1] = I.pf, cnt[1] = nf;
    base[2] = I.pi, cnt[2] = ni;
#pragma unroll
    for (int q = 0; q < 6; q++) base[3 + q] = I.pw + (long long)planes[q] * wn * 2, cnt[3 + q] = wn;
    const long T = nc + nf + ni + 6 * wn;
    const long lo = T * c / kFinChunks, hi = T * (c + 1) / kFinChunks;
    double v[kFinComp];
#pragma unroll
    for (int q = 0; q < kFinComp; q++) v[q] = 0.;
    const double *P = I.part;
    for (long q = lo + threadIdx.x; q < hi; q += kThreads) {
      long r0 = q;
      int rr = 0;
      while (rr < 8 && r0 >= cnt[rr]) r0 -= cnt[rr++];
      const double u = P[base[rr] + r0 * 2], d = P[base[rr] + r0 * 2 + 1];
#pragma unroll
      for (int r = 0; r < 9; r++)
        if (r == rr) {
          v[2 * r] += u;
          v[2 * r + 1] += d;
        }
    }
    // warp sums, then the warps' sums in warp order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kFinComp; q++) {
      double x = v[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sh[q][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < kFinComp) {
      double a = 0.;
      for (int q = 0; q < kThreads / 32; q++) a += sh[threadIdx.x][q];
      sh[threadIdx.x][0] = a;
    }
    __syncthreads();
    double *l2 = I.part + I.pl2;
    if (threadIdx.x == 0) {
      for (int q = 0; q < kFinComp; q++) l2[c * kFinComp + q] = sh[q][0];
      __threadfence();
      last = atomicAdd(count + I.slot, 1u) == (unsigned)(kFinChunks - 1);
    }
    __syncthreads();
    if (last) {
      __threadfence();
      // the chunk rows are loaded by the whole block at once, then summed in
      // chunk order by one thread each
      {
        const volatile double *L = l2;
        for (int q = threadIdx.x; q < kFinChunks * kFinComp; q += kThreads) sh[q % kFinComp][q / kFinComp] = L[q];
      }
      __syncthreads();
      double a = 0.;
      if (threadIdx.x < kFinComp)
        for (int q = 0; q < kFinChunks; q++) a += sh[threadIdx.x][q];
      __syncthreads();
      if (threadIdx.x < kFinComp) sh[threadIdx.x][0] = a;
      __syncthreads();
      if (threadIdx.x == 0) {
        double S[kFinComp];
        for (int q = 0; q < kFinComp; q++) S[q] = sh[q][0];
        DevState &X = state[I.slot];
        DevLog r;
        r.force = X.force;
        r.momentum = X.momentum;
        r.denst = X.denst;
        r.flowrate = X.momentum * I.flow_scale / X.denst;
        const double *U = S + 6;  // (U, D) per plane: lower k = 1, 2, 3; upper zdf-2, zdf-3, zdf-4
        const double stdown = ((-2. * U[0] + 3. * U[2] - U[4]) / I.norm2) * (I.mu * (U[1] / I.norm2));
        const double stup = (-(2. * U[6] - 3. * U[8] + U[10]) / I.norm2) * (I.mu * (U[11] / I.norm2));
        r.stup = stup;
        r.stdown = stdown;
        r.stress = 0.5 * (stup + stdown);
        r.pgrad = X.force * I.pgrad_scale;
        log[(size_t)I.slot * kLogRows + (size_t)(D.step % kLogRows)] = r;
        const double mom = (I.g3 * S[0] + 0.5 * I.g3 * S[4] + S[2]) / I.norm;
        const double den = (I.g3 * S[1] + 0.5 * I.g3 * S[5] + S[3] + I.den_offset) / I.norm;
        X.momentum = mom;
        X.denst = den;
        X.force = I.cfr ? I.ub - mom : I.gconst;
        // xcomputations.c:548-556 (history rotation); exchange.c / fexchange.c (pointer swaps)
        const int t = D.hpp;
        D.hpp = D.hp;
        D.hp = D.hn;
        D.hn = t;
        D.cc ^= 1;
        D.cf ^= (I.gr & 1);
        D.step += 1;
        D.remaining -= 1;
        dyn[I.slot] = D;
        count[I.slot] = 0u;
      }
    }
    __syncthreads();
  }
}

template <class K>
int occupancy_grid(K kernel, int *grid, int threads = kThreads) {
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0) != cudaSuccess) return -1;
  *grid = sms * (per > 0 ? per : 1);
  return 0;
}

}  // namespace

void tile_counts(const Inst &I, int c[PH_NPHASE]) {
  const int cb = I.cgx * I.cgy, fb = I.fgx * I.fgy;
  c[PH_STATS] = (I.nzc - 4) * cb + 2 * I.zds * fb;
  c[PH_SFINAL] = I.nzp;
  c[PH_COARSE] = I.nzc * cb;
  c[PH_FINE] = 2 * I.zds * fb;
  c[PH_ICORNER] = 2 * kAllCornerGroups * I.igx * I.igy;
  const int etx = I.gr == 2 ? IfTile<2>::TX : (I.gr == 3 ? IfTile<3>::TX : IfTile<4>::TX);
  const int ety = I.gr == 2 ? IfTile<2>::TY : (I.gr == 3 ? IfTile<3>::TY : IfTile<4>::TY);
  c[PH_IEVAL] = 2 * kEvalPopGroups * ((I.nx + etx - 1) / etx) * ((I.ny + ety - 1) / ety);
  c[PH_INJECT] = 2 * I.ny * I.egx;
  c[PH_FINAL] = kFinChunks;
}

int query_grids(int gr, Grids *g) {
  int rc = 0;
  rc |= occupancy_grid(b_stats, &g->stats);
  rc |= occupancy_grid(b_sfinal, &g->sfinal);
  rc |= occupancy_grid(b_coarse, &g->coarse);
  rc |= occupancy_grid(b_fine<3>, &g->fine);
  rc |= occupancy_grid(b_icorner_all, &g->icorner, kCornerThreads);
  if (gr == 2) rc |= occupancy_grid(b_ieval<2>, &g->ieval);
  else if (gr == 3) rc |= occupancy_grid(b_ieval<3>, &g->ieval);
  else rc |= occupancy_grid(b_ieval<4>, &g->ieval);
  rc |= occupancy_grid(b_inject, &g->inject);
  rc |= occupancy_grid(b_final, &g->final_);
  return rc;
}

static void launch_fine(const Mix *m, Dyn *dyn, DevState *state, int mode, int sub, const Grids &g,
                        cudaStream_t s) {
#define DNS_BFINE(M)                                                      \
  case M:                                                                 \
    b_fine<M><<<g.fine, kThreads, 0, s>>>(m, dyn, state, sub);            \
    break;
  switch (mode) {
    DNS_BFINE(0)
    DNS_BFINE(1)
    DNS_BFINE(2)
    DNS_BFINE(3)
  }
#undef DNS_BFINE
}

static TimeW time_weights(int sub, int gr) {
  const double t = (double)sub / (double)gr, t2 = t * t, t3 = t2 * t;
  const double h1 = 2. * t3 - 3. * t2 + 1., h2 = t3 - 2. * t2 + t, h3 = -2. * t3 + 3. * t2, h4 = t3 - t2;
  return TimeW{(float)(0.5 * h2 + h3 + 1.5 * h4), (float)(h1 - 2. * h4), (float)(-0.5 * h2 + 0.5 * h4)};
}

static void launch_eval(const Mix *m, Dyn *dyn, int gr, int sub, const Grids &g, cudaStream_t s) {
  const TimeW tw = time_weights(sub, gr);
  if (gr == 2) b_ieval<2><<<g.ieval, kThreads, 0, s>>>(m, dyn, sub, tw);
  else if (gr == 3) b_ieval<3><<<g.ieval, kThreads, 0, s>>>(m, dyn, sub, tw);
  else b_ieval<4><<<g.ieval, kThreads, 0, s>>>(m, dyn, sub, tw);
}

// One coarse step of every resident instance on two streams, with the
// dependency structure of the single-channel schedule:
//   s:   stats, sfinal, coarse, corners (every substep, with the extraction),
//        eval(1), [fine(1)] eval(2) ..., [inject] final
//   aux: [start] fine(1), [eval(1)] fine(2) ..., inject
// The statistics read the state fine(2) and eval(2) overwrite; both follow
// eval(1) on s.  ev: [0] start, [1..4] fine(sub), [5..8] eval(sub), [9] inject.
void launch_step(const Mix *m, Dyn *dyn, DevState *state, DevLog *log, unsigned int *count, int gr, const Grids &g,
                 cudaStream_t s, cudaStream_t aux, cudaEvent_t *ev, bool stats) {
  cudaEventRecord(ev[0], s);
  cudaStreamWaitEvent(aux, ev[0], 0);
  if (stats) {
    b_stats<<<g.stats, kThreads, 0, s>>>(m, dyn);
    b_sfinal<<<g.sfinal, kThreads, 0, s>>>(m, dyn);
  }
  b_coarse<<<g.coarse, kThreads, 0, s>>>(m, dyn, state);
  CornerTimes ct{};
  ct.gr = gr;
  for (int t = 0; t < gr && t < 4; t++) ct.w[t] = time_weights(t + 1, gr);
  b_icorner_all<<<g.icorner, kCornerThreads, 0, s>>>(m, dyn, ct);
  for (int sub = 1; sub <= gr; sub++) {
    const int mode = (sub == gr ? 1 : 0) | (sub == 1 ? 2 : 0);
    if (sub > 1) cudaStreamWaitEvent(aux, ev[5 + sub - 2], 0);
    launch_fine(m, dyn, state, mode, sub, g, aux);
    cudaEventRecord(ev[1 + sub - 1], aux);
    if (sub > 1) cudaStreamWaitEvent(s, ev[1 + sub - 2], 0);
    launch_eval(m, dyn, gr, sub, g, s);
    cudaEventRecord(ev[5 + sub - 1], s);
  }
  b_inject<<<g.inject, kThreads, 0, aux>>>(m, dyn);
  cudaEventRecord(ev[9], aux);
  cudaStreamWaitEvent(s, ev[9], 0);
  b_final<<<g.final_, kThreads, 0, s>>>(m, dyn, state, log, count);
}

}  // namespace batch
}  // namespace dns
