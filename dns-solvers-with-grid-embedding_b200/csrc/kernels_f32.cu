// FP32 deviation-storage form of the grid-embedded D3Q19 channel step: the
// kernels of one channel.  The device arithmetic (collision, streaming rules,
// interface evaluation) is in f32_core.cuh; layout, launch shapes and wall
// rules follow kernels_f64.cu.
#include "f32_core.cuh"
#include "kernels.h"
#include "lattice.cuh"
#include "quad_f32.cuh"

// DNS_F32_QUAD_SINGLE 1: the single-channel stream-collide uses the
// four-node kernels where the x extent allows (0: one node per thread).
#ifndef DNS_F32_QUAD_SINGLE
#define DNS_F32_QUAD_SINGLE 1
#endif
// rows per block of the four-node kernels: the scalar shape's jb
#ifndef DNS_QUAD_JB
#define DNS_QUAD_JB 2
#endif

namespace dns {

namespace {

using namespace f32;

// ------------------------------------------------------------------ coarse
template <bool STATS, bool BULK>
__global__ void __launch_bounds__(kThreads, BULK ? DNS_F32_BULK_MINB : 0) coarse_f32(const float *__restrict__ src, float *__restrict__ dst, Dims d,
                                                      int jb, float om, const DevState *st,
                                                      double *__restrict__ part, double *__restrict__ spart,
                                                      int k0) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // BULK: planes k0 + z for z < gridDim.z (k0 = 2); edge: planes 0, 1, zdc-2, zdc-1
  const int z = blockIdx.z;
  const int k = BULK ? k0 + z : (z < 2 ? z : nzc - 4 + z);
  const size_t pstride = (size_t)nzc * ny * nx;
  const float G = (float)st->force;
  double acc[2] = {0., 0.};
  PlaneStat sacc;
  sacc.init();
  for (int r = 0; r < jb; r++) {
    const int j = blockIdx.y * jb + r;
    if (i >= nx || j >= ny) continue;
    float fa[19];
    const size_t idx0 = ((size_t)k * ny + j) * nx + i;
    load19f(src, idx0, pstride, fa);
    if (BULK)
      coarse_bulk_f32<STATS>(fa, i, j, idx0, d, om, G, dst, pstride, acc, sacc);
    else
      coarse_node_f32<STATS>(fa, i, j, k, d, om, G, dst, pstride, acc, sacc);
  }
  const size_t blk = ((size_t)k * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce32<2>(acc, part + blk * 2);
  if (STATS) block_reduce_stat(sacc, spart + blk * kStatPart);
}

__global__ void __launch_bounds__(kThreads) extract_f32(const float *__restrict__ fc, float *__restrict__ hn, Dims d) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, w = blockIdx.z;
  if (i >= nx) return;
  const int k = w == 0 ? 1 : nzc - 2;
  const size_t pstride = (size_t)nzc * ny * nx, plane = (size_t)ny * nx;
  float f[19];
  load19f(fc, ((size_t)k * ny + j) * nx + i, pstride, f);
  const Mac32 m = macro_f32(f);
  float *o = hn + (size_t)w * 23 * plane + (size_t)j * nx + i;
  o[0] = m.drho;
  o[plane] = m.u0;
  o[2 * plane] = m.u1;
  o[3 * plane] = m.u2;
#pragma unroll
  for (int a = 0; a < 19; a++) o[(size_t)(4 + a) * plane] = f[a] - deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
}

// ------------------------------------------------------------------ fine
// The fine step is three launches over lists of planes: KIND 1 (bulk) the
// planes k = 2..zdf-3 of both blocks, where every push is regular; KIND 2 the
// two planes next to each interface, regular but for the pushes that leave the
// block; KIND 0 the two wall-adjacent planes (bounce-back / free-slip rules).
// blockIdx.z indexes the list; partial sums are stored at the plane's own
// block index, so the layout does not change.
struct PlaneList {
  int n;
  int p[64];
};

template <int MODE, int KIND>
__global__ void __launch_bounds__(kThreads, KIND ? DNS_F32_BULK_MINB : 0) fine_f32(const float *__restrict__ src, float *__restrict__ dst,
                                                    const int8_t *__restrict__ wf, Dims d, int jb, float om,
                                                    const DevState *st, double *__restrict__ part,
                                                    double *__restrict__ wpart, double *__restrict__ spart,
                                                    PlaneList pls) {
  const int nx = d.nxf, ny = d.nyf, zdf = d.zdf, zds = d.zds, gr = d.gr;
  const int P = 2 * zds;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = pls.p[blockIdx.z];
  const bool upper = p >= zds;
  const int k = upper ? p - zds : p + 1;
  const size_t pstride = (size_t)P * ny * nx;
  const float Gf = (float)((1. / (double)gr) * st->force);
  const bool wall_sum_plane =
      upper ? (k == zdf - 2 || k == zdf - 3 || k == zdf - 4) : (k == 1 || k == 2 || k == 3);
  const bool wall_rho_plane = upper ? (k == zdf - 4) : (k == 1);
  double acc[2] = {0., 0.}, wacc[2] = {0., 0.};
  PlaneStat sacc;
  sacc.init();
  float wz[3] = {0.f, 0.f, 0.f};
  {
    // destination planes k - 1, k, k + 1 (encalc2.c:33-53, 86-107)
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const int kd = k + q - 1;
      wz[q] = !upper ? ((kd >= 1 && kd < zdf - gr) ? 1.f : 0.f)
                     : ((kd >= gr && kd < zdf - 1) ? (kd == gr ? 0.5f : 1.f) : 0.f);
    }
  }
  for (int r = 0; r < jb; r++) {
    const int j = blockIdx.y * jb + r;
    if (i >= nx || j >= ny) continue;
    float fa[19];
    const size_t idx0 = ((size_t)p * ny + j) * nx + i;
    load19f(src, idx0, pstride, fa);
    if (KIND == 1)
      fine_bulk_f32<MODE>(fa, i, j, idx0, d, om, Gf, dst, pstride, wz, wall_sum_plane, wall_rho_plane, acc, wacc,
                          sacc);
    else if (KIND == 2 && !upper && k == zdf - 1)
      fine_bulk_f32<MODE, 2>(fa, i, j, idx0, d, om, Gf, dst, pstride, wz, wall_sum_plane, wall_rho_plane, acc,
                             wacc, sacc);
    else if (KIND == 2 && upper && k == 0)
      fine_bulk_f32<MODE, -2>(fa, i, j, idx0, d, om, Gf, dst, pstride, wz, wall_sum_plane, wall_rho_plane, acc,
                              wacc, sacc);
    else if (KIND == 2 && !upper)
      fine_bulk_f32<MODE, 1>(fa, i, j, idx0, d, om, Gf, dst, pstride, wz, wall_sum_plane, wall_rho_plane, acc, wacc,
                             sacc);
    else if (KIND == 2)
      fine_bulk_f32<MODE, -1>(fa, i, j, idx0, d, om, Gf, dst, pstride, wz, wall_sum_plane, wall_rho_plane, acc,
                              wacc, sacc);
    else if (!upper)
      fine_wall_f32<MODE, false>(fa, i, j, idx0, d, om, Gf, wf, dst, pstride, wz, wall_sum_plane, wall_rho_plane,
                                 acc, wacc, sacc);
    else
      fine_wall_f32<MODE, true>(fa, i, j, idx0, d, om, Gf, wf, dst, pstride, wz, wall_sum_plane, wall_rho_plane,
                                acc, wacc, sacc);
  }
  const size_t blk = ((size_t)p * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (MODE & 1) block_reduce32<2>(acc, part + blk * 2);
  if ((MODE & 2) && wall_sum_plane) block_reduce32<2>(wacc, wpart + blk * 2);
  if (MODE & 4) block_reduce_stat(sacc, spart + blk * kStatPart);
}

// ------------------------------------------------------------------ four nodes per thread
// The stream-collide of one channel with the batched engine's four-node
// threads (quad_f32.cuh: 16-byte loads and stores, opposite populations
// collided in pairs) over the scalar kernels' blocks: 32 x jb threads cover a
// scalar block's 128 x jb nodes, so every partial sum lands at the same block
// index and the finalize, statistics and flow-rate paths are unchanged.  Used
// when the x extent is a multiple of 4 (rows start on 16-byte boundaries);
// every plane class is one launch.
constexpr int kQuadRow = 32;  // threads per row: 128 nodes

template <bool STATS>
__global__ void __launch_bounds__(kQuadRow * DNS_QUAD_JB, 512 / (kQuadRow * DNS_QUAD_JB))
    coarse_quad_f32(const float *__restrict__ src, float *__restrict__ dst, Dims d, float om,
                    const DevState *__restrict__ st, double *__restrict__ part, double *__restrict__ spart) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const int tx = threadIdx.x & (kQuadRow - 1), ty = threadIdx.x / kQuadRow;
  const int k = blockIdx.z, jr = blockIdx.y * (blockDim.x / kQuadRow) + ty;
  const bool row_ok = jr < ny;
  const int j = row_ok ? jr : 0;
  const size_t pstride = (size_t)nzc * ny * nx;
  const float G = (float)st->force;
  const float one[3] = {1.f, 1.f, 1.f};
  const int plane = ny * nx;
  double acc[2] = {0., 0.};
  PlaneStat sacc;
  sacc.init();
  const QuadPos P = quad_pos(tx, kQuadRow, blockIdx.x * 4 * kQuadRow, nx, row_ok);
  const long long rowoff = ((long long)k * ny + j) * nx;
  float q[19][4];
  quad_load(src, (size_t)(rowoff + P.x0), pstride, P.ok, q);
  Mac32 m[4];
  quad_collide(q, om, G, m);
  if (STATS && P.ok)
#pragma unroll
    for (int c = 0; c < 4; c++) sacc.add(m[c].u0, m[c].u1, m[c].u2, 1.0 + (double)m[c].drho);
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
  const size_t blk = ((size_t)k * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce32<2>(acc, part + blk * 2);
  if (STATS) block_reduce_stat(sacc, spart + blk * kStatPart);
}

template <int MODE>
__global__ void __launch_bounds__(kQuadRow * DNS_QUAD_JB, 512 / (kQuadRow * DNS_QUAD_JB))
    fine_quad_f32(const float *__restrict__ src, float *__restrict__ dst, const int8_t *__restrict__ wf, Dims d,
                  float om, const DevState *__restrict__ st, double *__restrict__ part, double *__restrict__ wpart,
                  double *__restrict__ spart) {
  const int nx = d.nxf, ny = d.nyf, zdf = d.zdf, zds = d.zds, gr = d.gr;
  const int tx = threadIdx.x & (kQuadRow - 1), ty = threadIdx.x / kQuadRow;
  const int p = blockIdx.z, jr = blockIdx.y * (blockDim.x / kQuadRow) + ty;
  const bool row_ok = jr < ny;
  const int j = row_ok ? jr : 0;
  const bool upper = p >= zds;
  const int k = upper ? p - zds : p + 1;
  const size_t pstride = (size_t)2 * zds * ny * nx;
  const float Gf = (float)((1. / (double)gr) * st->force);
  const bool wall_sum_plane =
      upper ? (k == zdf - 2 || k == zdf - 3 || k == zdf - 4) : (k == 1 || k == 2 || k == 3);
  const bool wall_rho_plane = upper ? (k == zdf - 4) : (k == 1);
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
  PlaneStat sacc;
  sacc.init();
  const QuadPos P = quad_pos(tx, kQuadRow, blockIdx.x * 4 * kQuadRow, nx, row_ok);
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
      if (MODE & 4) sacc.add(m[c].u0, m[c].u1, m[c].u2, 1.0 + (double)m[c].drho);
    }
  }
  const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
  switch (cls) {
    case 0:
      if ((MODE & 1) && wuni) {
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
      quad_wall<false, (MODE & 1) != 0>(q, dst, pstride, rowoff, j, nx, ny, wf, P, wz[1], acc);
      break;
    case 2:
      quad_push<0, 1, (MODE & 1) != 0>(q, dst, pstride, rowoff, plane, dym, dyp, P, nx, wz, acc);
      quad_wall<true, (MODE & 1) != 0>(q, dst, pstride, rowoff, j, nx, ny, wf, P, wz[1], acc);
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
  const size_t blk = ((size_t)p * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (MODE & 1) block_reduce32<2>(acc, part + blk * 2);
  if ((MODE & 2) && wall_sum_plane) block_reduce32<2>(wacc, wpart + blk * 2);
  if (MODE & 4) block_reduce_stat(sacc, spart + blk * kStatPart);
}

// ------------------------------------------------------------------ interface
// pass 1: one block per (tile, wall, field group); pass 2: one block per
// (tile, wall, population group)
__global__ void __launch_bounds__(kThreads) iface_corner_f32(IfParams32 P) {
  __shared__ IfCornerSmem S;
  const int w = blockIdx.z / kCornerFieldGroups, g = blockIdx.z - w * kCornerFieldGroups;
  iface_corner_tile32(S, P, blockIdx.x, blockIdx.y, w, corner_field(g), corner_field(g + 1));
}

template <int GR>
__global__ void __launch_bounds__(kThreads) iface_eval_f32(IfParams32 P) {
  __shared__ IfEvalSmem<GR> S;
  const int w = blockIdx.z / kEvalPopGroups, g = blockIdx.z - w * kEvalPopGroups;
  iface_eval_tile32<GR>(S, P, blockIdx.x, blockIdx.y, w, 19 * g / kEvalPopGroups, 19 * (g + 1) / kEvalPopGroups);
}

// ------------------------------------------------------------------ injection
template <bool FLT>
__global__ void __launch_bounds__(kThreads) inject_f32(const float *__restrict__ fsrc, float *__restrict__ cdst, Dims d,
                                                      float fac, double *__restrict__ part) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc, gr = d.gr, zdf = d.zdf, zds = d.zds;
  const int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y, w = blockIdx.z;
  double acc[2] = {0., 0.};
  if (FLT && ic < nx) {
    float fo[19];
    filtered_node_f32(fsrc, d.nxf, d.nyf, zds, zdf, gr, w, ic, jc, fac, fo);
    const int kc = w == 0 ? 0 : nzc - 1;
    const size_t cstride = (size_t)nzc * ny * nx;
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
  } else if (!FLT && ic < nx) {
    const int ps = w == 0 ? (zdf - 1 - gr) - 1 : zds + gr;
    const size_t fstride = (size_t)2 * zds * d.nyf * d.nxf;
    float f[19];
    load19f(fsrc, ((size_t)ps * d.nyf + (size_t)jc * gr) * d.nxf + (size_t)ic * gr, fstride, f);
    const Mac32 m = macro_f32(f);
    const int kc = w == 0 ? 0 : nzc - 1;
    const size_t cstride = (size_t)nzc * ny * nx;
    float mom = 0.f, den = 0.f;
#pragma unroll
    for (int a = 0; a < 19; a++) {
      const float deq = deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
      const float fn = deq + fac * (f[a] - deq);
      cdst[(size_t)a * cstride + ((size_t)kc * ny + jc) * nx + ic] = fn;
      den += fn;
      if (ex_of(a) > 0) mom += fn;
      if (ex_of(a) < 0) mom -= fn;
    }
    acc[0] = mom;
    acc[1] = den;
  }
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce32<2>(acc, part + blk * 2);
}

// ------------------------------------------------------------------ direct encalc2 sums
__global__ void __launch_bounds__(kThreads) flow_sums_f32_kernel(const float *__restrict__ fc,
                                                                const float *__restrict__ ff, Dims d, int jb,
                                                                double *__restrict__ part) {
  const int z = blockIdx.z;
  const bool coarse = z < d.nzc;
  const int nx = coarse ? d.nx : d.nxf, ny = coarse ? d.ny : d.nyf;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0., 0.};
  double wgt;
  const float *base;
  size_t pstride;
  int p;
  const double g3 = (double)d.gr * d.gr * d.gr;
  if (coarse) {
    p = z;
    wgt = (p == 0 || p == d.nzc - 1) ? 0.5 * g3 : g3;
    base = fc;
    pstride = (size_t)d.nzc * d.ny * d.nx;
  } else {
    p = z - d.nzc;
    const bool upper = p >= d.zds;
    const int k = upper ? p - d.zds : p + 1;
    if (!upper) wgt = (k >= 1 && k < d.zdf - d.gr) ? 1.0 : 0.0;
    else wgt = (k >= d.gr && k < d.zdf - 1) ? (k == d.gr ? 0.5 : 1.0) : 0.0;
    base = ff;
    pstride = (size_t)2 * d.zds * d.nyf * d.nxf;
  }
  if (i < nx) {
    for (int r = 0; r < jb; r++) {
      const int j = blockIdx.y * jb + r;
      if (j >= ny) break;
      float f[19];
      load19f(base, ((size_t)p * ny + j) * nx + i, pstride, f);
      float mom = 0.f, den = 0.f;
#pragma unroll
      for (int a = 0; a < 19; a++) {
        den += f[a];
        if (ex_of(a) > 0) mom += f[a];
        if (ex_of(a) < 0) mom -= f[a];
      }
      acc[0] += wgt * mom;
      acc[1] += wgt * den;
    }
  }
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce32<2>(acc, part + blk * 2);
}

// ------------------------------------------------------------------ seeded state
__device__ __forceinline__ void philox32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                                         uint32_t (&out)[4]) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// the same seeded state as the FP64 form (identical Philox draws and profile),
// with the deviation feq - w evaluated in FP64 and rounded once
__device__ __forceinline__ void seed_node32(float *dst, size_t stride, uint64_t seed, double uc, double amp, double H,
                                            double z, uint32_t i, uint32_t j, uint32_t k, uint32_t lvl, double *u_out) {
  uint32_t r[4];
  philox32(i, j, k, lvl, (uint32_t)seed, (uint32_t)(seed >> 32), r);
  const double zeta = z / H;
  const double prof = 4.0 * uc * zeta * (1.0 - zeta);
  double u[3];
#pragma unroll
  for (int c = 0; c < 3; c++) u[c] = amp * (2.0 * (((double)r[c] + 0.5) * (1.0 / 4294967296.0)) - 1.0);
  u[0] = prof + u[0];
  const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const double eu = (double)ex_of(a) * u[0] + (double)ey_of(a) * u[1] + (double)ez_of(a) * u[2];
    const double w = a == 0 ? 1. / 3. : (a <= 6 ? 1. / 18. : 1. / 36.);
    dst[(size_t)a * stride] = (float)(w * (3. * eu + 4.5 * eu * eu - 1.5 * usq));
  }
  if (u_out) {
    u_out[0] = u[0];
    u_out[1] = u[1];
    u_out[2] = u[2];
  }
}

__global__ void __launch_bounds__(kThreads) seed_f32(float *fc, float *ff, float *hist3, Dims d, uint64_t seed,
                                                    double uc, double amp) {
  const int z = blockIdx.z, j = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double H = d.nzs - 2.0;
  if (z < d.nzc) {
    const int k = z;
    if (i >= d.nx || j >= d.ny) return;
    const size_t stride = (size_t)d.nzc * d.ny * d.nx;
    double u[3];
    seed_node32(fc + ((size_t)k * d.ny + j) * d.nx + i, stride, seed, uc, amp, H, (d.zdf - 1.5) + d.gr * (k - 1.0), i,
                j, k, 0, u);
    if (k == 1 || k == d.nzc - 2) {
      const size_t plane = (size_t)d.ny * d.nx;
      const int w = k == 1 ? 0 : 1;
      for (int l = 0; l < 3; l++) {
        float *o = hist3 + ((size_t)l * 2 + w) * 23 * plane + (size_t)j * d.nx + i;
        o[0] = 0.f;
        o[plane] = (float)u[0];
        o[2 * plane] = (float)u[1];
        o[3 * plane] = (float)u[2];
        for (int b = 4; b < 23; b++) o[(size_t)b * plane] = 0.f;
      }
    }
  } else {
    const int p = z - d.nzc;
    if (i >= d.nxf || j >= d.nyf) return;
    const bool upper = p >= d.zds;
    const int k = upper ? p - d.zds : p + 1;
    const double zpos = upper ? (d.zdf - 1.5) + d.gr * (d.nzc - 3.0) + k : k - 0.5;
    seed_node32(ff + ((size_t)p * d.nyf + j) * d.nxf + i, (size_t)2 * d.zds * d.nyf * d.nxf, seed, uc, amp, H, zpos,
                i, j, k, upper ? 2 : 1, nullptr);
  }
}

// ------------------------------------------------------------------ transposes with conversion
__global__ void dev_to_aos_kernel(const float *__restrict__ soa, double *__restrict__ aos, int nx, int ny, int P,
                                  int p0, int nz_aos, int k0_aos, int i0, int i1) {
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= i1) return;
  const size_t stride = (size_t)P * ny * nx;
  const size_t s = ((size_t)(p0 + q) * ny + j) * nx + i;
  double *o = aos + (((size_t)i * ny + j) * nz_aos + k0_aos + q) * 19;
  for (int a = 0; a < 19; a++) {
    const double w = a == 0 ? 1. / 3. : (a <= 6 ? 1. / 18. : 1. / 36.);
    o[a] = w + (double)soa[s + (size_t)a * stride];
  }
}

__global__ void aos_to_dev_kernel(const double *__restrict__ aos, float *__restrict__ soa, int nx, int ny, int P,
                                  int p0, int nz_aos, int k0_aos, int i0, int i1) {
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= i1) return;
  const size_t stride = (size_t)P * ny * nx;
  const size_t s = ((size_t)(p0 + q) * ny + j) * nx + i;
  const double *o = aos + (((size_t)i * ny + j) * nz_aos + k0_aos + q) * 19;
  for (int a = 0; a < 19; a++) {
    const double w = a == 0 ? 1. / 3. : (a <= 6 ? 1. / 18. : 1. / 36.);
    soa[s + (size_t)a * stride] = (float)(o[a] - w);
  }
}

// ------------------------------------------------------------------ field output
// f = w + d in FP64, then the moments in population order as the FP64 form
template <bool PLANAR>
__global__ void fields_f32_kernel(const float *__restrict__ soa, double *__restrict__ vel, double *__restrict__ den,
                                  int nx, int ny, int P, int p0, int nz_aos, int k0_aos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= nx) return;
  const size_t stride = (size_t)P * ny * nx, s = ((size_t)(p0 + q) * ny + j) * nx + i;
  double dens = 0., mx = 0., my = 0., mz = 0.;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const double f = (a == 0 ? 1. / 3. : (a <= 6 ? 1. / 18. : 1. / 36.)) + (double)soa[s + (size_t)a * stride];
    dens += f;
    mx += (double)ex_of(a) * f;
    my += (double)ey_of(a) * f;
    mz += (double)ez_of(a) * f;
  }
  double ux = 0., uy = 0., uz = 0.;
  if (dens > 0.) {
    ux = mx / dens;
    uy = my / dens;
    uz = mz / dens;
  } else {
    dens = 0.;
  }
  if (PLANAR) {  // vel[c][k][j][i], c = u, v, w, den / 3
    const size_t plane = (size_t)nz_aos * ny * nx, o = ((size_t)(k0_aos + q) * ny + j) * nx + i;
    vel[o] = ux;
    vel[plane + o] = uy;
    vel[2 * plane + o] = uz;
    vel[3 * plane + o] = (1. / 3.) * dens;
    return;
  }
  const size_t o = ((size_t)i * ny + j) * nz_aos + k0_aos + q;
  vel[o * 3 + 0] = ux;
  vel[o * 3 + 1] = uy;
  vel[o * 3 + 2] = uz;
  den[o] = dens;
}

}  // namespace

// ====================================================================== host
// the four-node kernels cover the scalar blocks exactly: 128 nodes of jb rows
static bool quad_ok(const Dims &d, const LaunchShape &s) {
  return DNS_F32_QUAD_SINGLE && d.nx % 4 == 0 && s.bx == 4 * kQuadRow && s.jb == DNS_QUAD_JB;
}

void launch_coarse_f32(const float *src, float *dst, const Dims &d, const LaunchShape &s, double om,
                       const DevState *st, double *partials, const PartialLayout &pl, bool stats,
                       cudaStream_t stream) {
  dim3 gb(s.cgx, s.cgy, d.nzc - 4), ge(s.cgx, s.cgy, 4), block(s.bx);
  double *pc = partials + pl.coarse, *ps = partials + pl.stats_c;
  const float omf = (float)om;
  if (quad_ok(d, s)) {
    dim3 g(s.cgx, s.cgy, d.nzc), b(kQuadRow * s.jb);
    if (stats)
      coarse_quad_f32<true><<<g, b, 0, stream>>>(src, dst, d, omf, st, pc, ps);
    else
      coarse_quad_f32<false><<<g, b, 0, stream>>>(src, dst, d, omf, st, pc, ps);
    return;
  }
  if (stats) {
    coarse_f32<true, true><<<gb, block, 0, stream>>>(src, dst, d, s.jb, omf, st, pc, ps, 2);
    coarse_f32<true, false><<<ge, block, 0, stream>>>(src, dst, d, s.jb, omf, st, pc, ps, 0);
  } else {
    coarse_f32<false, true><<<gb, block, 0, stream>>>(src, dst, d, s.jb, omf, st, pc, ps, 2);
    coarse_f32<false, false><<<ge, block, 0, stream>>>(src, dst, d, s.jb, omf, st, pc, ps, 0);
  }
}

void launch_extract_f32(const float *fc, float *hist_n, const Dims &d, const LaunchShape &s, cudaStream_t stream) {
  dim3 grid(s.jgx, d.ny, 2), block(s.bx);
  extract_f32<<<grid, block, 0, stream>>>(fc, hist_n, d);
}

void launch_fine_f32(const float *src, float *dst, const int8_t *wflag, const Dims &d, const LaunchShape &s,
                     double om, const DevState *st, double *partials, const PartialLayout &pl, bool first, bool last,
                     bool stats, cudaStream_t stream) {
  PlaneList bulk{}, edge{}, adj{};
  for (int p = 0; p < 2 * d.zds; p++) {
    const bool upper = p >= d.zds;
    const int k = upper ? p - d.zds : p + 1;
    const bool wall = upper ? k == d.zdf - 2 : k == 1;
    PlaneList &L = (k >= 2 && k <= d.zdf - 3) ? bulk : (wall ? edge : adj);
    L.p[L.n++] = p;
  }
  const int mode = (last ? 1 : 0) | (first ? 2 : 0) | (stats ? 4 : 0);
  double *pf = partials + pl.fine, *pw = partials + pl.wall, *ps = partials + pl.stats_f;
  const float omf = (float)om;
  if (quad_ok(d, s)) {
    dim3 g(s.fgx, s.fgy, 2 * d.zds), b(kQuadRow * s.jb);
#define FINEQ_CASE(M) \
  case M: fine_quad_f32<M><<<g, b, 0, stream>>>(src, dst, wflag, d, omf, st, pf, pw, ps); break;
    switch (mode) {
      FINEQ_CASE(0) FINEQ_CASE(1) FINEQ_CASE(2) FINEQ_CASE(3) FINEQ_CASE(4) FINEQ_CASE(5) FINEQ_CASE(6) FINEQ_CASE(7)
    }
#undef FINEQ_CASE
    return;
  }
  dim3 gb(s.fgx, s.fgy, bulk.n), ge(s.fgx, s.fgy, edge.n), ga(s.fgx, s.fgy, adj.n), block(s.bx);
#define FINE32_CASE(M)                                                                                       \
  case M:                                                                                                    \
    if (bulk.n) fine_f32<M, 1><<<gb, block, 0, stream>>>(src, dst, wflag, d, s.jb, omf, st, pf, pw, ps, bulk); \
    fine_f32<M, 2><<<ga, block, 0, stream>>>(src, dst, wflag, d, s.jb, omf, st, pf, pw, ps, adj);      \
    fine_f32<M, 0><<<ge, block, 0, stream>>>(src, dst, wflag, d, s.jb, omf, st, pf, pw, ps, edge);     \
    break;
  switch (mode) {
    FINE32_CASE(0) FINE32_CASE(1) FINE32_CASE(2) FINE32_CASE(3) FINE32_CASE(4) FINE32_CASE(5) FINE32_CASE(6)
    FINE32_CASE(7)
  }
#undef FINE32_CASE
}

void launch_interface_f32(const float *hn, const float *hp, const float *hpp, float *corner, float *fdst,
                          const Dims &d, int substep, double omega_c, double omega_f, cudaStream_t stream) {
  IfParams32 P = iface_params32(hn, hp, hpp, reinterpret_cast<float4 *>(corner), fdst, d, substep, omega_c, omega_f);
  dim3 gc((d.nx + CTX - 1) / CTX, (d.ny + CTY - 1) / CTY, 2 * kCornerFieldGroups);
  iface_corner_f32<<<gc, kThreads, 0, stream>>>(P);
#define DNS_EVAL_LAUNCH(G)                                                                            \
  iface_eval_f32<G><<<dim3((d.nx + IfTile<G>::TX - 1) / IfTile<G>::TX, (d.ny + IfTile<G>::TY - 1) / IfTile<G>::TY, \
                           2 * kEvalPopGroups),                                                        \
                      kThreads, 0, stream>>>(P)
  if (d.gr == 2) DNS_EVAL_LAUNCH(2);
  else if (d.gr == 3) DNS_EVAL_LAUNCH(3);
  else DNS_EVAL_LAUNCH(4);
#undef DNS_EVAL_LAUNCH
}

void launch_inject_f32(const float *fsrc, float *cdst, const Dims &d, const LaunchShape &s, double omega_c,
                       double omega_f, double *partials, const PartialLayout &pl, bool filtered,
                       cudaStream_t stream) {
  dim3 grid(s.jgx, s.jgy, 2), block(s.bx);
  const float fac = (float)(d.gr * (omega_f / omega_c));
  if (filtered)
    inject_f32<true><<<grid, block, 0, stream>>>(fsrc, cdst, d, fac, partials + pl.inject);
  else
    inject_f32<false><<<grid, block, 0, stream>>>(fsrc, cdst, d, fac, partials + pl.inject);
}

void launch_flow_sums_f32(const float *fc, const float *ff, DevState *st, double *partials, const PartialLayout &pl,
                          const Dims &d, const LaunchShape &s, const StepParams &sp, cudaStream_t stream) {
  const int gx = s.fgx > s.cgx ? s.fgx : s.cgx, gy = s.fgy > s.cgy ? s.fgy : s.cgy;
  dim3 grid(gx, gy, d.nzc + 2 * d.zds), block(s.bx);
  flow_sums_f32_kernel<<<grid, block, 0, stream>>>(fc, ff, d, s.jb, partials + pl.flow);
  finalize_flow_sums(st, partials + pl.flow, flow_sums_pairs(d, s), d, s, sp, stream);
}

void launch_seed_f32(float *fc, float *ff, float *hist3, const Dims &d, uint64_t seed, double uc, double amp,
                     cudaStream_t stream) {
  const int nxm = d.nxf > d.nx ? d.nxf : d.nx, nym = d.nyf > d.ny ? d.nyf : d.ny;
  dim3 grid((nxm + kThreads - 1) / kThreads, nym, d.nzc + 2 * d.zds), block(kThreads);
  seed_f32<<<grid, block, 0, stream>>>(fc, ff, hist3, d, seed, uc, amp);
}

void launch_dev_to_aos_f32(const float *soa, double *aos, int nx, int ny, int P, int p0, int np, int nz_aos,
                           int k0_aos, cudaStream_t stream, int i0, int i1) {
  if (i1 < 0) i1 = nx;
  if (i1 <= i0) return;
  dim3 grid((i1 - i0 + 127) / 128, ny, np), block(128);
  dev_to_aos_kernel<<<grid, block, 0, stream>>>(soa, aos, nx, ny, P, p0, nz_aos, k0_aos, i0, i1);
}

void launch_aos_to_dev_f32(const double *aos, float *soa, int nx, int ny, int P, int p0, int np, int nz_aos,
                           int k0_aos, cudaStream_t stream, int i0, int i1) {
  if (i1 < 0) i1 = nx;
  if (i1 <= i0) return;
  dim3 grid((i1 - i0 + 127) / 128, ny, np), block(128);
  aos_to_dev_kernel<<<grid, block, 0, stream>>>(aos, soa, nx, ny, P, p0, nz_aos, k0_aos, i0, i1);
}

void launch_fields_f32(const float *soa, double *vel, double *den, int nx, int ny, int P, int p0, int np, int nz_aos,
                       int k0_aos, cudaStream_t stream) {
  dim3 grid((nx + 127) / 128, ny, np), block(128);
  fields_f32_kernel<false><<<grid, block, 0, stream>>>(soa, vel, den, nx, ny, P, p0, nz_aos, k0_aos);
}

void launch_fields_planar_f32(const float *soa, double *q, int nx, int ny, int P, int p0, int np, int nz, int k0,
                              cudaStream_t stream) {
  dim3 grid((nx + 127) / 128, ny, np), block(128);
  fields_f32_kernel<true><<<grid, block, 0, stream>>>(soa, q, nullptr, nx, ny, P, p0, nz, k0);
}

}  // namespace dns
