// Device arithmetic of the FP32 deviation-storage form, shared by the
// single-channel kernels (kernels_f32.cu) and the batched engine
// (batch_f32.cu).
//
// Populations are stored as float deviations d_a = f_a - w_a (reference
// density rho0 = 1) and collided in FP32; the constant-flow-rate momentum and
// mass sums, the wall-shear sums and the statistics are accumulated in FP64.
// Storing the deviation keeps the float mantissa on the part of f that varies
// (|d| ~ 1e-2..1e-4 instead of f ~ 0.03..0.33).
//
// Exact identities used:  rho = 1 + sum d,  rho u = sum e d  (sum e w = 0),
// feq_a - w_a = w_a (drho + rho (3 e.u + 4.5 (e.u)^2 - 1.5 u^2)), and the
// bounce-back / mirror rules move d exactly as f (w is invariant under
// opposite and mirror).  Layout and wall rules are those of kernels_f64.cu;
// the interface history holds [drho, ux, uy, uz, fneq_0..18] in FP32.
#pragma once

#include <cstddef>
#include <cstdint>

#include "kernels.h"
#include "lattice.cuh"

namespace dns {
namespace f32 {

constexpr int kThreads = 128;
// minimum resident blocks asked of the register allocator for the bulk-plane
// kernels (0: compiler's choice).  The fine bulk and wall kernels collide each
// population right before its store, so collided values die as they are written.
#ifndef DNS_F32_BULK_MINB
#define DNS_F32_BULK_MINB 6
#endif

__device__ __forceinline__ int wrapf(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

__host__ __device__ constexpr float w_of(int a) { return a == 0 ? 1.f / 3.f : (a <= 6 ? 1.f / 18.f : 1.f / 36.f); }
__host__ __device__ constexpr float bi_of(int a) { return a == 0 ? 0.f : (a <= 6 ? 1.f / 6.f : 1.f / 12.f); }

__device__ __forceinline__ float proj_f32(int a, float u0, float u1, float u2) {
  return (float)ex_of(a) * u0 + (float)ey_of(a) * u1 + (float)ez_of(a) * u2;
}

// deviation of the equilibrium from w_a
__device__ __forceinline__ float deq_f32(int a, float drho, float rho, float u0, float u1, float u2, float usq) {
  const float eu = proj_f32(a, u0, u1, u2);
  return w_of(a) * (drho + rho * (3.f * eu + 4.5f * eu * eu - 1.5f * usq));
}

struct Mac32 {
  float drho, rho, u0, u1, u2, usq;
};

__device__ __forceinline__ Mac32 macro_f32(const float (&d)[19]) {
  float dr = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    dr += d[a];
    if (ex_of(a) > 0) mx += d[a];
    if (ex_of(a) < 0) mx -= d[a];
    if (ey_of(a) > 0) my += d[a];
    if (ey_of(a) < 0) my -= d[a];
    if (ez_of(a) > 0) mz += d[a];
    if (ez_of(a) < 0) mz -= d[a];
  }
  Mac32 m;
  m.drho = dr;
  m.rho = 1.f + dr;
  const float inv = 1.f / m.rho;
  m.u0 = mx * inv;
  m.u1 = my * inv;
  m.u2 = mz * inv;
  m.usq = m.u0 * m.u0 + m.u1 * m.u1 + m.u2 * m.u2;
  return m;
}

__device__ __forceinline__ Mac32 collide_f32(float (&d)[19], float om, float G) {
  const Mac32 m = macro_f32(d);
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const float deq = deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
    float dn = d[a] - om * (d[a] - deq);
    if (ex_of(a) != 0) dn += (float)ex_of(a) * bi_of(a) * m.rho * G;
    d[a] = dn;
  }
  return m;
}

template <int N>
__device__ __forceinline__ void block_reduce32(double (&v)[N], double *out) {
  __shared__ double red[N][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < N; q++) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < N; q++) {
      double s = red[q][0];
      for (int w = 1; w < nw; w++) s += red[q][w];
      out[q] = s;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void load19f(const float *__restrict__ src, size_t idx, size_t stride, float (&d)[19]) {
#pragma unroll
  for (int a = 0; a < 19; a++) d[a] = __ldg(src + idx + (size_t)a * stride);
}

// ------------------------------------------------------------------ filtered transfer
// One coarse vertex of the filtered fine-to-coarse transfer (FLTR,
// ftcdtransfer_lesfltr.c:163-363, GR = 4) in deviation form: the trapezoid-
// weighted (1/2, 1, 1, 1, 1/2 per axis) sum over the 5 x 5 x 5 fine nodes around
// the vertex (planes kb-2..kb+2, x and y wrapped) of w f^neq / GR^3, added as
// fac x sum to the deviation equilibrium of the vertex node's density and
// momentum (the reference's equilibrium takes the momentum as the velocity).
// Output: f - w of the coarse node.
__device__ __forceinline__ void filtered_node_f32(const float *__restrict__ fs, int nxf, int nyf, int zds, int zdf,
                                                  int gr, int wall, int ic, int jc, float fac, float (&out)[19]) {
  const int kb = wall == 0 ? zdf - 1 - gr : gr;
  const size_t fstride = (size_t)2 * zds * nyf * nxf;
  const float inv_g3 = 1.f / (float)(gr * gr * gr);
  const int i = ic * gr, j = jc * gr;
  float t[19];
#pragma unroll
  for (int a = 0; a < 19; a++) t[a] = 0.f;
  Mac32 c{};
#pragma unroll 1
  for (int ii = -2; ii < 3; ii++) {
    const int x = wrapf(i + ii, nxf);
#pragma unroll 1
    for (int jj = -2; jj < 3; jj++) {
      const int y = wrapf(j + jj, nyf);
      const float wxy = ((ii == -2 || ii == 2) ? 0.5f : 1.f) * ((jj == -2 || jj == 2) ? 0.5f : 1.f) * inv_g3;
#pragma unroll 1
      for (int kk = -2; kk < 3; kk++) {
        const int k = kb + kk;
        const int p = wall == 0 ? k - 1 : zds + k;
        float f[19];
        load19f(fs, ((size_t)p * nyf + y) * nxf + x, fstride, f);
        const Mac32 m = macro_f32(f);
        if (ii == 0 && jj == 0 && kk == 0) c = m;
        const float wq = wxy * ((kk == -2 || kk == 2) ? 0.5f : 1.f);
#pragma unroll
        for (int a = 0; a < 19; a++) t[a] += wq * (f[a] - deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq));
      }
    }
  }
  const float U0 = c.u0 * c.rho, U1 = c.u1 * c.rho, U2 = c.u2 * c.rho;
  const float Usq = U0 * U0 + U1 * U1 + U2 * U2;
#pragma unroll
  for (int a = 0; a < 19; a++) out[a] = deq_f32(a, c.drho, c.rho, U0, U1, U2, Usq) + fac * t[a];
}

// ------------------------------------------------------------------ coarse
template <bool STATS>
__device__ __forceinline__ void coarse_node_f32(float (&f)[19], int i, int j, int k, const Dims &d, float om,
                                                float G, float *__restrict__ dst, size_t pstride, double (&acc)[2],
                                                PlaneStat &sacc) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const Mac32 m = collide_f32(f, om, G);
  if (STATS) sacc.add(m.u0, m.u1, m.u2, 1.0 + (double)m.drho);
  const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
  const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
  float mom = 0.f, den = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int k2 = k + ez_of(a);
    if (k2 < 1 || k2 > nzc - 2) continue;
    const int i2 = ex_of(a) > 0 ? ip : (ex_of(a) < 0 ? im : i);
    const int j2 = ey_of(a) > 0 ? jp : (ey_of(a) < 0 ? jm : j);
    (dst + (size_t)a * pstride)[(unsigned)((k2 * ny + j2) * nx + i2)] = f[a];
    den += f[a];
    if (ex_of(a) > 0) mom += f[a];
    if (ex_of(a) < 0) mom -= f[a];
  }
  acc[0] += mom;
  acc[1] += den;
}

template <bool STATS>
__device__ __forceinline__ void coarse_bulk_f32(float (&f)[19], int i, int j, size_t idx0, const Dims &d, float om,
                                                float G, float *__restrict__ dst, size_t pstride, double (&acc)[2],
                                                PlaneStat &sacc) {
  const int nx = d.nx, ny = d.ny;
  const Mac32 m = collide_f32(f, om, G);
  if (STATS) sacc.add(m.u0, m.u1, m.u2, 1.0 + (double)m.drho);
  const int plane = ny * nx;
  const int dxm = i == 0 ? nx - 1 : -1, dxp = i == nx - 1 ? 1 - nx : 1;
  const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
  // each population array holds fewer than 2^31 floats: 32-bit offsets from
  // the population's (thread-uniform) base
  const unsigned u0 = (unsigned)idx0;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int off = (ez_of(a) > 0 ? plane : (ez_of(a) < 0 ? -plane : 0)) + (ey_of(a) > 0 ? dyp : (ey_of(a) < 0 ? dym : 0)) +
                    (ex_of(a) > 0 ? dxp : (ex_of(a) < 0 ? dxm : 0));
    (dst + (size_t)a * pstride)[u0 + (unsigned)off] = f[a];
  }
  // every push of a bulk node lands on a plane of equal flow-rate weight, so
  // the partials are the node's post-collision moments: the collision keeps
  // mass and momentum and the force adds rho G to sum e_x f (sum e_x^2 B = 1)
  acc[0] += (double)(m.rho * m.u0 + m.rho * G);
  acc[1] += (double)m.drho;
}

// the pushes of one bulk node (fused collision); ACC: accumulate the flow-rate
// partials per destination plane weight
template <bool ACC, int ZSKIP>
__device__ __forceinline__ void fine_push_f32(float (&f)[19], const Mac32 &m, float om, float Gf,
                                              float *__restrict__ dst, size_t pstride, unsigned u0, int plane, int dxm,
                                              int dxp, int dym, int dyp, const float (&wz)[3], double (&acc)[2]) {
  float mom = 0.f, den = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    if ((ZSKIP == 1 && ez_of(a) > 0) || (ZSKIP == 2 && ez_of(a) >= 0) || (ZSKIP == -1 && ez_of(a) < 0) ||
        (ZSKIP == -2 && ez_of(a) <= 0))
      continue;
    const int off = (ez_of(a) > 0 ? plane : (ez_of(a) < 0 ? -plane : 0)) + (ey_of(a) > 0 ? dyp : (ey_of(a) < 0 ? dym : 0)) +
                    (ex_of(a) > 0 ? dxp : (ex_of(a) < 0 ? dxm : 0));
    {
      const float deq = deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
      float dn = f[a] - om * (f[a] - deq);
      if (ex_of(a) != 0) dn += (float)ex_of(a) * bi_of(a) * m.rho * Gf;
      f[a] = dn;
    }
    (dst + (size_t)a * pstride)[u0 + (unsigned)off] = f[a];
    if (ACC) {
      const float wgt = wz[ez_of(a) + 1];
      den += wgt * f[a];
      if (ex_of(a) > 0) mom += wgt * f[a];
      if (ex_of(a) < 0) mom -= wgt * f[a];
    }
  }
  if (ACC) {
    acc[0] += mom;
    acc[1] += den;
  }
}

// ------------------------------------------------------------------ fine
// Bulk planes (every push lands on a fluid plane of the same block: no wall,
// no interface): destinations from precomputed +-1 / +-row / +-plane offsets
// with the periodic wrap folded in; encalc2 weights per destination plane.
// ZSKIP drops the pushes that land on or beyond the block's interface plane,
// as the node rule's block-boundary test does (xfcomputations.c:843-897): the
// interface plane of the destination belongs to the coarse-to-fine transfer,
// which runs concurrently.  +1: e_z > 0 (lower k = zdf-2); +2: e_z >= 0
// (lower k = zdf-1, the interface plane); -1: e_z < 0 (upper k = 1);
// -2: e_z <= 0 (upper k = 0, the interface plane).
template <int MODE, int ZSKIP = 0>
__device__ __forceinline__ void fine_bulk_f32(float (&f)[19], int i, int j, size_t idx0, const Dims &d, float om,
                                              float Gf, float *__restrict__ dst, size_t pstride, const float (&wz)[3],
                                              bool wall_sum_plane, bool wall_rho_plane, double (&acc)[2],
                                              double (&wacc)[2], PlaneStat &sacc) {
  const int nx = d.nxf, ny = d.nyf;
  const Mac32 m = macro_f32(f);
  if (MODE & 2) {
    if (wall_sum_plane) wacc[0] += (double)m.u0;
    if (wall_rho_plane) wacc[1] += 1.0 + (double)m.drho;
  }
  if (MODE & 4) sacc.add(m.u0, m.u1, m.u2, 1.0 + (double)m.drho);
  const int plane = ny * nx;
  const int dxm = i == 0 ? nx - 1 : -1, dxp = i == nx - 1 ? 1 - nx : 1;
  const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
  // each population array holds fewer than 2^31 floats: 32-bit offsets from
  // the population's (thread-uniform) base
  const unsigned u0 = (unsigned)idx0;
  // planes whose three destination planes weigh the same: the flow-rate
  // partials are the node's post-collision moments (as in coarse_bulk_f32)
  const bool wuni = ZSKIP == 0 && wz[0] == wz[1] && wz[1] == wz[2];
  if ((MODE & 1) && wuni) {
    acc[0] += (double)(wz[1] * (m.rho * m.u0 + m.rho * Gf));
    acc[1] += (double)(wz[1] * m.drho);
  }
  if ((MODE & 1) && !wuni)
    fine_push_f32<true, ZSKIP>(f, m, om, Gf, dst, pstride, u0, plane, dxm, dxp, dym, dyp, wz, acc);
  else
    fine_push_f32<false, ZSKIP>(f, m, om, Gf, dst, pstride, u0, plane, dxm, dxp, dym, dyp, wz, acc);
}

// Wall-adjacent planes (lower k = 1, upper k = zdf-2): the regular pushes as
// in the bulk planes; the five populations heading into the wall plane follow
// the node rule (xfcomputations.c:226-240): half-way bounce-back onto the
// node itself when both the destination column and the node's own column are
// solid (flag -1), else specular reflection into the destination column.
template <int MODE, bool UPPER>
__device__ __forceinline__ void fine_wall_f32(float (&f)[19], int i, int j, size_t idx0, const Dims &d, float om,
                                              float Gf, const int8_t *__restrict__ wf, float *__restrict__ dst,
                                              size_t pstride, const float (&wz)[3], bool wall_sum_plane,
                                              bool wall_rho_plane, double (&acc)[2], double (&wacc)[2],
                                              PlaneStat &sacc) {
  const int nx = d.nxf, ny = d.nyf;
  const Mac32 m = macro_f32(f);
  if (MODE & 2) {
    if (wall_sum_plane) wacc[0] += (double)m.u0;
    if (wall_rho_plane) wacc[1] += 1.0 + (double)m.drho;
  }
  if (MODE & 4) sacc.add(m.u0, m.u1, m.u2, 1.0 + (double)m.drho);
  const int plane = ny * nx;
  const int dxm = i == 0 ? nx - 1 : -1, dxp = i == nx - 1 ? 1 - nx : 1;
  const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
  const unsigned u0 = (unsigned)idx0, c0 = (unsigned)(j * nx + i);
  const int8_t own = __ldg(wf + c0);
  float mom = 0.f, den = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int coff = (ey_of(a) > 0 ? dyp : (ey_of(a) < 0 ? dym : 0)) + (ex_of(a) > 0 ? dxp : (ex_of(a) < 0 ? dxm : 0));
    {
      const float deq = deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
      float dn = f[a] - om * (f[a] - deq);
      if (ex_of(a) != 0) dn += (float)ex_of(a) * bi_of(a) * m.rho * Gf;
      f[a] = dn;
    }
    if ((UPPER && ez_of(a) > 0) || (!UPPER && ez_of(a) < 0)) {
      const int8_t sld = __ldg(wf + (c0 + (unsigned)coff));  // 32-bit wrap before the pointer add
      int exd;
      if (sld == -1 && own == -1) {
        (dst + (size_t)opp_of(a) * pstride)[u0] = f[a];
        exd = -ex_of(a);
      } else {
        (dst + (size_t)mir_of(a) * pstride)[u0 + (unsigned)coff] = f[a];
        exd = ex_of(a);
      }
      if (MODE & 1) {
        const float wgt = wz[1];  // stays on the node's plane
        den += wgt * f[a];
        if (exd > 0) mom += wgt * f[a];
        if (exd < 0) mom -= wgt * f[a];
      }
    } else {
      const int off = (ez_of(a) > 0 ? plane : (ez_of(a) < 0 ? -plane : 0)) + coff;
      (dst + (size_t)a * pstride)[u0 + (unsigned)off] = f[a];
      if (MODE & 1) {
        const float wgt = wz[ez_of(a) + 1];
        den += wgt * f[a];
        if (ex_of(a) > 0) mom += wgt * f[a];
        if (ex_of(a) < 0) mom -= wgt * f[a];
      }
    }
  }
  acc[0] += mom;
  acc[1] += den;
}

// ------------------------------------------------------------------ interface
// Coarse-to-fine transfer (ctfdtransfer_opt.c, tinterpolate_hrmt.c,
// derivative.c, bcucof_opt.c) in two fully parallel passes per substep:
//
//  1. corner data: for every (tile, wall, field) the three history levels are
//     combined with the Hermite-in-time weights and the fourth-order x, y and
//     cross derivatives formed in shared memory; each coarse interface node
//     gets C = (value, d/dx, d/dy, d2/dxdy) as one float4 [2][23][ny][nx].
//  2. evaluation: one thread per fine interface node reads its cell's four
//     corners per field and evaluates the bicubic patch as the tensor product
//     of the cubic Hermite basis
//       h00(t) = 2t^3 - 3t^2 + 1, h01(t) = -2t^3 + 3t^2, h10(t) = t^3 - 2t^2 + t, h11(t) = t^3 - t^2,
//       p(t, u) = sum_{a,b in 0,1} [h0a(t) h0b(u) V + h1a(t) h0b(u) Dx + h0a(t) h1b(u) Dy + h1a(t) h1b(u) Dxy],
//     the polynomial the reference's 16-coefficient map gives at unit spacing
//     (20 multiply-adds per node instead of 256 + 16); then
//     f_a = feq_a(rho^, u^) + fac fneq^_a into the wall's interface plane.
// The FP32 form keeps its own rounding order (it is compared with the FP64
// oracle within a tolerance, not bit for bit).
struct IfParams32 {
  const float *hn, *hp, *hpp;  // history slots of levels n, p, pp: [2 walls][23][ny][nx]
  float4 *corner;              // corner data [2 walls][23][ny][nx]
  float *fdst;                 // fine lattice receiving the interface planes
  int nx, ny, nxf, nyf, zds;
  float an, ap, app;           // Hermite-in-time weights of levels n, p, pp
  float fac;                   // omega_c / (GR omega_f): non-equilibrium rescaling
};

// launch parameters of one substep's transfer (substep s of GR: time s/GR)
inline IfParams32 iface_params32(const float *hn, const float *hp, const float *hpp, float4 *corner, float *fdst,
                                 const Dims &d, int substep, double omega_c, double omega_f) {
  // value = h00 p + h10 (n - pp)/2 + h01 n + h11 (3n - 4p + pp)/2 (tinterpolate_hrmt.c:28-34),
  // gathered per level
  const double t = (double)substep / (double)d.gr, t2 = t * t, t3 = t2 * t;
  const double h1 = 2. * t3 - 3. * t2 + 1., h2 = t3 - 2. * t2 + t, h3 = -2. * t3 + 3. * t2, h4 = t3 - t2;
  IfParams32 P;
  P.hn = hn;
  P.hp = hp;
  P.hpp = hpp;
  P.corner = corner;
  P.fdst = fdst;
  P.nx = d.nx;
  P.ny = d.ny;
  P.nxf = d.nxf;
  P.nyf = d.nyf;
  P.zds = d.zds;
  P.an = (float)(0.5 * h2 + h3 + 1.5 * h4);
  P.ap = (float)(h1 - 2. * h4);
  P.app = (float)(-0.5 * h2 + 0.5 * h4);
  P.fac = (float)(omega_c / ((double)d.gr * omega_f));
  return P;
}

// pass 1 tile: CTX x CTY interface nodes; a work item covers a group of fields
constexpr int CTX = 32, CTY = 8;
#ifndef DNS_CORNER_FIELD_GROUPS
#define DNS_CORNER_FIELD_GROUPS 3
#endif
constexpr int kCornerFieldGroups = DNS_CORNER_FIELD_GROUPS;  // work items per (tile, wall): field groups
__host__ __device__ constexpr int corner_field(int g) { return 23 * g / kCornerFieldGroups; }
struct IfCornerSmem {
  float V[CTY + 4][CTX + 4];
  float DY[CTY][CTX + 4];
};

// Fields [f0, f1) of one (tile, wall): the next field's history values are
// loaded into registers while the current one is differentiated.
__device__ __forceinline__ void iface_corner_tile32(IfCornerSmem &S, const IfParams32 &P, int tx, int ty, int w,
                                                    int f0, int f1) {
  constexpr int QX = CTX + 4, QY = CTY + 4, NV = (QX * QY + kThreads - 1) / kThreads;
  const float c2o3 = 2.f / 3.f, c1o12 = 1.f / 12.f;
  const int i0 = tx * CTX, j0 = ty * CTY;
  const size_t plane = (size_t)P.ny * P.nx;
  // the last substep (t = 1) is level n alone
  const bool one = P.ap == 0.f && P.app == 0.f;
  int off[NV];
  float vn[NV], vp[NV], vpp[NV];
#pragma unroll
  for (int s = 0; s < NV; s++) {
    const int q = threadIdx.x + s * kThreads;
    off[s] = -1;
    vn[s] = vp[s] = vpp[s] = 0.f;
    if (q < QX * QY) off[s] = wrapf(j0 - 2 + q / QX, P.ny) * P.nx + wrapf(i0 - 2 + q % QX, P.nx);
  }
  auto fetch = [&](int f) {
    const size_t fo = ((size_t)w * 23 + f) * plane;
#pragma unroll
    for (int s = 0; s < NV; s++)
      if (off[s] >= 0) {
        vn[s] = __ldg(P.hn + fo + off[s]);
        if (!one) {
          vp[s] = __ldg(P.hp + fo + off[s]);
          vpp[s] = __ldg(P.hpp + fo + off[s]);
        }
      }
  };
  fetch(f0);
  float *V = &S.V[0][0];
  for (int f = f0; f < f1; f++) {
#pragma unroll
    for (int s = 0; s < NV; s++)
      if (off[s] >= 0) V[threadIdx.x + s * kThreads] = one ? vn[s] : P.an * vn[s] + P.ap * vp[s] + P.app * vpp[s];
    if (f + 1 < f1) fetch(f + 1);
    __syncthreads();
#pragma unroll
    for (int s = 0; s < (QX * CTY + kThreads - 1) / kThreads; s++) {
      const int q = threadIdx.x + s * kThreads;
      if (q < QX * CTY) {
        const int pi = q % QX, r = q / QX;
        S.DY[r][pi] = c2o3 * (S.V[r + 3][pi] - S.V[r + 1][pi]) - c1o12 * (S.V[r + 4][pi] - S.V[r][pi]);
      }
    }
    __syncthreads();
    float4 *out = P.corner + ((size_t)w * 23 + f) * plane;
#pragma unroll
    for (int s = 0; s < CTX * CTY / kThreads; s++) {
      const int q = threadIdx.x + s * kThreads;
      const int c = q % CTX, r = q / CTX;
      if (i0 + c < P.nx && j0 + r < P.ny) {
        const float dx =
            c2o3 * (S.V[r + 2][c + 3] - S.V[r + 2][c + 1]) - c1o12 * (S.V[r + 2][c + 4] - S.V[r + 2][c]);
        const float dxy = c2o3 * (S.DY[r][c + 3] - S.DY[r][c + 1]) - c1o12 * (S.DY[r][c + 4] - S.DY[r][c]);
        out[(size_t)(j0 + r) * P.nx + i0 + c] = make_float4(S.V[r + 2][c + 2], dx, S.DY[r][c + 2], dxy);
      }
    }
    __syncthreads();  // V and DY are rewritten for the next field (or the next item)
  }
}

struct Herm {
  float a0, a1, b0, b1;  // h00, h01, h10, h11
};

// e_x, e_y, e_z, w of each population, for loops over a run-time population
#define DNS_POP_ROW(a) {(float)ex_of(a), (float)ey_of(a), (float)ez_of(a), w_of(a)}
static __constant__ float c_pop[19][4] = {
    DNS_POP_ROW(0),  DNS_POP_ROW(1),  DNS_POP_ROW(2),  DNS_POP_ROW(3),  DNS_POP_ROW(4),
    DNS_POP_ROW(5),  DNS_POP_ROW(6),  DNS_POP_ROW(7),  DNS_POP_ROW(8),  DNS_POP_ROW(9),
    DNS_POP_ROW(10), DNS_POP_ROW(11), DNS_POP_ROW(12), DNS_POP_ROW(13), DNS_POP_ROW(14),
    DNS_POP_ROW(15), DNS_POP_ROW(16), DNS_POP_ROW(17), DNS_POP_ROW(18)};
#undef DNS_POP_ROW
__device__ __forceinline__ Herm herm_at(float t) {
  const float t2 = t * t, t3 = t2 * t;
  return Herm{2.f * t3 - 3.f * t2 + 1.f, -2.f * t3 + 3.f * t2, t3 - 2.f * t2 + t, t3 - t2};
}

// pass 2 tile: TX x TY interface cells; the fine tile is GR*TX (<= 64) columns
// wide and thread t evaluates fine column (t & 63) of rows (t >> 6) + 2r.
template <int GR>
struct IfTile;
template <>
struct IfTile<2> {
  static constexpr int TX = 32, TY = 8;
};
template <>
struct IfTile<3> {
  static constexpr int TX = 21, TY = 6;
};
template <>
struct IfTile<4> {
  static constexpr int TX = 16, TY = 4;
};
constexpr int kEvalStages = 4;     // corner tiles in flight
#ifndef DNS_EVAL_POP_GROUPS
#define DNS_EVAL_POP_GROUPS 2
#endif
constexpr int kEvalPopGroups = DNS_EVAL_POP_GROUPS;  // population groups per (tile, wall)

template <int GR>
struct IfEvalSmem {
  static constexpr int CW = IfTile<GR>::TX + 1, CH = IfTile<GR>::TY + 1;
  float4 C[kEvalStages][CH][CW];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int GR>
__device__ __forceinline__ void if_rowpass32(const float4 (&C)[IfTile<GR>::TY + 1][IfTile<GR>::TX + 1], int cx,
                                             int cr, const Herm &hx, float &p, float &q) {
  const float4 c0 = C[cr][cx], c1 = C[cr][cx + 1];
  p = hx.a0 * c0.x + hx.a1 * c1.x + hx.b0 * c0.y + hx.b1 * c1.y;
  q = hx.a0 * c0.z + hx.a1 * c1.z + hx.b0 * c0.w + hx.b1 * c1.w;
}

// GR = 2, a warp's nodes all at sub-position (II, JJ) of their cells: the
// Hermite basis is (1, 0, 0, 0) at t = 0 and (1/2, 1/2, 1/8, -1/8) at t = 1/2,
// so II = 0 needs no x-pass and JJ = 0 no y-pass; cell row r is node r.
template <int II, int JJ, int NR, int CH, int CW>
__device__ __forceinline__ void if_col2(const float4 (&C)[CH][CW], int cx, float (&val)[NR]) {
  auto xpass = [&](int r, float &p, float &q) {
    const float4 c0 = C[r][cx];
    if (II == 0) {
      p = c0.x;
      q = c0.z;
    } else {
      const float4 c1 = C[r][cx + 1];
      p = 0.5f * (c0.x + c1.x) + 0.125f * (c0.y - c1.y);
      q = 0.5f * (c0.z + c1.z) + 0.125f * (c0.w - c1.w);
    }
  };
  if (JJ == 0) {
#pragma unroll
    for (int r = 0; r < NR; r++) {
      float p, q;
      xpass(r, p, q);
      val[r] = p;
    }
  } else {
    float p0, q0;
    xpass(0, p0, q0);
#pragma unroll
    for (int r = 0; r < NR; r++) {
      float p1, q1;
      xpass(r + 1, p1, q1);
      val[r] = 0.5f * (p0 + p1) + 0.125f * (q0 - q1);
      p0 = p1;
      q0 = q1;
    }
  }
}

// the NR node values of the thread's fine column (cell column cx, basis hx;
// for GR = 2 the sub-position ii and jj = fy0 are warp-uniform)
template <int GR, int NR>
__device__ __forceinline__ void if_column32(const float4 (&C)[IfTile<GR>::TY + 1][IfTile<GR>::TX + 1], int cx, int ii,
                                           int fy0, const Herm &hx, float (&val)[NR]) {
  constexpr int CH = IfTile<GR>::TY + 1, CW = IfTile<GR>::TX + 1;
  if constexpr (GR == 2) {
    switch (ii * 2 + fy0) {
      case 0: if_col2<0, 0, NR, CH, CW>(C, cx, val); break;
      case 1: if_col2<0, 1, NR, CH, CW>(C, cx, val); break;
      case 2: if_col2<1, 0, NR, CH, CW>(C, cx, val); break;
      default: if_col2<1, 1, NR, CH, CW>(C, cx, val); break;
    }
  } else {
#pragma unroll
    for (int r = 0; r < NR; r++) {
      const int fy = fy0 + 2 * r, cy = fy / GR, jj = fy - cy * GR;
      const Herm hy = herm_at((float)jj * (1.f / GR));
      float p0, q0, p1, q1;
      if_rowpass32<GR>(C, cx, cy, hx, p0, q0);
      if_rowpass32<GR>(C, cx, cy + 1, hx, p1, q1);
      val[r] = hy.a0 * p0 + hy.a1 * p1 + hy.b0 * q0 + hy.b1 * q1;
    }
  }
}

// GR = 2, both fine columns of cell column cx (sub-positions 0 and 1) at
// sub-row JJ of the NR cell rows cy0, cy0 + 2, ...: v[r][0] / v[r][1] (the
// arithmetic of if_col2 for II = 0 and II = 1).
template <int JJ, int NR, int CH, int CW>
__device__ __forceinline__ void if_pair2(const float4 (&C)[CH][CW], int cx, int cy0, float (&v)[NR][2]) {
  auto xpass = [&](int r, float &p0, float &q0, float &p1, float &q1) {
    const float4 c0 = C[r][cx], c1 = C[r][cx + 1];
    p0 = c0.x;
    q0 = c0.z;
    p1 = 0.5f * (c0.x + c1.x) + 0.125f * (c0.y - c1.y);
    q1 = 0.5f * (c0.z + c1.z) + 0.125f * (c0.w - c1.w);
  };
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int cy = cy0 + 2 * r;
    float pa0, qa0, pa1, qa1;
    xpass(cy, pa0, qa0, pa1, qa1);
    if (JJ == 0) {
      v[r][0] = pa0;
      v[r][1] = pa1;
    } else {
      float pb0, qb0, pb1, qb1;
      xpass(cy + 1, pb0, qb0, pb1, qb1);
      v[r][0] = 0.5f * (pa0 + pb0) + 0.125f * (qa0 - qb0);
      v[r][1] = 0.5f * (pa1 + pb1) + 0.125f * (qa1 - qb1);
    }
  }
}

// GR = 2 form of iface_eval_tile32: a thread takes both fine columns of one
// cell column and the fine rows w, w + 4, ... of its warp w, so that a warp
// stores 32 consecutive column pairs (256 contiguous bytes) per row.
__device__ __forceinline__ void iface_eval_tile32_gr2(IfEvalSmem<2> &S, const IfParams32 &P, int tx, int ty, int w,
                                                      int a0, int a1) {
  constexpr int TX = IfTile<2>::TX, TY = IfTile<2>::TY, NR = TY / 2;  // rows per thread
  constexpr int CW = TX + 1, CH = TY + 1, NC = CW * CH, NCS = (NC + kThreads - 1) / kThreads;
  static_assert(kThreads == 128 && TX == 32, "four warps of 32 cell columns");
  const int i0 = tx * TX, j0 = ty * TY;
  const int t = threadIdx.x, cx = t & 31, wp = t >> 5;
  const int jj = wp & 1, cy0 = wp >> 1;  // fine rows 2 (cy0 + 2 r) + jj
  const bool colok = i0 + cx < P.nx;
  const size_t plane = (size_t)P.ny * P.nx;
  int goff[NCS];
#pragma unroll
  for (int s = 0; s < NCS; s++) {
    const int c = t + s * kThreads;
    goff[s] = c < NC ? wrapf(j0 + c / CW, P.ny) * P.nx + wrapf(i0 + c % CW, P.nx) : -1;
  }
  const int nf = 4 + (a1 - a0);
  auto issue = [&](int k) {
    if (k < nf) {
      const int f = k < 4 ? k : 4 + a0 + (k - 4);
      const float4 *src = P.corner + ((size_t)w * 23 + f) * plane;
      float4 *dst = &S.C[k % kEvalStages][0][0];
#pragma unroll
      for (int s = 0; s < NCS; s++)
        if (goff[s] >= 0) cp_async16(dst + t + s * kThreads, src + goff[s]);
    }
    cp_async_commit();
  };
  auto column = [&](int k, float (&v)[NR][2]) {
    if (jj == 0)
      if_pair2<0, NR, CH, CW>(S.C[k % kEvalStages], cx, cy0, v);
    else
      if_pair2<1, NR, CH, CW>(S.C[k % kEvalStages], cx, cy0, v);
  };
#pragma unroll
  for (int k = 0; k < kEvalStages - 1; k++) issue(k);
  float mac[4][NR][2];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    cp_async_wait<kEvalStages - 2>();
    __syncthreads();
    issue(k + kEvalStages - 1);
    column(k, mac[k]);
  }
  float usq[NR][2];
#pragma unroll
  for (int r = 0; r < NR; r++)
#pragma unroll
    for (int h = 0; h < 2; h++)
      usq[r][h] = mac[1][r][h] * mac[1][r][h] + mac[2][r][h] * mac[2][r][h] + mac[3][r][h] * mac[3][r][h];
  const size_t fplane = (size_t)P.nyf * P.nxf, fstride = (size_t)2 * P.zds * fplane;
  const int pf = w == 0 ? P.zds - 1 : P.zds;
  float *out = P.fdst + (size_t)pf * fplane;
  for (int k = 4; k < nf; k++) {
    cp_async_wait<kEvalStages - 2>();
    __syncthreads();
    issue(k + kEvalStages - 1);
    const int a = a0 + (k - 4);
    float fv[NR][2];
    column(k, fv);
    const float ex = c_pop[a][0], ey = c_pop[a][1], ez = c_pop[a][2], wa = c_pop[a][3];
    float *oa = out + (size_t)a * fstride;
#pragma unroll
    for (int r = 0; r < NR; r++) {
      const int cy = cy0 + 2 * r;
      if (colok && j0 + cy < P.ny) {
        float o[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const float dr = mac[0][r][h], eu = ex * mac[1][r][h] + ey * mac[2][r][h] + ez * mac[3][r][h];
          const float deq = wa * (dr + (1.f + dr) * (3.f * eu + 4.5f * eu * eu - 1.5f * usq[r][h]));
          o[h] = deq + P.fac * fv[r][h];
        }
        *reinterpret_cast<float2 *>(oa + (size_t)((j0 + cy) * 2 + jj) * P.nxf + (i0 + cx) * 2) =
            make_float2(o[0], o[1]);
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // the ring may be reused by the next item
}

// One (tile, wall) and populations [a0, a1) (the macroscopic fields always):
// the corner tiles of successive fields stream into shared memory through a
// cp.async ring while earlier ones are evaluated.  blockDim.x == kThreads.
template <int GR>
__device__ __forceinline__ void iface_eval_tile32(IfEvalSmem<GR> &S, const IfParams32 &P, int tx, int ty, int w,
                                                  int a0, int a1) {
  if constexpr (GR == 2) {
    iface_eval_tile32_gr2(S, P, tx, ty, w, a0, a1);
    return;
  }
  constexpr int TX = IfTile<GR>::TX, TY = IfTile<GR>::TY, NR = GR * TY / 2;
  constexpr int CW = TX + 1, CH = TY + 1, NC = CW * CH, NCS = (NC + kThreads - 1) / kThreads;
  const int i0 = tx * TX, j0 = ty * TY;
  // GR = 2: lanes take consecutive cells and a warp one sub-position ii, so
  // the fine column is 2 cx + ii; otherwise lanes take consecutive fine columns
  const int t = threadIdx.x, fy0 = (t >> 6) & 1;
  const int fx = GR == 2 ? 2 * (t & 31) + ((t >> 5) & 1) : (t & 63);
  const bool colok = fx < GR * TX && i0 + fx / GR < P.nx;
  const int cx = colok ? fx / GR : 0, ii = colok ? fx - cx * GR : 0;  // idle lanes read in bounds
  const Herm hx = herm_at((float)ii * (1.f / GR));
  const size_t plane = (size_t)P.ny * P.nx;
  int goff[NCS];
#pragma unroll
  for (int s = 0; s < NCS; s++) {
    const int c = t + s * kThreads;
    goff[s] = c < NC ? wrapf(j0 + c / CW, P.ny) * P.nx + wrapf(i0 + c % CW, P.nx) : -1;
  }
  const int nf = 4 + (a1 - a0);
  auto issue = [&](int k) {
    if (k < nf) {
      const int f = k < 4 ? k : 4 + a0 + (k - 4);
      const float4 *src = P.corner + ((size_t)w * 23 + f) * plane;
      float4 *dst = &S.C[k % kEvalStages][0][0];
#pragma unroll
      for (int s = 0; s < NCS; s++)
        if (goff[s] >= 0) cp_async16(dst + t + s * kThreads, src + goff[s]);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int k = 0; k < kEvalStages - 1; k++) issue(k);
  float mac[4][NR];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    cp_async_wait<kEvalStages - 2>();
    __syncthreads();
    issue(k + kEvalStages - 1);
    if_column32<GR, NR>(S.C[k % kEvalStages], cx, ii, fy0, hx, mac[k]);
  }
  float usq[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) usq[r] = mac[1][r] * mac[1][r] + mac[2][r] * mac[2][r] + mac[3][r] * mac[3][r];
  const size_t fplane = (size_t)P.nyf * P.nxf, fstride = (size_t)2 * P.zds * fplane;
  const int pf = w == 0 ? P.zds - 1 : P.zds;
  float *out = P.fdst + (size_t)pf * fplane;
  for (int k = 4; k < nf; k++) {
    cp_async_wait<kEvalStages - 2>();
    __syncthreads();
    issue(k + kEvalStages - 1);
    const int a = a0 + (k - 4);
    float fv[NR];
    if_column32<GR, NR>(S.C[k % kEvalStages], cx, ii, fy0, hx, fv);
    const float ex = c_pop[a][0], ey = c_pop[a][1], ez = c_pop[a][2], wa = c_pop[a][3];
    float *oa = out + (size_t)a * fstride;
#pragma unroll
    for (int r = 0; r < NR; r++) {
      const int fy = fy0 + 2 * r, cy = fy / GR, jj = fy - cy * GR;
      if (colok && j0 + cy < P.ny) {
        const float dr = mac[0][r], eu = ex * mac[1][r] + ey * mac[2][r] + ez * mac[3][r];
        const float deq = wa * (dr + (1.f + dr) * (3.f * eu + 4.5f * eu * eu - 1.5f * usq[r]));
        oa[(size_t)((j0 + cy) * GR + jj) * P.nxf + (i0 + cx) * GR + ii] = deq + P.fac * fv[r];
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // the ring may be reused by the next item
}

}  // namespace f32
}  // namespace dns
