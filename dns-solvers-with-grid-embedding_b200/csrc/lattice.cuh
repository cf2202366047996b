// D3Q19 lattice arithmetic shared by the kernels.
//
// Population order, weights and forcing weights are the reference's
// (src/globals.c:3-13): 0 rest; 1/2 +-x; 3/4 +-y; 5/6 +-z; 7..10 xy diagonals
// (+,+) (-,+) (-,-) (+,-); 11..14 xz (+,+) (+,-) (-,-) (-,+); 15..18 yz
// (+,+) (+,-) (-,-) (-,+).  opposite / mirror are the reference's tables.
//
// The FP64 helpers evaluate every expression in the reference's order
// (xcomputations.c:61-86): moments summed in population order, the velocity
// projection e.u, feq = (w rho) (((1 + 3u) + (4.5u)u) - 1.5v) and the update
// f + (F - omega (f - feq)).  The translation unit that includes them is built
// with -fmad=false, so with IEEE division the results are bit-identical to the
// reference compiled without fused multiply-add.  Terms the reference
// multiplies by a zero velocity component are dropped: adding an exact zero
// cannot change a non-zero sum, and a zero-valued velocity only changes the
// sign of a zero that is later added to 1.
#pragma once

#include <cstddef>

#include "kernels.h"

namespace dns {

__host__ __device__ constexpr int ex_of(int a) {
  return (a == 1 || a == 7 || a == 10 || a == 11 || a == 12) ? 1
         : (a == 2 || a == 8 || a == 9 || a == 13 || a == 14) ? -1 : 0;
}
__host__ __device__ constexpr int ey_of(int a) {
  return (a == 3 || a == 7 || a == 8 || a == 15 || a == 16) ? 1
         : (a == 4 || a == 9 || a == 10 || a == 17 || a == 18) ? -1 : 0;
}
__host__ __device__ constexpr int ez_of(int a) {
  return (a == 5 || a == 11 || a == 14 || a == 15 || a == 18) ? 1
         : (a == 6 || a == 12 || a == 13 || a == 16 || a == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp_of(int a) {
  return a == 0 ? 0 : (a <= 6 ? (a % 2 ? a + 1 : a - 1) : (a <= 10 ? (a <= 8 ? a + 2 : a - 2) : (a <= 14 ? (a <= 12 ? a + 2 : a - 2) : (a <= 16 ? a + 2 : a - 2))));
}
__host__ __device__ constexpr int mir_of(int a) {
  return (a == 5) ? 6 : (a == 6) ? 5 : (a == 11) ? 12 : (a == 12) ? 11 : (a == 13) ? 14 : (a == 14) ? 13
         : (a == 15) ? 16 : (a == 16) ? 15 : (a == 17) ? 18 : (a == 18) ? 17 : a;
}
// weight class: 0 rest, 1 axis, 2 diagonal
__host__ __device__ constexpr int wclass_of(int a) { return a == 0 ? 0 : (a <= 6 ? 1 : 2); }

static_assert(opp_of(7) == 9 && opp_of(8) == 10 && opp_of(11) == 13 && opp_of(12) == 14 && opp_of(15) == 17 &&
                  opp_of(16) == 18 && opp_of(1) == 2 && opp_of(6) == 5,
              "opposite table");

// Moments of one node: dens = sum f_a, m = sum e_a f_a, each in population order.
__device__ __forceinline__ void moments_f64(const double (&f)[19], double &dens, double &mx, double &my,
                                            double &mz) {
  double d = f[0];
#pragma unroll
  for (int a = 1; a < 19; a++) d = d + f[a];
  double x = f[1];
  x = x - f[2]; x = x + f[7]; x = x - f[8]; x = x - f[9]; x = x + f[10];
  x = x + f[11]; x = x + f[12]; x = x - f[13]; x = x - f[14];
  double y = f[3];
  y = y - f[4]; y = y + f[7]; y = y + f[8]; y = y - f[9]; y = y - f[10];
  y = y + f[15]; y = y + f[16]; y = y - f[17]; y = y - f[18];
  double z = f[5];
  z = z - f[6]; z = z + f[11]; z = z - f[12]; z = z - f[13]; z = z + f[14];
  z = z + f[15]; z = z - f[16]; z = z - f[17]; z = z + f[18];
  dens = d;
  mx = x;
  my = y;
  mz = z;
}

// e_a . u for every population, as the reference forms it
// (E0 u0 + E1 u1) + E2 u2 with the zero terms dropped.
__device__ __forceinline__ double proj_f64(int a, double u0, double u1, double u2) {
  switch (a) {
    case 0: return 0.0;
    case 1: return u0;
    case 2: return -u0;
    case 3: return u1;
    case 4: return -u1;
    case 5: return u2;
    case 6: return -u2;
    case 7: return u0 + u1;
    case 8: return -u0 + u1;
    case 9: return -u0 - u1;
    case 10: return u0 - u1;
    case 11: return u0 + u2;
    case 12: return u0 - u2;
    case 13: return -u0 - u2;
    case 14: return -u0 + u2;
    case 15: return u1 + u2;
    case 16: return u1 - u2;
    case 17: return -u1 - u2;
    default: return -u1 + u2;
  }
}

// Equilibrium of population a given wr = w_a rho and t15v = 1.5 v.
__device__ __forceinline__ double feq_f64(double wr, double u, double t15v) {
  return wr * (1. + 3. * u + 4.5 * u * u - t15v);
}

struct Weighted {
  double w0, w1, w2;  // w_a rho per weight class
};

__device__ __forceinline__ Weighted weighted_rho(double dens) {
  Weighted r;
  r.w0 = (1. / 3.) * dens;
  r.w1 = (1. / 18.) * dens;
  r.w2 = (1. / 36.) * dens;
  return r;
}

// BGK collision with body force G in place; returns the pre-collision
// moments (dens, velocity) for the reductions.
__device__ __forceinline__ void collide_f64(double (&f)[19], double om, double G, double &dens, double &u0,
                                            double &u1, double &u2) {
  double mx, my, mz;
  moments_f64(f, dens, mx, my, mz);
  u0 = mx / dens;
  u1 = my / dens;
  u2 = mz / dens;
  const double v = u0 * u0 + u1 * u1 + u2 * u2;
  const double t15v = 1.5 * v;
  const Weighted wr = weighted_rho(dens);
  const double q1 = (1. / 6.) * dens * G;   // BI_a rho G, axis directions
  const double q2 = (1. / 12.) * dens * G;  // diagonals
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int c = wclass_of(a);
    const double wra = c == 0 ? wr.w0 : (c == 1 ? wr.w1 : wr.w2);
    const double feq = feq_f64(wra, proj_f64(a, u0, u1, u2), t15v);
    const double t = om * (f[a] - feq);
    const int ex = ex_of(a);
    if (ex == 0) {
      f[a] = f[a] - t;                                   // f + (0 - t)
    } else {
      const double q = c == 1 ? q1 : q2;
      f[a] = ex > 0 ? f[a] + (q - t) : f[a] - (q + t);   // f + (+-q - t)
    }
  }
}


// ------------------------------------------------------------------ sampled statistics
// Moments of a set of nodes' u, v, w, rho: count n, means m and sums of
// squared deviations from the means q = (uu, vv, ww, uw, rr).  add() is
// Welford's update, merge() the pairwise combination of Chan, Golub and
// LeVeque (1979); neither forms E[x^2] - E[x]^2, so a small variance under a
// large mean keeps its digits.
struct PlaneStat {
  double n, m[4], q[5];
  __device__ __forceinline__ void init() {
    n = 0.;
#pragma unroll
    for (int c = 0; c < 4; c++) m[c] = 0.;
#pragma unroll
    for (int c = 0; c < 5; c++) q[c] = 0.;
  }
  __device__ __forceinline__ void add(double u0, double u1, double u2, double rho) {
    n += 1.;
    const double inv = 1. / n;
    const double d0 = u0 - m[0], d1 = u1 - m[1], d2 = u2 - m[2], d3 = rho - m[3];
    m[0] += d0 * inv;
    m[1] += d1 * inv;
    m[2] += d2 * inv;
    m[3] += d3 * inv;
    q[0] += d0 * (u0 - m[0]);
    q[1] += d1 * (u1 - m[1]);
    q[2] += d2 * (u2 - m[2]);
    q[3] += d0 * (u2 - m[2]);
    q[4] += d3 * (rho - m[3]);
  }
  __device__ __forceinline__ void merge(double nb, const double (&mb)[4], const double (&qb)[5]) {
    if (nb == 0.) return;
    if (n == 0.) {
      n = nb;
#pragma unroll
      for (int c = 0; c < 4; c++) m[c] = mb[c];
#pragma unroll
      for (int c = 0; c < 5; c++) q[c] = qb[c];
      return;
    }
    const double nt = n + nb, f = nb / nt, g = n * f;
    const double d0 = mb[0] - m[0], d1 = mb[1] - m[1], d2 = mb[2] - m[2], d3 = mb[3] - m[3];
    q[0] += qb[0] + d0 * d0 * g;
    q[1] += qb[1] + d1 * d1 * g;
    q[2] += qb[2] + d2 * d2 * g;
    q[3] += qb[3] + d0 * d2 * g;
    q[4] += qb[4] + d3 * d3 * g;
    m[0] += d0 * f;
    m[1] += d1 * f;
    m[2] += d2 * f;
    m[3] += d3 * f;
    n = nt;
  }
  __device__ __forceinline__ void merge(const double *p) {  // a stored (n, m[4], q[5])
    const double mb[4] = {p[1], p[2], p[3], p[4]}, qb[5] = {p[5], p[6], p[7], p[8], p[9]};
    merge(p[0], mb, qb);
  }
  __device__ __forceinline__ void store(double *p) const {
    p[0] = n;
#pragma unroll
    for (int c = 0; c < 4; c++) p[1 + c] = m[c];
#pragma unroll
    for (int c = 0; c < 5; c++) p[5 + c] = q[c];
  }
};

// Merge the block's PlaneStats in a fixed order (warp shuffles, then the
// warps in order) and store the result (kStatPart doubles) at out.  Every
// thread of the block must call it; blockDim.x is a multiple of 32, at most 1024.
__device__ __forceinline__ void block_reduce_stat(PlaneStat st, double *out) {
  __shared__ double red[32][kStatPart];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double nb = __shfl_down_sync(0xffffffffu, st.n, o);
    double mb[4], qb[5];
#pragma unroll
    for (int c = 0; c < 4; c++) mb[c] = __shfl_down_sync(0xffffffffu, st.m[c], o);
#pragma unroll
    for (int c = 0; c < 5; c++) qb[c] = __shfl_down_sync(0xffffffffu, st.q[c], o);
    if (lane + o < 32) st.merge(nb, mb, qb);
  }
  if (lane == 0) st.store(red[warp]);
  __syncthreads();
  if (threadIdx.x == 0) {
    PlaneStat t;
    t.init();
    for (int w = 0; w < nw; w++) t.merge(red[w]);
    t.store(out);
  }
  __syncthreads();
}

// Add one sample's plane moments s (n, means, sums of squared deviations) to
// the running-statistics row o (layout in kernels.h).  The first sample after
// a reset sets the reference c of the plane means.
__device__ __forceinline__ void stat_row_add(double *o, const PlaneStat &s) {
  if (o[15] == 0.) {
#pragma unroll
    for (int c = 0; c < 4; c++) o[16 + c] = s.m[c];
  }
  const double d0 = s.m[0] - o[16], d1 = s.m[1] - o[17], d2 = s.m[2] - o[18], d3 = s.m[3] - o[19];
  o[0] += d0;
  o[1] += d1;
  o[2] += d2;
  o[3] += d3;
  o[4] += d0 * d0;
  o[5] += d1 * d1;
  o[6] += d2 * d2;
  o[7] += d0 * d2;
  o[8] += d3 * d3;
  const double inv = 1. / s.n;
#pragma unroll
  for (int c = 0; c < 5; c++) o[9 + c] += s.q[c] * inv;
  o[14] = s.n;
  o[15] += 1.0;
}

// Per-plane finalize of one sample: merge the plane's nb block partials (each
// kStatPart doubles) in a fixed order (thread t takes blocks t, t + T, ...,
// then the threads in order) and add the plane's moments to the row.
__device__ __forceinline__ void stat_plane_finalize(const double *parts, long nb, double *row) {
  PlaneStat st;
  st.init();
  for (long q = threadIdx.x; q < nb; q += blockDim.x) st.merge(parts + q * kStatPart);
  __shared__ double part[kStatPart];
  block_reduce_stat(st, part);
  if (threadIdx.x == 0) {
    PlaneStat t;
    t.init();
    t.merge(part);
    stat_row_add(row, t);
  }
}

}  // namespace dns
