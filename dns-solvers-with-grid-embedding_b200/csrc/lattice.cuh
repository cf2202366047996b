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
// Composite-profile index of coarse plane k (k = 2..zdc-3) and of fine device
// plane p (lower block k = p + 1, upper block k = p - zds), statistics.c:52-146;
// profile_plane inverts them: level (0 coarse, 1 fine) and plane (coarse k or
// fine device plane) of index idx, or level -1 for the two wall points.
__host__ __device__ __forceinline__ int profile_index_coarse(int k, int zdf) { return zdf - 2 + k; }
__host__ __device__ __forceinline__ int profile_index_fine(int p, int zds, int zdf, int nzc) {
  return p < zds ? p + 1 : zdf + nzc - 4 + (p - zds);
}
__host__ __device__ __forceinline__ void profile_plane(int idx, int zds, int zdf, int nzc, int &level, int &plane) {
  level = -1;
  plane = 0;
  if (idx >= 1 && idx <= zdf - 1) {
    level = 1;
    plane = idx - 1;
  } else if (idx >= zdf && idx <= zdf + nzc - 5) {
    level = 0;
    plane = idx - zdf + 2;
  } else if (idx >= zdf + nzc - 4 && idx <= 2 * zdf + nzc - 6) {
    level = 1;
    plane = zds + idx - (zdf + nzc - 4);
  }
}

// One block's sums of the sampled moments of its nodes, taken about the plane's
// shift (the running-statistics row's entries 16..19).
struct PlaneStat {
  double s[9];
  double sh[4];
  __device__ __forceinline__ void init(const double *rows, int idx, bool on) {
#pragma unroll
    for (int c = 0; c < 9; c++) s[c] = 0.;
#pragma unroll
    for (int c = 0; c < 4; c++) sh[c] = on ? rows[(size_t)idx * kStatRow + 16 + c] : 0.;
  }
  __device__ __forceinline__ void add(double u0, double u1, double u2, double rho) {
    const double a = u0 - sh[0], b = u1 - sh[1], c = u2 - sh[2], r = rho - sh[3];
    s[0] += a; s[1] += b; s[2] += c; s[3] += r;
    s[4] += a * a; s[5] += b * b; s[6] += c * c; s[7] += a * c; s[8] += r * r;
  }
};

// Add one sample's plane sums s9 (taken about the row's shift) to the row o of
// nn nodes.  A row without a shift (o[19], the mean density, still zero: the
// single-channel forms set the shift from the state before their first sample,
// the batched engine does not) took this sample about zero: its sums are
// re-centred on its own plane means, which become the shift of every later
// sample.  The per-sample variances do not depend on the shift.
__device__ __forceinline__ void stat_row_add(double *o, const double (&s9)[9], double nn) {
  const double mu = s9[0] / nn, mv = s9[1] / nn, mw = s9[2] / nn, mr = s9[3] / nn;
  const double var[5] = {s9[4] / nn - mu * mu, s9[5] / nn - mv * mv, s9[6] / nn - mw * mw, s9[7] / nn - mu * mw,
                         s9[8] / nn - mr * mr};
  double t[9];
#pragma unroll
  for (int c = 0; c < 9; c++) t[c] = s9[c];
  if (o[19] == 0.) {
    t[0] = s9[0] - nn * mu;
    t[1] = s9[1] - nn * mv;
    t[2] = s9[2] - nn * mw;
    t[3] = s9[3] - nn * mr;
    t[4] = s9[4] - nn * (mu * mu);
    t[5] = s9[5] - nn * (mv * mv);
    t[6] = s9[6] - nn * (mw * mw);
    t[7] = s9[7] - nn * (mu * mw);
    t[8] = s9[8] - nn * (mr * mr);
    o[16] = mu;
    o[17] = mv;
    o[18] = mw;
    o[19] = mr;
  }
#pragma unroll
  for (int c = 0; c < 9; c++) o[c] += t[c];
#pragma unroll
  for (int c = 0; c < 5; c++) o[9 + c] += var[c];
  o[14] = nn;
  o[15] += 1.0;
}

}  // namespace dns
