// Four nodes per thread: the FP32 stream-collide of the batched engine with
// 128-bit memory operations.
//
// A thread owns four consecutive nodes along x (x0 = 4t .. 4t + 3 of a row) and
// moves each population of them with one 16-byte load and, after the
// collision, one 16-byte store: the structure-of-arrays layout keeps the four
// values adjacent, and every row starts on a 16-byte boundary because the
// x extent is a multiple of 4 (the batched engine requires it).  Pushes along
// e_x = 0 keep that alignment.  The +-x pushes move the four values one node
// along the row, so the aligned four-node group a thread stores takes one value
// from its x-neighbour thread by a warp shuffle; where the neighbour is in
// another warp, block or across the periodic wrap, the thread stores the
// three values that stay inside its group one by one and the crossing value
// is stored by the thread it leaves.  Every destination node of every row is
// written exactly once.
//
// The arithmetic per node is f32_core.cuh's (collide_f32, the deviation
// equilibrium, the wall rules), so a node's post-collision populations are the
// single-channel FP32 form's.
#pragma once

#include <cstddef>
#include <cstdint>

#include "f32_core.cuh"
#include "lattice.cuh"

namespace dns {
namespace f32 {

// Position of a thread's four-node group in its row and whether the groups
// beside it are held by the neighbouring lanes of the same warp.
struct QuadPos {
  int x0;          // first node along x (a multiple of 4)
  bool ok;         // the group lies inside the grid (else: loads and stores are skipped)
  bool has_left;   // the group at x0 - 4 is lane - 1's
  bool has_right;  // the group at x0 + 4 is lane + 1's
};

// tx: thread index along the row segment of W threads (W a power of two);
// the segment's first group starts at node gx0.
__device__ __forceinline__ QuadPos quad_pos(int tx, int W, int gx0, int nx, bool row_ok) {
  const int lane = threadIdx.x & 31;
  QuadPos q;
  q.x0 = gx0 + 4 * tx;
  q.ok = row_ok && q.x0 < nx;
  q.has_left = tx > 0 && lane > 0;
  q.has_right = tx < W - 1 && lane < 31 && q.x0 + 4 < nx;
  return q;
}

__device__ __forceinline__ void quad_load(const float *__restrict__ src, size_t idx0, size_t pstride, bool ok,
                                          float (&q)[19][4]) {
#pragma unroll
  for (int a = 0; a < 19; a++) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ok) v = __ldg(reinterpret_cast<const float4 *>(src + (size_t)a * pstride + idx0));
    q[a][0] = v.x;
    q[a][1] = v.y;
    q[a][2] = v.z;
    q[a][3] = v.w;
  }
}

// The BGK collision of collide_f32 with opposite populations taken in pairs:
// e_b = -e_a gives e_b.u = -e_a.u, so the equilibrium deviations are
// S + A and S - A with the even part S = w drho + w rho (4.5 (e.u)^2 - 1.5 u^2)
// and the odd part A = 3 w rho e.u, and the forcing terms are opposite;
// d' = (1 - omega) d + omega deq is formed once per pair for both.  (The
// same deviation equilibrium and update, grouped so that the pair's common
// terms are computed once.)
#ifndef DNS_F32_PAIRS
#define DNS_F32_PAIRS 1
#endif
__device__ __forceinline__ Mac32 collide_f32_pairs(float (&d)[19], float om, float G) {
  const Mac32 m = macro_f32(d);
  const float omc = 1.f - om, usq15 = 1.5f * m.usq;
  d[0] = omc * d[0] + om * (w_of(0) * (m.drho - m.rho * usq15));
#pragma unroll
  for (int a = 1; a < 19; a++) {
    const int b = opp_of(a);
    if (b < a) continue;  // each pair once, from its smaller index
    const float eu = proj_f32(a, m.u0, m.u1, m.u2);
    const float wr = w_of(a) * m.rho;
    const float t = om * (w_of(a) * m.drho + wr * (4.5f * eu * eu - usq15));
    const float ta = om * (3.f * wr * eu);
    const float f = (float)ex_of(a) * bi_of(a) * m.rho * G;  // force on a; b gets -f
    d[a] = omc * d[a] + (t + ta) + f;
    d[b] = omc * d[b] + (t - ta) - f;
  }
  return m;
}

// BGK collision of the four nodes in place; returns their pre-collision moments.
__device__ __forceinline__ void quad_collide(float (&q)[19][4], float om, float G, Mac32 (&m)[4]) {
#pragma unroll
  for (int n = 0; n < 4; n++) {
    float d[19];
#pragma unroll
    for (int a = 0; a < 19; a++) d[a] = q[a][n];
    m[n] = DNS_F32_PAIRS ? collide_f32_pairs(d, om, G) : collide_f32(d, om, G);
#pragma unroll
    for (int a = 0; a < 19; a++) q[a][n] = d[a];
  }
}

__device__ __forceinline__ void st4(float *p, float a, float b, float c, float d) {
  *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}

// Store population a's four post-collision values, pushed by e_x(a) along
// the row: row is the population array plus the destination row's offset
// (its node x0 at row[x0]).  All lanes of the warp must call it (shuffles).
template <int EX>
__device__ __forceinline__ void quad_store(float *__restrict__ row, const float (&v)[4], const QuadPos &P, int nx) {
  if (EX == 0) {
    if (P.ok) st4(row + P.x0, v[0], v[1], v[2], v[3]);
  } else if (EX > 0) {
    const float w = __shfl_up_sync(0xffffffffu, v[3], 1);
    if (P.ok) {
      if (P.has_left) {
        st4(row + P.x0, w, v[0], v[1], v[2]);
      } else {
        row[P.x0 + 1] = v[0];
        row[P.x0 + 2] = v[1];
        row[P.x0 + 3] = v[2];
      }
      if (!P.has_right) row[P.x0 + 4 == nx ? 0 : P.x0 + 4] = v[3];
    }
  } else {
    const float w = __shfl_down_sync(0xffffffffu, v[0], 1);
    if (P.ok) {
      if (P.has_right) {
        st4(row + P.x0, v[1], v[2], v[3], w);
      } else {
        row[P.x0] = v[1];
        row[P.x0 + 1] = v[2];
        row[P.x0 + 2] = v[3];
      }
      if (!P.has_left) row[P.x0 == 0 ? nx - 1 : P.x0 - 1] = v[0];
    }
  }
}

// Does a push of population a leave the plane set?  ZSKIP as fine_push_f32:
// +1 e_z > 0, +2 e_z >= 0, -1 e_z < 0, -2 e_z <= 0 are dropped.
template <int ZSKIP>
__host__ __device__ constexpr bool zskip(int a) {
  return (ZSKIP == 1 && ez_of(a) > 0) || (ZSKIP == 2 && ez_of(a) >= 0) || (ZSKIP == -1 && ez_of(a) < 0) ||
         (ZSKIP == -2 && ez_of(a) <= 0);
}

// Regular pushes of the four nodes (no wall): destination row of population a
// is the node's row shifted by e_y (periodic) and its plane by e_z.  rowoff:
// offset of the node's row (p ny + j) nx in the population arrays; plane = nx ny;
// dym / dyp: row offsets to j - 1 / j + 1 with the wrap folded in.  SKIPWALL
// (0: none, -1 / +1): populations heading into the lower / upper wall plane are
// left to the wall rule.  ACC: flow-rate partials per destination plane weight
// wz[e_z + 1], summed per node in float, then added to acc in node order.
template <int ZSKIP, int SKIPWALL, bool ACC>
__device__ __forceinline__ void quad_push(const float (&q)[19][4], float *__restrict__ dst, size_t pstride,
                                          long long rowoff, int plane, int dym, int dyp, const QuadPos &P, int nx,
                                          const float (&wz)[3], double (&acc)[2]) {
  float mom[4] = {0.f, 0.f, 0.f, 0.f}, den[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < 19; a++) {
    if (zskip<ZSKIP>(a)) continue;
    if ((SKIPWALL < 0 && ez_of(a) < 0) || (SKIPWALL > 0 && ez_of(a) > 0)) continue;
    const int off = (ez_of(a) > 0 ? plane : (ez_of(a) < 0 ? -plane : 0)) + (ey_of(a) > 0 ? dyp : (ey_of(a) < 0 ? dym : 0));
    float *row = dst + (size_t)a * pstride + (rowoff + off);
    const float v[4] = {q[a][0], q[a][1], q[a][2], q[a][3]};
    // (a is a constant once the loop is unrolled: one branch survives)
    if (ex_of(a) > 0)
      quad_store<1>(row, v, P, nx);
    else if (ex_of(a) < 0)
      quad_store<-1>(row, v, P, nx);
    else
      quad_store<0>(row, v, P, nx);
    if (ACC) {
      const float wgt = wz[ez_of(a) + 1];
#pragma unroll
      for (int n = 0; n < 4; n++) {
        den[n] += wgt * v[n];
        if (ex_of(a) > 0) mom[n] += wgt * v[n];
        if (ex_of(a) < 0) mom[n] -= wgt * v[n];
      }
    }
  }
  if (ACC && P.ok) {
#pragma unroll
    for (int n = 0; n < 4; n++) {
      acc[0] += mom[n];
      acc[1] += den[n];
    }
  }
}

// The five populations of a wall-adjacent plane's nodes that head into the
// wall plane (xfcomputations.c:226-240): half-way bounce-back onto the node
// itself when the destination column and the node's own column are both solid
// (flag -1), else specular reflection into the destination column; both stay
// in the node's plane (flow-rate weight wz[1]).  Scalar stores, one per node.
template <bool UPPER, bool ACC>
__device__ __forceinline__ void quad_wall(const float (&q)[19][4], float *__restrict__ dst, size_t pstride,
                                          long long rowoff, int j, int nx, int ny, const int8_t *__restrict__ wf,
                                          const QuadPos &P, float wgt, double (&acc)[2]) {
  if (!P.ok) return;
  const char4 own4 = *reinterpret_cast<const char4 *>(wf + (size_t)j * nx + P.x0);
  const int8_t own[4] = {(int8_t)own4.x, (int8_t)own4.y, (int8_t)own4.z, (int8_t)own4.w};
  const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
  float mom[4] = {0.f, 0.f, 0.f, 0.f}, den[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < 19; a++) {
    if (!((UPPER && ez_of(a) > 0) || (!UPPER && ez_of(a) < 0))) continue;
    const int j2 = ey_of(a) > 0 ? jp : (ey_of(a) < 0 ? jm : j);
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const int x = P.x0 + n;
      const int i2 = ex_of(a) > 0 ? (x == nx - 1 ? 0 : x + 1) : (ex_of(a) < 0 ? (x == 0 ? nx - 1 : x - 1) : x);
      const int8_t sld = __ldg(wf + (size_t)j2 * nx + i2);
      const float f = q[a][n];
      int exd;
      if (sld == -1 && own[n] == -1) {
        dst[(size_t)opp_of(a) * pstride + (size_t)(rowoff + x)] = f;
        exd = -ex_of(a);
      } else {
        dst[(size_t)mir_of(a) * pstride + (size_t)(rowoff + (long long)(j2 - j) * nx + i2)] = f;
        exd = ex_of(a);
      }
      if (ACC) {
        den[n] += wgt * f;
        if (exd > 0) mom[n] += wgt * f;
        if (exd < 0) mom[n] -= wgt * f;
      }
    }
  }
  if (ACC) {
#pragma unroll
    for (int n = 0; n < 4; n++) {
      acc[0] += mom[n];
      acc[1] += den[n];
    }
  }
}

}  // namespace f32
}  // namespace dns
