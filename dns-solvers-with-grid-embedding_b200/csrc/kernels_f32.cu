// FP32 deviation-storage form of the grid-embedded D3Q19 channel step.
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
// opposite and mirror).  Layout, launch shapes, wall rules and the interface
// algorithm are those of kernels_f64.cu; the interface history holds
// [drho, ux, uy, uz, fneq_0..18] in FP32.
#include "bicubic_gen.cuh"
#include "kernels.h"
#include "lattice.cuh"

namespace dns {

namespace {

constexpr int kThreads = 128;
// minimum resident blocks asked of the register allocator for the bulk-plane
// kernels (0: compiler's choice); fused: collide each population right before
// its store so collided values die as they are written
#ifndef DNS_F32_BULK_MINB
#define DNS_F32_BULK_MINB 6
#endif
#ifndef DNS_F32_FUSED
#define DNS_F32_FUSED 1
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

// ------------------------------------------------------------------ coarse
template <bool STATS>
__device__ __forceinline__ void coarse_node_f32(float (&f)[19], int i, int j, int k, const Dims &d, float om,
                                                float G, float *__restrict__ dst, size_t pstride, double (&acc)[2],
                                                double (&sacc)[9]) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const Mac32 m = collide_f32(f, om, G);
  if (STATS) {
    const double u0 = m.u0, u1 = m.u1, u2 = m.u2, rho = 1.0 + (double)m.drho;
    sacc[0] += u0; sacc[1] += u1; sacc[2] += u2; sacc[3] += rho;
    sacc[4] += u0 * u0; sacc[5] += u1 * u1; sacc[6] += u2 * u2; sacc[7] += u0 * u2; sacc[8] += rho * rho;
  }
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
                                                double (&sacc)[9]) {
  const int nx = d.nx, ny = d.ny;
  const Mac32 m = collide_f32(f, om, G);
  if (STATS) {
    const double u0 = m.u0, u1 = m.u1, u2 = m.u2, rho = 1.0 + (double)m.drho;
    sacc[0] += u0; sacc[1] += u1; sacc[2] += u2; sacc[3] += rho;
    sacc[4] += u0 * u0; sacc[5] += u1 * u1; sacc[6] += u2 * u2; sacc[7] += u0 * u2; sacc[8] += rho * rho;
  }
  const int plane = ny * nx;
  const int dxm = i == 0 ? nx - 1 : -1, dxp = i == nx - 1 ? 1 - nx : 1;
  const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
  // each population array holds fewer than 2^31 floats: 32-bit offsets from
  // the population's (thread-uniform) base
  const unsigned u0 = (unsigned)idx0;
  float mom = 0.f, den = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int off = (ez_of(a) > 0 ? plane : (ez_of(a) < 0 ? -plane : 0)) + (ey_of(a) > 0 ? dyp : (ey_of(a) < 0 ? dym : 0)) +
                    (ex_of(a) > 0 ? dxp : (ex_of(a) < 0 ? dxm : 0));
    (dst + (size_t)a * pstride)[u0 + (unsigned)off] = f[a];
    den += f[a];
    if (ex_of(a) > 0) mom += f[a];
    if (ex_of(a) < 0) mom -= f[a];
  }
  acc[0] += mom;
  acc[1] += den;
}

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
  double sacc[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
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
  if (STATS) block_reduce32<9>(sacc, spart + blk * 9);
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
template <int MODE>
__device__ __forceinline__ void fine_node_f32(float (&f)[19], int i, int j, int p, int k, bool upper, int kwall,
                                              const Dims &d, float om, float Gf, const int8_t *__restrict__ wf,
                                              float *__restrict__ dst, size_t pstride, bool wall_sum_plane,
                                              bool wall_rho_plane, double (&acc)[2], double (&wacc)[2],
                                              double (&sacc)[9]) {
  const int nx = d.nxf, ny = d.nyf, zdf = d.zdf, zds = d.zds, gr = d.gr;
  const Mac32 m = collide_f32(f, om, Gf);
  if (MODE & 2) {
    if (wall_sum_plane) wacc[0] += (double)m.u0;
    if (wall_rho_plane) wacc[1] += 1.0 + (double)m.drho;
  }
  if (MODE & 4) {
    const double u0 = m.u0, u1 = m.u1, u2 = m.u2, rho = 1.0 + (double)m.drho;
    sacc[0] += u0; sacc[1] += u1; sacc[2] += u2; sacc[3] += rho;
    sacc[4] += u0 * u0; sacc[5] += u1 * u1; sacc[6] += u2 * u2; sacc[7] += u0 * u2; sacc[8] += rho * rho;
  }
  const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
  const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
  const bool wall_adjacent = upper ? (k == zdf - 2) : (k == 1);
  const int8_t own = wall_adjacent ? wf[(size_t)j * nx + i] : (int8_t)-1;
  float mom = 0.f, den = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int k2 = k + ez_of(a);
    const int i2 = ex_of(a) > 0 ? ip : (ex_of(a) < 0 ? im : i);
    const int j2 = ey_of(a) > 0 ? jp : (ey_of(a) < 0 ? jm : j);
    int pd, id, jd, ad, kd, exd;
    if (k2 == kwall) {
      const int8_t sld = wf[(size_t)j2 * nx + i2];
      if (sld == -1 && own == -1) {
        pd = p; id = i; jd = j; ad = opp_of(a); exd = -ex_of(a);
      } else {
        pd = p; id = i2; jd = j2; ad = mir_of(a); exd = ex_of(a);
      }
      kd = k;
    } else {
      if (!upper && k2 >= zdf - 1) continue;
      if (upper && k2 <= 0) continue;
      pd = upper ? zds + k2 : k2 - 1; id = i2; jd = j2; ad = a; kd = k2; exd = ex_of(a);
    }
    (dst + (size_t)ad * pstride)[(unsigned)((pd * ny + jd) * nx + id)] = f[a];
    if (MODE & 1) {
      const float wgt = !upper ? ((kd >= 1 && kd < zdf - gr) ? 1.f : 0.f)
                               : ((kd >= gr && kd < zdf - 1) ? (kd == gr ? 0.5f : 1.f) : 0.f);
      den += wgt * f[a];
      if (exd > 0) mom += wgt * f[a];
      if (exd < 0) mom -= wgt * f[a];
    }
  }
  acc[0] += mom;
  acc[1] += den;
}

// Bulk planes (every push lands on a fluid plane of the same block: no wall,
// no interface): destinations from precomputed +-1 / +-row / +-plane offsets
// with the periodic wrap folded in; encalc2 weights per destination plane.
template <int MODE>
__device__ __forceinline__ void fine_bulk_f32(float (&f)[19], int i, int j, size_t idx0, const Dims &d, float om,
                                              float Gf, float *__restrict__ dst, size_t pstride, const float (&wz)[3],
                                              bool wall_sum_plane, bool wall_rho_plane, double (&acc)[2],
                                              double (&wacc)[2], double (&sacc)[9]) {
  const int nx = d.nxf, ny = d.nyf;
#if DNS_F32_FUSED
  const Mac32 m = macro_f32(f);
#else
  const Mac32 m = collide_f32(f, om, Gf);
#endif
  if (MODE & 2) {
    if (wall_sum_plane) wacc[0] += (double)m.u0;
    if (wall_rho_plane) wacc[1] += 1.0 + (double)m.drho;
  }
  if (MODE & 4) {
    const double u0 = m.u0, u1 = m.u1, u2 = m.u2, rho = 1.0 + (double)m.drho;
    sacc[0] += u0; sacc[1] += u1; sacc[2] += u2; sacc[3] += rho;
    sacc[4] += u0 * u0; sacc[5] += u1 * u1; sacc[6] += u2 * u2; sacc[7] += u0 * u2; sacc[8] += rho * rho;
  }
  const int plane = ny * nx;
  const int dxm = i == 0 ? nx - 1 : -1, dxp = i == nx - 1 ? 1 - nx : 1;
  const int dym = j == 0 ? (ny - 1) * nx : -nx, dyp = j == ny - 1 ? -(ny - 1) * nx : nx;
  // each population array holds fewer than 2^31 floats: 32-bit offsets from
  // the population's (thread-uniform) base
  const unsigned u0 = (unsigned)idx0;
  float mom = 0.f, den = 0.f;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int off = (ez_of(a) > 0 ? plane : (ez_of(a) < 0 ? -plane : 0)) + (ey_of(a) > 0 ? dyp : (ey_of(a) < 0 ? dym : 0)) +
                    (ex_of(a) > 0 ? dxp : (ex_of(a) < 0 ? dxm : 0));
#if DNS_F32_FUSED
    {
      const float deq = deq_f32(a, m.drho, m.rho, m.u0, m.u1, m.u2, m.usq);
      float dn = f[a] - om * (f[a] - deq);
      if (ex_of(a) != 0) dn += (float)ex_of(a) * bi_of(a) * m.rho * Gf;
      f[a] = dn;
    }
#endif
    (dst + (size_t)a * pstride)[u0 + (unsigned)off] = f[a];
    if (MODE & 1) {
      const float wgt = wz[ez_of(a) + 1];
      den += wgt * f[a];
      if (ex_of(a) > 0) mom += wgt * f[a];
      if (ex_of(a) < 0) mom -= wgt * f[a];
    }
  }
  acc[0] += mom;
  acc[1] += den;
}

// The fine step is two launches: BULK over planes k = 2..zdf-3 of both blocks
// (every push regular) and the edge planes (wall-adjacent, interface, and the
// planes next to them).  blockIdx.z indexes a list of planes; partial sums
// are stored at the plane's own block index, so the layout does not change.
struct PlaneList {
  int n;
  int p[64];
};

template <int MODE, bool BULK>
__global__ void __launch_bounds__(kThreads, BULK ? DNS_F32_BULK_MINB : 0) fine_f32(const float *__restrict__ src, float *__restrict__ dst,
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
  const int kwall = upper ? zdf - 1 : 0;
  const size_t pstride = (size_t)P * ny * nx;
  const float Gf = (float)((1. / (double)gr) * st->force);
  const bool wall_sum_plane =
      upper ? (k == zdf - 2 || k == zdf - 3 || k == zdf - 4) : (k == 1 || k == 2 || k == 3);
  const bool wall_rho_plane = upper ? (k == zdf - 4) : (k == 1);
  double acc[2] = {0., 0.}, wacc[2] = {0., 0.};
  double sacc[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  float wz[3] = {0.f, 0.f, 0.f};
  if (BULK) {
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
    if (BULK)
      fine_bulk_f32<MODE>(fa, i, j, idx0, d, om, Gf, dst, pstride, wz, wall_sum_plane, wall_rho_plane, acc, wacc,
                          sacc);
    else
      fine_node_f32<MODE>(fa, i, j, p, k, upper, kwall, d, om, Gf, wf, dst, pstride, wall_sum_plane,
                          wall_rho_plane, acc, wacc, sacc);
  }
  const size_t blk = ((size_t)p * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (MODE & 1) block_reduce32<2>(acc, part + blk * 2);
  if ((MODE & 2) && wall_sum_plane) block_reduce32<2>(wacc, wpart + blk * 2);
  if (MODE & 4) block_reduce32<9>(sacc, spart + blk * 9);
}

// ------------------------------------------------------------------ interface
constexpr int JTX = 32, JTY = 16, JPX = 16, JPY = 8;
constexpr int QX = JTX + 5, QY = JTY + 5;

struct IfaceArgs32 {
  float h1, h2, h3, h4, fac;
};

struct IfaceSmem32 {
  float V[QY][QX];
  float Dy[JTY + 1][QX];
  float Dx[JTY + 1][JTX + 1];
  float Dxy[JTY + 1][JTX + 1];
};

__device__ __forceinline__ void stage32(IfaceSmem32 &S, const float *__restrict__ hn, const float *__restrict__ hp,
                                        const float *__restrict__ hpp, size_t fo, int i0, int j0, int nx, int ny,
                                        const IfaceArgs32 &ia) {
  const float c2o3 = 2.f / 3.f, c1o12 = 1.f / 12.f;
  for (int q = threadIdx.x; q < QX * QY; q += blockDim.x) {
    const int pi = q % QX, pj = q / QX;
    const size_t g = fo + (size_t)wrapf(j0 - 2 + pj, ny) * nx + wrapf(i0 - 2 + pi, nx);
    const float n = hn[g], pv = hp[g], pp = hpp[g];
    S.V[pj][pi] = ia.h1 * pv + ia.h2 * ((n - pp) * 0.5f) + ia.h3 * n + ia.h4 * ((3.f * n - 4.f * pv + pp) * 0.5f);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < QX * (JTY + 1); q += blockDim.x) {
    const int pi = q % QX, r = q / QX, pj = r + 2;
    S.Dy[r][pi] = c2o3 * (S.V[pj + 1][pi] - S.V[pj - 1][pi]) - c1o12 * (S.V[pj + 2][pi] - S.V[pj - 2][pi]);
    if (pi >= 2 && pi < JTX + 3)
      S.Dx[r][pi - 2] = c2o3 * (S.V[pj][pi + 1] - S.V[pj][pi - 1]) - c1o12 * (S.V[pj][pi + 2] - S.V[pj][pi - 2]);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < (JTX + 1) * (JTY + 1); q += blockDim.x) {
    const int c = q % (JTX + 1), r = q / (JTX + 1), pi = c + 2;
    S.Dxy[r][c] = c2o3 * (S.Dy[r][pi + 1] - S.Dy[r][pi - 1]) - c1o12 * (S.Dy[r][pi + 2] - S.Dy[r][pi - 2]);
  }
  __syncthreads();
}

__device__ __forceinline__ void coeffs32(const IfaceSmem32 &S, int cx, int cy, float (&cf)[16]) {
  float x[16];
  const int ci[4] = {0, 1, 1, 0}, cj[4] = {0, 0, 1, 1};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cx + ci[q], r = cy + cj[q];
    x[q] = S.V[r + 2][c + 2];
    x[4 + q] = S.Dx[r][c];
    x[8 + q] = S.Dy[r][c + 2];
    x[12 + q] = S.Dxy[r][c];
  }
  DNS_BICUBIC_COEFFS_F32(cf, x);
}

template <int GR>
__device__ __forceinline__ float eval32(const float (&cf)[16], int ii, int jj) {
  const float tt = (float)ii / (float)GR, uu = (float)jj / (float)GR;
  float val = 0.f;
#pragma unroll
  for (int nn = 3; nn > -1; nn--)
    val = tt * val + ((cf[nn * 4 + 3] * uu + cf[nn * 4 + 2]) * uu + cf[nn * 4 + 1]) * uu + cf[nn * 4 + 0];
  return val;
}

template <int GR>
__global__ void __launch_bounds__(JPX *JPY) iface_macro_f32(const float *__restrict__ hn, const float *__restrict__ hp,
                                                            const float *__restrict__ hpp, float *__restrict__ mac,
                                                            Dims d, IfaceArgs32 ia) {
  __shared__ IfaceSmem32 S;
  const int nx = d.nx, ny = d.ny, nxf = d.nxf, nyf = d.nyf;
  const int w = blockIdx.z >> 2, b = blockIdx.z & 3;
  const int i0 = blockIdx.x * JTX, j0 = blockIdx.y * JTY;
  const int tx = threadIdx.x % JPX, ty = threadIdx.x / JPX;
  const size_t plane = (size_t)ny * nx, fplane = (size_t)nyf * nxf;
  stage32(S, hn, hp, hpp, ((size_t)w * 23 + b) * plane, i0, j0, nx, ny, ia);
  float *o = mac + ((size_t)w * 4 + b) * fplane;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int cx = tx + JPX * (q & 1), cy = ty + JPY * (q >> 1);
    const int ic = i0 + cx, jc = j0 + cy;
    if (ic < nx && jc < ny) {
      float cf[16];
      coeffs32(S, cx, cy, cf);
#pragma unroll
      for (int ii = 0; ii < GR; ii++)
#pragma unroll
        for (int jj = 0; jj < GR; jj++) o[(size_t)(jc * GR + jj) * nxf + ic * GR + ii] = eval32<GR>(cf, ii, jj);
    }
  }
}

template <int GR>
__global__ void __launch_bounds__(JPX *JPY) iface_pop_f32(const float *__restrict__ hn, const float *__restrict__ hp,
                                                          const float *__restrict__ hpp, const float *__restrict__ mac,
                                                          float *__restrict__ fdst, Dims d, IfaceArgs32 ia) {
  __shared__ IfaceSmem32 S;
  const int nx = d.nx, ny = d.ny, nxf = d.nxf, nyf = d.nyf, zds = d.zds;
  const int w = blockIdx.z / 19, a = blockIdx.z % 19;
  const int i0 = blockIdx.x * JTX, j0 = blockIdx.y * JTY;
  const int tx = threadIdx.x % JPX, ty = threadIdx.x / JPX;
  const size_t plane = (size_t)ny * nx, fplane = (size_t)nyf * nxf;
  const int pf = w == 0 ? zds - 1 : zds;
  const size_t fstride = (size_t)2 * zds * fplane;
  stage32(S, hn, hp, hpp, ((size_t)w * 23 + 4 + a) * plane, i0, j0, nx, ny, ia);
  const float *m = mac + (size_t)w * 4 * fplane;
  float *out = fdst + (size_t)a * fstride + (size_t)pf * fplane;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int cx = tx + JPX * (q & 1), cy = ty + JPY * (q >> 1);
    const int ic = i0 + cx, jc = j0 + cy;
    if (ic < nx && jc < ny) {
      float cf[16];
      coeffs32(S, cx, cy, cf);
#pragma unroll
      for (int ii = 0; ii < GR; ii++)
#pragma unroll
        for (int jj = 0; jj < GR; jj++) {
          const size_t qn = (size_t)(jc * GR + jj) * nxf + ic * GR + ii;
          const float dr = m[qn], u0 = m[fplane + qn], u1 = m[2 * fplane + qn], u2 = m[3 * fplane + qn];
          const float usq = u0 * u0 + u1 * u1 + u2 * u2;
          out[qn] = deq_f32(a, dr, 1.f + dr, u0, u1, u2, usq) + ia.fac * eval32<GR>(cf, ii, jj);
        }
    }
  }
}

// ------------------------------------------------------------------ injection
__global__ void __launch_bounds__(kThreads) inject_f32(const float *__restrict__ fsrc, float *__restrict__ cdst, Dims d,
                                                      float fac, double *__restrict__ part) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc, gr = d.gr, zdf = d.zdf, zds = d.zds;
  const int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y, w = blockIdx.z;
  double acc[2] = {0., 0.};
  if (ic < nx) {
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
                                  int p0, int nz_aos, int k0_aos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= nx) return;
  const size_t stride = (size_t)P * ny * nx;
  const size_t s = ((size_t)(p0 + q) * ny + j) * nx + i;
  double *o = aos + (((size_t)i * ny + j) * nz_aos + k0_aos + q) * 19;
  for (int a = 0; a < 19; a++) {
    const double w = a == 0 ? 1. / 3. : (a <= 6 ? 1. / 18. : 1. / 36.);
    o[a] = w + (double)soa[s + (size_t)a * stride];
  }
}

__global__ void aos_to_dev_kernel(const double *__restrict__ aos, float *__restrict__ soa, int nx, int ny, int P,
                                  int p0, int nz_aos, int k0_aos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= nx) return;
  const size_t stride = (size_t)P * ny * nx;
  const size_t s = ((size_t)(p0 + q) * ny + j) * nx + i;
  const double *o = aos + (((size_t)i * ny + j) * nz_aos + k0_aos + q) * 19;
  for (int a = 0; a < 19; a++) {
    const double w = a == 0 ? 1. / 3. : (a <= 6 ? 1. / 18. : 1. / 36.);
    soa[s + (size_t)a * stride] = (float)(o[a] - w);
  }
}

}  // namespace

// ====================================================================== host
void launch_coarse_f32(const float *src, float *dst, const Dims &d, const LaunchShape &s, double om,
                       const DevState *st, double *partials, const PartialLayout &pl, bool stats,
                       cudaStream_t stream) {
  dim3 gb(s.cgx, s.cgy, d.nzc - 4), ge(s.cgx, s.cgy, 4), block(s.bx);
  double *pc = partials + pl.coarse, *ps = partials + pl.stats_c;
  const float omf = (float)om;
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
  PlaneList bulk{}, edge{};
  for (int p = 0; p < 2 * d.zds; p++) {
    const int k = p >= d.zds ? p - d.zds : p + 1;
    PlaneList &L = (k >= 2 && k <= d.zdf - 3) ? bulk : edge;
    L.p[L.n++] = p;
  }
  const int mode = (last ? 1 : 0) | (first ? 2 : 0) | (stats ? 4 : 0);
  double *pf = partials + pl.fine, *pw = partials + pl.wall, *ps = partials + pl.stats_f;
  const float omf = (float)om;
  dim3 gb(s.fgx, s.fgy, bulk.n), ge(s.fgx, s.fgy, edge.n), block(s.bx);
#define FINE32_CASE(M)                                                                                         \
  case M:                                                                                                      \
    if (bulk.n) fine_f32<M, true><<<gb, block, 0, stream>>>(src, dst, wflag, d, s.jb, omf, st, pf, pw, ps, bulk); \
    fine_f32<M, false><<<ge, block, 0, stream>>>(src, dst, wflag, d, s.jb, omf, st, pf, pw, ps, edge);        \
    break;
  switch (mode) {
    FINE32_CASE(0) FINE32_CASE(1) FINE32_CASE(2) FINE32_CASE(3) FINE32_CASE(4) FINE32_CASE(5) FINE32_CASE(6)
    FINE32_CASE(7)
  }
#undef FINE32_CASE
}

void launch_interface_f32(const float *hn, const float *hp, const float *hpp, float *mac, float *fdst, const Dims &d,
                          int substep, double omega_c, double omega_f, cudaStream_t stream) {
  const double tmp = (((double)substep) / ((double)d.gr));
  IfaceArgs32 ia;
  ia.h1 = (float)(2. * tmp * tmp * tmp - 3. * tmp * tmp + 1.);
  ia.h2 = (float)(tmp * tmp * tmp - 2. * tmp * tmp + tmp);
  ia.h3 = (float)(-2. * tmp * tmp * tmp + 3. * tmp * tmp);
  ia.h4 = (float)(tmp * tmp * tmp - tmp * tmp);
  ia.fac = (float)(omega_c / ((double)d.gr * omega_f));
  const int gx = (d.nx + JTX - 1) / JTX, gy = (d.ny + JTY - 1) / JTY;
  dim3 gm(gx, gy, 2 * 4), gp(gx, gy, 2 * 19), block(JPX * JPY);
  if (d.gr == 2) {
    iface_macro_f32<2><<<gm, block, 0, stream>>>(hn, hp, hpp, mac, d, ia);
    iface_pop_f32<2><<<gp, block, 0, stream>>>(hn, hp, hpp, mac, fdst, d, ia);
  } else if (d.gr == 3) {
    iface_macro_f32<3><<<gm, block, 0, stream>>>(hn, hp, hpp, mac, d, ia);
    iface_pop_f32<3><<<gp, block, 0, stream>>>(hn, hp, hpp, mac, fdst, d, ia);
  } else {
    iface_macro_f32<4><<<gm, block, 0, stream>>>(hn, hp, hpp, mac, d, ia);
    iface_pop_f32<4><<<gp, block, 0, stream>>>(hn, hp, hpp, mac, fdst, d, ia);
  }
}

void launch_inject_f32(const float *fsrc, float *cdst, const Dims &d, const LaunchShape &s, double omega_c,
                       double omega_f, double *partials, const PartialLayout &pl, cudaStream_t stream) {
  dim3 grid(s.jgx, s.jgy, 2), block(s.bx);
  inject_f32<<<grid, block, 0, stream>>>(fsrc, cdst, d, (float)(d.gr * (omega_f / omega_c)), partials + pl.inject);
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
                           int k0_aos, cudaStream_t stream) {
  dim3 grid((nx + 127) / 128, ny, np), block(128);
  dev_to_aos_kernel<<<grid, block, 0, stream>>>(soa, aos, nx, ny, P, p0, nz_aos, k0_aos);
}

void launch_aos_to_dev_f32(const double *aos, float *soa, int nx, int ny, int P, int p0, int np, int nz_aos,
                           int k0_aos, cudaStream_t stream) {
  dim3 grid((nx + 127) / 128, ny, np), block(128);
  aos_to_dev_kernel<<<grid, block, 0, stream>>>(aos, soa, nx, ny, P, p0, nz_aos, k0_aos);
}

}  // namespace dns
