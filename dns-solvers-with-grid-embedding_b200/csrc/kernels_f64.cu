// FP64 plain-form kernels of the grid-embedded D3Q19 channel step.
//
// Built with -fmad=false: together with the operation order of lattice.cuh the
// per-node arithmetic is bit-identical to the reference compiled without fused
// multiply-add.  Only the constant-flow-rate reduction (a sum over the whole
// domain) is associated differently from the reference's sequential loop.
//
// Device layout (structure of arrays, x fastest, one array per population):
//   coarse  fc[a][k][j][i]   k = 0..zdc-1, j < ydv, i < xdv
//   fine    ff[a][p][j][i]   p = 0..zds-1 : lower block k = p + 1 (1..zdf-1)
//                            p = zds..2zds-1 : upper block k = p - zds (0..zdf-2)
//   wall flags wf[j][i] (-1 no-slip, -2 slip), identical on both walls
//   interface history h[wall][field][j][i], fields [rho, ux, uy, uz, fneq_0..18]
// The state between coarse steps is the post-stream state S (the reference's
// ftemp arrays after exchange); kernels read S from one buffer, collide, and
// push into the other (ping-pong), with the periodic wrap in x and y replacing
// the reference's ghost column/row and halo exchange.
#include "bicubic_gen.cuh"
#include "kernels.h"
#include "lattice.cuh"

namespace dns {

namespace {

// Launch-shape tuning knobs (compile-time): threads per block along x, rows per
// block, and the minimum resident blocks per SM asked of the register
// allocator for the two stream-collide kernels (0 = let the compiler choose).
#ifndef DNS_BX
#define DNS_BX 128
#endif
#ifndef DNS_JB
#define DNS_JB 2
#endif
#ifndef DNS_MINB_FINE
#define DNS_MINB_FINE 0
#endif
#ifndef DNS_MINB_COARSE
#define DNS_MINB_COARSE 0
#endif
constexpr int kMaxThreads = DNS_BX;

// periodic index for any offset (an interface tile can be wider than the domain)
__device__ __forceinline__ int wrapi(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Fixed-order block reduction of N doubles; thread 0 returns the sums.
template <int N>
__device__ __forceinline__ void block_reduce(double (&v)[N], double *out) {
  __shared__ double red[N][kMaxThreads / 32];
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

// Fixed-order block reduction of N doubles into shared out[N] (visible to all
// threads on return); NT threads per block.
template <int N, int NT>
__device__ __forceinline__ void block_reduce_n(double (&v)[N], double *out) {
  __shared__ double red[N][NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; q++) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double s = red[threadIdx.x][0];
#pragma unroll
    for (int w = 1; w < NT / 32; w++) s += red[threadIdx.x][w];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

__device__ __forceinline__ void load19(const double *__restrict__ src, size_t idx, size_t stride, double (&f)[19]) {
#pragma unroll
  for (int a = 0; a < 19; a++) f[a] = __ldg(src + idx + (size_t)a * stride);
}

// ------------------------------------------------------------------ coarse
// Collide every coarse plane (xcomputations.c:49-86, 291-342) and push into
// planes 1..zdc-2 (:135-204, 353-420).  Planes 0 and zdc-1 of dst are
// rewritten by the fine-to-coarse injection, so pushes into them are dropped.
// Partials: constant-flow-rate momentum/mass of what lands in dst (all weight
// GR^3 in encalc2.c:57-84); with STATS the pre-collision plane moments.
template <bool STATS>
__global__ void __launch_bounds__(kMaxThreads, DNS_MINB_COARSE) coarse_kernel(const double *__restrict__ src, double *__restrict__ dst,
                                                            Dims d, int jb, double om, const DevState *st,
                                                            double *__restrict__ part, double *__restrict__ spart) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.z;
  const size_t pstride = (size_t)nzc * ny * nx;
  const double G = st->force;
  double acc[2] = {0., 0.};
  PlaneStat sacc;  // planes 2..zdc-3 are profile points; the others' moments are not read
  sacc.init();
  const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
  for (int r = 0; r < jb; r++) {
    const int j = blockIdx.y * jb + r;
    if (i >= nx || j >= ny) continue;
    double f[19];
    load19(src, ((size_t)k * ny + j) * nx + i, pstride, f);
    double dens, u0, u1, u2;
    collide_f64(f, om, G, dens, u0, u1, u2);
    if (STATS) sacc.add(u0, u1, u2, dens);
    const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
#pragma unroll
    for (int a = 0; a < 19; a++) {
      const int k2 = k + ez_of(a);
      if (k2 < 1 || k2 > nzc - 2) continue;
      const int i2 = ex_of(a) > 0 ? ip : (ex_of(a) < 0 ? im : i);
      const int j2 = ey_of(a) > 0 ? jp : (ey_of(a) < 0 ? jm : j);
      dst[(size_t)a * pstride + ((size_t)k2 * ny + j2) * nx + i2] = f[a];
      acc[1] += f[a];
      if (ex_of(a) > 0) acc[0] += f[a];
      if (ex_of(a) < 0) acc[0] -= f[a];
    }
  }
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce<2>(acc, part + blk * 2);
  if (STATS) block_reduce_stat(sacc, spart + blk * kStatPart);
}

// Interface planes of the new coarse state into history level n
// (xcomputations.c:558-625): [rho, u, f - feq] at k = 1 (lower) and zdc-2.
__global__ void __launch_bounds__(kMaxThreads) extract_kernel(const double *__restrict__ fc, double *__restrict__ hn,
                                                             Dims d) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, w = blockIdx.z;
  if (i >= nx) return;
  const int k = w == 0 ? 1 : nzc - 2;
  const size_t pstride = (size_t)nzc * ny * nx, plane = (size_t)ny * nx;
  double f[19];
  load19(fc, ((size_t)k * ny + j) * nx + i, pstride, f);
  double dens, mx, my, mz;
  moments_f64(f, dens, mx, my, mz);
  const double u0 = mx / dens, u1 = my / dens, u2 = mz / dens;
  const double t15v = 1.5 * (u0 * u0 + u1 * u1 + u2 * u2);
  const Weighted wr = weighted_rho(dens);
  double *o = hn + (size_t)w * 23 * plane + (size_t)j * nx + i;
  o[0] = dens;
  o[plane] = u0;
  o[2 * plane] = u1;
  o[3 * plane] = u2;
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int c = wclass_of(a);
    const double feq = feq_f64(c == 0 ? wr.w0 : (c == 1 ? wr.w1 : wr.w2), proj_f64(a, u0, u1, u2), t15v);
    o[(size_t)(4 + a) * plane] = f[a] - feq;
  }
}

// ------------------------------------------------------------------ fine
// Both near-wall blocks in one launch (xfcomputations.c:43-214, 599-712
// collision with force G/GR; :215-442, 724-897 streaming).  At a wall plane
// destination d = x + e_a with flags sld = flag(d), sld1 = flag(column of x):
//   sld = -1 and sld1 = -1 : half-way bounce-back into f(x, opposite a)
//   otherwise (slip involved): specular reflection into f(d_i, d_j, x_k, mirror a)
// Pushes into the interface planes are dropped (the coarse-to-fine transfer
// rewrites them).  MODE bits: 1 constant-flow-rate partials of dst (last
// substep; encalc2.c:33-53, 86-107 weights), 2 wall-shear plane sums of the
// pre-collision state (first substep; wshearstr.c:37-134), 4 plane statistics.
template <int MODE>
__global__ void __launch_bounds__(kMaxThreads, DNS_MINB_FINE) fine_kernel(const double *__restrict__ src, double *__restrict__ dst,
                                                          const int8_t *__restrict__ wf, Dims d, int jb, double om,
                                                          const DevState *st, double *__restrict__ part,
                                                          double *__restrict__ wpart, double *__restrict__ spart) {
  const int nx = d.nxf, ny = d.nyf, zdf = d.zdf, zds = d.zds, gr = d.gr;
  const int P = 2 * zds;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.z;
  const bool upper = p >= zds;
  const int k = upper ? p - zds : p + 1;  // reference k inside the block
  const int kwall = upper ? zdf - 1 : 0;
  const size_t pstride = (size_t)P * ny * nx;
  const double Gf = (1. / ((double)gr)) * st->force;
  // encalc2 weights of the destination planes k - 1, k, k + 1 (block-uniform;
  // a push into the wall plane stays on plane k)
  double wz[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int kd = k + c - 1;
    wz[c] = !upper ? ((kd >= 1 && kd < zdf - gr) ? 1.0 : 0.0)
                   : ((kd >= gr && kd < zdf - 1) ? (kd == gr ? 0.5 : 1.0) : 0.0);
  }
  const bool wall_sum_plane =
      upper ? (k == zdf - 2 || k == zdf - 3 || k == zdf - 4) : (k == 1 || k == 2 || k == 3);
  const bool wall_rho_plane = upper ? (k == zdf - 4) : (k == 1);
  // Planes whose pushes all land on planes of encalc2 weight 1 (no wall, no
  // dropped push into the interface plane): a node's flow-rate partials are
  // its post-collision moments, mass dens and momentum dens u0 + dens Gf (the
  // collision keeps both; the forcing adds rho G to sum e_x f, since
  // sum_a e_x^2 BI_a = 1).  Other planes sum the pushes with their weights.
  const bool unit_plane = upper ? (k >= gr + 2 && k <= zdf - 3) : (k >= 2 && k <= zdf - gr - 2);
  double acc[2] = {0., 0.}, wacc[2] = {0., 0.};
  PlaneStat sacc;
  sacc.init();
  const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
  for (int r = 0; r < jb; r++) {
    const int j = blockIdx.y * jb + r;
    if (i >= nx || j >= ny) continue;
    double f[19];
    load19(src, ((size_t)p * ny + j) * nx + i, pstride, f);
    double dens, u0, u1, u2;
    collide_f64(f, om, Gf, dens, u0, u1, u2);
    if (MODE & 2) {
      if (wall_sum_plane) wacc[0] += u0;
      if (wall_rho_plane) wacc[1] += dens;
    }
    if (MODE & 4) sacc.add(u0, u1, u2, dens);
    if ((MODE & 1) && unit_plane) {
      acc[0] += dens * u0 + dens * Gf;
      acc[1] += dens;
    }
    const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
    const int8_t own = wf[(size_t)j * nx + i];
#pragma unroll
    for (int a = 0; a < 19; a++) {
      const int k2 = k + ez_of(a);
      const int i2 = ex_of(a) > 0 ? ip : (ex_of(a) < 0 ? im : i);
      const int j2 = ey_of(a) > 0 ? jp : (ey_of(a) < 0 ? jm : j);
      int pd, id, jd, ad, exd;
      double wgt;  // encalc2 weight of the destination plane
      if (k2 == kwall) {
        const int8_t sld = wf[(size_t)j2 * nx + i2];
        if (sld == -1 && own == -1) {
          pd = p; id = i; jd = j; ad = opp_of(a); exd = -ex_of(a);
        } else {
          pd = p; id = i2; jd = j2; ad = mir_of(a); exd = ex_of(a);
        }
        wgt = wz[1];
      } else {
        if (!upper && k2 >= zdf - 1) continue;
        if (upper && k2 <= 0) continue;
        pd = upper ? zds + k2 : k2 - 1; id = i2; jd = j2; ad = a; exd = ex_of(a);
        wgt = wz[ez_of(a) + 1];
      }
      dst[(size_t)ad * pstride + ((size_t)pd * ny + jd) * nx + id] = f[a];
      if ((MODE & 1) && !unit_plane) {
        acc[1] += wgt * f[a];
        if (exd > 0) acc[0] += wgt * f[a];
        if (exd < 0) acc[0] -= wgt * f[a];
      }
    }
  }
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (MODE & 1) block_reduce<2>(acc, part + blk * 2);
  if ((MODE & 2) && wall_sum_plane) block_reduce<2>(wacc, wpart + blk * 2);
  if (MODE & 4) block_reduce_stat(sacc, spart + blk * kStatPart);
}

// ------------------------------------------------------------------ interface
// Coarse-to-fine transfer for one substep, both walls (tinterpolate_hrmt.c,
// derivative.c, bcucof_opt.c, ctfdtransfer_opt.c): Hermite interpolation in
// time of the three history levels, 4th-order central derivatives d/dx, d/dy,
// d2/dxdy, bicubic coefficients per coarse cell, Horner evaluation at the
// GR x GR fine nodes and f = feq + omega_c/(GR omega_f) fneq.  A tile of
// ITX x ITY coarse cells stages the (ITX+5) x (ITY+5) periodic patch of one
// field at a time in shared memory; each thread owns CPT coarse cells.  The
// tile is 32 x 8 cells (2 per thread): twice the blocks of 32 x 16 tiles, so
// the last of the ~5 waves of population blocks is a smaller share of the
// launch (a 2 x 19 x 64-tile grid at 7 blocks per SM leaves the third of 2.35
// waves a third full).
#ifndef DNS_ITY
#define DNS_ITY 8
#endif
constexpr int ITX = 32, ITY = DNS_ITY;     // coarse cells per tile
constexpr int TPX = 16, TPY = 8;           // threads per tile
constexpr int CPT = (ITX / TPX) * (ITY / TPY);  // cells per thread
static_assert(ITX % TPX == 0 && ITY % TPY == 0, "tile / thread layout");
constexpr int PX = ITX + 5, PY = ITY + 5;  // staged periodic patch

struct IfaceArgs {
  double h1, h2, h3, h4, fac;
};

struct IfaceSmem {
  double V[PY][PX];
  double Dy[ITY + 1][PX];
  double Dx[ITY + 1][ITX + 1];
  double Dxy[ITY + 1][ITX + 1];
};

// Stage field `fo` (offset of one wall's field in the history slots) of the
// tile's periodic patch: Hermite value, then d/dy, d/dx, d2/dxdy.
__device__ __forceinline__ void iface_stage(IfaceSmem &S, const double *__restrict__ hn,
                                            const double *__restrict__ hp, const double *__restrict__ hpp,
                                            size_t fo, int i0, int j0, int nx, int ny, const IfaceArgs &ia) {
  const double c2o3 = 2. / 3., c1o12 = 1. / 12.;
  for (int q = threadIdx.x; q < PX * PY; q += blockDim.x) {
    const int pi = q % PX, pj = q / PX;
    const int gi = wrapi(i0 - 2 + pi, nx), gj = wrapi(j0 - 2 + pj, ny);
    const size_t g = fo + (size_t)gj * nx + gi;
    const double n = hn[g], pv = hp[g], pp = hpp[g];
    const double c1 = pv;
    const double c2 = (n - pp) * 0.5;
    const double c3 = n;
    const double c4 = (3. * n - 4. * pv + pp) * 0.5;
    S.V[pj][pi] = ia.h1 * c1 + ia.h2 * c2 + ia.h3 * c3 + ia.h4 * c4;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < PX * (ITY + 1); q += blockDim.x) {
    const int pi = q % PX, r = q / PX, pj = r + 2;
    S.Dy[r][pi] = c2o3 * (S.V[pj + 1][pi] - S.V[pj - 1][pi]) - c1o12 * (S.V[pj + 2][pi] - S.V[pj - 2][pi]);
    if (pi >= 2 && pi < ITX + 3)
      S.Dx[r][pi - 2] = c2o3 * (S.V[pj][pi + 1] - S.V[pj][pi - 1]) - c1o12 * (S.V[pj][pi + 2] - S.V[pj][pi - 2]);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < (ITX + 1) * (ITY + 1); q += blockDim.x) {
    const int c = q % (ITX + 1), r = q / (ITX + 1), pi = c + 2;
    S.Dxy[r][c] = c2o3 * (S.Dy[r][pi + 1] - S.Dy[r][pi - 1]) - c1o12 * (S.Dy[r][pi + 2] - S.Dy[r][pi - 2]);
  }
  __syncthreads();
}

// Bicubic coefficients of tile cell (cx, cy) of the staged field.
__device__ __forceinline__ void iface_coeffs(const IfaceSmem &S, int cx, int cy, double (&cf)[16]) {
  double x[16];
  const int ci[4] = {0, 1, 1, 0}, cj[4] = {0, 0, 1, 1};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cx + ci[q], r = cy + cj[q];
    x[q] = S.V[r + 2][c + 2];
    x[4 + q] = S.Dx[r][c];
    x[8 + q] = S.Dy[r][c + 2];
    x[12 + q] = S.Dxy[r][c];
  }
  DNS_BICUBIC_COEFFS(cf, x);
}

// Horner evaluation at (t, u) = (ii/GR, jj/GR), ctfdtransfer_opt.c:62-97 order:
// val = t val + ((c3 u + c2) u + c1) u + c0 for nn = 3..0, starting from 0.
// At t = 0 every t val term is an exact zero, so val is the nn = 0 polynomial;
// at u = 0 each inner polynomial is its constant term.  Adding an exact zero
// leaves a non-zero value unchanged, so the shortcuts give the same value
// (a zero result can only differ in the sign of the zero).
// For GR = 2 the only non-zero t and u are 1/2: every product is exact, so a
// product and the sum it feeds become one fused multiply-add with the same
// result.  The outer step is (t val + p u) + c0 in that association: the
// reference adds the row's constant term last.
template <int GR>
__device__ __forceinline__ double iface_eval(const double (&cf)[16], int ii, int jj) {
  const double tt = ((double)ii) / ((double)GR);
  const double uu = ((double)jj) / ((double)GR);
  if (ii == 0 && jj == 0) return cf[0];
  if (GR == 2) {
    if (ii == 0) return fma(fma(fma(cf[3], uu, cf[2]), uu, cf[1]), uu, cf[0]);
    if (jj == 0) return fma(tt, fma(tt, fma(tt, cf[12], cf[8]), cf[4]), cf[0]);
    double val = fma(fma(fma(cf[15], uu, cf[14]), uu, cf[13]), uu, cf[12]);
#pragma unroll
    for (int nn = 2; nn > -1; nn--) {
      const double p = fma(fma(cf[nn * 4 + 3], uu, cf[nn * 4 + 2]), uu, cf[nn * 4 + 1]);
      val = fma(p, uu, tt * val) + cf[nn * 4];
    }
    return val;
  }
  if (ii == 0) return ((cf[3] * uu + cf[2]) * uu + cf[1]) * uu + cf[0];
  if (jj == 0) {
    double val = cf[12];
    val = tt * val + cf[8];
    val = tt * val + cf[4];
    return tt * val + cf[0];
  }
  double val = ((cf[15] * uu + cf[14]) * uu + cf[13]) * uu + cf[12];
#pragma unroll
  for (int nn = 2; nn > -1; nn--)
    val = tt * val + ((cf[nn * 4 + 3] * uu + cf[nn * 4 + 2]) * uu + cf[nn * 4 + 1]) * uu + cf[nn * 4 + 0];
  return val;
}

// Phase 1: macroscopic fields.  Block (tile, wall, field b < 4) writes field b
// (rho, ux, uy, uz) at the tile's fine interface nodes into mac[wall][b][j][i].
template <int GR>
__global__ void __launch_bounds__(TPX *TPY) interface_macro_kernel(const double *__restrict__ hn,
                                                                   const double *__restrict__ hp,
                                                                   const double *__restrict__ hpp,
                                                                   double *__restrict__ mac, Dims d, IfaceArgs ia) {
  __shared__ IfaceSmem S;
  const int nx = d.nx, ny = d.ny, nxf = d.nxf, nyf = d.nyf;
  const int w = blockIdx.z >> 2, b = blockIdx.z & 3;
  const int i0 = blockIdx.x * ITX, j0 = blockIdx.y * ITY;
  const int tx = threadIdx.x % TPX, ty = threadIdx.x / TPX;
  const size_t plane = (size_t)ny * nx, fplane = (size_t)nyf * nxf;
  iface_stage(S, hn, hp, hpp, ((size_t)w * 23 + b) * plane, i0, j0, nx, ny, ia);
  double *o = mac + ((size_t)w * 4 + b) * fplane;
#pragma unroll
  for (int q = 0; q < CPT; q++) {
    const int cx = tx + TPX * (q % (ITX / TPX)), cy = ty + TPY * (q / (ITX / TPX));
    const int ic = i0 + cx, jc = j0 + cy;
    if (ic < nx && jc < ny) {
      double cf[16];
      iface_coeffs(S, cx, cy, cf);
      if constexpr (GR == 2) {
        // both fine columns of the cell in one 16-byte store
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
          *reinterpret_cast<double2 *>(o + (size_t)(jc * 2 + jj) * nxf + ic * 2) =
              make_double2(iface_eval<2>(cf, 0, jj), iface_eval<2>(cf, 1, jj));
      } else {
#pragma unroll
        for (int ii = 0; ii < GR; ii++)
#pragma unroll
          for (int jj = 0; jj < GR; jj++)
            o[(size_t)(jc * GR + jj) * nxf + ic * GR + ii] = iface_eval<GR>(cf, ii, jj);
      }
    }
  }
}

// Phase 2: one population per block (tile, wall, a): feq(rho, u) of phase 1
// plus omega_c / (GR omega_f) times the interpolated fneq, into the fine
// block's interface plane.
template <int GR>
__global__ void __launch_bounds__(TPX *TPY) interface_pop_kernel(const double *__restrict__ hn,
                                                                 const double *__restrict__ hp,
                                                                 const double *__restrict__ hpp,
                                                                 const double *__restrict__ mac,
                                                                 double *__restrict__ fdst, Dims d, IfaceArgs ia) {
  __shared__ IfaceSmem S;
  const int nx = d.nx, ny = d.ny, nxf = d.nxf, nyf = d.nyf, zds = d.zds;
  const int w = blockIdx.z / 19, a = blockIdx.z % 19;
  const int i0 = blockIdx.x * ITX, j0 = blockIdx.y * ITY;
  const int tx = threadIdx.x % TPX, ty = threadIdx.x / TPX;
  const size_t plane = (size_t)ny * nx, fplane = (size_t)nyf * nxf;
  const int pf = w == 0 ? zds - 1 : zds;  // interface plane of the fine block
  const size_t fstride = (size_t)2 * zds * fplane;
  iface_stage(S, hn, hp, hpp, ((size_t)w * 23 + 4 + a) * plane, i0, j0, nx, ny, ia);
  const int cls = a == 0 ? 0 : (a <= 6 ? 1 : 2);
  const double wa = cls == 0 ? 1. / 3. : (cls == 1 ? 1. / 18. : 1. / 36.);
  const double *m = mac + (size_t)w * 4 * fplane;
  double *out = fdst + (size_t)a * fstride + (size_t)pf * fplane;
#pragma unroll
  for (int q = 0; q < CPT; q++) {
    const int cx = tx + TPX * (q % (ITX / TPX)), cy = ty + TPY * (q / (ITX / TPX));
    const int ic = i0 + cx, jc = j0 + cy;
    if (ic < nx && jc < ny) {
      double cf[16];
      iface_coeffs(S, cx, cy, cf);
      if constexpr (GR == 2) {
        // both fine columns of the cell: 16-byte loads of the fields and one
        // 16-byte store (the same arithmetic per node)
#pragma unroll
        for (int jj = 0; jj < 2; jj++) {
          const size_t q0 = (size_t)(jc * 2 + jj) * nxf + ic * 2;
          const double2 r2 = *reinterpret_cast<const double2 *>(m + q0);
          const double2 x2 = *reinterpret_cast<const double2 *>(m + fplane + q0);
          const double2 y2 = *reinterpret_cast<const double2 *>(m + 2 * fplane + q0);
          const double2 z2 = *reinterpret_cast<const double2 *>(m + 3 * fplane + q0);
          double o2[2];
#pragma unroll
          for (int ii = 0; ii < 2; ii++) {
            const double rho = ii ? r2.y : r2.x, u0 = ii ? x2.y : x2.x, u1 = ii ? y2.y : y2.x, u2 = ii ? z2.y : z2.x;
            const double t15v = 1.5 * (u0 * u0 + u1 * u1 + u2 * u2);
            const double val = iface_eval<2>(cf, ii, jj);
            const double feq = feq_f64(wa * rho, proj_f64(a, u0, u1, u2), t15v);
            o2[ii] = feq + ia.fac * val;
          }
          *reinterpret_cast<double2 *>(out + q0) = make_double2(o2[0], o2[1]);
        }
      } else {
#pragma unroll
        for (int ii = 0; ii < GR; ii++)
#pragma unroll
          for (int jj = 0; jj < GR; jj++) {
            const size_t qn = (size_t)(jc * GR + jj) * nxf + ic * GR + ii;
            const double rho = m[qn], u0 = m[fplane + qn], u1 = m[2 * fplane + qn], u2 = m[3 * fplane + qn];
            const double t15v = 1.5 * (u0 * u0 + u1 * u1 + u2 * u2);
            const double val = iface_eval<GR>(cf, ii, jj);
            const double feq = feq_f64(wa * rho, proj_f64(a, u0, u1, u2), t15v);
            out[qn] = feq + ia.fac * val;
          }
      }
    }
  }
}

// ------------------------------------------------------------------ injection
// Fine-to-coarse transfer (ftcdtransfer.c:28-115): the fine node on the coarse
// vertex at lower k = zdf-1-GR / upper k = GR gives the coarse planes 0 and
// zdc-1 as feq + GR omega_f/omega_c (f - feq).  Partials: what this writes into
// the state weighs GR^3 / 2 in encalc2.
//
// Filtered form (FLTR, ftcdtransfer_lesfltr.c:163-363, GR = 4): f - feq of each
// of the 5 x 5 x 5 fine nodes around the vertex (planes kb-2..kb+2, x and y
// wrapped), summed as (w f^neq) / GR^3 with the trapezoid weights
// (1/2, 1, 1, 1, 1/2) per axis, x outer, z inner; the equilibrium is that of
// the vertex node's density and momentum sums (the reference keeps the
// momentum where it reads the velocity back, :185-188, :222-225).
__device__ __forceinline__ double trapezoid5(int q) { return (q == -2 || q == 2) ? 0.5 : 1.0; }

__device__ __forceinline__ void filtered_node_f64(const double *__restrict__ fsrc, const Dims &d, int w, int ic,
                                                  int jc, double fac, double (&out)[19]) {
  const int gr = d.gr, zds = d.zds, nxf = d.nxf, nyf = d.nyf;
  const int kb = w == 0 ? d.zdf - 1 - gr : gr;
  const size_t fstride = (size_t)2 * zds * nyf * nxf;
  const double g3 = (double)gr * gr * gr;
  const int i = ic * gr, j = jc * gr;
  double t[19];
#pragma unroll
  for (int a = 0; a < 19; a++) t[a] = 0.;
  double cdens = 0., cmx = 0., cmy = 0., cmz = 0.;
#pragma unroll 1
  for (int ii = -2; ii < 3; ii++) {
    int x = i + ii;
    x = x < 0 ? x + nxf : (x >= nxf ? x - nxf : x);
#pragma unroll 1
    for (int jj = -2; jj < 3; jj++) {
      int y = j + jj;
      y = y < 0 ? y + nyf : (y >= nyf ? y - nyf : y);
      const double wxy = trapezoid5(ii) * trapezoid5(jj);
#pragma unroll 1
      for (int kk = -2; kk < 3; kk++) {
        const int k = kb + kk;
        const int p = w == 0 ? k - 1 : zds + k;
        double f[19];
        load19(fsrc, ((size_t)p * nyf + y) * nxf + x, fstride, f);
        double dens, mx, my, mz;
        moments_f64(f, dens, mx, my, mz);
        if (ii == 0 && jj == 0 && kk == 0) {
          cdens = dens;
          cmx = mx;
          cmy = my;
          cmz = mz;
        }
        const double u0 = mx / dens, u1 = my / dens, u2 = mz / dens;
        const double t15v = 1.5 * (u0 * u0 + u1 * u1 + u2 * u2);
        const Weighted wr = weighted_rho(dens);
        const double wgt = wxy * trapezoid5(kk);
#pragma unroll
        for (int a = 0; a < 19; a++) {
          const int c = wclass_of(a);
          const double feq = feq_f64(c == 0 ? wr.w0 : (c == 1 ? wr.w1 : wr.w2), proj_f64(a, u0, u1, u2), t15v);
          t[a] += (wgt * (f[a] - feq)) / g3;
        }
      }
    }
  }
  const double t15v = 1.5 * (cmx * cmx + cmy * cmy + cmz * cmz);
  const Weighted wr = weighted_rho(cdens);
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int c = wclass_of(a);
    const double feq = feq_f64(c == 0 ? wr.w0 : (c == 1 ? wr.w1 : wr.w2), proj_f64(a, cmx, cmy, cmz), t15v);
    out[a] = feq + fac * t[a];
  }
}

template <bool FLT>
__global__ void __launch_bounds__(kMaxThreads) inject_kernel(const double *__restrict__ fsrc,
                                                            double *__restrict__ cdst, Dims d, double fac,
                                                            double *__restrict__ part) {
  const int nx = d.nx, ny = d.ny, nzc = d.nzc, gr = d.gr, zdf = d.zdf, zds = d.zds;
  const int ic = blockIdx.x * blockDim.x + threadIdx.x, jc = blockIdx.y, w = blockIdx.z;
  double acc[2] = {0., 0.};
  if (FLT && ic < nx) {
    double fo[19];
    filtered_node_f64(fsrc, d, w, ic, jc, fac, fo);
    const int kc = w == 0 ? 0 : nzc - 1;
    const size_t cstride = (size_t)nzc * ny * nx;
#pragma unroll
    for (int a = 0; a < 19; a++) {
      cdst[(size_t)a * cstride + ((size_t)kc * ny + jc) * nx + ic] = fo[a];
      acc[1] += fo[a];
      if (ex_of(a) > 0) acc[0] += fo[a];
      if (ex_of(a) < 0) acc[0] -= fo[a];
    }
  } else if (!FLT && ic < nx) {
    const int ps = w == 0 ? (zdf - 1 - gr) - 1 : zds + gr;  // lower k = zdf-1-GR, upper k = GR
    const size_t fstride = (size_t)2 * zds * d.nyf * d.nxf;
    double f[19];
    load19(fsrc, ((size_t)ps * d.nyf + (size_t)jc * gr) * d.nxf + (size_t)ic * gr, fstride, f);
    double dens, mx, my, mz;
    moments_f64(f, dens, mx, my, mz);
    const double u0 = mx / dens, u1 = my / dens, u2 = mz / dens;
    const double t15v = 1.5 * (u0 * u0 + u1 * u1 + u2 * u2);
    const Weighted wr = weighted_rho(dens);
    const int kc = w == 0 ? 0 : nzc - 1;
    const size_t cstride = (size_t)nzc * ny * nx;
#pragma unroll
    for (int a = 0; a < 19; a++) {
      const int c = wclass_of(a);
      const double feq = feq_f64(c == 0 ? wr.w0 : (c == 1 ? wr.w1 : wr.w2), proj_f64(a, u0, u1, u2), t15v);
      const double fn = feq + fac * (f[a] - feq);
      cdst[(size_t)a * cstride + ((size_t)kc * ny + jc) * nx + ic] = fn;
      acc[1] += fn;
      if (ex_of(a) > 0) acc[0] += fn;
      if (ex_of(a) < 0) acc[0] -= fn;
    }
  }
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce<2>(acc, part + blk * 2);
}

// ------------------------------------------------------------------ direct encalc2
// encalc2 sums of a stored state (used after a load / seed and by dns_get_force):
// one block partial per (plane, row-block) of each level.
__global__ void __launch_bounds__(kMaxThreads) flow_sums_kernel(const double *__restrict__ fc,
                                                               const double *__restrict__ ff, Dims d, int jb,
                                                               int ncoarse_planes, double *__restrict__ part) {
  const int z = blockIdx.z;
  const bool coarse = z < ncoarse_planes;
  const int nx = coarse ? d.nx : d.nxf, ny = coarse ? d.ny : d.nyf;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0., 0.};
  double wgt;
  const double *base;
  size_t pstride;
  int p;
  const double g3 = (double)d.gr * d.gr * d.gr;
  if (coarse) {
    p = z;
    wgt = (p == 0 || p == d.nzc - 1) ? 0.5 * g3 : g3;
    base = fc;
    pstride = (size_t)d.nzc * d.ny * d.nx;
  } else {
    p = z - ncoarse_planes;
    const bool upper = p >= d.zds;
    const int k = upper ? p - d.zds : p + 1;
    if (!upper) wgt = (k >= 1 && k < d.zdf - d.gr) ? 1.0 : 0.0;
    else wgt = (k >= d.gr && k < d.zdf - 1) ? (k == d.gr ? 0.5 : 1.0) : 0.0;
    base = ff;
    pstride = (size_t)2 * d.zds * d.nyf * d.nxf;
  }
  if (i < nx && blockIdx.x * blockDim.x < nx) {
    for (int r = 0; r < jb; r++) {
      const int j = blockIdx.y * jb + r;
      if (j >= ny) break;
      double f[19];
      load19(base, ((size_t)p * ny + j) * nx + i, pstride, f);
      double dens, mx, my, mz;
      moments_f64(f, dens, mx, my, mz);
      acc[0] += wgt * mx;
      acc[1] += wgt * dens;
    }
  }
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_reduce<2>(acc, part + blk * 2);
}

// ------------------------------------------------------------------ finalize
// Deterministic reduction of the block partials (fixed order, one block) into
// the next step's encalc2 values and force, plus this step's log row.
constexpr int kFinThreads = 1024;

__device__ double fixed_sum(const double *p, long n, int stride, int comp) {
  __shared__ double sh[kFinThreads];
  double s = 0.;
  for (long q = threadIdx.x; q < n; q += blockDim.x) s += p[q * stride + comp];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

struct FinArgs {
  long nc, nf, ni;             // partial counts (pairs)
  long wb[6];                  // wall-shear plane block offsets (pairs), lower k=1,2,3 then upper zdf-2,-3,-4
  long wn;                     // blocks per plane
  double g3, norm, norm2, mu, ub, gconst, pgrad_scale, flow_scale, den_offset;
  int cfr, with_log;
};

__global__ void __launch_bounds__(kFinThreads) finalize_kernel(DevState *st, DevLog *lg, const double *part_c,
                                                              const double *part_f, const double *part_i,
                                                              const double *part_w, FinArgs a) {
  double momc = fixed_sum(part_c, a.nc, 2, 0), denc = fixed_sum(part_c, a.nc, 2, 1);
  double momf = fixed_sum(part_f, a.nf, 2, 0), denf = fixed_sum(part_f, a.nf, 2, 1);
  double momi = fixed_sum(part_i, a.ni, 2, 0), deni = fixed_sum(part_i, a.ni, 2, 1);
  double U[6], D[6];
  if (a.with_log) {
    for (int q = 0; q < 6; q++) {
      U[q] = fixed_sum(part_w + a.wb[q] * 2, a.wn, 2, 0);
      D[q] = fixed_sum(part_w + a.wb[q] * 2, a.wn, 2, 1);
    }
  }
  if (threadIdx.x == 0) {
    if (a.with_log) {
      DevLog r;
      r.force = st->force;
      r.momentum = st->momentum;
      r.denst = st->denst;
      r.flowrate = st->momentum * a.flow_scale / st->denst;
      const double stdown = ((-2. * U[0] + 3. * U[1] - U[2]) / a.norm2) * (a.mu * (D[0] / a.norm2));
      const double stup = (-(2. * U[3] - 3. * U[4] + U[5]) / a.norm2) * (a.mu * (D[5] / a.norm2));
      r.stup = stup;
      r.stdown = stdown;
      r.stress = 0.5 * (stup + stdown);
      r.pgrad = st->force * a.pgrad_scale;
      *lg = r;
    }
    const double mom = (a.g3 * momc + 0.5 * a.g3 * momi + momf) / a.norm;
    const double den = (a.g3 * denc + 0.5 * a.g3 * deni + denf + a.den_offset) / a.norm;
    st->momentum = mom;
    st->denst = den;
    st->force = a.cfr ? a.ub - mom : a.gconst;
  }
}

// Per-step finalize in two levels: kFin2Blocks blocks each reduce a fixed
// chunk of every partial region (fixed order), the last block to finish sums
// the chunk results in block order.  Deterministic, one launch, no waiting.
constexpr int kFin2Blocks = 64, kFin2Threads = 256, kFin2Comp = 18;

__global__ void __launch_bounds__(kFin2Threads) finalize2_kernel(DevState *st, DevLog *lg, const double *part_c,
                                                                const double *part_f, const double *part_i,
                                                                const double *part_w, double *level2,
                                                                unsigned int *counter, FinArgs a) {
  __shared__ double sh[kFin2Comp];
  __shared__ bool last;
  const int b = blockIdx.x, nb = gridDim.x;
  double v[kFin2Comp];
#pragma unroll
  for (int c = 0; c < kFin2Comp; c++) v[c] = 0.;
  // the nine regions (coarse, fine, injection, six wall planes) as one run of
  // (U, D) pairs; this block takes a fixed slice of it, so that a thread's
  // loads are issued together whatever region they fall in
  const double *base[9] = {part_c, part_f, part_i, part_w + a.wb[0] * 2, part_w + a.wb[1] * 2,
                           part_w + a.wb[2] * 2, part_w + a.wb[3] * 2, part_w + a.wb[4] * 2, part_w + a.wb[5] * 2};
  const long cnt[9] = {a.nc, a.nf, a.ni, a.wn, a.wn, a.wn, a.wn, a.wn, a.wn};
  const long T = a.nc + a.nf + a.ni + 6 * a.wn;
  const long lo = T * b / nb, hi = T * (b + 1) / nb;
  for (long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
    long r0 = q;
    int rr = 0;
    while (rr < 8 && r0 >= cnt[rr]) r0 -= cnt[rr++];
    const double u = base[rr][r0 * 2], dd = base[rr][r0 * 2 + 1];
#pragma unroll
    for (int r = 0; r < 9; r++)
      if (r == rr) {
        v[2 * r] += u;
        v[2 * r + 1] += dd;
      }
  }
  block_reduce_n<kFin2Comp, kFin2Threads>(v, sh);
  if (threadIdx.x == 0) {
    for (int c = 0; c < kFin2Comp; c++) level2[b * kFin2Comp + c] = sh[c];
    __threadfence();
    last = atomicAdd(counter, 1u) == (unsigned)(nb - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  __syncthreads();
  // the level-2 rows are loaded by the whole block at once, then summed in
  // block order by one thread per component
  __shared__ double rows[kFin2Blocks * kFin2Comp];
  {
    const volatile double *l2 = level2;
    for (int q = threadIdx.x; q < nb * kFin2Comp; q += blockDim.x) rows[q] = l2[q];
  }
  __syncthreads();
  if (threadIdx.x < kFin2Comp) {
    double s = 0.;
    for (int q = 0; q < nb; q++) s += rows[q * kFin2Comp + threadIdx.x];
    sh[threadIdx.x] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double *S = sh;
    DevLog r;
    r.force = st->force;
    r.momentum = st->momentum;
    r.denst = st->denst;
    r.flowrate = st->momentum * a.flow_scale / st->denst;
    const double *U = S + 6;  // (U, D) pairs per plane: lower k=1,2,3, upper zdf-2,-3,-4
    const double stdown = ((-2. * U[0] + 3. * U[2] - U[4]) / a.norm2) * (a.mu * (U[1] / a.norm2));
    const double stup = (-(2. * U[6] - 3. * U[8] + U[10]) / a.norm2) * (a.mu * (U[11] / a.norm2));
    r.stup = stup;
    r.stdown = stdown;
    r.stress = 0.5 * (stup + stdown);
    r.pgrad = st->force * a.pgrad_scale;
    *lg = r;
    const double mom = (a.g3 * S[0] + 0.5 * a.g3 * S[4] + S[2]) / a.norm;
    const double den = (a.g3 * S[1] + 0.5 * a.g3 * S[5] + S[3] + a.den_offset) / a.norm;
    st->momentum = mom;
    st->denst = den;
    st->force = a.cfr ? a.ub - mom : a.gconst;
    *counter = 0u;
  }
}

// per-plane statistics of one sample, added to the running rows acc[NZ][kStatRow]
// (layout in kernels.h)
struct StatsArgs {
  int nzp;          // composite profile length
  int zdf, nzc, zds;
  long bc, bf;      // blocks per plane (coarse, fine)
  double nc, nf;    // nodes per plane (coarse, fine)
};

__global__ void __launch_bounds__(256) stats_finalize_kernel(double *acc, const double *spc, const double *spf,
                                                            StatsArgs a) {
  const int idx = blockIdx.x;
  const double *src = nullptr;
  long nb = 0;
  const int zdf = a.zdf, nzc = a.nzc;
  if (idx >= 1 && idx <= zdf - 1) {  // lower fine k = idx
    src = spf + (size_t)(idx - 1) * a.bf * kStatPart; nb = a.bf;
  } else if (idx >= zdf && idx <= zdf + nzc - 5) {  // coarse k = idx - zdf + 2
    src = spc + (size_t)(idx - zdf + 2) * a.bc * kStatPart; nb = a.bc;
  } else if (idx >= zdf + nzc - 4 && idx <= 2 * zdf + nzc - 6) {  // upper fine k
    const int k = idx - (zdf + nzc - 4);
    src = spf + (size_t)(a.zds + k) * a.bf * kStatPart; nb = a.bf;
  }
  if (!src) return;
  stat_plane_finalize(src, nb, acc + (size_t)idx * kStatRow);
}

// ------------------------------------------------------------------ seeded state
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                              uint32_t k1, uint32_t (&out)[4]) {
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

__device__ __forceinline__ void seeded_node(double *dst, size_t stride, uint64_t seed, double uc, double amp,
                                            double H, double z, uint32_t i, uint32_t j, uint32_t k, uint32_t lvl,
                                            double *u_out) {
  uint32_t r[4];
  philox4x32_10(i, j, k, lvl, (uint32_t)seed, (uint32_t)(seed >> 32), r);
  const double zeta = z / H;
  const double prof = 4.0 * uc * zeta * (1.0 - zeta);
  double u[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double x = ((double)r[c] + 0.5) * (1.0 / 4294967296.0);
    u[c] = amp * (2.0 * x - 1.0);
  }
  u[0] = prof + u[0];
  const double t15v = 1.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int c = wclass_of(a);
    const double wr = (c == 0 ? 1. / 3. : (c == 1 ? 1. / 18. : 1. / 36.)) * 1.0;
    dst[(size_t)a * stride] = feq_f64(wr, proj_f64(a, u[0], u[1], u[2]), t15v);
  }
  if (u_out) {
    u_out[0] = u[0];
    u_out[1] = u[1];
    u_out[2] = u[2];
  }
}

__global__ void __launch_bounds__(kMaxThreads) seed_kernel(double *fc, double *ff, double *hist3, Dims d,
                                                          uint64_t seed, double uc, double amp) {
  const int z = blockIdx.z, j = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double H = d.nzs - 2.0;
  if (z < d.nzc) {
    const int k = z;
    if (i >= d.nx || j >= d.ny) return;
    const size_t stride = (size_t)d.nzc * d.ny * d.nx;
    const double zpos = (d.zdf - 1.5) + d.gr * (k - 1.0);
    double u[3];
    seeded_node(fc + ((size_t)k * d.ny + j) * d.nx + i, stride, seed, uc, amp, H, zpos, i, j, k, 0, u);
    if (k == 1 || k == d.nzc - 2) {
      const size_t plane = (size_t)d.ny * d.nx;
      const int w = k == 1 ? 0 : 1;
      for (int l = 0; l < 3; l++) {
        double *o = hist3 + ((size_t)l * 2 + w) * 23 * plane + (size_t)j * d.nx + i;
        o[0] = 1.0;
        o[plane] = u[0];
        o[2 * plane] = u[1];
        o[3 * plane] = u[2];
        for (int b = 4; b < 23; b++) o[(size_t)b * plane] = 0.0;
      }
    }
  } else {
    const int p = z - d.nzc;
    if (i >= d.nxf || j >= d.nyf) return;
    const bool upper = p >= d.zds;
    const int k = upper ? p - d.zds : p + 1;
    const double zpos = upper ? (d.zdf - 1.5) + d.gr * (d.nzc - 3.0) + k : k - 0.5;
    const size_t stride = (size_t)2 * d.zds * d.nyf * d.nxf;
    seeded_node(ff + ((size_t)p * d.nyf + j) * d.nxf + i, stride, seed, uc, amp, H, zpos, i, j, k,
                upper ? 2 : 1, nullptr);
  }
}

// ------------------------------------------------------------------ transposes
__global__ void soa_to_aos_kernel(const double *__restrict__ soa, double *__restrict__ aos, int nx, int ny, int P,
                                  int p0, int nz_aos, int k0_aos, int i0, int i1) {
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= i1) return;
  const size_t stride = (size_t)P * ny * nx;
  const size_t s = ((size_t)(p0 + q) * ny + j) * nx + i;
  double *o = aos + (((size_t)i * ny + j) * nz_aos + k0_aos + q) * 19;
  for (int a = 0; a < 19; a++) o[a] = soa[s + (size_t)a * stride];
}

__global__ void aos_to_soa_kernel(const double *__restrict__ aos, double *__restrict__ soa, int nx, int ny, int P,
                                  int p0, int nz_aos, int k0_aos, int i0, int i1) {
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= i1) return;
  const size_t stride = (size_t)P * ny * nx;
  const size_t s = ((size_t)(p0 + q) * ny + j) * nx + i;
  const double *o = aos + (((size_t)i * ny + j) * nz_aos + k0_aos + q) * 19;
  for (int a = 0; a < 19; a++) soa[s + (size_t)a * stride] = o[a];
}

// Wall plane kw of an AoS level [nx][ny][nz][19] <-> the compact wall array
// [nx][ny][19] (TO_AOS: wall -> aos).
template <bool TO_AOS>
__global__ void wall_plane_kernel(double *__restrict__ aos, double *__restrict__ wall, long long nodes, int nz,
                                  int kw) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nodes * 19) return;
  const long long c = t / 19, a = t - c * 19;
  double *o = aos + (c * nz + kw) * 19 + a;
  if (TO_AOS)
    *o = wall[t];
  else
    wall[t] = *o;
}

// ------------------------------------------------------------------ field output
// vel_print.c:86-125: per node u = (sum E f) / rho, rho = sum f, both summed in
// population order (moments_f64 is that order); zero where rho <= 0
template <bool PLANAR>
__global__ void fields_kernel(const double *__restrict__ soa, double *__restrict__ vel, double *__restrict__ den,
                              int nx, int ny, int P, int p0, int nz_aos, int k0_aos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, q = blockIdx.z;
  if (i >= nx) return;
  const size_t stride = (size_t)P * ny * nx;
  double f[19];
  load19(soa, ((size_t)(p0 + q) * ny + j) * nx + i, stride, f);
  double dens, mx, my, mz;
  moments_f64(f, dens, mx, my, mz);
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
LaunchShape make_shape(const Dims &d) {
  LaunchShape s;
  s.bx = DNS_BX;
  s.jb = DNS_JB;
  s.cgx = (d.nx + s.bx - 1) / s.bx;
  s.cgy = (d.ny + s.jb - 1) / s.jb;
  s.fgx = (d.nxf + s.bx - 1) / s.bx;
  s.fgy = (d.nyf + s.jb - 1) / s.jb;
  s.igx = (d.nx + ITX - 1) / ITX;
  s.igy = (d.ny + ITY - 1) / ITY;
  s.jgx = (d.nx + s.bx - 1) / s.bx;
  s.jgy = d.ny;
  return s;
}

PartialLayout partial_layout(const Dims &d, const LaunchShape &s) {
  PartialLayout pl;
  const long nbc = s.n_coarse_blocks() * d.nzc, nbf = s.n_fine_blocks() * 2 * d.zds;
  const long nbi = (long)s.jgx * s.jgy * 2;
  long o = 0;
  pl.coarse = o; o += nbc * 2;
  pl.fine = o; o += nbf * 2;
  pl.inject = o; o += nbi * 2;
  pl.wall = o; o += nbf * 2;
  pl.stats_c = o; o += nbc * kStatPart;
  pl.stats_f = o; o += nbf * kStatPart;
  const long gx = s.fgx > s.cgx ? s.fgx : s.cgx, gy = s.fgy > s.cgy ? s.fgy : s.cgy;
  pl.flow = o; o += gx * gy * (d.nzc + 2 * d.zds) * 2;
  pl.level2 = o; o += kFin2Blocks * kFin2Comp;
  pl.total = o;
  return pl;
}

void launch_coarse_f64(const double *src, double *dst, const Dims &d, const LaunchShape &s, double om,
                       const DevState *st, double *partials, const PartialLayout &pl, bool stats,
                       cudaStream_t stream) {
  dim3 grid(s.cgx, s.cgy, d.nzc), block(s.bx);
  if (stats)
    coarse_kernel<true><<<grid, block, 0, stream>>>(src, dst, d, s.jb, om, st, partials + pl.coarse,
                                                    partials + pl.stats_c);
  else
    coarse_kernel<false><<<grid, block, 0, stream>>>(src, dst, d, s.jb, om, st, partials + pl.coarse,
                                                     partials + pl.stats_c);
}

void launch_extract_f64(const double *fc, double *hist_n, const Dims &d, const LaunchShape &s, cudaStream_t stream) {
  dim3 grid(s.jgx, d.ny, 2), block(s.bx);
  extract_kernel<<<grid, block, 0, stream>>>(fc, hist_n, d);
}

void launch_fine_f64(const double *src, double *dst, const int8_t *wflag, const Dims &d, const LaunchShape &s,
                     double om, const DevState *st, double *partials, const PartialLayout &pl, bool first,
                     bool last, bool stats, cudaStream_t stream) {
  dim3 grid(s.fgx, s.fgy, 2 * d.zds), block(s.bx);
  const int mode = (last ? 1 : 0) | (first ? 2 : 0) | (stats ? 4 : 0);
  double *pf = partials + pl.fine, *pw = partials + pl.wall, *ps = partials + pl.stats_f;
#define FINE_CASE(M) \
  case M: fine_kernel<M><<<grid, block, 0, stream>>>(src, dst, wflag, d, s.jb, om, st, pf, pw, ps); break;
  switch (mode) {
    FINE_CASE(0) FINE_CASE(1) FINE_CASE(2) FINE_CASE(3) FINE_CASE(4) FINE_CASE(5) FINE_CASE(6) FINE_CASE(7)
  }
#undef FINE_CASE
}

void launch_interface_f64(const double *hn, const double *hp, const double *hpp, double *mac, double *fdst,
                          const Dims &d, const LaunchShape &s, int substep, double omega_c, double omega_f,
                          cudaStream_t stream) {
  // Hermite basis at tau = substep / GR, evaluated as the reference writes it
  // (tinterpolate_hrmt.c:34); rescaling factor of ctfdtransfer_opt.c:101.
  const double tmp = (((double)substep) / ((double)d.gr));
  IfaceArgs ia;
  ia.h1 = 2. * tmp * tmp * tmp - 3. * tmp * tmp + 1.;
  ia.h2 = tmp * tmp * tmp - 2. * tmp * tmp + tmp;
  ia.h3 = -2. * tmp * tmp * tmp + 3. * tmp * tmp;
  ia.h4 = tmp * tmp * tmp - tmp * tmp;
  ia.fac = omega_c / ((double)d.gr * omega_f);
  dim3 gm(s.igx, s.igy, 2 * 4), gp(s.igx, s.igy, 2 * 19), block(TPX * TPY);
  if (d.gr == 2) {
    interface_macro_kernel<2><<<gm, block, 0, stream>>>(hn, hp, hpp, mac, d, ia);
    interface_pop_kernel<2><<<gp, block, 0, stream>>>(hn, hp, hpp, mac, fdst, d, ia);
  } else if (d.gr == 3) {
    interface_macro_kernel<3><<<gm, block, 0, stream>>>(hn, hp, hpp, mac, d, ia);
    interface_pop_kernel<3><<<gp, block, 0, stream>>>(hn, hp, hpp, mac, fdst, d, ia);
  } else {
    interface_macro_kernel<4><<<gm, block, 0, stream>>>(hn, hp, hpp, mac, d, ia);
    interface_pop_kernel<4><<<gp, block, 0, stream>>>(hn, hp, hpp, mac, fdst, d, ia);
  }
}

void launch_inject_f64(const double *fsrc, double *cdst, const Dims &d, const LaunchShape &s, double omega_c,
                       double omega_f, double *partials, const PartialLayout &pl, bool filtered,
                       cudaStream_t stream) {
  const double fac = d.gr * (omega_f / omega_c);
  dim3 grid(s.jgx, s.jgy, 2), block(s.bx);
  if (filtered)
    inject_kernel<true><<<grid, block, 0, stream>>>(fsrc, cdst, d, fac, partials + pl.inject);
  else
    inject_kernel<false><<<grid, block, 0, stream>>>(fsrc, cdst, d, fac, partials + pl.inject);
}

static FinArgs fin_args(const PartialLayout &pl, const Dims &d, const LaunchShape &s, const StepParams &sp) {
  FinArgs a;
  a.nc = s.n_coarse_blocks() * d.nzc;
  a.nf = s.n_fine_blocks() * 2 * d.zds;
  a.ni = (long)s.jgx * s.jgy * 2;
  a.wn = s.n_fine_blocks();
  const int zds = d.zds, zdf = d.zdf;
  const int planes[6] = {0, 1, 2, zds + zdf - 2, zds + zdf - 3, zds + zdf - 4};
  for (int q = 0; q < 6; q++) a.wb[q] = (long)planes[q] * s.n_fine_blocks();
  a.g3 = (double)d.gr * d.gr * d.gr;
  a.norm = (double)((double)d.nxf * (double)d.nyf * (d.nzs - 2.));
  a.norm2 = (double)d.nxf * (double)d.nyf;
  a.mu = (1. / 6.) * (2. / sp.omega_f - 1);
  a.ub = sp.ub;
  a.gconst = sp.gconst;
  a.pgrad_scale = (d.nzs - 2.) / (2. * d.gr);
  a.flow_scale = (double)((long)d.nyf * (d.nzs - 2));
  a.cfr = sp.cfr;
  a.den_offset = sp.den_offset;
  a.with_log = 1;
  (void)pl;
  return a;
}

void launch_finalize(DevState *st, DevLog *log_row, double *partials, unsigned int *counter,
                     const PartialLayout &pl, const Dims &d, const LaunchShape &s, const StepParams &sp,
                     cudaStream_t stream) {
  FinArgs a = fin_args(pl, d, s, sp);
  finalize2_kernel<<<kFin2Blocks, kFin2Threads, 0, stream>>>(st, log_row, partials + pl.coarse, partials + pl.fine,
                                                             partials + pl.inject, partials + pl.wall,
                                                             partials + pl.level2, counter, a);
}

void launch_stats_finalize(double *acc, const double *partials, const PartialLayout &pl, const Dims &d,
                           const LaunchShape &s, cudaStream_t stream) {
  StatsArgs a;
  a.nzp = 2 * d.zdf + d.nzc - 4;
  a.zdf = d.zdf;
  a.nzc = d.nzc;
  a.zds = d.zds;
  a.bc = s.n_coarse_blocks();
  a.bf = s.n_fine_blocks();
  a.nc = (double)d.nx * d.ny;
  a.nf = (double)d.nxf * d.nyf;
  stats_finalize_kernel<<<a.nzp, 256, 0, stream>>>(acc, partials + pl.stats_c, partials + pl.stats_f, a);
}

void launch_flow_sums_f64(const double *fc, const double *ff, DevState *st, double *partials,
                          const PartialLayout &pl, const Dims &d, const LaunchShape &s, const StepParams &sp,
                          cudaStream_t stream) {
  // coarse planes then fine planes; one pair per block into the coarse+fine partial areas
  const int gx = s.fgx > s.cgx ? s.fgx : s.cgx, gy = s.fgy > s.cgy ? s.fgy : s.cgy;
  const int nz = d.nzc + 2 * d.zds;
  const long nblocks = (long)gx * gy * nz;
  double *scratch = partials + pl.flow;
  dim3 grid(gx, gy, nz), block(s.bx);
  flow_sums_kernel<<<grid, block, 0, stream>>>(fc, ff, d, s.jb, d.nzc, scratch);
  FinArgs a = fin_args(pl, d, s, sp);
  a.nc = 0;
  a.ni = 0;
  a.nf = nblocks;
  a.with_log = 0;
  // the fine path of finalize sums with weight 1: the kernel already applied
  // every encalc2 weight, so feed everything through the fine slot
  finalize_kernel<<<1, kFinThreads, 0, stream>>>(st, nullptr, scratch, scratch, scratch, scratch, a);
}

void finalize_flow_sums(DevState *st, const double *pairs, long npairs, const Dims &d, const LaunchShape &s,
                        const StepParams &sp, cudaStream_t stream) {
  PartialLayout unused{};
  FinArgs a = fin_args(unused, d, s, sp);
  a.nc = 0;
  a.ni = 0;
  a.nf = npairs;
  a.with_log = 0;
  finalize_kernel<<<1, kFinThreads, 0, stream>>>(st, nullptr, pairs, pairs, pairs, pairs, a);
}

double encalc2_weight_sum(const Dims &d) {
  const double g3 = (double)d.gr * d.gr * d.gr;
  const double cplane = (double)d.nx * d.ny, fplane = (double)d.nxf * d.nyf;
  // coarse: planes 1..zdc-2 weigh GR^3, planes 0 and zdc-1 half that;
  // lower fine k in [1, zdf-GR); upper fine k in [GR, zdf-1) with k = GR halved
  return g3 * cplane * (d.nzc - 1) + fplane * ((d.zdf - d.gr - 1) + (d.zdf - 2 - d.gr) + 0.5);
}

long flow_sums_pairs(const Dims &d, const LaunchShape &s) {
  const long gx = s.fgx > s.cgx ? s.fgx : s.cgx, gy = s.fgy > s.cgy ? s.fgy : s.cgy;
  return gx * gy * (d.nzc + 2 * d.zds);
}

void launch_flow_sums_scratch(const double *fc, const double *ff, DevState *out, double *scratch, const Dims &d,
                              const LaunchShape &s, const StepParams &sp, cudaStream_t stream) {
  const int gx = s.fgx > s.cgx ? s.fgx : s.cgx, gy = s.fgy > s.cgy ? s.fgy : s.cgy;
  dim3 grid(gx, gy, d.nzc + 2 * d.zds), block(s.bx);
  flow_sums_kernel<<<grid, block, 0, stream>>>(fc, ff, d, s.jb, d.nzc, scratch);
  PartialLayout unused{};
  FinArgs a = fin_args(unused, d, s, sp);
  a.nc = 0;
  a.ni = 0;
  a.nf = flow_sums_pairs(d, s);
  a.with_log = 0;
  finalize_kernel<<<1, kFinThreads, 0, stream>>>(out, nullptr, scratch, scratch, scratch, scratch, a);
}

void launch_seed_f64(double *fc, double *ff, double *hist3, const Dims &d, uint64_t seed, double uc, double amp,
                     cudaStream_t stream) {
  const int nxm = d.nxf > d.nx ? d.nxf : d.nx, nym = d.nyf > d.ny ? d.nyf : d.ny;
  dim3 grid((nxm + 127) / 128, nym, d.nzc + 2 * d.zds), block(128);
  seed_kernel<<<grid, block, 0, stream>>>(fc, ff, hist3, d, seed, uc, amp);
}

void launch_soa_to_aos(const double *soa, double *aos, int nx, int ny, int P, int p0, int np, int nz_aos, int k0_aos,
                       cudaStream_t stream, int i0, int i1) {
  if (i1 < 0) i1 = nx;
  if (i1 <= i0) return;
  dim3 grid((i1 - i0 + 127) / 128, ny, np), block(128);
  soa_to_aos_kernel<<<grid, block, 0, stream>>>(soa, aos, nx, ny, P, p0, nz_aos, k0_aos, i0, i1);
}

void launch_aos_to_soa(const double *aos, double *soa, int nx, int ny, int P, int p0, int np, int nz_aos, int k0_aos,
                       cudaStream_t stream, int i0, int i1) {
  if (i1 < 0) i1 = nx;
  if (i1 <= i0) return;
  dim3 grid((i1 - i0 + 127) / 128, ny, np), block(128);
  aos_to_soa_kernel<<<grid, block, 0, stream>>>(aos, soa, nx, ny, P, p0, nz_aos, k0_aos, i0, i1);
}

void launch_wall_plane(double *aos, double *wall, long long nodes, int nz, int kw, bool to_aos, cudaStream_t stream) {
  const unsigned blocks = (unsigned)((nodes * 19 + 255) / 256);
  if (to_aos)
    wall_plane_kernel<true><<<blocks, 256, 0, stream>>>(aos, wall, nodes, nz, kw);
  else
    wall_plane_kernel<false><<<blocks, 256, 0, stream>>>(aos, wall, nodes, nz, kw);
}

void launch_fields_f64(const double *soa, double *vel, double *den, int nx, int ny, int P, int p0, int np, int nz_aos,
                       int k0_aos, cudaStream_t stream) {
  dim3 grid((nx + 127) / 128, ny, np), block(128);
  fields_kernel<false><<<grid, block, 0, stream>>>(soa, vel, den, nx, ny, P, p0, nz_aos, k0_aos);
}

void launch_fields_planar_f64(const double *soa, double *q, int nx, int ny, int P, int p0, int np, int nz,
                              int k0, cudaStream_t stream) {
  dim3 grid((nx + 127) / 128, ny, np), block(128);
  fields_kernel<true><<<grid, block, 0, stream>>>(soa, q, nullptr, nx, ny, P, p0, nz, k0);
}

// ------------------------------------------------------------------ mode -i start
// Uniform grid -> embedded grid (initializer.c:303-533, the pass over the first half,
// sp_interpolate_qd.c:22-45): tri-quadratic Lagrange interpolation of all 19
// populations at the level's node, then f = feq + fac (f_int - feq) with feq of
// the interpolated moments.  Every expression is the reference's, in its order
// (this unit is built without fused multiply-add).  The reference reads the
// uniform state into an array with a two-deep ghost layer below and four above
// in x and y, filled periodically; the periodic wrap here reads the same values
// wherever that halo reaches.
namespace {

__device__ __forceinline__ int wrap_periodic(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// 0.5 d (d - 1) F0 - (d - 1)(d + 1) F1 + 0.5 (d + 1) d F2  (sp_interpolate_qd.c:34,41,44)
__device__ __forceinline__ double lagrange3(double d, double f0, double f1, double f2) {
  return 0.5 * d * (d - 1.) * f0 - (d - 1.) * (d + 1.) * f1 + 0.5 * (d + 1.) * d * f2;
}

__global__ void __launch_bounds__(128) uniform_interp_kernel(const double *__restrict__ uni, UniformMap m,
                                                             double *__restrict__ out, int *__restrict__ bad) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nodes = (long long)m.nxl * m.nyl * m.nzl;
  if (t >= nodes) return;
  const int k = (int)(t % m.nzl);
  const int j = (int)((t / m.nzl) % m.nyl);
  const int i = (int)(t / ((long long)m.nzl * m.nyl));
  double *o = out + t * 19;
  const bool wall = (m.level == 1 && k == 0) || (m.level == 2 && k == m.zdf - 1);
  if (wall) {
    // init.c:18-53 runs before the wall flags exist in mode -i: rest equilibrium
#pragma unroll
    for (int a = 0; a < 19; a++) {
      const int c = wclass_of(a);
      o[a] = c == 0 ? 1. / 3. : (c == 1 ? 1. / 18. : 1. / 36.);
    }
    return;
  }
  const double dxf = m.dxf, dxc = m.dxc, dxr = m.dxr;
  const int GR = m.gr, zdf = m.zdf, zdc = m.zdc;
  int iref, jref, kref, k0;
  double dx, dy, dz;
  if (m.level == 1) {  // initializer.c:326-399
    iref = (int)floor((i + 0.5) * (dxf / dxr) - 0.5);
    jref = (int)floor((j + 0.5) * (dxf / dxr) - 0.5);
    kref = (int)floor((k - 0.5) * (dxf / dxr) + 0.5);
    dx = (i + 0.5) * dxf - (iref + 0.5) * dxr;
    dy = (j + 0.5) * dxf - (jref + 0.5) * dxr;
    if (kref == 0) {
      k0 = kref;
      dz = -dxr + (k - 0.5) * dxf + 0.5 * dxr - kref * dxr;
    } else {
      k0 = kref - 1;
      dz = (k - 0.5) * dxf + 0.5 * dxr - kref * dxr;
    }
  } else if (m.level == 0) {  // initializer.c:402-468
    iref = (int)floor((i + 0.5) * dxc / dxr - 0.5);
    jref = (int)floor((j + 0.5) * dxc / dxr - 0.5);
    kref = (int)floor(0.5 + (k * GR + (zdf - GR - 1 - 0.5)) * dxf / dxr);
    dx = (i + 0.5) * dxc - (iref + 0.5) * dxr;
    dy = (j + 0.5) * dxc - (jref + 0.5) * dxr;
    k0 = kref - 1;
    dz = (k * GR + (zdf - GR - 1 - 0.5)) * dxf - (kref - 0.5) * dxr;
  } else {  // initializer.c:470-533
    iref = (int)floor((i + 0.5) * dxf / dxr - 0.5);
    jref = (int)floor((j + 0.5) * dxf / dxr - 0.5);
    kref = (int)floor(0.5 + (k + GR * (zdc - 3) + zdf - 1 - 0.5) * dxf / dxr);
    dx = (i + 0.5) * dxf - (iref + 0.5) * dxr;
    dy = (j + 0.5) * dxf - (jref + 0.5) * dxr;
    k0 = kref - 1;
    dz = (k + GR * (zdc - 3) + zdf - 1 - 0.5) * dxf - (kref - 0.5) * dxr;
  }
  dx = dx / dxr;
  dy = dy / dxr;
  dz = dz / dxr;
  if (iref - 1 < -2 || iref + 1 > m.xu + 3 || jref - 1 < -2 || jref + 1 > m.yu + 3 || k0 < 0 || k0 + 2 >= m.zd) {
    atomicOr(bad, 1);
#pragma unroll
    for (int a = 0; a < 19; a++) o[a] = __longlong_as_double(0x7ff8000000000000LL);
    return;
  }
  // row offsets of the 3 x 3 stencil columns (ind[i] x jnd[j]), z-runs of 3 x 19 doubles
  size_t col[3][3];
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int q = 0; q < 3; q++)
      col[p][q] = (((size_t)wrap_periodic(iref - 1 + p, m.xu) * m.yu + wrap_periodic(jref - 1 + q, m.yu)) * m.zd + k0) * 19;
  double fi[19];
#pragma unroll 1
  for (int a = 0; a < 19; a++) {
    double cy[3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      double cz[3];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const double *u = uni + col[p][q] + a;
        cz[q] = lagrange3(dz, __ldg(u), __ldg(u + 19), __ldg(u + 38));
      }
      cy[p] = lagrange3(dy, cz[0], cz[1], cz[2]);
    }
    fi[a] = lagrange3(dx, cy[0], cy[1], cy[2]);
  }
  double dens, mx, my, mz;
  moments_f64(fi, dens, mx, my, mz);
  const double u0 = mx / dens, u1 = my / dens, u2 = mz / dens;
  const double t15v = 1.5 * (u0 * u0 + u1 * u1 + u2 * u2);
  const Weighted wr = weighted_rho(dens);
#pragma unroll
  for (int a = 0; a < 19; a++) {
    const int c = wclass_of(a);
    const double feq = feq_f64(c == 0 ? wr.w0 : (c == 1 ? wr.w1 : wr.w2), proj_f64(a, u0, u1, u2), t15v);
    o[a] = feq + m.fac * (fi[a] - feq);
  }
}

}  // namespace

void launch_uniform_interp_f64(const double *uni, const UniformMap &m, double *out, int *bad, cudaStream_t stream) {
  const long long nodes = (long long)m.nxl * m.nyl * m.nzl;
  uniform_interp_kernel<<<(unsigned)((nodes + 127) / 128), 128, 0, stream>>>(uni, m, out, bad);
}

}  // namespace dns
