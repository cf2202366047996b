// Turbulence statistics and kinetic-energy budget of one snapshot, on the
// device: the reference's offline program TKE-budget/computations
// (budget-no-slip-mgrd.c:95-105 loop body: reading.c, budget2D.c:13-1736,
// uv_fluc.c:15-49) applied to the vel-* / den-* fields of the three levels.
//
// Pipeline (all FP64):
//   1. planar copy of each level's fields, q[c][k][j][i] with c = u, v, w and
//      den / 3 (the reference's pressure, budget2D.c:184);
//   2. plane means of the composite profile (budget2D.c:178-241): lower fine
//      planes 0..zdf-1, coarse planes 2..zdc-3, upper fine planes 0..zdf-1,
//      each summed in the reference's order, so they are bit-identical;
//   3. per-plane sums of the 44 products of fluctuations and their gradients
//      (budget2D.c:448-1002): 4th-order central differences in x and y,
//      the reference's plane-dependent rules in z (one-sided at the walls,
//      mixed-spacing at the level joins, reading the neighbouring level);
//   4. on the host, the O(NZ) finalisation of budget2D.c:1004-1550: plane
//      averages, rms, skewness, flatness, vorticity rms, production,
//      turbulent / pressure / viscous transport, pressure strain, dissipation.
// Block partials of the 44 products are summed in a fixed order, so results are
// deterministic; they differ from the reference's sequential plane sums by
// rounding only.
// This unit is built without fused multiply-add, like the reference.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "host.h"
#include "kernels.h"

namespace dns {

namespace {

constexpr int kT = 128;  // threads per block
constexpr int kNS = 44;  // per-plane sums of the budget pass

// accumulator order (the reference's reduction order, budget2D.c:1070-1244)
enum {
  S_UU, S_UV, S_UW, S_VV, S_VW, S_WW, S_DD,
  S_SKU, S_SKV, S_SKW, S_SKP, S_SKUW, S_SKUV, S_SKVW,
  S_KUU, S_KUV, S_KUW, S_KUP, S_KUUW, S_KUVW, S_KUUV,
  S_WX, S_WY, S_WZ, S_UUW, S_VVW, S_WWW, S_UWW, S_PU, S_PV, S_PW,
  S_PAIUU, S_PAIVV, S_PAIWW, S_PAIUW, S_EPUU, S_EPVV, S_EPWW, S_EPUW,
  S_USUW, S_VSVW, S_WSWW, S_WSUW, S_USWW, S_COUNT
};
static_assert(S_COUNT == kNS, "44 budget sums");

struct TkeArgs {
  const double *q[3];  // planar fields per level (0 coarse, 1 lower fine, 2 upper fine)
  const double *mean;  // [NZ][4] plane means of u, v, w, den/3
  double *part;        // [NZ][nymax][W] row partials
  int nx[3], ny[3], nz[3];
  int gr, zdf, zdc, NZ, nymax;
  double coef;         // 1 / GR
};

template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *out) {
  __shared__ double red[N][kT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; q++) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < N; q += blockDim.x) {
    double s = red[q][0];
#pragma unroll
    for (int w = 1; w < kT / 32; w++) s += red[q][w];
    out[q] = s;
  }
  __syncthreads();
}

// reference file layout vel[i][j][k][3], den[i][j][k] -> q[c][k][j][i]
__global__ void __launch_bounds__(kT) tke_planar_kernel(const double *__restrict__ vel,
                                                        const double *__restrict__ den, int nx, int ny, int nz,
                                                        double *__restrict__ q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= nx) return;
  const size_t node = ((size_t)i * ny + j) * nz + k, plane = (size_t)nz * ny * nx;
  const size_t o = ((size_t)k * ny + j) * nx + i;
  q[o] = vel[node * 3];
  q[plane + o] = vel[node * 3 + 1];
  q[2 * plane + o] = vel[node * 3 + 2];
  q[3 * plane + o] = (1. / 3.) * den[node];
}

// composite-profile plane of (level, k)
__device__ __forceinline__ int profile_of(const TkeArgs &A, int l, int k) {
  return l == 1 ? k : (l == 0 ? A.zdf - 2 + k : A.zdf + A.zdc - 4 + k);
}

// plane means of the four fields of the profile planes k0.. of level L, each
// summed in the reference's order (j outer, i inner: the plane's memory order)
// and divided by the plane's node count (budget2D.c:178-241): the means, and
// with them every fluctuation, are the reference's to the last bit.  The block
// stages the plane through shared memory in coalesced chunks; threads 0..3
// (u, v, w, den / 3) add each chunk in order.
constexpr int kMeanChunk = 1024;

template <int L>
__device__ __forceinline__ void mean_plane(const TkeArgs &A, int k, double (*buf)[kMeanChunk],
                                           double *__restrict__ mean) {
  const int nx = A.nx[L], ny = A.ny[L], nz = A.nz[L];
  const size_t n = (size_t)nx * ny, field = (size_t)nz * n;
  const double *q = A.q[L] + (size_t)k * n;
  double s = 0.;
  for (size_t base = 0; base < n; base += kMeanChunk) {
    const int len = (int)(n - base < (size_t)kMeanChunk ? n - base : (size_t)kMeanChunk);
#pragma unroll
    for (int c = 0; c < 4; c++)
      for (int t = threadIdx.x; t < len; t += blockDim.x) buf[c][t] = q[c * field + base + t];
    __syncthreads();
    if (threadIdx.x < 4) {
      // unrolled so the shared-memory loads run ahead of the (ordered) adds
#pragma unroll 16
      for (int t = 0; t < len; t++) s += buf[threadIdx.x][t];
    }
    __syncthreads();
  }
  if (threadIdx.x < 4) mean[(size_t)profile_of(A, L, k) * 4 + threadIdx.x] = s / (double)(nx * ny);
}

// one block per profile plane K
__global__ void __launch_bounds__(kT) tke_mean_seq(TkeArgs A, double *__restrict__ mean) {
  __shared__ double buf[4][kMeanChunk];
  const int K = blockIdx.x;
  if (K < A.zdf) mean_plane<1>(A, K, buf, mean);
  else if (K < A.zdf + A.zdc - 4) mean_plane<0>(A, K - A.zdf + 2, buf, mean);
  else mean_plane<2>(A, K - (A.zdf + A.zdc - 4), buf, mean);
}

// plane totals of W row partials in row order
__global__ void tke_sum_rows(const double *__restrict__ part, int nymax, int W, const int *__restrict__ rows,
                             double *__restrict__ out) {
  const int K = blockIdx.x;
  for (int q = threadIdx.x; q < W; q += blockDim.x) {
    double s = 0.;
    for (int j = 0; j < rows[K]; j++) s += part[((size_t)K * nymax + j) * W + q];
    out[(size_t)K * W + q] = s;
  }
}

// fluctuation of field c at (i, j, k) of level l (budget2D.c:243-291)
__device__ __forceinline__ double fl(const TkeArgs &A, int l, int c, int i, int j, int k) {
  const int nx = A.nx[l], ny = A.ny[l], nz = A.nz[l];
  return A.q[l][(((size_t)c * nz + k) * ny + j) * nx + i] - A.mean[profile_of(A, l, k) * 4 + c];
}

__device__ __forceinline__ int wrapn(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// d/dz of field c at (i, j, k) of level l by the reference's plane rules
// (lower budget2D.c:548-599, coarse :732-761, upper :924-975)
__device__ __forceinline__ double ddz(const TkeArgs &A, int l, int c, int i, int j, int k) {
  const int gr = A.gr, zdf = A.zdf, zdc = A.zdc;
  const double coef = A.coef;
  if (l == 1) {
    if (k == 1) {
      const double q0 = fl(A, 1, c, i, j, k), q1 = fl(A, 1, c, i, j, k + 1), q2 = fl(A, 1, c, i, j, k + 2);
      const double q3 = fl(A, 1, c, i, j, k + 3), q4 = fl(A, 1, c, i, j, k + 4);
      const double tmp = (2. / 3.) * (q3 - q1) - (1. / 12.) * (q4 - q0);
      return -(7. / 3.) * q0 + 6. * q1 - 3. * q2 - (2. / 3.) * q3 + 3. * tmp;
    }
    if (k == zdf - 1) {
      const double qc = fl(A, 0, c, i / gr, j / gr, 2);
      const double q0 = fl(A, 1, c, i, j, k), qm = fl(A, 1, c, i, j, k - 1);
      return (coef * (qc - q0) + gr * (q0 - qm)) * 1. / (1. + gr);
    }
    return 0.5 * (fl(A, 1, c, i, j, k + 1) - fl(A, 1, c, i, j, k - 1));
  }
  if (l == 0) {
    if (k == 2) return 0.5 * coef * (fl(A, 0, c, i, j, k + 1) - fl(A, 1, c, i * gr, j * gr, zdf - 1));
    if (k == 3 || k == zdc - 4) return 0.5 * coef * (fl(A, 0, c, i, j, k + 1) - fl(A, 0, c, i, j, k - 1));
    if (k == zdc - 3) return 0.5 * coef * (fl(A, 2, c, i * gr, j * gr, 0) - fl(A, 0, c, i, j, k - 1));
    return 0.5 * coef * (fl(A, 0, c, i, j, k + 1) - fl(A, 0, c, i, j, k - 1));
  }
  if (k == 0) {
    const double q0 = fl(A, 2, c, i, j, 0), q1 = fl(A, 2, c, i, j, 1);
    const double qc = fl(A, 0, c, i / gr, j / gr, zdc - 3);
    return (gr * (q1 - q0) + coef * (q0 - qc)) * 1. / (1. + gr);
  }
  if (k == zdf - 2) {
    const double q0 = fl(A, 2, c, i, j, k), q1 = fl(A, 2, c, i, j, k - 1), q2 = fl(A, 2, c, i, j, k - 2);
    const double q3 = fl(A, 2, c, i, j, k - 3), q4 = fl(A, 2, c, i, j, k - 4);
    const double tmp = (2. / 3.) * (q1 - q3) - (1. / 12.) * (q0 - q4);
    return (7. / 3.) * q0 - 6. * q1 + 3. * q2 + (2. / 3.) * q3 + 3. * tmp;
  }
  return 0.5 * (fl(A, 2, c, i, j, k + 1) - fl(A, 2, c, i, j, k - 1));
}

// the 44 per-node terms of budget2D.c:448-624 (and the identical coarse and
// upper bodies), summed over rows of the planes k0.. of level L (lower fine
// 1..zdf-1, coarse 2..zdc-3, upper fine 0..zdf-2); grid (ny, planes)
template <int L>
__global__ void __launch_bounds__(kT) tke_budget_rows(TkeArgs A, int k0) {
  constexpr int l = L;
  const int j = blockIdx.x, k = k0 + blockIdx.y, K = profile_of(A, L, k);
  double s[kNS];
#pragma unroll
  for (int q = 0; q < kNS; q++) s[q] = 0.;
  {
    const int nx = A.nx[l], ny = A.ny[l];
    const int jp = wrapn(j - 1, ny), jpp = wrapn(j - 2, ny), jn = wrapn(j + 1, ny), jnn = wrapn(j + 2, ny);
    const double cx = l == 0 ? A.coef : 1.;
    const double davg = A.mean[K * 4 + 3];
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      const int ip = wrapn(i - 1, nx), ipp = wrapn(i - 2, nx), in = wrapn(i + 1, nx), inn = wrapn(i + 2, nx);
      const double u = fl(A, l, 0, i, j, k), v = fl(A, l, 1, i, j, k), w = fl(A, l, 2, i, j, k);
      const double dfl = A.q[l][(((size_t)3 * A.nz[l] + k) * ny + j) * nx + i] - davg;
      double gx[3], gy[3], gz[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double dx = (2. / 3.) * (fl(A, l, c, in, j, k) - fl(A, l, c, ip, j, k)) -
                          (1. / 12.) * (fl(A, l, c, inn, j, k) - fl(A, l, c, ipp, j, k));
        const double dy = (2. / 3.) * (fl(A, l, c, i, jn, k) - fl(A, l, c, i, jp, k)) -
                          (1. / 12.) * (fl(A, l, c, i, jnn, k) - fl(A, l, c, i, jpp, k));
        gx[c] = l == 0 ? cx * dx : dx;
        gy[c] = l == 0 ? cx * dy : dy;
        gz[c] = ddz(A, l, c, i, j, k);
      }
      const double dudx = gx[0], dvdx = gx[1], dwdx = gx[2];
      const double dudy = gy[0], dvdy = gy[1], dwdy = gy[2];
      const double dudz = gz[0], dvdz = gz[1], dwdz = gz[2];
      s[S_UU] += u * u;
      s[S_UV] += u * v;
      s[S_UW] += u * w;
      s[S_VV] += v * v;
      s[S_VW] += v * w;
      s[S_WW] += w * w;
      s[S_SKU] += u * u * u;
      s[S_SKV] += v * v * v;
      s[S_SKW] += w * w * w;
      s[S_SKP] += dfl * dfl * dfl;
      s[S_SKUW] += u * u * u * w * w * w;
      s[S_SKUV] += u * u * u * v * v * v;
      s[S_SKVW] += v * v * v * w * w * w;
      s[S_KUU] += u * u * u * u;
      s[S_KUV] += v * v * v * v;
      s[S_KUW] += w * w * w * w;
      s[S_KUP] += dfl * dfl * dfl * dfl;
      s[S_KUUW] += u * u * u * u * w * w * w * w;
      s[S_KUVW] += v * v * v * v * w * w * w * w;
      s[S_KUUV] += u * u * u * u * v * v * v * v;
      s[S_DD] += dfl * dfl;
      s[S_UUW] += u * u * w;
      s[S_VVW] += v * v * w;
      s[S_WWW] += w * w * w;
      s[S_UWW] += u * w * w;
      s[S_PU] += u * dfl;
      s[S_PV] += v * dfl;
      s[S_PW] += w * dfl;
      const double ox = (dwdy - dvdz), oy = (dudz - dwdx), oz = (dvdx - dudy);
      s[S_WX] += ox * ox;
      s[S_WY] += oy * oy;
      s[S_WZ] += oz * oz;
      s[S_PAIUU] += dfl * dudx;
      s[S_PAIVV] += dfl * dvdy;
      s[S_PAIWW] += dfl * dwdz;
      s[S_PAIUW] += dfl * (dudz + dwdx);
      s[S_USUW] += 0.5 * u * (dudz + dwdx);
      s[S_VSVW] += 0.5 * v * (dvdz + dwdy);
      s[S_WSWW] += 0.5 * w * (dwdz + dwdz);
      s[S_WSUW] += 0.5 * w * (dudz + dwdx);
      s[S_USWW] += 0.5 * u * (dwdz + dwdz);
      s[S_EPUU] += dudx * (dudx + dudx) + dudy * (dudy + dvdx) + dudz * (dudz + dwdx);
      s[S_EPVV] += dvdx * (dvdx + dudy) + dvdy * (dvdy + dvdy) + dvdz * (dvdz + dwdy);
      s[S_EPWW] += dwdx * (dwdx + dudz) + dwdy * (dwdy + dvdz) + dwdz * (dwdz + dwdz);
      s[S_EPUW] += dudx * (dwdx + dudz) + dudy * (dwdy + dvdz) + dudz * (dwdz + dwdz) + dwdx * (dudx + dudx) +
                   dwdy * (dudy + dvdx) + dwdz * (dudz + dwdx);
    }
  }
  block_sum<kNS>(s, A.part + ((size_t)K * A.nymax + j) * kNS);
}

// ------------------------------------------------------------ finalisation
// budget2D.c:1004-1550 on the plane sums; profile rows in the order of the
// three output files (turb-fld-2d :1555-1579, vort-fluc-2d :1585-1587,
// KE-Budget-2d :1592-1639).
enum {
  P_UAVG, P_VAVG, P_WAVG, P_UTIN, P_VTIN, P_WTIN, P_UW, P_DAVG, P_DTIN, P_SKU, P_SKV, P_SKW, P_SKUW, P_SKP,
  P_KUU, P_KUV, P_KUW, P_KUUW, P_KUP,
  P_WX, P_WY, P_WZ,
  P_PII, P_PUU, P_PVV, P_PWW, P_PUW, P_TIIR, P_TUUR, P_TVVR, P_TWWR, P_TUWR, P_TIIPAI, P_TUUPAI, P_TVVPAI,
  P_TWWPAI, P_TUWPAI, P_PAIUU, P_PAIVV, P_PAIWW, P_PAIUW, P_TIIS, P_TUUS, P_TVVS, P_TWWS, P_TUWS, P_EPII,
  P_EPUU, P_EPVV, P_EPWW, P_EPUW, P_KE, P_COUNT
};
static_assert(P_COUNT == DNS_TKE_NPROF, "profile count");

// the reference's profile-derivative macros (TKE-budget/computations/definitions.h:56-94)
inline double ddz1f(const std::vector<double> &a, int k) { return (a[k + 1]) - (a[k]); }
inline double ddz1b(const std::vector<double> &a, int k) { return (a[k]) - (a[k - 1]); }
inline double ddz2c(const std::vector<double> &a, int k) { return ((a[k + 1]) - (a[k - 1])) * 0.5; }
inline double ddz2cnul(const std::vector<double> &a, int k, double r) {
  return (1. / (1. + r)) * ((1. / r) * ((a[k + 1]) - (a[k])) + r * ((a[k]) - (a[k - 1])));
}
inline double ddz2cnuu(const std::vector<double> &a, int k, double r) {
  return (1. / (1. + r)) * ((1. / r) * ((a[k]) - (a[k - 1])) + r * ((a[k + 1]) - (a[k])));
}

void finalize(const TkeArgs &A, double nu, const double *mean, const double *sums, double *prof) {
  const int NZ = A.NZ, zdf = A.zdf, zdc = A.zdc, GR = A.gr;
  const double coef = A.coef;
  auto col = [&](int q) {
    std::vector<double> v(NZ);
    for (int K = 0; K < NZ; K++) v[K] = sums[(size_t)K * kNS + q];
    return v;
  };
  std::vector<double> U(NZ), V(NZ), W(NZ), D(NZ);
  for (int K = 0; K < NZ; K++) {
    U[K] = mean[K * 4];
    V[K] = mean[K * 4 + 1];
    W[K] = mean[K * 4 + 2];
    D[K] = mean[K * 4 + 3];
  }
  std::vector<double> uu = col(S_UU), uv = col(S_UV), uw = col(S_UW), vv = col(S_VV), vw = col(S_VW),
                      ww = col(S_WW), dd = col(S_DD), SKu = col(S_SKU), SKv = col(S_SKV), SKw = col(S_SKW),
                      SKp = col(S_SKP), SKuw = col(S_SKUW), SKuv = col(S_SKUV), SKvw = col(S_SKVW),
                      KUu = col(S_KUU), KUv = col(S_KUV), KUw = col(S_KUW), KUp = col(S_KUP), KUuw = col(S_KUUW),
                      KUvw = col(S_KUVW), KUuv = col(S_KUUV), wx = col(S_WX), wy = col(S_WY), wz = col(S_WZ),
                      uuw = col(S_UUW), vvw = col(S_VVW), www = col(S_WWW), uww = col(S_UWW), pu = col(S_PU),
                      pv = col(S_PV), pw = col(S_PW), Paiuu = col(S_PAIUU), Paivv = col(S_PAIVV),
                      Paiww = col(S_PAIWW), Paiuw = col(S_PAIUW), Epuu = col(S_EPUU), Epvv = col(S_EPVV),
                      Epww = col(S_EPWW), Epuw = col(S_EPUW), usuw = col(S_USUW), vsvw = col(S_VSVW),
                      wsww = col(S_WSWW), wsuw = col(S_WSUW), usww = col(S_USWW);
  std::vector<double *> all = {uu.data(),   uv.data(),    uw.data(),    vv.data(),    vw.data(),   ww.data(),
                               dd.data(),   SKu.data(),   SKv.data(),   SKw.data(),   SKp.data(),  SKuw.data(),
                               SKuv.data(), SKvw.data(),  KUu.data(),   KUv.data(),   KUw.data(),  KUp.data(),
                               KUuw.data(), KUuv.data(),  KUvw.data(),  wx.data(),    wy.data(),   wz.data(),
                               uuw.data(),  vvw.data(),   www.data(),   uww.data(),   pu.data(),   pv.data(),
                               pw.data(),   Paiuu.data(), Paivv.data(), Paiww.data(), Paiuw.data(), Epuu.data(),
                               Epvv.data(), Epww.data(),  Epuw.data(),  usuw.data(),  vsvw.data(), wsww.data(),
                               wsuw.data(), usww.data()};
  // :1004-1064 plane averages
  for (int K = 0; K < NZ; K++) {
    long num;
    if (K < zdf) num = (long)A.nx[1] * A.ny[1];
    else if (K < zdf + zdc - 4) num = (long)A.nx[0] * A.ny[0];
    else num = (long)A.nx[2] * A.ny[2];
    for (double *a : all) a[K] /= (double)(num);
  }
  // mean shear (:295-444)
  std::vector<double> dUdz(NZ, 0.);
  for (int k = 1; k < zdf; k++) {
    if (k == 1) {
      const double tmp = (2. / 3.) * (U[k + 3] - U[k + 1]) - (1. / 12.) * (U[k + 4] - U[k]);
      dUdz[k] = -(7. / 3.) * U[k] + 6. * U[k + 1] - 3. * U[k + 2] - (2. / 3.) * U[k + 3] + 3. * tmp;
    } else if (k == zdf - 1) {
      dUdz[k] = (coef * (U[k + 1] - U[k]) + GR * (U[k] - U[k - 1])) * 1. / (1. + GR);
    } else if (k == 2 || k == zdf - 2) {
      dUdz[k] = 0.5 * (U[k + 1] - U[k - 1]);
    } else {
      dUdz[k] = (2. / 3.) * (U[k + 1] - U[k - 1]) - (1. / 12.) * (U[k + 2] - U[k - 2]);
    }
  }
  for (int k = 2; k < zdc - 2; k++) {
    const int K = zdf - 2 + k;
    if (k == 2 || k == 3 || k == zdc - 4 || k == zdc - 3)
      dUdz[K] = 0.5 * coef * (U[K + 1] - U[K - 1]);
    else
      dUdz[K] = coef * ((2. / 3.) * (U[K + 1] - U[K - 1]) - (1. / 12.) * (U[K + 2] - U[K - 2]));
  }
  for (int k = 0; k < zdf - 1; k++) {
    const int K = zdf + zdc - 4 + k;
    if (k == 0) {
      dUdz[K] = (GR * (U[K + 1] - U[K]) + coef * (U[K] - U[K - 1])) * 1. / (1. + GR);
    } else if (k == zdf - 2) {
      const double tmp = (2. / 3.) * (U[K - 1] - U[K - 3]) - (1. / 12.) * (U[K] - U[K - 4]);
      dUdz[K] = (7. / 3.) * U[K] - 6. * U[K - 1] + 3. * U[K - 2] + (2. / 3.) * U[K - 3] + 3. * tmp;
    } else if (k == 1 || k == zdf - 3) {
      dUdz[K] = 0.5 * (U[K + 1] - U[K - 1]);
    } else {
      dUdz[K] = (2. / 3.) * (U[K + 1] - U[K - 1]) - (1. / 12.) * (U[K + 2] - U[K - 2]);
    }
  }
  std::vector<double> UTIN(NZ, 0.), VTIN(NZ, 0.), WTIN(NZ, 0.), DTIN(NZ, 0.), KE(NZ, 0.), Epii(NZ, 0.);
  // :1249-1284
  for (int k = 1; k < NZ - 1; k++) {
    const double siu = UTIN[k] = std::sqrt(uu[k]);
    const double siv = VTIN[k] = std::sqrt(vv[k]);
    const double siw = WTIN[k] = std::sqrt(ww[k]);
    const double sip = DTIN[k] = std::sqrt(dd[k]);
    KE[k] += (uu[k] + vv[k] + ww[k]);
    wx[k] = std::sqrt(wx[k]);
    wy[k] = std::sqrt(wy[k]);
    wz[k] = std::sqrt(wz[k]);
    SKu[k] /= (siu * siu * siu);
    SKv[k] /= (siv * siv * siv);
    SKw[k] /= (siw * siw * siw);
    SKp[k] /= (sip * sip * sip);
    SKuw[k] /= (siu * siu * siu * siw * siw * siw);
    SKvw[k] /= (siv * siv * siv * siw * siw * siw);
    SKuv[k] /= (siu * siu * siu * siv * siv * siv);
    KUu[k] /= (siu * siu * siu * siu);
    KUv[k] /= (siv * siv * siv * siv);
    KUw[k] /= (siw * siw * siw * siw);
    KUp[k] /= (sip * sip * sip * sip);
    KUuw[k] /= (siu * siu * siu * siu * siw * siw * siw * siw);
    KUuv[k] /= (siu * siu * siu * siu * siv * siv * siv * siv);
    KUvw[k] /= (siv * siv * siv * siv * siw * siw * siw * siw);
    Epuu[k] *= nu;
    Epvv[k] *= nu;
    Epww[k] *= nu;
    Epuw[k] *= (2. * nu);
    Epii[k] = (Epuu[k]) + (Epvv[k]) + (Epww[k]);
  }
  std::vector<double> Pii(NZ, 0.), Puu(NZ, 0.), Pvv(NZ, 0.), Pww(NZ, 0.), Puw(NZ, 0.), Tiir(NZ, 0.), Tuur(NZ, 0.),
      Tvvr(NZ, 0.), Twwr(NZ, 0.), Tuwr(NZ, 0.), Tiipai(NZ, 0.), Tuupai(NZ, 0.), Tvvpai(NZ, 0.), Twwpai(NZ, 0.),
      Tuwpai(NZ, 0.), Tiis(NZ, 0.), Tuus(NZ, 0.), Tvvs(NZ, 0.), Twws(NZ, 0.), Tuws(NZ, 0.);
  auto production = [&](int K) {
    Pii[K] = -(uw[K]) * (dUdz[K]);
    Puu[K] = 2. * (Pii[K]);
    Pvv[K] = 0.;
    Pww[K] = 0.;
    Puw[K] = -(ww[K]) * (dUdz[K]);
    Tuupai[K] = 0.;
    Tvvpai[K] = 0.;
  };
  // one transport rule: D is the profile derivative, h the factor of the
  // diagonal turbulent-transport terms
  auto fine_rule = [&](int K, auto Dz, double h) {
    Tuur[K] = h * Dz(uuw, K);
    Tvvr[K] = h * Dz(vvw, K);
    Twwr[K] = h * Dz(www, K);
    Tuwr[K] = -Dz(uww, K);
    Tiipai[K] = -Dz(pw, K);
    Twwpai[K] = -2. * Dz(pw, K);
    Tuwpai[K] = -Dz(pu, K);
    Tuus[K] = 2. * nu * Dz(usuw, K);
    Tvvs[K] = 2. * nu * Dz(vsvw, K);
    Twws[K] = 2. * nu * Dz(wsww, K);
    Tuws[K] = 2. * nu * Dz(wsuw, K) + 2. * nu * Dz(wsww, K);
  };
  auto d1f = [](const std::vector<double> &a, int K) { return ddz1f(a, K); };
  auto d1b = [](const std::vector<double> &a, int K) { return ddz1b(a, K); };
  auto d2c = [](const std::vector<double> &a, int K) { return ddz2c(a, K); };
  auto nul = [GR](const std::vector<double> &a, int K) { return ddz2cnul(a, K, GR); };
  auto nuu = [GR](const std::vector<double> &a, int K) { return ddz2cnuu(a, K, GR); };
  // lower fine (:1286-1381)
  for (int k = 1; k < zdf; k++) {
    production(k);
    if (k == 1) fine_rule(k, d1f, -1.);
    else if (k == zdf - 1) fine_rule(k, nul, -1.);
    else if (k == 2 || k == zdf - 2) fine_rule(k, d2c, -1.);
    else fine_rule(k, d2c, -0.5);
    Tiis[k] = 0.5 * (Tuus[k] + Tvvs[k] + Twws[k]);
    Tiir[k] = 0.5 * (Tuur[k] + Tvvr[k] + Twwr[k]);
  }
  // coarse (:1383-1465): the rules at k = 2, 3, zdc-4, zdc-3 coincide
  for (int k = 2; k < zdc - 2; k++) {
    const int K = zdf - 2 + k;
    production(K);
    if (k == 2 || k == 3 || k == zdc - 4 || k == zdc - 3) {
      Tuur[K] = -coef * ddz2c(uuw, K);
      Tvvr[K] = -coef * ddz2c(vvw, K);
      Twwr[K] = -coef * ddz2c(www, K);
      Tuwr[K] = -coef * ddz2c(uww, K);
      Tiipai[K] = -coef * ddz2c(pw, K);
      Twwpai[K] = -2. * coef * ddz2c(pw, K);
      Tuwpai[K] = -coef * ddz2c(pu, K);
      Tuus[K] = 2. * nu * coef * ddz2c(usuw, K);
      Tvvs[K] = 2. * nu * coef * ddz2c(vsvw, K);
      Twws[K] = 2. * nu * coef * ddz2c(wsww, K);
      Tuws[K] = 2. * nu * coef * ddz2c(wsuw, K) + 2. * nu * coef * ddz2c(wsww, K);
    } else {
      Tuur[K] = -coef * 0.5 * ddz2c(uuw, K);
      Tvvr[K] = -coef * 0.5 * ddz2c(vvw, K);
      Twwr[K] = -coef * 0.5 * ddz2c(www, K);
      Tuwr[K] = -coef * ddz2c(uww, K);
      Tiipai[K] = -coef * ddz2c(pw, K);
      Twwpai[K] = -2. * coef * ddz2c(pw, K);
      Tuwpai[K] = -coef * ddz2c(pu, K);
      Tuus[K] = coef * 2. * nu * ddz2c(usuw, K);
      Tvvs[K] = coef * 2. * nu * ddz2c(vsvw, K);
      Twws[K] = coef * 2. * nu * ddz2c(wsww, K);
      Tuws[K] = coef * 2. * nu * ddz2c(wsuw, K) + coef * 2. * nu * ddz2c(wsww, K);
    }
    Tiis[K] = 0.5 * (Tuus[K] + Tvvs[K] + Twws[K]);
    Tiir[K] = 0.5 * (Tuur[K] + Tvvr[K] + Twwr[K]);
  }
  // upper fine (:1467-1548)
  for (int k = 0; k < zdf - 1; k++) {
    const int K = zdf + zdc - 4 + k;
    production(K);
    if (k == 0) fine_rule(K, nuu, -1.);
    else if (k == zdf - 2) fine_rule(K, d1b, -1.);
    else if (k == 2 || k == zdf - 3) fine_rule(K, d2c, -1.);
    else fine_rule(K, d2c, -0.5);
    Tiis[K] = 0.5 * (Tuus[K] + Tvvs[K] + Twws[K]);
    Tiir[K] = 0.5 * (Tuur[K] + Tvvr[K] + Twwr[K]);
  }
  const std::vector<double> *rows[P_COUNT] = {
      &U,    &V,      &W,      &UTIN,   &VTIN,   &WTIN,   &uw,     &D,     &DTIN,  &SKu,  &SKv,  &SKw,  &SKuw,
      &SKp,  &KUu,    &KUv,    &KUw,    &KUuw,   &KUp,    &wx,     &wy,    &wz,    &Pii,  &Puu,  &Pvv,  &Pww,
      &Puw,  &Tiir,   &Tuur,   &Tvvr,   &Twwr,   &Tuwr,   &Tiipai, &Tuupai, &Tvvpai, &Twwpai, &Tuwpai, &Paiuu,
      &Paivv, &Paiww, &Paiuw,  &Tiis,   &Tuus,   &Tvvs,   &Twws,   &Tuws,  &Epii,  &Epuu, &Epvv, &Epww, &Epuw,
      &KE};
  for (int r = 0; r < P_COUNT; r++) std::memcpy(prof + (size_t)r * NZ, rows[r]->data(), (size_t)NZ * 8);
}

}  // namespace

int tke_validate(const dns_params &p) {
  if (p.zds < 5) return fail_with(DNS_EINVAL, "the budget needs zds >= 5 (its wall stencils reach 4 planes)");
  if (p.zdv < 7) return fail_with(DNS_EINVAL, "the budget needs zdv >= 7 (coarse planes 2..zdc-3 with 4-point rules)");
  if (p.ydv < 4 || p.xdv < 4) return fail_with(DNS_EINVAL, "the budget needs xdv, ydv >= 4 (5-point stencils)");
  return DNS_OK;
}

size_t tke_workspace_bytes(const dns_geometry &g) {
  const size_t NZ = g.nz_profile;
  return (NZ * g.nyf * kNS + NZ * 4 + NZ * kNS) * 8 + NZ * sizeof(int);
}

int tke_budget_planar(const dns_params &p, const dns_geometry &g, const double *const q[3], double *prof,
                      double *ufl, double *vfl, cudaStream_t st, void *work) {
  int rc = tke_validate(p);
  if (rc) return rc;
  TkeArgs A{};
  A.nx[0] = g.nx;
  A.ny[0] = g.ny;
  A.nz[0] = g.nzc;
  for (int l = 1; l < 3; l++) {
    A.nx[l] = g.nxf;
    A.ny[l] = g.nyf;
    A.nz[l] = g.zdf;
  }
  for (int l = 0; l < 3; l++) A.q[l] = q[l];
  A.gr = g.gr;
  A.zdf = g.zdf;
  A.zdc = g.nzc;
  A.NZ = g.nz_profile;
  A.nymax = g.nyf;
  A.coef = (1. / ((double)g.gr));
  const int NZ = A.NZ;
  // budget2D.c:57-60, tauf the fine relaxation time
  const double tauf = (3. / p.Rebs) * p.ub * (g.nzs - 2.) + 0.5;
  const double nu = (1. / 6.) * (2. * tauf - 1.);
  const size_t npart = (size_t)NZ * A.nymax * kNS;
  const size_t nbuf = npart + (size_t)NZ * 4 + (size_t)NZ * kNS;
  void *owned = nullptr;
  if (!work) {
    if (cudaMalloc(&owned, tke_workspace_bytes(g)) != cudaSuccess) return fail_with(DNS_ENOMEM, "budget work space");
    work = owned;
  }
  double *buf = static_cast<double *>(work);
  int *dims = reinterpret_cast<int *>(buf + nbuf);
  double *part = buf, *mean = part + npart, *sums = mean + (size_t)NZ * 4;
  std::vector<int> hdims(NZ);
  for (int K = 0; K < NZ; K++) hdims[K] = (K >= g.zdf && K < g.zdf + g.nzc - 4) ? g.ny : g.nyf;
  A.part = part;
  A.mean = mean;
  const int nyc = g.ny, nyf = g.nyf;
  cudaError_t e = cudaMemcpyAsync(dims, hdims.data(), NZ * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    tke_mean_seq<<<NZ, kT, 0, st>>>(A, mean);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(part, 0, npart * 8, st);  // profile planes 0, NZ-1: no products
  if (e == cudaSuccess) {
    tke_budget_rows<1><<<dim3(nyf, g.zdf - 1), kT, 0, st>>>(A, 1);
    tke_budget_rows<0><<<dim3(nyc, g.nzc - 4), kT, 0, st>>>(A, 2);
    tke_budget_rows<2><<<dim3(nyf, g.zdf - 1), kT, 0, st>>>(A, 0);
    tke_sum_rows<<<NZ, 64, 0, st>>>(part, A.nymax, kNS, dims, sums);
    e = cudaGetLastError();
  }
  std::vector<double> hmean((size_t)NZ * 4), hsums((size_t)NZ * kNS);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hmean.data(), mean, hmean.size() * 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hsums.data(), sums, hsums.size() * 8, cudaMemcpyDeviceToHost, st);
  // uv_fluc.c:24-33: fluctuations of the lower fine plane k = 4
  const size_t pl = (size_t)g.nyf * g.nxf;
  std::vector<double> plane;
  if (e == cudaSuccess && (ufl || vfl)) {
    plane.resize(2 * pl);
    e = cudaMemcpyAsync(plane.data(), q[1] + 4 * pl, pl * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(plane.data() + pl, q[1] + (size_t)g.zdf * pl + 4 * pl, pl * 8, cudaMemcpyDeviceToHost,
                          st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (owned) cudaFree(owned);
  if (e != cudaSuccess) return fail_with(DNS_ECUDA, cudaGetErrorString(e));
  finalize(A, nu, hmean.data(), hsums.data(), prof);
  if (ufl || vfl) {
    for (int i = 0; i < g.nxf; i++)
      for (int j = 0; j < g.nyf; j++) {
        if (ufl) ufl[(size_t)i * g.nyf + j] = plane[(size_t)j * g.nxf + i] - hmean[4 * 4 + 0];
        if (vfl) vfl[(size_t)i * g.nyf + j] = plane[pl + (size_t)j * g.nxf + i] - hmean[4 * 4 + 1];
      }
  }
  return DNS_OK;
}

int tke_budget_device(const dns_params &p, const dns_geometry &g, const double *const vel[3],
                      const double *const den[3], double *prof, double *ufl, double *vfl, cudaStream_t st) {
  int rc = tke_validate(p);
  if (rc) return rc;
  const int nx[3] = {g.nx, g.nxf, g.nxf}, ny[3] = {g.ny, g.nyf, g.nyf}, nz[3] = {g.nzc, g.zdf, g.zdf};
  size_t nq = 0;
  for (int l = 0; l < 3; l++) nq += 4ull * nx[l] * ny[l] * nz[l];
  double *buf = nullptr;
  if (cudaMalloc(&buf, nq * 8) != cudaSuccess) return fail_with(DNS_ENOMEM, "budget planar fields");
  const double *q[3];
  double *ql = buf;
  cudaError_t e = cudaSuccess;
  for (int l = 0; l < 3 && e == cudaSuccess; l++) {
    q[l] = ql;
    dim3 grid((nx[l] + kT - 1) / kT, ny[l], nz[l]);
    tke_planar_kernel<<<grid, kT, 0, st>>>(vel[l], den[l], nx[l], ny[l], nz[l], ql);
    ql += 4ull * nx[l] * ny[l] * nz[l];
    e = cudaGetLastError();
  }
  rc = e == cudaSuccess ? tke_budget_planar(p, g, q, prof, ufl, vfl, st) : fail_with(DNS_ECUDA, cudaGetErrorString(e));
  cudaStreamSynchronize(st);
  cudaFree(buf);
  return rc;
}

}  // namespace dns
