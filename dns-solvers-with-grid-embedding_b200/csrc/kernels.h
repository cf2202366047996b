// Host-side launchers of the device kernels (internal to libdnsembed).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/dns_embed.h"

namespace dns {

// Running statistics of one composite-profile plane, kStatRow doubles.  Each
// sample's plane moments are exact two-pass quantities: every block keeps a
// running (count, means, sums of squared deviations) per thread (Welford) and
// merges them pairwise (Chan, Golub and LeVeque's parallel update), so a
// plane's variance is never formed as E[x^2] - E[x]^2.  The row holds:
//   0..3   sums over samples of (m - c) for the plane means m of u, v, w, rho;
//   4..8   sums over samples of (mu - cu)^2, (mv - cv)^2, (mw - cw)^2,
//          (mu - cu)(mw - cw), (mr - cr)^2 (the plane means' time variation);
//   9..13  sums over samples of the per-sample plane variances of u, v, w, the
//          covariance uw and the variance of rho;
//   14     nodes per plane; 15 samples;
//   16..19 c = (cu, cv, cw, cr): the plane means of the first sample after a
//          reset, about which the plane means are summed.
// Per-block partials of one sample: kStatPart doubles, (n, 4 means, 5 sums of
// squared deviations).
constexpr int kStatPart = 10;
constexpr int kStatRow = 20;

// Device-side scalar state carried between steps (one instance per handle).
struct DevState {
  double force;     // force[0] of the next step
  double momentum;  // encalc2 momentum of the current state
  double denst;     // encalc2 mass of the current state
  double pad;
};

// One row of the per-step log, filled on the device (time is added on the host).
struct DevLog {
  double force, momentum, denst, flowrate, stup, stdown, stress, pgrad;
};

struct Dims {
  int nx, ny, nzc;        // coarse
  int nxf, nyf, zdf, zds; // fine block; zds planes stored per block
  int gr, nzs;
};

// Launch geometry shared by the kernels and the reductions.
struct LaunchShape {
  int bx;          // threads per block along x
  int jb;          // rows (y) per block
  int cgx, cgy;    // coarse grid x/y blocks (z = nzc planes)
  int fgx, fgy;    // fine grid x/y blocks (z = 2 zds planes)
  int igx, igy;    // interface tile grid
  int jgx, jgy;    // injection / extraction grid (x, y) per wall
  long n_coarse_blocks() const { return (long)cgx * cgy; }  // per plane
  long n_fine_blocks() const { return (long)fgx * fgy; }    // per plane
};

LaunchShape make_shape(const Dims &d);

// record a message for dns_last_error() on the calling thread (dns_api.cu)
void set_last_error(const std::string &msg);

// Reduction scratch sizes (doubles) for a given shape.
struct PartialLayout {
  long coarse, fine, inject, wall, stats_c, stats_f, flow, level2;  // offsets into one buffer
  long total;
};
PartialLayout partial_layout(const Dims &d, const LaunchShape &s);

struct StepParams {
  double omega_c, omega_f;
  double ub;        // bulk velocity (constant flow rate target)
  double gconst;    // constant body force
  int cfr;          // 1: force = ub - momentum
  double den_offset;  // encalc2 weight sum added to the mass partials (FP32 form: they sum deviations)
};

// --- FP64 kernels (kernels_f64.cu) ---
// stats: also the per-block moments of the sampled statistics (kStatPart doubles per block)
void launch_coarse_f64(const double *src, double *dst, const Dims &d, const LaunchShape &s, double om,
                       const DevState *st, double *partials, const PartialLayout &pl, bool stats,
                       cudaStream_t stream);
void launch_extract_f64(const double *fc, double *hist_n, const Dims &d, const LaunchShape &s,
                        cudaStream_t stream);
void launch_fine_f64(const double *src, double *dst, const int8_t *wflag, const Dims &d, const LaunchShape &s,
                     double om, const DevState *st, double *partials, const PartialLayout &pl, bool first,
                     bool last, bool stats, cudaStream_t stream);
// two launches: macroscopic fields into mac[2 walls][4][nyf][nxf], then one
// block per (tile, wall, population) into the interface planes of fdst
void launch_interface_f64(const double *hn, const double *hp, const double *hpp, double *mac, double *fdst,
                          const Dims &d, const LaunchShape &s, int substep, double omega_c, double omega_f,
                          cudaStream_t stream);
// filtered: the FLTR transfer (ftcdtransfer_lesfltr.c) instead of ftcdtransfer.c
void launch_inject_f64(const double *fsrc, double *cdst, const Dims &d, const LaunchShape &s, double omega_c,
                       double omega_f, double *partials, const PartialLayout &pl, bool filtered,
                       cudaStream_t stream);
// counter: one device unsigned int, zero between launches (the kernel resets it)
void launch_finalize(DevState *st, DevLog *log_row, double *partials, unsigned int *counter,
                     const PartialLayout &pl, const Dims &d, const LaunchShape &s, const StepParams &sp,
                     cudaStream_t stream);
void launch_stats_finalize(double *acc, const double *partials, const PartialLayout &pl, const Dims &d,
                           const LaunchShape &s, cudaStream_t stream);
// direct encalc2 reduction of the stored state into st (momentum, denst, force)
void launch_flow_sums_f64(const double *fc, const double *ff, DevState *st, double *partials,
                          const PartialLayout &pl, const Dims &d, const LaunchShape &s, const StepParams &sp,
                          cudaStream_t stream);
// the same reduction over a caller-held state, with caller-provided block scratch
// (scratch_pairs = flow_sums_pairs(d, s) pairs of doubles), result into *out
long flow_sums_pairs(const Dims &d, const LaunchShape &s);
void launch_flow_sums_scratch(const double *fc, const double *ff, DevState *out, double *scratch, const Dims &d,
                              const LaunchShape &s, const StepParams &sp, cudaStream_t stream);
// finalize a direct (flow_sums) reduction of npairs block partials into *st
void finalize_flow_sums(DevState *st, const double *pairs, long npairs, const Dims &d, const LaunchShape &s,
                        const StepParams &sp, cudaStream_t stream);
// encalc2 weight of every node summed (the mass of a state with rho = 1)
double encalc2_weight_sum(const Dims &d);
void launch_seed_f64(double *fc, double *ff, double *hist3, const Dims &d, uint64_t seed, double uc, double amp,
                     cudaStream_t stream);
// vel_print field records of np device planes p0.. into vel[i][j][k][3] and
// den[i][j][k] (nz_aos planes, device plane p0 + q at k = k0_aos + q)
void launch_fields_f64(const double *soa, double *vel, double *den, int nx, int ny, int P, int p0, int np, int nz_aos,
                       int k0_aos, cudaStream_t stream);
void launch_fields_f32(const float *soa, double *vel, double *den, int nx, int ny, int P, int p0, int np, int nz_aos,
                       int k0_aos, cudaStream_t stream);
// the same moments as planar fields q[c][k][j][i] (c = u, v, w, den / 3) of a
// level with nz planes, device plane p0 + s at k = k0 + s
void launch_fields_planar_f64(const double *soa, double *q, int nx, int ny, int P, int p0, int np, int nz,
                              int k0, cudaStream_t stream);
void launch_fields_planar_f32(const float *soa, double *q, int nx, int ny, int P, int p0, int np, int nz, int k0,
                              cudaStream_t stream);
// Mode -i start: one level of the embedded grid interpolated from a uniform-grid
// state.  uni is the uniform state in reference AoS order [xu][yu][zd][19]; out
// receives the level in reference AoS order [nxl][nyl][nzl][19] (wall plane of a
// fine block = the rest equilibrium w_a).  *bad is set when a stencil index
// leaves the reference's two-deep halo in x or y, or the grid in z (those
// nodes are not read).  level: 0 coarse, 1 lower fine, 2 upper fine.
struct UniformMap {
  int level, nxl, nyl, nzl;  // output level extents (nzl = zdc or zdf)
  int xu, yu, zd;            // uniform grid: xdu, ydu, zdu + 2
  int gr, zdf, zdc;
  double dxf, dxc, dxr;      // node spacings as the reference's initializer forms them
  double fac;                // (dxr / dx_level) (omega / omega_level), the f^neq rescaling
};
void launch_uniform_interp_f64(const double *uni, const UniformMap &m, double *out, int *bad, cudaStream_t stream);
// Turbulence statistics / kinetic-energy budget of one snapshot (tke.cu) from
// the device field arrays of the three levels in the reference file layout
// (0 coarse vel[i][j][k][3] / den[i][j][k], 1 lower fine, 2 upper fine);
// prof on the host, [DNS_TKE_NPROF][nz_profile]; ufl / vfl optional.
int tke_validate(const dns_params &p);
int tke_budget_device(const dns_params &p, const dns_geometry &g, const double *const vel[3],
                      const double *const den[3], double *prof, double *ufl, double *vfl, cudaStream_t st);
// the same from planar fields q[l] = [4][nz][ny][nx] (u, v, w, den / 3) per level
// work: device space of tke_workspace_bytes(g) (8-byte aligned), or null to
// allocate per call
size_t tke_workspace_bytes(const dns_geometry &g);
int tke_budget_planar(const dns_params &p, const dns_geometry &g, const double *const q[3], double *prof,
                      double *ufl, double *vfl, cudaStream_t st, void *work = nullptr);
// wall plane kw of a level in reference AoS order [nodes = nx ny][nz][19] to
// (to_aos) or from the compact wall array [nodes][19]
void launch_wall_plane(double *aos, double *wall, long long nodes, int nz, int kw, bool to_aos, cudaStream_t stream);
// layout transposes between the device SoA state and the reference AoS order
// [i0, i1): the x indices to move (i1 < 0: all); the AoS side is i-major, so
// an x range is one contiguous run of it
void launch_soa_to_aos(const double *soa, double *aos, int nx, int ny, int P, int p0, int np, int nz_aos,
                       int k0_aos, cudaStream_t stream, int i0 = 0, int i1 = -1);
void launch_aos_to_soa(const double *aos, double *soa, int nx, int ny, int P, int p0, int np, int nz_aos,
                       int k0_aos, cudaStream_t stream, int i0 = 0, int i1 = -1);

// --- FP32 deviation-storage kernels (kernels_f32.cu); same layouts in float ---
void launch_coarse_f32(const float *src, float *dst, const Dims &d, const LaunchShape &s, double om,
                       const DevState *st, double *partials, const PartialLayout &pl, bool stats,
                       cudaStream_t stream);
void launch_extract_f32(const float *fc, float *hist_n, const Dims &d, const LaunchShape &s, cudaStream_t stream);
void launch_fine_f32(const float *src, float *dst, const int8_t *wflag, const Dims &d, const LaunchShape &s,
                     double om, const DevState *st, double *partials, const PartialLayout &pl, bool first, bool last,
                     bool stats, cudaStream_t stream);
// corner: scratch of 2 x 23 x ny x nx float4 (corner values and derivatives)
void launch_interface_f32(const float *hn, const float *hp, const float *hpp, float *corner, float *fdst,
                          const Dims &d, int substep, double omega_c, double omega_f, cudaStream_t stream);
void launch_inject_f32(const float *fsrc, float *cdst, const Dims &d, const LaunchShape &s, double omega_c,
                       double omega_f, double *partials, const PartialLayout &pl, bool filtered,
                       cudaStream_t stream);
void launch_flow_sums_f32(const float *fc, const float *ff, DevState *st, double *partials, const PartialLayout &pl,
                          const Dims &d, const LaunchShape &s, const StepParams &sp, cudaStream_t stream);
void launch_seed_f32(float *fc, float *ff, float *hist3, const Dims &d, uint64_t seed, double uc, double amp,
                     cudaStream_t stream);
// device float deviations <-> reference AoS doubles (f = w + d)
void launch_dev_to_aos_f32(const float *soa, double *aos, int nx, int ny, int P, int p0, int np, int nz_aos,
                           int k0_aos, cudaStream_t stream, int i0 = 0, int i1 = -1);
void launch_aos_to_dev_f32(const double *aos, float *soa, int nx, int ny, int P, int p0, int np, int nz_aos,
                           int k0_aos, cudaStream_t stream, int i0 = 0, int i1 = -1);

}  // namespace dns
