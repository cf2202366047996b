// Batched FP32 engine: many independent channels stepped by one set of
// persistent kernels over a per-instance block table (internal to
// libdnsembed; the C ABI is dns_batch_* in include/dns_embed.h).
//
// Every phase of the coarse step (statistics, coarse collide-stream, interface
// history and corner data, fine substeps, interface evaluation, injection,
// finalize) is one
// persistent kernel: a grid sized to the machine walks the phase's work items
// of all resident instances.  Instance s owns items [start[ph][s],
// start[ph][s+1]); an item is one tile of one instance, decoded against that
// instance's own sizes and tile shape.  Everything a step needs that changes
// from step to step (ping-pong parity, history ring, step count, remaining
// budget) lives in device memory and is advanced by the finalize kernel, so a
// captured CUDA graph of a step group replays unchanged while instances join
// and leave (only the tables it reads are rewritten between groups).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "kernels.h"

namespace dns {
namespace batch {

constexpr int kMaxInst = 1024;  // resident instances per batch
constexpr int kLogRows = 64;    // per-instance log ring (>= steps per graph replay)
constexpr int kFinChunks = 32;  // blocks per instance in the finalize

enum Phase {
  PH_STATS = 0,  // plane statistics of the sampled state (coarse 2..zdc-3, every fine plane)
  PH_SFINAL,     // per-plane accumulation of those sums
  PH_COARSE,     // every coarse plane
  PH_FINE,       // every fine plane of both blocks (wall-adjacent, interface-adjacent, then bulk)
  PH_ICORNER,    // interface history level n and every substep's corner data: tiles x walls x field groups
  PH_IEVAL,      // interface evaluation: fine rows x walls
  PH_INJECT,     // fine-to-coarse injection rows
  PH_FINAL,      // reduction chunks of the finalize
  PH_NPHASE
};

// Constant while the instance is resident.
struct Inst {
  int nx, ny, nzc, nxf, nyf, zdf, zds, gr;
  // tiles of the stream-collide kernels: width (threads along x, each updating
  // four consecutive nodes), row iterations, and items per plane in x and y
  int cw, cjb, cgx, cgy;  // coarse
  int fw, fjb, fgx, fgy;  // fine
  int igx, igy;           // interface corner tiles
  int egx;                // injection blocks per row
  int nzp;                // composite profile planes
  int slot;               // row of the batch-level dyn / state / log arrays
  long long sample_every; // statistics every n steps of the instance (0: none)
  float om_c, om_f, fac_if, fac_inj;
  // finalize constants (encalc2.c, wshearstr.c)
  double g3, norm, norm2, mu, ub, gconst, pgrad_scale, flow_scale, den_offset;
  int cfr, fltr;          // constant flow rate; filtered fine-to-coarse transfer (FLTR)
  float *fc[2], *ff[2];   // coarse / fine SoA deviations, ping-pong
  float *hist;            // 3 ring slots x [2 walls][23][ny][nx]
  float4 *corner;         // interface corner data of each substep [GR][2 walls][23][ny][nx]
  int8_t *wflag;          // [nyf][nxf]
  double *part;           // block partials
  long long pc, pf, pi, pw, psc, psf, pl2;  // region offsets (doubles) in part; pl2: finalize level 2
  double *stats;          // [nzp][kStatRow] running statistics (kernels.h)
};

// Advanced on the device by the finalize kernel.
struct Dyn {
  int cc, cf;             // coarse / fine buffer holding the post-stream state
  int hn, hp, hpp;        // history ring slots of levels n, p, pp
  int pad;
  long long step;         // coarse steps done
  long long remaining;    // steps left in the budget
};

struct Mix {
  int n;                  // resident instances (entries of inst)
  int pad[3];
  int start[PH_NPHASE][kMaxInst + 1];
  Inst inst[kMaxInst];
};

// Hermite-in-time weights of one substep (same for every instance of a batch)
struct TimeW {
  float an, ap, app;
};

// Interface corner tile (coarse nodes): CTX x CTY of f32_core.cuh.
#ifndef DNS_CORNER_TY
#define DNS_CORNER_TY 8
#endif
constexpr int kCornerTX = 32, kCornerTY = DNS_CORNER_TY;

// Launch helpers (batch_f32.cu).  grid = persistent blocks of each kernel.
struct Grids {
  int stats, sfinal, coarse, fine, icorner, ieval, inject, final_;
};
int query_grids(int gr, Grids *g);
// count: one zeroed counter per slot (the finalize resets it)
// stats: launch the statistics phases (some resident instance samples)
void launch_step(const Mix *m, Dyn *dyn, DevState *state, DevLog *log, unsigned int *count, int gr, const Grids &g,
                 cudaStream_t s, cudaStream_t aux, cudaEvent_t *ev, bool stats);  // ev: 10 events (fork/join of the two streams)
void tile_counts(const Inst &I, int counts[PH_NPHASE]);

}  // namespace batch
}  // namespace dns
