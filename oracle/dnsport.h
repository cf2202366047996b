/*
 * CPU restatement of the reference's grid-embedded D3Q19 channel step —
 * TEST INFRASTRUCTURE ONLY (the oracle; never linked by the product).
 *
 * One periodic domain (no per-rank ghost columns), push streaming exactly as
 * the reference, every floating-point expression evaluated in the reference's
 * order so that results are bit-identical to the reference compiled with
 * -ffp-contract=off (checked against oracle/_ref builds by the tests).
 *
 * State layout: the reference's own AoS order f[i][j][k][a] (a fastest), the
 * global domain without ghosts:
 *   coarse  xdv x ydv x zdc
 *   lower / upper fine  (GR xdv) x (GR ydv) x (zds + 1)   (wall plane included)
 * Interface history: 3 levels (n, p, pp) x 2 walls (0 lower/lin, 1 upper/uin)
 *   x xdv x ydv x 23 fields [rho, ux, uy, uz, fneq_0..18].
 */
#ifndef ORACLE_DNSPORT_H
#define ORACLE_DNSPORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PORT_PATTERN_NONE = 0, PORT_PATTERN_RSLIP = 1, PORT_PATTERN_PSLIP = 2, PORT_PATTERN_SSLIP = 3 };

typedef struct port_cfg {
  int xdv, ydv, zdc, zds, gr;
  double Reb, ub, CFL;
  int pattern;
  int gy, wy, gx, wx; /* gyplussize, wyplussize, gxplussize, wxplussize */
  int fltr;           /* 1: filtered fine-to-coarse transfer (FLTR), GR = 4 */
} port_cfg;

/* one coarse step's log values (reference encalc2.c / wshearstr.c) */
typedef struct port_log {
  double force;     /* force[0] used by this step's collisions */
  double momentum;  /* normalised streamwise momentum of the pre-step state */
  double denst;     /* normalised mass */
  double flowrate;  /* momentum * (ydf-1)(NZs-2) / denst */
  double stup, stdown, stress, pgrad;
} port_log;

typedef struct port_state port_state;

port_state *port_create(const port_cfg *cfg);
void port_destroy(port_state *s);
int port_load_restart(port_state *s, const char *dir, int cntr);
int port_save_restart(port_state *s, const char *dir, int cntr);
/* seeded initial condition: rho = 1, laminar profile with centreline uc plus
   Philox4x32-10 uniform perturbations of amplitude amp; force[0] = force */
void port_init_seeded(port_state *s, uint64_t seed, double uc, double amp, double force);
/* mode -i start from a uniform-grid state u, the first half of lbf.TTTT in the
   reference's order [xu][yu][zu + 2][19]; -1 when a stencil leaves the
   reference's halo (x, y) or the uniform grid (z) */
int port_init_uniform(port_state *s, const double *u, int xu, int yu, int zu);
/* cfr != 0: constant flow rate (force from encalc2 every step); else fixed g */
void port_set_forcing(port_state *s, int cfr, double g);
/* advance n coarse steps; log (may be NULL) receives n entries */
void port_step(port_state *s, long n, port_log *log);
/* S (post-stream state) in reference AoS order; level 0 coarse, 1 lower, 2 upper */
long port_export(const port_state *s, int level, double *out);
long port_export_history(const port_state *s, double *out); /* [3][2][xdv][ydv][23] */
void port_import_history(port_state *s, const double *in);
double port_force(const port_state *s);
/* instantaneous plane statistics exactly as reference statistics.c:
   out[9][NZ] = UAVG VAVG WAVG UTIN VTIN WTIN REYS DAVG DTIN, NZ = 2 zdf + zdc - 4 */
int port_plane_stats(const port_state *s, double *out);
/* Philox4x32-10 (Salmon et al. 2011) for known-answer tests */
void port_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* relaxation rates and derived sizes as the reference main computes them */
void port_params(const port_state *s, double *omega_c, double *omega_f, int *nzs);

#ifdef __cplusplus
}
#endif
#endif
