/*
 * CPU restatement of the reference's grid-embedded D3Q19 channel step —
 * TEST INFRASTRUCTURE ONLY (the oracle).  See dnsport.h.
 *
 * Every routine cites the reference function it restates (paths relative to
 * DNS-solver-with-grid-embedding/src/).  Compile with -ffp-contract=off.
 */
#include "dnsport.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* D3Q19 velocity set and weights, in the reference's population order
   (globals.c:3-11); opposite/mirror are derived from the velocities. */
static const int EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0};
static const int EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
static const int EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static double EXd[19], EYd[19], EZd[19], WT[19], BIW[19];
static int OPP[19], MIR[19];
static int BICUBIC_W[16][16];
static int tables_ready = 0;

/* the 16x16 map from (values, d/dt, d/du, d2/dtdu at the four cell corners)
   to the coefficients c[n*4+m] of t^n u^m, obtained by inverting the
   Hermite constraint matrix (corners counter-clockwise from (0,0)). */
static void derive_bicubic(void) {
  static const int ct[4] = {0, 1, 1, 0}, cu[4] = {0, 0, 1, 1};
  double M[16][32];
  memset(M, 0, sizeof M);
  for (int typ = 0; typ < 4; typ++)
    for (int q = 0; q < 4; q++) {
      int r = typ * 4 + q;
      for (int n = 0; n < 4; n++)
        for (int m = 0; m < 4; m++) {
          int dn = (typ == 1 || typ == 3), dm = (typ == 2 || typ == 3);
          if (n < dn || m < dm) continue;
          double v = 1.0;
          if (dn) v *= n;
          if (dm) v *= m;
          for (int e = 0; e < n - dn; e++) v *= ct[q];
          for (int e = 0; e < m - dm; e++) v *= cu[q];
          M[r][n * 4 + m] = v;
        }
      M[r][16 + r] = 1.0;
    }
  for (int col = 0; col < 16; col++) { /* Gauss-Jordan, partial pivoting */
    int piv = col;
    for (int r = col + 1; r < 16; r++)
      if (fabs(M[r][col]) > fabs(M[piv][col])) piv = r;
    if (piv != col)
      for (int c = 0; c < 32; c++) {
        double t = M[col][c];
        M[col][c] = M[piv][c];
        M[piv][c] = t;
      }
    double d = M[col][col];
    for (int c = 0; c < 32; c++) M[col][c] /= d;
    for (int r = 0; r < 16; r++)
      if (r != col && M[r][col] != 0.0) {
        double f = M[r][col];
        for (int c = 0; c < 32; c++) M[r][c] -= f * M[col][c];
      }
  }
  for (int r = 0; r < 16; r++)
    for (int c = 0; c < 16; c++) BICUBIC_W[r][c] = (int)lround(M[r][16 + c]);
}

static void init_tables(void) {
  if (tables_ready) return;
  for (int a = 0; a < 19; a++) {
    EXd[a] = EX[a];
    EYd[a] = EY[a];
    EZd[a] = EZ[a];
    int n2 = EX[a] * EX[a] + EY[a] * EY[a] + EZ[a] * EZ[a];
    WT[a] = n2 == 0 ? 1. / 3. : (n2 == 1 ? 1. / 18. : 1. / 36.);
    BIW[a] = n2 == 0 ? 0. : (n2 == 1 ? 1. / 6. : 1. / 12.);
    for (int b = 0; b < 19; b++) {
      if (EX[b] == -EX[a] && EY[b] == -EY[a] && EZ[b] == -EZ[a]) OPP[a] = b;
      if (EX[b] == EX[a] && EY[b] == EY[a] && EZ[b] == -EZ[a]) MIR[a] = b;
    }
  }
  derive_bicubic();
  tables_ready = 1;
}

struct port_state {
  port_cfg c;
  int nx, ny, zdc, nxf, nyf, zdf, gr, nzs;
  double omc, omf;
  double *fc[2], *fl[2], *fu[2]; /* [0] current S, [1] scratch */
  double *hist[3];               /* ring slots, each [2][nx][ny][23] */
  int hn, hp, hpp;               /* slot indices of levels n, p, pp */
  signed char *wflag;            /* wall plane flags [nxf][nyf] (-1 no-slip, -2 slip) */
  double force, g;
  int cfr;
  double *plane, *dx, *dy, *dxy; /* interface work planes [nx][ny] */
};

#define CIDX(s, i, j, k) ((((size_t)(i) * (s)->ny + (j)) * (s)->zdc + (k)) * 19)
#define FIDX(s, i, j, k) ((((size_t)(i) * (s)->nyf + (j)) * (s)->zdf + (k)) * 19)
#define HIDX(s, w, i, j) ((((size_t)(w) * (s)->nx + (i)) * (s)->ny + (j)) * 23)

static int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

/* ------------------------------------------------------------ parameters */
/* dns-q-mgrd-all-patterns-xyc.c:139-155 (sizes), :443-451 (relaxation rates) */
static void derive(port_state *s) {
  const port_cfg *c = &s->c;
  s->gr = c->gr;
  s->nx = c->xdv;
  s->ny = c->ydv;
  s->zdc = c->zdc;
  s->nxf = c->gr * c->xdv;
  s->nyf = c->gr * c->ydv;
  s->zdf = c->zds + 1;
  s->nzs = 2 * s->zdf + s->gr * (s->zdc - 4) + s->gr - 1;
  double tauf = (3. / c->Reb) * c->ub * (s->nzs - 2.) + 0.5;
  double tauc = (1. / ((double)s->gr)) * (3. / c->Reb) * c->ub * (s->nzs - 2.) + 0.5;
  s->omf = 1. / tauf;
  s->omc = 1. / tauc;
}

void port_params(const port_state *s, double *omega_c, double *omega_f, int *nzs) {
  if (omega_c) *omega_c = s->omc;
  if (omega_f) *omega_f = s->omf;
  if (nzs) *nzs = s->nzs;
}

/* wall flags: solid_init.c:46-69 (walls start no-slip), slip_ridges_init.c:35-66,
   slip_posts_init.c:45-117, slip_spanwise_init.c:34-66; periodic in the global
   index, pattern writes that would fall past the end of the span are dropped */
static void init_walls(port_state *s) {
  const port_cfg *c = &s->c;
  int nxf = s->nxf, nyf = s->nyf;
  signed char *sx = (signed char *)malloc((size_t)nxf), *sy = (signed char *)malloc((size_t)nyf);
  for (int i = 0; i < nxf; i++) sx[i] = -1;
  for (int j = 0; j < nyf; j++) sy[j] = -1;
  if (c->pattern == PORT_PATTERN_RSLIP || c->pattern == PORT_PATTERN_PSLIP)
    for (int j = c->wy / 2; j < nyf; j += c->gy + c->wy)
      for (int a = 0; a < c->gy && j + a < nyf; a++) sy[j + a] = -2;
  if (c->pattern == PORT_PATTERN_SSLIP || c->pattern == PORT_PATTERN_PSLIP)
    for (int i = c->wx / 2; i < nxf; i += c->gx + c->wx)
      for (int a = 0; a < c->gx && i + a < nxf; a++) sx[i + a] = -2;
  for (int i = 0; i < nxf; i++)
    for (int j = 0; j < nyf; j++) {
      signed char f = -1;
      if (c->pattern == PORT_PATTERN_RSLIP) f = sy[j];
      else if (c->pattern == PORT_PATTERN_SSLIP) f = sx[i];
      else if (c->pattern == PORT_PATTERN_PSLIP) f = (sx[i] == -2 || sy[j] == -2) ? -2 : -1;
      s->wflag[(size_t)i * nyf + j] = f;
    }
  free(sx);
  free(sy);
}

port_state *port_create(const port_cfg *cfg) {
  init_tables();
  port_state *s = (port_state *)calloc(1, sizeof(*s));
  s->c = *cfg;
  derive(s);
  size_t nc = (size_t)s->nx * s->ny * s->zdc * 19, nf = (size_t)s->nxf * s->nyf * s->zdf * 19;
  size_t nh = (size_t)2 * s->nx * s->ny * 23, npl = (size_t)s->nx * s->ny;
  for (int h = 0; h < 2; h++) {
    s->fc[h] = (double *)calloc(nc, sizeof(double));
    s->fl[h] = (double *)calloc(nf, sizeof(double));
    s->fu[h] = (double *)calloc(nf, sizeof(double));
  }
  for (int h = 0; h < 3; h++) s->hist[h] = (double *)calloc(nh, sizeof(double));
  s->hn = 0;
  s->hp = 1;
  s->hpp = 2;
  s->wflag = (signed char *)malloc((size_t)s->nxf * s->nyf);
  s->plane = (double *)calloc(npl, sizeof(double));
  s->dx = (double *)calloc(npl, sizeof(double));
  s->dy = (double *)calloc(npl, sizeof(double));
  s->dxy = (double *)calloc(npl, sizeof(double));
  init_walls(s);
  s->cfr = 1;
  return s;
}

void port_destroy(port_state *s) {
  if (!s) return;
  for (int h = 0; h < 2; h++) {
    free(s->fc[h]);
    free(s->fl[h]);
    free(s->fu[h]);
  }
  for (int h = 0; h < 3; h++) free(s->hist[h]);
  free(s->wflag);
  free(s->plane);
  free(s->dx);
  free(s->dy);
  free(s->dxy);
  free(s);
}

void port_set_forcing(port_state *s, int cfr, double g) {
  s->cfr = cfr;
  s->g = g;
  if (!cfr) s->force = g;
}

/* the force a restart written now would hold: with constant flow rate the
   reference recomputes it (encalc2) at the top of the iteration that writes
   the restart (dns-q-mgrd-all-patterns-xyc.c:1256-1306) */
static void flow_sums(const port_state *s, double *mom_out, double *den_out);
double port_force(const port_state *s) {
  if (!s->cfr) return s->force;
  double mom, den;
  flow_sums(s, &mom, &den);
  return s->c.ub - mom;
}

/* ------------------------------------------------------------ node physics */
/* moments accumulated in population order (xcomputations.c:61-67) */
static void moments(const double *f, double *dens, double *ux, double *uy, double *uz) {
  double d = 0., x = 0., y = 0., z = 0.;
  for (int a = 0; a < 19; a++) {
    x += EXd[a] * f[a];
    y += EYd[a] * f[a];
    z += EZd[a] * f[a];
    d += f[a];
  }
  *dens = d;
  *ux = x;
  *uy = y;
  *uz = z;
}

static double feq_of(int a, double dens, double u0, double u1, double u2, double v) {
  double u = EXd[a] * u0 + EYd[a] * u1 + EZd[a] * u2;
  return WT[a] * dens * (1. + 3. * u + 4.5 * u * u - 1.5 * v);
}

/* BGK collision with body force, in place (xcomputations.c:49-86) */
static void collide(double *f, double om, double G) {
  double dens, ux, uy, uz;
  moments(f, &dens, &ux, &uy, &uz);
  double u0 = ux / dens, u1 = uy / dens, u2 = uz / dens;
  double v = u0 * u0 + u1 * u1 + u2 * u2;
  for (int a = 0; a < 19; a++) {
    double feq = feq_of(a, dens, u0, u1, u2, v);
    double Fi = BIW[a] * dens * (EXd[a] * G);
    f[a] += (Fi - om * (f[a] - feq));
  }
}

/* ------------------------------------------------------------ reductions */
/* encalc2.c:33-129 in its loop order */
static void flow_sums(const port_state *s, double *mom_out, double *den_out) {
  int gr = s->gr, zdf = s->zdf;
  double momentum = 0., denst = 0., dens, ux, uy, uz, coef;
  const double *fl = s->fl[0], *fc = s->fc[0], *fu = s->fu[0];
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++)
      for (int k = 1; k < zdf - gr; k++) {
        moments(fl + FIDX(s, i, j, k), &dens, &ux, &uy, &uz);
        coef = (k == (zdf - gr)) ? 0.5 : 1.;
        momentum += coef * ux;
        denst += coef * dens;
      }
  for (int i = 0; i < s->nx; i++)
    for (int j = 0; j < s->ny; j++)
      for (int k = 0; k < s->zdc; k++) {
        moments(fc + CIDX(s, i, j, k), &dens, &ux, &uy, &uz);
        coef = ((k == 0) || (k == (s->zdc - 1))) ? 0.5 * gr * gr * gr : 1. * gr * gr * gr;
        momentum += coef * ux;
        denst += coef * dens;
      }
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++)
      for (int k = gr; k < zdf - 1; k++) {
        moments(fu + FIDX(s, i, j, k), &dens, &ux, &uy, &uz);
        coef = (k == gr) ? 0.5 : 1.;
        momentum += coef * ux;
        denst += coef * dens;
      }
  double norm = (double)((s->nxf - 0.) * (s->nyf - 0.) * 1 * 1 * (s->nzs - 2.));
  *mom_out = momentum / norm;
  *den_out = denst / norm;
}

/* wshearstr.c:33-137 in its loop order */
static void wall_shear(const port_state *s, port_log *lg) {
  int zdf = s->zdf;
  double mu = (1. / 6.) * (2. / s->omf - 1);
  double stdown = 0., stup = 0., davg = 0., dens, ux, uy, uz, ux1, ux2, ux3;
  const double *fl = s->fl[0], *fu = s->fu[0];
  double norm = (double)((s->nxf - 0.) * (s->nyf - 0.) * 1 * 1);
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++) {
      moments(fl + FIDX(s, i, j, 1), &dens, &ux, &uy, &uz);
      ux1 = ux / dens;
      davg += dens;
      moments(fl + FIDX(s, i, j, 2), &dens, &ux, &uy, &uz);
      ux2 = ux / dens;
      moments(fl + FIDX(s, i, j, 3), &dens, &ux, &uy, &uz);
      ux3 = ux / dens;
      stdown += (-2. * ux1 + 3. * ux2 - ux3);
    }
  davg /= norm;
  stdown /= norm;
  stdown *= mu * davg;
  davg = 0.;
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++) {
      moments(fu + FIDX(s, i, j, zdf - 2), &dens, &ux, &uy, &uz);
      ux1 = ux / dens;
      moments(fu + FIDX(s, i, j, zdf - 3), &dens, &ux, &uy, &uz);
      ux2 = ux / dens;
      moments(fu + FIDX(s, i, j, zdf - 4), &dens, &ux, &uy, &uz);
      ux3 = ux / dens;
      stup += -(2. * ux1 - 3. * ux2 + ux3);
      davg += dens;
    }
  davg /= norm;
  stup /= norm;
  stup *= mu * davg;
  lg->stup = stup;
  lg->stdown = stdown;
  lg->stress = 0.5 * (stup + stdown);
  lg->pgrad = s->force * (s->nzs - 2.) / (2. * s->gr);
}

/* ------------------------------------------------------------ streaming */
/* coarse: collide every plane, push into planes 1..zdc-2 (xcomputations.c:135-420);
   planes 0 and zdc-1 are rewritten by the fine-to-coarse transfer */
static void coarse_collide_push(port_state *s) {
  double P[19];
  for (int i = 0; i < s->nx; i++)
    for (int j = 0; j < s->ny; j++)
      for (int k = 0; k < s->zdc; k++) {
        memcpy(P, s->fc[0] + CIDX(s, i, j, k), sizeof P);
        collide(P, s->omc, s->force);
        for (int a = 0; a < 19; a++) {
          int k2 = k + EZ[a];
          if (k2 < 1 || k2 > s->zdc - 2) continue;
          int i2 = wrap(i + EX[a], s->nx), j2 = wrap(j + EY[a], s->ny);
          s->fc[1][CIDX(s, i2, j2, k2) + a] = P[a];
        }
      }
}

/* fine: both blocks, half-way bounce-back and specular reflection at the wall
   planes (xfcomputations.c:226-240); pushes into the interface plane are
   dropped because the coarse-to-fine transfer rewrites it */
static void fine_collide_push(port_state *s, double Gf) {
  double P[19];
  int zdf = s->zdf, nxf = s->nxf, nyf = s->nyf;
  for (int blk = 0; blk < 2; blk++) {
    double *cur = blk == 0 ? s->fl[0] : s->fu[0];
    double *nxt = blk == 0 ? s->fl[1] : s->fu[1];
    int klo = blk == 0 ? 1 : 0, khi = blk == 0 ? zdf - 1 : zdf - 2;
    int kwall = blk == 0 ? 0 : zdf - 1;
    for (int i = 0; i < nxf; i++)
      for (int j = 0; j < nyf; j++)
        for (int k = klo; k <= khi; k++) {
          memcpy(P, cur + FIDX(s, i, j, k), sizeof P);
          collide(P, s->omf, Gf);
          for (int a = 0; a < 19; a++) {
            int k2 = k + EZ[a];
            int i2 = wrap(i + EX[a], nxf), j2 = wrap(j + EY[a], nyf);
            if (k2 == kwall) {
              int sld = s->wflag[(size_t)i2 * nyf + j2], sld1 = s->wflag[(size_t)i * nyf + j];
              if (sld == -1 && sld1 == -1)
                nxt[FIDX(s, i, j, k) + OPP[a]] = P[a];
              else if ((sld == -1 && sld1 == -2) || sld == -2)
                nxt[FIDX(s, i2, j2, k) + MIR[a]] = P[a];
              continue;
            }
            if (blk == 0 && k2 >= zdf - 1) continue;
            if (blk == 1 && k2 <= 0) continue;
            nxt[FIDX(s, i2, j2, k2) + a] = P[a];
          }
        }
  }
}

/* interface planes of the new coarse state (xcomputations.c:548-625) */
static void extract_planes(port_state *s) {
  int t = s->hpp;
  s->hpp = s->hp;
  s->hp = s->hn;
  s->hn = t;
  double *h = s->hist[s->hn];
  for (int w = 0; w < 2; w++) {
    int k = w == 0 ? 1 : s->zdc - 2;
    for (int i = 0; i < s->nx; i++)
      for (int j = 0; j < s->ny; j++) {
        const double *f = s->fc[1] + CIDX(s, i, j, k);
        double dens, ux, uy, uz;
        moments(f, &dens, &ux, &uy, &uz);
        double u0 = ux / dens, u1 = uy / dens, u2 = uz / dens;
        double v = u0 * u0 + u1 * u1 + u2 * u2;
        double *o = h + HIDX(s, w, i, j);
        o[0] = dens;
        o[1] = u0;
        o[2] = u1;
        o[3] = u2;
        for (int a = 0; a < 19; a++) o[4 + a] = f[a] - feq_of(a, dens, u0, u1, u2, v);
      }
  }
}

/* coarse-to-fine transfer at substep `it` (tinterpolate_hrmt.c, derivative.c,
   bcucof_opt.c, ctfdtransfer_opt.c): Hermite in time, 4th-order derivatives,
   bicubic in space, feq + omega_c/(GR omega_f) fneq into both interface planes */
static void interface_transfer(port_state *s, int it) {
  int nx = s->nx, ny = s->ny, gr = s->gr, zdf = s->zdf;
  double tmp = (((double)it) / ((double)gr));
  double h1 = 2. * tmp * tmp * tmp - 3. * tmp * tmp + 1.;
  double h2 = tmp * tmp * tmp - 2. * tmp * tmp + tmp;
  double h3 = -2. * tmp * tmp * tmp + 3. * tmp * tmp;
  double h4 = tmp * tmp * tmp - tmp * tmp;
  double fac = s->omc / ((double)gr * s->omf);
  const double *Hn = s->hist[s->hn], *Hp = s->hist[s->hp], *Hpp = s->hist[s->hpp];
  double *coef = (double *)malloc(sizeof(double) * (size_t)nx * ny * 23 * 16);
  for (int w = 0; w < 2; w++) {
    for (int b = 0; b < 23; b++) {
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
          size_t q = HIDX(s, w, i, j) + b;
          double c1 = Hp[q];
          double c2 = (Hn[q] - Hpp[q]) * 0.5;
          double c3 = Hn[q];
          double c4 = (3. * Hn[q] - 4. * Hp[q] + Hpp[q]) * 0.5;
          s->plane[(size_t)i * ny + j] = h1 * c1 + h2 * c2 + h3 * c3 + h4 * c4;
        }
#define PL(A, I, J) (A)[(size_t)wrap((I), nx) * ny + wrap((J), ny)]
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
          s->dx[(size_t)i * ny + j] = (2. / 3.) * (PL(s->plane, i + 1, j) - PL(s->plane, i - 1, j)) -
                                      (1. / 12.) * (PL(s->plane, i + 2, j) - PL(s->plane, i - 2, j));
          s->dy[(size_t)i * ny + j] = (2. / 3.) * (PL(s->plane, i, j + 1) - PL(s->plane, i, j - 1)) -
                                      (1. / 12.) * (PL(s->plane, i, j + 2) - PL(s->plane, i, j - 2));
        }
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
          s->dxy[(size_t)i * ny + j] = (2. / 3.) * (PL(s->dy, i + 1, j) - PL(s->dy, i - 1, j)) -
                                       (1. / 12.) * (PL(s->dy, i + 2, j) - PL(s->dy, i - 2, j));
      for (int ic = 0; ic < nx; ic++)
        for (int jc = 0; jc < ny; jc++) {
          static const int ci[4] = {0, 1, 1, 0}, cj[4] = {0, 0, 1, 1};
          double x[16];
          for (int q = 0; q < 4; q++) {
            x[q] = PL(s->plane, ic + ci[q], jc + cj[q]);
            x[4 + q] = PL(s->dx, ic + ci[q], jc + cj[q]);
            x[8 + q] = PL(s->dy, ic + ci[q], jc + cj[q]);
            x[12 + q] = PL(s->dxy, ic + ci[q], jc + cj[q]);
          }
          double *cc = coef + (((size_t)ic * ny + jc) * 23 + b) * 16;
          for (int r = 0; r < 16; r++) {
            double xx = 0.0;
            for (int k = 0; k < 16; k++) xx += BICUBIC_W[r][k] * x[k];
            cc[r] = xx;
          }
        }
#undef PL
    }
    double *nxt = w == 0 ? s->fl[1] : s->fu[1];
    int kf = w == 0 ? zdf - 1 : 0;
    for (int ic = 0; ic < nx; ic++)
      for (int jc = 0; jc < ny; jc++) {
        const double *cc = coef + ((size_t)ic * ny + jc) * 23 * 16;
        for (int ii = 0; ii < gr; ii++)
          for (int jj = 0; jj < gr; jj++) {
            int i = ic * gr + ii, j = jc * gr + jj;
            double tt = ((double)(i % gr)) / ((double)gr);
            double uu = ((double)(j % gr)) / ((double)gr);
            double val[23];
            for (int b = 0; b < 23; b++) {
              const double *c = cc + b * 16;
              double r = 0.;
              for (int nn = 3; nn > -1; nn--)
                r = tt * r + ((c[nn * 4 + 3] * uu + c[nn * 4 + 2]) * uu + c[nn * 4 + 1]) * uu + c[nn * 4 + 0];
              val[b] = r;
            }
            double dens = val[0], u0 = val[1], u1 = val[2], u2 = val[3];
            double v = u0 * u0 + u1 * u1 + u2 * u2;
            double *o = nxt + FIDX(s, i, j, kf);
            for (int a = 0; a < 19; a++) o[a] = feq_of(a, dens, u0, u1, u2, v) + fac * val[4 + a];
          }
      }
  }
  free(coef);
}

/* fine-to-coarse injection (ftcdtransfer.c:28-115) */
static void inject(port_state *s) {
  int gr = s->gr;
  double fac = gr * (s->omf / s->omc);
  for (int w = 0; w < 2; w++) {
    const double *src = w == 0 ? s->fl[0] : s->fu[0];
    int ks = w == 0 ? s->zdf - 1 - gr : gr;
    int kc = w == 0 ? 0 : s->zdc - 1;
    for (int ic = 0; ic < s->nx; ic++)
      for (int jc = 0; jc < s->ny; jc++) {
        const double *f = src + FIDX(s, ic * gr, jc * gr, ks);
        double dens, ux, uy, uz;
        moments(f, &dens, &ux, &uy, &uz);
        double u0 = ux / dens, u1 = uy / dens, u2 = uz / dens;
        double v = u0 * u0 + u1 * u1 + u2 * u2;
        double *o = s->fc[1] + CIDX(s, ic, jc, kc);
        for (int a = 0; a < 19; a++) {
          double feq = feq_of(a, dens, u0, u1, u2, v);
          double fneq = f[a] - feq;
          o[a] = feq + fac * fneq;
        }
      }
  }
}

/* filtered fine-to-coarse transfer (ftcdtransfer_lesfltr.c:163-363, FLTR),
   for GR = 4: f^neq of every fine node of the five planes kb-2..kb+2 around the
   transfer plane kb (:166-196), a sum over the 5 x 5 x 5 nodes around the coarse
   vertex of weight x f^neq / GR^3 with the trapezoid weights (1/2, 1, 1, 1, 1/2)
   per axis (:22-27, :232-246), in the order (x, y, z) outer, population inner,
   and the equilibrium of the centre node's density and MOMENTUM: the reference
   stores the momentum sums where it later reads the velocity (:185-188,
   :222-225).  x and y wrap periodically, as the halo exchange does. */
static void inject_filtered(port_state *s) {
  static const double c5[5] = {0.5, 1., 1., 1., 0.5};
  int gr = s->gr, nxf = s->nxf, nyf = s->nyf;
  double fac = gr * (s->omf / s->omc);
  double *fq = (double *)malloc(sizeof(double) * (size_t)nxf * nyf * 5 * 19);
  double *mc = (double *)malloc(sizeof(double) * (size_t)nxf * nyf * 4);
  for (int w = 0; w < 2; w++) {
    const double *src = w == 0 ? s->fl[0] : s->fu[0];
    int kb = w == 0 ? s->zdf - 1 - gr : gr;
    int kc = w == 0 ? 0 : s->zdc - 1;
    for (int i = 0; i < nxf; i++)
      for (int j = 0; j < nyf; j++)
        for (int kk = -2; kk < 3; kk++) {
          const double *f = src + FIDX(s, i, j, kb + kk);
          double dens, ux, uy, uz;
          moments(f, &dens, &ux, &uy, &uz);
          double u0 = ux / dens, u1 = uy / dens, u2 = uz / dens;
          double v = u0 * u0 + u1 * u1 + u2 * u2;
          double *o = fq + (((size_t)i * nyf + j) * 5 + (kk + 2)) * 19;
          for (int a = 0; a < 19; a++) o[a] = f[a] - feq_of(a, dens, u0, u1, u2, v);
          if (kk == 0) {
            double *m = mc + ((size_t)i * nyf + j) * 4;
            m[0] = dens;
            m[1] = ux;
            m[2] = uy;
            m[3] = uz;
          }
        }
    for (int ic = 0; ic < s->nx; ic++)
      for (int jc = 0; jc < s->ny; jc++) {
        int i = ic * gr, j = jc * gr;
        const double *m = mc + ((size_t)i * nyf + j) * 4;
        double dens = m[0], u0 = m[1], u1 = m[2], u2 = m[3];
        double v = u0 * u0 + u1 * u1 + u2 * u2;
        double t[19] = {0.};
        for (int ii = -2; ii < 3; ii++)
          for (int jj = -2; jj < 3; jj++)
            for (int kk = -2; kk < 3; kk++) {
              double wgt = c5[ii + 2] * c5[jj + 2] * c5[kk + 2];
              const double *q = fq + (((size_t)wrap(i + ii, nxf) * nyf + wrap(j + jj, nyf)) * 5 + (kk + 2)) * 19;
              for (int a = 0; a < 19; a++) t[a] += (wgt * q[a]) / ((double)gr * gr * gr);
            }
        double *o = s->fc[1] + CIDX(s, ic, jc, kc);
        for (int a = 0; a < 19; a++) o[a] = feq_of(a, dens, u0, u1, u2, v) + fac * t[a];
      }
  }
  free(fq);
  free(mc);
}

static void swap2(double **p) {
  double *t = p[0];
  p[0] = p[1];
  p[1] = t;
}

/* one coarse step: main loop body dns-q-mgrd-all-patterns-xyc.c:1256-1374 */
void port_step(port_state *s, long n, port_log *log) {
  for (long st = 0; st < n; st++) {
    port_log lg;
    memset(&lg, 0, sizeof lg);
    flow_sums(s, &lg.momentum, &lg.denst);
    if (s->cfr) s->force = s->c.ub - lg.momentum;
    lg.force = s->force;
    lg.flowrate = lg.momentum * ((s->nyf) * (s->nzs - 2)) / lg.denst;
    wall_shear(s, &lg);
    coarse_collide_push(s);
    extract_planes(s);
    double Gf = (1. / ((double)s->gr)) * s->force;
    for (int it = 1; it <= s->gr; it++) {
      fine_collide_push(s, Gf);
      interface_transfer(s, it);
      swap2(s->fl);
      swap2(s->fu);
    }
    if (s->c.fltr) inject_filtered(s);
    else inject(s);
    swap2(s->fc);
    if (log) log[st] = lg;
  }
}

/* ------------------------------------------------------------ seeded IC */
static uint32_t mulhilo(uint32_t a, uint32_t b, uint32_t *hi) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  return (uint32_t)p;
}

void port_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, hi1;
    uint32_t lo0 = mulhilo(0xD2511F53u, c0, &hi0);
    uint32_t lo1 = mulhilo(0xCD9E8D57u, c2, &hi1);
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* velocity of the seeded state at wall-normal position z (fine units) */
static void seeded_velocity(uint64_t seed, double uc, double amp, double H, double z, uint32_t i,
                            uint32_t j, uint32_t k, uint32_t level, double u[3]) {
  uint32_t ctr[4] = {i, j, k, level}, key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)}, r[4];
  port_philox4x32_10(ctr, key, r);
  double zeta = z / H;
  double prof = 4.0 * uc * zeta * (1.0 - zeta);
  for (int c = 0; c < 3; c++) {
    double x = ((double)r[c] + 0.5) * (1.0 / 4294967296.0);
    u[c] = amp * (2.0 * x - 1.0);
  }
  u[0] = prof + u[0];
}

static void seeded_node(double *f, const double u[3]) {
  double v = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  for (int a = 0; a < 19; a++) f[a] = feq_of(a, 1.0, u[0], u[1], u[2], v);
}

void port_init_seeded(port_state *s, uint64_t seed, double uc, double amp, double force) {
  int zdf = s->zdf, gr = s->gr;
  double H = s->nzs - 2.0;
  double u[3];
  for (int h = 0; h < 2; h++) {
    memset(s->fc[h], 0, sizeof(double) * (size_t)s->nx * s->ny * s->zdc * 19);
    memset(s->fl[h], 0, sizeof(double) * (size_t)s->nxf * s->nyf * zdf * 19);
    memset(s->fu[h], 0, sizeof(double) * (size_t)s->nxf * s->nyf * zdf * 19);
  }
  for (int i = 0; i < s->nx; i++)
    for (int j = 0; j < s->ny; j++)
      for (int k = 0; k < s->zdc; k++) {
        double z = (zdf - 1.5) + gr * (k - 1.0);
        seeded_velocity(seed, uc, amp, H, z, i, j, k, 0, u);
        seeded_node(s->fc[0] + CIDX(s, i, j, k), u);
        if (k == 1 || k == s->zdc - 2) {
          for (int l = 0; l < 3; l++) {
            double *o = s->hist[l] + HIDX(s, k == 1 ? 0 : 1, i, j);
            memset(o, 0, 23 * sizeof(double));
            o[0] = 1.0;
            o[1] = u[0];
            o[2] = u[1];
            o[3] = u[2];
          }
        }
      }
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++) {
      for (int k = 1; k < zdf; k++) {
        double z = k - 0.5;
        seeded_velocity(seed, uc, amp, H, z, i, j, k, 1, u);
        seeded_node(s->fl[0] + FIDX(s, i, j, k), u);
      }
      for (int k = 0; k < zdf - 1; k++) {
        double z = (zdf - 1.5) + gr * (s->zdc - 3.0) + k;
        seeded_velocity(seed, uc, amp, H, z, i, j, k, 2, u);
        seeded_node(s->fu[0] + FIDX(s, i, j, k), u);
      }
    }
  s->hn = 0;
  s->hp = 1;
  s->hpp = 2;
  s->force = force;
}

/* ------------------------------------------------------------ mode -i start */
/* sp_interpolate_qd.c:22-45: quadratic Lagrange in z, then y, then x over the
   3 x 3 x 3 stencil ind x jnd x knd of the uniform state u ([xu][yu][zd][19]);
   x and y wrap periodically, which is what the reference's halo holds */
static void qd_interp(const double *u, int xu, int yu, int zd, const int *ind, const int *jnd, const int *knd,
                      double dx, double dy, double dz, double *ans) {
  double cz[3][3][19], cy[3][19];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      int ii = ((ind[i] % xu) + xu) % xu, jj = ((jnd[j] % yu) + yu) % yu;
      const double *col = u + ((size_t)ii * yu + jj) * zd * 19;
      for (int a = 0; a < 19; a++)
        cz[i][j][a] = 0.5 * dz * (dz - 1.) * col[knd[0] * 19 + a] - (dz - 1.) * (dz + 1.) * col[knd[1] * 19 + a] +
                      0.5 * (dz + 1.) * dz * col[knd[2] * 19 + a];
    }
  for (int i = 0; i < 3; i++)
    for (int a = 0; a < 19; a++)
      cy[i][a] = 0.5 * dy * (dy - 1.) * cz[i][0][a] - (dy - 1.) * (dy + 1.) * cz[i][1][a] +
                 0.5 * (dy + 1.) * dy * cz[i][2][a];
  for (int a = 0; a < 19; a++)
    ans[a] = 0.5 * dx * (dx - 1.) * cy[0][a] - (dx - 1.) * (dx + 1.) * cy[1][a] + 0.5 * (dx + 1.) * dx * cy[2][a];
}

/* interpolated populations -> feq + fac (f - feq) (initializer.c:372-395) */
static void rescale_node(const double *fi, double fac, double *out) {
  double dens, ux, uy, uz;
  moments(fi, &dens, &ux, &uy, &uz);
  double u0 = ux / dens, u1 = uy / dens, u2 = uz / dens;
  double v = u0 * u0 + u1 * u1 + u2 * u2;
  for (int a = 0; a < 19; a++) {
    double feq = feq_of(a, dens, u0, u1, u2, v);
    out[a] = feq + fac * (fi[a] - feq);
  }
}

static int stencil_ok(const int *ind, const int *jnd, const int *knd, int xu, int yu, int zd) {
  return ind[0] >= -2 && ind[2] <= xu + 3 && jnd[0] >= -2 && jnd[2] <= yu + 3 && knd[0] >= 0 && knd[2] < zd;
}

/* dns-q-mgrd-all-patterns-xyc.c:978-997 (mode -i): init.c before the wall flags
   exist (every node w_a), initializer.c:303-533 (first half of lbf.TTTT onto the
   post-stream lattices), inter_init.c (interface history from the coarse
   state).  Two slips of inter_init are not reproduced: levels p and pp get all
   23 fields of level n (the reference copies 19 of every 23, :237-248), and the
   upper plane's density and velocity go to the upper history (the reference
   writes them into the lower one, :202-205). */
int port_init_uniform(port_state *s, const double *u, int xu, int yu, int zu) {
  const int zd = zu + 2, GR = s->gr, zdf = s->zdf, zdc = s->zdc;
  const double dxf = 2. / ((double)(s->nzs - 2.));
  const double dxc = GR * dxf;
  const double dxr = 2. / ((double)(zd - 2.));
  double tau = (3. / s->c.Reb) * s->c.ub * (zd - 2.) + 0.5;
  tau = 1. / tau;
  const double tauf = s->omf, tauc = s->omc;
  int ind[3], jnd[3], knd[3], iref, jref, kref;
  double dx, dy, dz, fi[19];
  size_t nc = (size_t)s->nx * s->ny * zdc * 19, nf = (size_t)s->nxf * s->nyf * zdf * 19;
  for (int h = 0; h < 2; h++) {
    for (size_t q = 0; q < nc; q++) s->fc[h][q] = WT[q % 19];
    for (size_t q = 0; q < nf; q++) s->fl[h][q] = s->fu[h][q] = WT[q % 19];
  }
  /* lower fine block, k = 1..zdf-1 (initializer.c:326-399) */
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++)
      for (int k = 1; k < zdf; k++) {
        iref = (int)floor((i + 0.5) * (dxf / dxr) - 0.5);
        jref = (int)floor((j + 0.5) * (dxf / dxr) - 0.5);
        kref = (int)floor((k - 0.5) * (dxf / dxr) + 0.5);
        ind[0] = iref - 1; ind[1] = iref; ind[2] = iref + 1;
        jnd[0] = jref - 1; jnd[1] = jref; jnd[2] = jref + 1;
        dx = (i + 0.5) * dxf - (iref + 0.5) * dxr;
        dy = (j + 0.5) * dxf - (jref + 0.5) * dxr;
        if (kref == 0) {
          knd[0] = kref; knd[1] = kref + 1; knd[2] = kref + 2;
          dz = -dxr + (k - 0.5) * dxf + 0.5 * dxr - kref * dxr;
        } else {
          knd[0] = kref - 1; knd[1] = kref; knd[2] = kref + 1;
          dz = (k - 0.5) * dxf + 0.5 * dxr - kref * dxr;
        }
        dx = dx / dxr; dy = dy / dxr; dz = dz / dxr;
        if (!stencil_ok(ind, jnd, knd, xu, yu, zd)) return -1;
        qd_interp(u, xu, yu, zd, ind, jnd, knd, dx, dy, dz, fi);
        rescale_node(fi, (dxr / dxf) * (tau / tauf), s->fl[0] + FIDX(s, i, j, k));
      }
  /* coarse grid, k = 0..zdc-1 (initializer.c:402-468) */
  for (int i = 0; i < s->nx; i++)
    for (int j = 0; j < s->ny; j++)
      for (int k = 0; k < zdc; k++) {
        iref = (int)floor((i + 0.5) * dxc / dxr - 0.5);
        jref = (int)floor((j + 0.5) * dxc / dxr - 0.5);
        kref = (int)floor(0.5 + (k * GR + (zdf - GR - 1 - 0.5)) * dxf / dxr);
        ind[0] = iref - 1; ind[1] = iref; ind[2] = iref + 1;
        jnd[0] = jref - 1; jnd[1] = jref; jnd[2] = jref + 1;
        knd[0] = kref - 1; knd[1] = kref; knd[2] = kref + 1;
        dx = (i + 0.5) * dxc - (iref + 0.5) * dxr;
        dy = (j + 0.5) * dxc - (jref + 0.5) * dxr;
        dz = (k * GR + (zdf - GR - 1 - 0.5)) * dxf - (kref - 0.5) * dxr;
        dx = dx / dxr; dy = dy / dxr; dz = dz / dxr;
        if (!stencil_ok(ind, jnd, knd, xu, yu, zd)) return -1;
        qd_interp(u, xu, yu, zd, ind, jnd, knd, dx, dy, dz, fi);
        rescale_node(fi, (dxr / dxc) * (tau / tauc), s->fc[0] + CIDX(s, i, j, k));
      }
  /* upper fine block, k = 0..zdf-2 (initializer.c:470-533) */
  for (int i = 0; i < s->nxf; i++)
    for (int j = 0; j < s->nyf; j++)
      for (int k = 0; k < zdf - 1; k++) {
        iref = (int)floor((i + 0.5) * dxf / dxr - 0.5);
        jref = (int)floor((j + 0.5) * dxf / dxr - 0.5);
        kref = (int)floor(0.5 + (k + GR * (zdc - 3) + zdf - 1 - 0.5) * dxf / dxr);
        ind[0] = iref - 1; ind[1] = iref; ind[2] = iref + 1;
        jnd[0] = jref - 1; jnd[1] = jref; jnd[2] = jref + 1;
        knd[0] = kref - 1; knd[1] = kref; knd[2] = kref + 1;
        dx = (i + 0.5) * dxf - (iref + 0.5) * dxr;
        dy = (j + 0.5) * dxf - (jref + 0.5) * dxr;
        dz = (k + GR * (zdc - 3) + zdf - 1 - 0.5) * dxf - (kref - 0.5) * dxr;
        dx = dx / dxr; dy = dy / dxr; dz = dz / dxr;
        if (!stencil_ok(ind, jnd, knd, xu, yu, zd)) return -1;
        qd_interp(u, xu, yu, zd, ind, jnd, knd, dx, dy, dz, fi);
        rescale_node(fi, (dxr / dxf) * (tau / tauf), s->fu[0] + FIDX(s, i, j, k));
      }
  memcpy(s->fl[1], s->fl[0], nf * sizeof(double));
  memcpy(s->fu[1], s->fu[0], nf * sizeof(double));
  /* inter_init.c:150-226 on the new coarse state, then all three levels */
  s->hn = 0;
  s->hp = 1;
  s->hpp = 2;
  for (int w = 0; w < 2; w++) {
    int k = w == 0 ? 1 : zdc - 2;
    for (int i = 0; i < s->nx; i++)
      for (int j = 0; j < s->ny; j++) {
        const double *f = s->fc[0] + CIDX(s, i, j, k);
        double dens, ux, uy, uz;
        moments(f, &dens, &ux, &uy, &uz);
        double u0 = ux / dens, u1 = uy / dens, u2 = uz / dens;
        double v = u0 * u0 + u1 * u1 + u2 * u2;
        double *o = s->hist[0] + HIDX(s, w, i, j);
        o[0] = dens;
        o[1] = u0;
        o[2] = u1;
        o[3] = u2;
        for (int a = 0; a < 19; a++) o[4 + a] = f[a] - feq_of(a, dens, u0, u1, u2, v);
      }
  }
  size_t nh = (size_t)2 * s->nx * s->ny * 23;
  memcpy(s->hist[1], s->hist[0], nh * sizeof(double));
  memcpy(s->hist[2], s->hist[0], nh * sizeof(double));
  s->force = s->cfr ? 0. : s->g;
  return 0;
}

/* ------------------------------------------------------------ restart I/O */
static int read_block(FILE *fp, double *dst, size_t n) { return fread(dst, sizeof(double), n, fp) == n ? 0 : -1; }

int port_load_restart(port_state *s, const char *dir, int cntr) {
  char fn[4096];
  size_t nc = (size_t)s->nx * s->ny * s->zdc * 19, nf = (size_t)s->nxf * s->nyf * s->zdf * 19;
  const char *names[3] = {"lbf-c", "lbf-slf", "lbf-suf"};
  double *dst[3] = {s->fc[0], s->fl[0], s->fu[0]};
  size_t cnt[3] = {nc, nf, nf};
  for (int q = 0; q < 3; q++) {
    snprintf(fn, sizeof fn, "%s/%s.%.4d", dir, names[q], cntr);
    FILE *fp = fopen(fn, "rb");
    if (!fp || read_block(fp, dst[q], cnt[q])) {
      if (fp) fclose(fp);
      return -1;
    }
    fclose(fp);
  }
  memcpy(s->fl[1], s->fl[0], nf * sizeof(double));
  memcpy(s->fu[1], s->fu[0], nf * sizeof(double));
  snprintf(fn, sizeof fn, "%s/force.%.4d", dir, cntr);
  FILE *fp = fopen(fn, "rb");
  if (!fp || read_block(fp, &s->force, 1)) {
    if (fp) fclose(fp);
    return -1;
  }
  fclose(fp);
  const char *hn[2] = {"lbf-lin", "lbf-uin"};
  size_t per = (size_t)s->nx * s->ny * 23;
  for (int w = 0; w < 2; w++) {
    snprintf(fn, sizeof fn, "%s/%s.%.4d", dir, hn[w], cntr);
    fp = fopen(fn, "rb");
    if (!fp) return -1;
    for (int l = 0; l < 3; l++)
      if (read_block(fp, s->hist[l] + (size_t)w * per, per)) {
        fclose(fp);
        return -1;
      }
    fclose(fp);
  }
  s->hn = 0;
  s->hp = 1;
  s->hpp = 2;
  return 0;
}

int port_save_restart(port_state *s, const char *dir, int cntr) {
  char fn[4096];
  size_t nc = (size_t)s->nx * s->ny * s->zdc * 19, nf = (size_t)s->nxf * s->nyf * s->zdf * 19;
  const char *names[3] = {"lbf-c", "lbf-slf", "lbf-suf"};
  double *src[3] = {s->fc[0], s->fl[0], s->fu[0]};
  size_t cnt[3] = {nc, nf, nf};
  for (int q = 0; q < 3; q++) {
    snprintf(fn, sizeof fn, "%s/%s.%.4d", dir, names[q], cntr);
    FILE *fp = fopen(fn, "wb");
    if (!fp) return -1;
    /* [ftemp | f]: the second half is scratch the reference never reads before
       overwriting it; the post-stream state is written to both halves */
    int bad = fwrite(src[q], sizeof(double), cnt[q], fp) != cnt[q] ||
              fwrite(src[q], sizeof(double), cnt[q], fp) != cnt[q];
    fclose(fp);
    if (bad) return -1;
  }
  snprintf(fn, sizeof fn, "%s/force.%.4d", dir, cntr);
  FILE *fp = fopen(fn, "wb");
  if (!fp) return -1;
  double fnext = port_force(s);
  fwrite(&fnext, sizeof(double), 1, fp);
  fclose(fp);
  const char *hn[2] = {"lbf-lin", "lbf-uin"};
  size_t per = (size_t)s->nx * s->ny * 23;
  int lv[3] = {s->hn, s->hp, s->hpp};
  for (int w = 0; w < 2; w++) {
    snprintf(fn, sizeof fn, "%s/%s.%.4d", dir, hn[w], cntr);
    fp = fopen(fn, "wb");
    if (!fp) return -1;
    for (int l = 0; l < 3; l++) fwrite(s->hist[lv[l]] + (size_t)w * per, sizeof(double), per, fp);
    fclose(fp);
  }
  return 0;
}

long port_export(const port_state *s, int level, double *out) {
  size_t n = level == 0 ? (size_t)s->nx * s->ny * s->zdc * 19 : (size_t)s->nxf * s->nyf * s->zdf * 19;
  const double *src = level == 0 ? s->fc[0] : (level == 1 ? s->fl[0] : s->fu[0]);
  if (out) memcpy(out, src, n * sizeof(double));
  return (long)n;
}

long port_export_history(const port_state *s, double *out) {
  size_t per = (size_t)2 * s->nx * s->ny * 23;
  if (out) {
    memcpy(out, s->hist[s->hn], per * sizeof(double));
    memcpy(out + per, s->hist[s->hp], per * sizeof(double));
    memcpy(out + 2 * per, s->hist[s->hpp], per * sizeof(double));
  }
  return (long)(3 * per);
}

/* the inverse of port_export_history; all zeros leaves the history as main's
   mode s does (dns-q-mgrd-all-patterns-xyc.c:961-977 never sets it) */
void port_import_history(port_state *s, const double *in) {
  size_t per = (size_t)2 * s->nx * s->ny * 23;
  memcpy(s->hist[s->hn], in, per * sizeof(double));
  memcpy(s->hist[s->hp], in + per, per * sizeof(double));
  memcpy(s->hist[s->hpp], in + 2 * per, per * sizeof(double));
}

/* ------------------------------------------------------------ statistics */
/* statistics.c:48-300: per-plane means, then rms of the deviation from the
   plane mean, over the composite profile of NZ = 2 zdf + zdc - 4 planes */
int port_plane_stats(const port_state *s, double *out) {
  int zdf = s->zdf, zdc = s->zdc, NZ = 2 * zdf + zdc - 4;
  double *U = out, *Vv = out + NZ, *Wv = out + 2 * NZ, *UT = out + 3 * NZ, *VT = out + 4 * NZ,
         *WT_ = out + 5 * NZ, *RE = out + 6 * NZ, *DA = out + 7 * NZ, *DT = out + 8 * NZ;
  memset(out, 0, sizeof(double) * 9 * (size_t)NZ);
  struct seg { const double *arr; int fine, k0, k1, off; } segs[3] = {
      {s->fl[0], 1, 1, zdf, 0}, {s->fc[0], 0, 2, zdc - 2, zdf - 2}, {s->fu[0], 1, 0, zdf - 1, zdf + zdc - 4}};
  for (int pass = 0; pass < 2; pass++) {
    for (int g = 0; g < 3; g++) {
      int ex = segs[g].fine ? s->nxf : s->nx, ey = segs[g].fine ? s->nyf : s->ny;
      for (int i = 0; i < ex; i++)
        for (int j = 0; j < ey; j++)
          for (int k = segs[g].k0; k < segs[g].k1; k++) {
            const double *f = segs[g].arr + (segs[g].fine ? FIDX(s, i, j, k) : CIDX(s, i, j, k));
            double u = 0., v = 0., w = 0., dens = 0.;
            for (int a = 0; a < 19; a++) {
              dens += f[a];
              u += EXd[a] * f[a];
              v += EYd[a] * f[a];
              w += EZd[a] * f[a];
            }
            int p = segs[g].off + k;
            if (pass == 0) {
              U[p] += (u / dens);
              Vv[p] += (v / dens);
              Wv[p] += (w / dens);
              DA[p] += dens;
            } else {
              double uf = (u / dens) - U[p], vf = (v / dens) - Vv[p], wf = (w / dens) - Wv[p], df = dens - DA[p];
              UT[p] += uf * uf;
              VT[p] += vf * vf;
              WT_[p] += wf * wf;
              RE[p] += uf * wf;
              DT[p] += df * df;
            }
          }
      /* the reference normalises a fine block over k = 0..zdf-1 and the coarse over 2..zdc-3 */
      int d0 = g == 1 ? segs[g].off + 2 : segs[g].off, d1 = g == 1 ? segs[g].off + zdc - 2 : segs[g].off + zdf;
      double norm = (double)(ex * ey * 1 * 1);
      for (int p = d0; p < d1; p++) {
        if (pass == 0) {
          U[p] /= norm;
          Vv[p] /= norm;
          Wv[p] /= norm;
          DA[p] /= norm;
        } else {
          UT[p] /= norm;
          VT[p] /= norm;
          WT_[p] /= norm;
          RE[p] /= norm;
          DT[p] /= norm;
        }
      }
    }
  }
  for (int p = 0; p < NZ; p++) {
    UT[p] = sqrt(UT[p]);
    VT[p] = sqrt(VT[p]);
    WT_[p] = sqrt(WT_[p]);
    DT[p] = sqrt(DT[p]);
  }
  return NZ;
}
