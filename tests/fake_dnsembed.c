/*
 * A fake of libdnsembed's C ABI for testing the host driver dns_run without a
 * GPU — TEST INFRASTRUCTURE ONLY.  The channel is held by the oracle's CPU
 * restatement (oracle/dnsport.c, which is pinned to the reference); the
 * host-only calls (parameters, geometry, error strings) are forwarded to the
 * real library named by DNS_FAKE_REAL.  tests/test_driver.py builds it into a
 * temporary libdnsembed.so that the driver loads through LD_LIBRARY_PATH, so
 * that the driver's own work (modes, loop cadence, files, log lines) can be
 * compared with the unmodified reference main on the host.  The product never
 * loads it.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dns_embed.h"
#include "dnsport.h"

struct dns_handle {
  port_state *s;
  dns_params p;
  dns_geometry g;
  long ss;  /* coarse steps since the start */
};

static char g_err[512];

static void *real(const char *sym) {
  static void *lib;
  if (!lib) {
    const char *path = getenv("DNS_FAKE_REAL");
    lib = path ? dlopen(path, RTLD_NOW | RTLD_LOCAL) : NULL;
    if (!lib) {
      fprintf(stderr, "fake: cannot load the real library (DNS_FAKE_REAL)\n");
      exit(3);
    }
  }
  void *f = dlsym(lib, sym);
  if (!f) {
    fprintf(stderr, "fake: %s missing\n", sym);
    exit(3);
  }
  return f;
}

static int failf(int code, const char *msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

int dns_params_default(dns_params *p) { return ((int (*)(dns_params *))real("dns_params_default"))(p); }
int dns_params_from_definitions(const char *path, dns_params *p) {
  return ((int (*)(const char *, dns_params *))real("dns_params_from_definitions"))(path, p);
}
int dns_geometry_of(const dns_params *p, dns_geometry *g) {
  return ((int (*)(const dns_params *, dns_geometry *))real("dns_geometry_of"))(p, g);
}
const char *dns_error_string(int code) { return ((const char *(*)(int))real("dns_error_string"))(code); }
const char *dns_last_error(void) {
  return g_err[0] ? g_err : ((const char *(*)(void))real("dns_last_error"))();
}

int dns_create(const dns_params *p, dns_handle **out) {
  dns_geometry g;
  int rc = dns_geometry_of(p, &g);
  if (rc) return rc;
  port_cfg c = {p->xdv, p->ydv, p->zdv, p->zds, p->gratio, p->Rebs, p->ub, p->CFL, p->pattern,
                p->gyplussize, p->wyplussize, p->gxplussize, p->wxplussize, p->fltr};
  dns_handle *h = (dns_handle *)calloc(1, sizeof *h);
  if (!h || !(h->s = port_create(&c))) {
    free(h);
    return failf(DNS_ENOMEM, "fake: port_create");
  }
  h->p = *p;
  h->g = g;
  *out = h;
  return DNS_OK;
}

void dns_destroy(dns_handle *h) {
  if (!h) return;
  port_destroy(h->s);
  free(h);
}

int dns_init_seeded(dns_handle *h, uint64_t seed, double uc, double amp) {
  port_init_seeded(h->s, seed, uc, amp, 0.0);
  port_set_forcing(h->s, 1, 0.0);
  h->ss = 0;
  return DNS_OK;
}

int dns_import_history(dns_handle *h, const double *in) {
  port_import_history(h->s, in);
  return DNS_OK;
}

int dns_load_restart(dns_handle *h, const char *dir, int cntr) {
  if (port_load_restart(h->s, dir, cntr)) return failf(DNS_EIO, "fake: restart files");
  port_set_forcing(h->s, 1, 0.0);
  h->ss = 0;
  return DNS_OK;
}

int dns_load_uniform(dns_handle *h, const char *dir, int cntr) {
  const dns_params *p = &h->p;
  const size_t n = (size_t)19 * p->xdu * p->ydu * (p->zdu + 2);
  char fn[4096];
  snprintf(fn, sizeof fn, "%s/lbf.%.4d", dir, cntr);
  double *u = (double *)malloc(n * sizeof(double));
  FILE *fp = fopen(fn, "rb");
  const int ok = u && fp && fread(u, sizeof(double), n, fp) == n;
  if (fp) fclose(fp);
  const int rc = ok ? port_init_uniform(h->s, u, p->xdu, p->ydu, p->zdu) : -1;
  free(u);
  if (rc) return failf(ok ? DNS_EINVAL : DNS_EIO, "fake: uniform-grid start");
  port_set_forcing(h->s, 1, 0.0);
  h->ss = 0;
  return DNS_OK;
}

int dns_write_restart(dns_handle *h, const char *dir, int cntr) {
  return port_save_restart(h->s, dir, cntr) ? failf(DNS_EIO, "fake: writing restart files") : DNS_OK;
}

/* vel_print.c:95-125 on each level of the post-stream state */
int dns_write_fields(dns_handle *h, const char *dir, int cntr) {
  static const double EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0};
  static const double EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
  static const double EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  const char *names[3] = {"c", "slf", "suf"};
  for (int lvl = 0; lvl < 3; lvl++) {
    const long n = port_export(h->s, lvl, NULL);
    const size_t nodes = (size_t)n / 19;
    double *f = (double *)malloc((size_t)n * sizeof(double));
    double *vel = (double *)malloc(nodes * 3 * sizeof(double));
    double *den = (double *)malloc(nodes * sizeof(double));
    if (!f || !vel || !den) return failf(DNS_ENOMEM, "fake: fields");
    port_export(h->s, lvl, f);
    for (size_t c = 0; c < nodes; c++) {
      double ux = 0., uy = 0., uz = 0., dens = 0.;
      for (int a = 0; a < 19; a++) {
        ux += EX[a] * f[c * 19 + a];
        uy += EY[a] * f[c * 19 + a];
        uz += EZ[a] * f[c * 19 + a];
        dens += f[c * 19 + a];
      }
      if (dens > 0.) {
        ux /= dens;
        uy /= dens;
        uz /= dens;
      } else {
        ux = uy = uz = dens = 0.;
      }
      vel[3 * c] = ux;
      vel[3 * c + 1] = uy;
      vel[3 * c + 2] = uz;
      den[c] = dens;
    }
    char fn[4096];
    int bad = 0;
    snprintf(fn, sizeof fn, "%s/vel-%s.%.4d", dir, names[lvl], cntr);
    FILE *fp = fopen(fn, "wb");
    bad |= !fp || fwrite(vel, sizeof(double), nodes * 3, fp) != nodes * 3;
    if (fp) fclose(fp);
    snprintf(fn, sizeof fn, "%s/den-%s.%.4d", dir, names[lvl], cntr);
    fp = fopen(fn, "wb");
    bad |= !fp || fwrite(den, sizeof(double), nodes, fp) != nodes;
    if (fp) fclose(fp);
    free(f);
    free(vel);
    free(den);
    if (bad) return failf(DNS_EIO, "fake: writing fields");
  }
  return DNS_OK;
}

int dns_plane_stats(dns_handle *h, double *out) {
  return port_plane_stats(h->s, out) > 0 ? DNS_OK : failf(DNS_EINVAL, "fake: plane statistics");
}

/* time stamps as encalc2.c:31,138: TM + dt ss with dt = GR / (0.5 (NZs - 2) / CFL) */
int dns_step(dns_handle *h, long n, dns_step_log *log) {
  port_log *pl = (port_log *)malloc(sizeof(port_log) * (size_t)(n > 0 ? n : 1));
  if (!pl) return failf(DNS_ENOMEM, "fake: step");
  port_step(h->s, n, pl);
  const double dt = h->g.gr * 1. / ((double)(0.5 * (h->g.nzs - 2.) / h->p.CFL));
  int rc = DNS_OK;
  for (long q = 0; q < n; q++) {
    dns_step_log *o = &log[q];
    o->time = (double)h->p.TSTR + dt * (double)(h->ss + q);
    o->force = pl[q].force;
    o->momentum = pl[q].momentum;
    o->denst = pl[q].denst;
    o->flowrate = pl[q].flowrate;
    o->stup = pl[q].stup;
    o->stdown = pl[q].stdown;
    o->stress = pl[q].stress;
    o->pgrad = pl[q].pgrad;
    if (rc == DNS_OK && isnan(o->stress)) rc = failf(DNS_ENAN, "fake: NaN wall shear stress");
  }
  h->ss += n;
  free(pl);
  return rc;
}
