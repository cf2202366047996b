/*
 * dns_run — host driver of the B200 channel solver through the C ABI of
 * dns_embed.h.  It stands in for the reference's program (run-dns-mgrd,
 * DNS-solver-with-grid-embedding/src/dns-q-mgrd-all-patterns-xyc.c, main):
 * the same start modes, the same parameters (a reference-style
 * definitions.h, read at run time instead of compiled in), the same loop and
 * the same files, with one GPU in place of the MPI ranks.
 *
 *   dns_run -s|-i|-p [-D definitions.h] [-C dir] [-n steps] [--fp32]
 *                    [--seed N --uc U --amp A] [--plan]
 *
 *   -s  start from rest, as main's mode s (init.c: f = w at every non-solid
 *       node; the interface history left at zero, as main leaves it); with
 *       --seed/--uc/--amp a seeded laminar profile plus noise instead, its
 *       history set from that state;
 *   -i  start from a uniform-grid run's lbf.TSTR (main's mode i);
 *   -p  resume from the restart files of counter TSTR (main's mode p).
 *   -D  parameters (default ./definitions.h); -C  directory of every file read
 *   or written (default .); -n  number of loop iterations minus one, as
 *   #define ITER; --fp32  the FP32 deviation-storage form; --plan  print the
 *   loop's output schedule and exit (no GPU used).
 *
 * The loop (main :1254-1375): for ss = 0 .. up (up = ITER, else
 * (TEND - TSTR) utime), the logs of the pre-step state are appended to
 * flowrate.txt, density.txt (encalc2.c:135-144), str-up.txt, str-do.txt,
 * w-str.txt and p-grad.txt (wshearstr.c:145-166); when ss is a multiple of
 * utime the restart files (every 50 unit times, :1262-1341), the vel-* / den-*
 * files (vel_print, :1342) and the plane statistics turb-fld.000.TTT with
 * uavg-temp.dat and uavg-exact-lam.dat (statistics.c:303-351) of the
 * pre-step state are written under counter TM + ss / utime; then the step.
 * After the loop the statistics are written once more (:1381).  A non-finite
 * wall shear stress ends the run with status 1 (the reference aborts,
 * wshearstr.c:139-143).  report.code records the run (:1383-1421).
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "dns_embed.h"

typedef struct {
  char mode;               /* 's', 'i' or 'p' */
  const char *defs;        /* definitions.h */
  const char *dir;         /* directory of every file read or written */
  long steps;              /* -n: overrides the loop bound (>= 0), else -1 */
  int fp32;                /* --fp32 */
  int seeded;              /* --seed / --uc / --amp given */
  unsigned long long seed;
  double uc, amp;
  int plan;                /* --plan */
} options;

static void usage(FILE *to) {
  fprintf(to,
          "usage: dns_run -s|-i|-p [-D definitions.h] [-C dir] [-n steps] [--fp32]\n"
          "               [--seed N --uc U --amp A] [--plan]\n");
}

/* 0 on success, 2 on a usage error */
static int parse_args(int argc, char **argv, options *o) {
  memset(o, 0, sizeof *o);
  o->defs = "definitions.h";
  o->dir = ".";
  o->steps = -1;
  if (argc < 2 || argv[1][0] != '-' || argv[1][1] == '\0' || argv[1][2] != '\0') return 2;
  o->mode = argv[1][1];
  if (o->mode != 's' && o->mode != 'i' && o->mode != 'p') return 2;
  for (int a = 2; a < argc; a++) {
    const char *s = argv[a];
    const char *v = a + 1 < argc ? argv[a + 1] : NULL;
    char *end = NULL;
    if (!strcmp(s, "--fp32")) {
      o->fp32 = 1;
    } else if (!strcmp(s, "--plan")) {
      o->plan = 1;
    } else if (!v) {
      return 2;
    } else if (!strcmp(s, "-D")) {
      o->defs = v, a++;
    } else if (!strcmp(s, "-C")) {
      o->dir = v, a++;
    } else if (!strcmp(s, "-n")) {
      o->steps = strtol(v, &end, 10), a++;
      if (*end || o->steps < 0) return 2;
    } else if (!strcmp(s, "--seed")) {
      o->seed = strtoull(v, &end, 10), a++, o->seeded = 1;
      if (*end) return 2;
    } else if (!strcmp(s, "--uc")) {
      o->uc = strtod(v, &end), a++, o->seeded = 1;
      if (*end) return 2;
    } else if (!strcmp(s, "--amp")) {
      o->amp = strtod(v, &end), a++, o->seeded = 1;
      if (*end) return 2;
    } else {
      return 2;
    }
  }
  if (o->seeded && o->mode != 's') return 2;
  return 0;
}

/* ------------------------------------------------------------------ files */
static char *path_in(const char *dir, const char *name) {
  const size_t n = strlen(dir) + strlen(name) + 2;
  char *p = (char *)malloc(n);
  if (p) snprintf(p, n, "%s/%s", dir, name);
  return p;
}

/* the six per-step logs (encalc2.c:135-144, wshearstr.c:145-166), each
   opened in append mode at its first line and kept open for the run */
static const char *const kLogNames[6] = {"flowrate.txt", "density.txt", "str-up.txt",
                                         "str-do.txt",   "w-str.txt",   "p-grad.txt"};
typedef struct {
  const char *dir;
  FILE *fp[6];
} logs;

static int log_line(logs *L, int which, double t, double v) {
  if (!L->fp[which]) {
    char *p = path_in(L->dir, kLogNames[which]);
    L->fp[which] = p ? fopen(p, "a") : NULL;
    free(p);
    if (!L->fp[which]) return -1;
  }
  /* encalc2.c:138, wshearstr.c:149 */
  return fprintf(L->fp[which], "%f %.12f\n", t, v) > 0 ? 0 : -1;
}

static int append_logs(logs *L, const dns_step_log *r) {
  int rc = 0;
  rc |= log_line(L, 0, r->time, r->flowrate);
  rc |= log_line(L, 1, r->time, r->denst);
  if (isnan(r->stress)) return rc; /* the reference aborts before the wall logs (NaN only) */
  rc |= log_line(L, 2, r->time, r->stup);
  rc |= log_line(L, 3, r->time, r->stdown);
  rc |= log_line(L, 4, r->time, r->stress);
  rc |= log_line(L, 5, r->time, r->pgrad);
  return rc;
}

static int flush_logs(logs *L) {
  int rc = 0;
  for (int q = 0; q < 6; q++)
    if (L->fp[q] && fflush(L->fp[q]) != 0) rc = -1;
  return rc;
}

static int close_logs(logs *L) {
  int rc = 0;
  for (int q = 0; q < 6; q++)
    if (L->fp[q]) {
      if (fclose(L->fp[q]) != 0) rc = -1;
      L->fp[q] = NULL;
    }
  return rc;
}

/* statistics.c:303-351: the 9 x NZ record turb-fld.000.TTT (the rank field is
   0: one process holds the domain), the mean-velocity profile at the composite
   profile's z/H (uavg-temp.dat) and the laminar Poiseuille profile at every
   fine z/H (uavg-exact-lam.dat) */
static int write_statistics(dns_handle *h, const dns_params *p, const dns_geometry *g, const char *dir,
                            long ts) {
  const int NZ = g->nz_profile, zdf = g->zdf, zdc = g->nzc, GR = g->gr, NZs = g->nzs;
  const double H = (double)(NZs - 2.);
  double *rec = (double *)calloc((size_t)9 * NZ, sizeof(double));
  double *zps = (double *)calloc((size_t)NZ, sizeof(double));
  double *zpsf = (double *)calloc((size_t)NZs, sizeof(double));
  double *lam = (double *)calloc((size_t)NZs, sizeof(double));
  int rc = (!rec || !zps || !zpsf || !lam) ? -1 : 0;
  if (!rc && dns_plane_stats(h, rec) != DNS_OK) rc = 1;
  char name[64];
  snprintf(name, sizeof name, "turb-fld.%.3d.%.3ld", 0, ts);
  char *fn = rc ? NULL : path_in(dir, name);
  FILE *fp = fn ? fopen(fn, "wb") : NULL;
  free(fn);
  if (!rc && (!fp || fwrite(rec, sizeof(double), (size_t)9 * NZ, fp) != (size_t)9 * NZ)) rc = -1;
  if (fp && fclose(fp) != 0) rc = -1;
  if (!rc) {
    for (int k = 1; k < zdf; k++) zps[k] = k - 0.5;
    for (int k = 2; k < zdc - 2; k++) zps[zdf - 2 + k] = GR * (k - 1) + (zdf - 1 - 0.5);
    for (int k = 0; k < zdf - 1; k++) zps[zdf + zdc - 4 + k] = k + GR * (zdc - 3) + zdf - 1. - 0.5;
    zps[2 * zdf + zdc - 5] = 2 * zdf + GR * (zdc - 4) + GR - 3;
    for (int k = 0; k < NZ; k++) zps[k] /= H;
    for (int k = 1; k < NZs - 1; k++) lam[k] = -6. * p->ub * ((k - 0.5) / H) * ((k - 0.5) / H - 1);
    for (int k = 1; k < NZs - 1; k++) zpsf[k] = k - 0.5;
    zpsf[NZs - 1] = NZs - 2;
    for (int k = 0; k < NZs; k++) zpsf[k] /= H;
    fn = path_in(dir, "uavg-temp.dat");
    fp = fn ? fopen(fn, "w") : NULL;
    free(fn);
    if (!fp) rc = -1;
    for (int k = 0; fp && k < NZ; k++) fprintf(fp, "%.12f %.12f\n", zps[k], rec[k]);
    if (fp && fclose(fp) != 0) rc = -1;
    fn = path_in(dir, "uavg-exact-lam.dat");
    fp = fn ? fopen(fn, "w") : NULL;
    free(fn);
    if (!fp) rc = -1;
    for (int k = 0; fp && k < NZs; k++) fprintf(fp, "%.12f %.12f \n", zpsf[k], lam[k]);
    if (fp && fclose(fp) != 0) rc = -1;
  }
  free(rec);
  free(zps);
  free(zpsf);
  free(lam);
  return rc;
}

/* ------------------------------------------------------------------ schedule */
/* main :439-468: utime = (int)((0.5 (NZs - 2) / CFL) / GR) coarse steps per
   unit time; the loop runs ss = 0 .. up with up = ITER, else (TEND - TSTR) utime */
static long loop_bound(const dns_params *p, const dns_geometry *g, const options *o) {
  if (o->steps >= 0) return o->steps;
  if (p->ITER >= 0) return p->ITER;
  return (long)(p->TEND - p->TSTR) * (long)g->utime;
}

/* what iteration ss writes before its step: bit 1 restart, bit 2 fields and
   statistics */
static int outputs_at(long ss, long utime) {
  if (ss % utime) return 0;
  return 2 | ((ss % (50 * utime)) == 0 ? 1 : 0);
}

static void print_plan(const dns_params *p, const dns_geometry *g, const options *o) {
  const long up = loop_bound(p, g, o), ut = g->utime;
  printf("mode %c utime %ld iterations %ld (steps 0..%ld)\n", o->mode, ut, up + 1, up);
  for (long ss = 0; ss <= up; ss++) {
    const int w = outputs_at(ss, ut);
    if (w & 1) printf("ss %ld restart %04ld\n", ss, p->TSTR + ss / ut);
    if (w & 2) printf("ss %ld fields %04ld statistics %03ld\n", ss, p->TSTR + ss / ut, p->TSTR + ss / ut);
  }
  printf("end statistics %03ld\n", p->TSTR + (up + 1) / ut);
}

/* ------------------------------------------------------------------ run */
static int fail_call(const char *what, int rc) {
  fprintf(stderr, "dns_run: %s: %s (%s)\n", what, dns_error_string(rc), dns_last_error());
  return 1;
}

static void write_report(const char *dir, const dns_params *p, const dns_geometry *g, const options *o, long up,
                         double seconds) {
  char *fn = path_in(dir, "report.code");
  FILE *fp = fn ? fopen(fn, "w") : NULL;
  free(fn);
  if (!fp) return;
  const char *pat[] = {"none", "RSLIP", "PSLIP", "SSLIP"};
  fprintf(fp, "coarse nodes %d x %d x %d, Reb=%f, tauc=%f, Ub=%f, CFLnumber=%f\n", g->nx, g->ny, g->nzc, p->Rebs,
          1. / g->omega_c, p->ub, p->CFL);
  fprintf(fp, "fine nodes per block %d x %d x %d, tauf=%f, GR=%d, NZs=%d\n", g->nxf, g->nyf, g->zdf,
          1. / g->omega_f, g->gr, g->nzs);
  fprintf(fp, "slip option: %s\n", pat[p->pattern >= 0 && p->pattern <= 3 ? p->pattern : 0]);
  fprintf(fp, "start mode: %c, precision: %s, one GPU (device %d)\n", o->mode, o->fp32 ? "FP32" : "FP64",
          p->device);
  fprintf(fp, "Total computational time is: %f s\n", seconds);
  fprintf(fp, "Unit non-dimensional time is: %d iterations\n", g->utime);
  fprintf(fp, "Loop iterations: %ld\n", up + 1);
  fprintf(fp, "Starting time: %d\n", p->TSTR);
  fprintf(fp, "Current Time is: %d\n", p->TEND);
  fprintf(fp, "node updates per coarse step: %lld, MLUPS: %f\n", g->updates_per_step,
          seconds > 0 ? (double)g->updates_per_step * (double)(up + 1) / seconds / 1e6 : 0.);
  fclose(fp);
}

static double now_seconds(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int main(int argc, char **argv) {
  options o;
  if (parse_args(argc, argv, &o)) {
    usage(stderr);
    return 2;
  }
  dns_params p;
  int rc = dns_params_from_definitions(o.defs, &p);
  if (rc) return fail_call("reading the parameters", rc);
  p.precision = o.fp32 ? DNS_FP32 : DNS_FP64;
  p.forcing = DNS_FORCING_CFR; /* main keeps encalc2's constant-flow-rate force */
  dns_geometry g;
  if ((rc = dns_geometry_of(&p, &g))) return fail_call("parameters", rc);
  if (g.utime < 1) {
    fprintf(stderr, "dns_run: utime = (0.5 (NZs - 2) / CFL) / GR is below one coarse step; lower CFL\n");
    return 1;
  }
  const long up = loop_bound(&p, &g, &o), ut = g.utime;
  if (o.plan) {
    print_plan(&p, &g, &o);
    return 0;
  }
  dns_handle *h = NULL;
  if ((rc = dns_create(&p, &h))) return fail_call("creating the channel", rc);
  switch (o.mode) {
    case 's':
      if (o.seeded) {
        rc = dns_init_seeded(h, o.seed, o.uc, o.amp);
      } else {
        /* init.c: f = w at the non-solid nodes (the seeded form with no flow and
           no noise is exactly that); the history stays zero as in main */
        rc = dns_init_seeded(h, 0, 0., 0.);
        if (!rc) {
          const size_t nh = (size_t)3 * 2 * g.nx * g.ny * 23;
          double *zero = (double *)calloc(nh, sizeof(double));
          rc = zero ? dns_import_history(h, zero) : DNS_ENOMEM;
          free(zero);
        }
      }
      break;
    case 'i':
      rc = dns_load_uniform(h, o.dir, p.TSTR);
      break;
    default:
      rc = dns_load_restart(h, o.dir, p.TSTR);
      break;
  }
  if (rc) {
    dns_destroy(h);
    return fail_call(o.mode == 's' ? "initial state" : (o.mode == 'i' ? "uniform-grid start" : "restart"), rc);
  }
  printf("dns_run: mode %c, %d x %d x %d coarse, GR %d, utime %ld, %ld iterations, %s\n", o.mode, g.nx, g.ny,
         g.nzc, g.gr, ut, up + 1, o.fp32 ? "FP32" : "FP64");
  dns_step_log *rows = (dns_step_log *)malloc(sizeof(dns_step_log) * (size_t)ut);
  if (!rows) {
    dns_destroy(h);
    fprintf(stderr, "dns_run: out of host memory\n");
    return 1;
  }
  logs L = {o.dir, {NULL, NULL, NULL, NULL, NULL, NULL}};
  const double t0 = now_seconds();
  int status = 0;
  for (long ss = 0; ss <= up && !status;) {
    const int w = outputs_at(ss, ut);
    const int cntr = p.TSTR + (int)(ss / ut);
    if ((w & 1) && (rc = dns_write_restart(h, o.dir, cntr))) status = fail_call("writing the restart files", rc);
    if (!status && (w & 2) && (rc = dns_write_fields(h, o.dir, cntr))) status = fail_call("writing the fields", rc);
    if (!status && (w & 2) && write_statistics(h, &p, &g, o.dir, (long)cntr))
      status = fail_call("writing the statistics", DNS_EIO);
    if (status) break;
    /* steps up to the next output boundary (or the end of the loop) in one call */
    const long n = (up + 1 - ss) < (ut - ss % ut) ? (up + 1 - ss) : (ut - ss % ut);
    rc = dns_step(h, n, rows);
    long done = rc == DNS_OK ? n : 0; /* any other failure leaves the rows unset */
    if (rc == DNS_ENAN) {
      done = 0;
      while (done < n && !isnan(rows[done].stress)) done++;
      if (done < n) done++; /* the failing step's flow-rate logs are written, as encalc2 runs first */
    }
    for (long q = 0; q < done && !status; q++)
      if (append_logs(&L, &rows[q])) status = fail_call("appending the logs", DNS_EIO);
    if (!status && flush_logs(&L)) status = fail_call("appending the logs", DNS_EIO);
    if (!status && rc == DNS_ENAN) {
      fprintf(stderr, "Error: NAN in wall shear stress (step %ld)\n", ss + done - 1);
      status = 1;
    } else if (!status && rc) {
      status = fail_call("step", rc);
    }
    ss += n;
  }
  if (close_logs(&L) && !status) status = fail_call("closing the logs", DNS_EIO);
  const double seconds = now_seconds() - t0;
  if (!status && write_statistics(h, &p, &g, o.dir, (long)p.TSTR + (up + 1) / ut))
    status = fail_call("writing the statistics", DNS_EIO);
  if (!status) write_report(o.dir, &p, &g, &o, up, seconds);
  free(rows);
  dns_destroy(h);
  if (!status)
    printf("dns_run: %ld iterations in %.3f s (%.1f MLUPS)\n", up + 1, seconds,
           seconds > 0 ? (double)g.updates_per_step * (double)(up + 1) / seconds / 1e6 : 0.);
  return status;
}
