/*
 * dns_budget — the turbulence-statistics / kinetic-energy budget program on
 * the GPU, through the C ABI of dns_embed.h.  It stands in for the
 * reference's offline program (TKE-budget/computations,
 * budget-no-slip-mgrd.c:14-122), which runs in a subdirectory of the solver's
 * run: for every snapshot counter tst = TSTR, TSTR + DT, ..., TEND it reads
 * the solver's vel-* / den-* files of counter tst from the parent directory
 * (reading.c:35-200), computes the 52 profiles of budget2D.c and writes
 * turb-fld-2d.000.TTTT, vort-fluc-2d.000.TTTT and KE-Budget-2d.000.TTTT into
 * the current one; when tst is a multiple of 200 it also writes the
 * fluctuation plane ufl4.TTTT / vfl4.TTTT (uv_fluc.c, plane 4 of the lower
 * block).
 *
 *   dns_budget [-D definitions.h] [-F fields-dir] [-O output-dir] [--plan]
 *
 * The parameters are the budget program's definitions.h macros (grid, Rebs,
 * ub, TSTR, TEND, DT), read at run time.  -F is where the vel-* / den-* files
 * are (default .., as the reference reads them), -O where the profiles go
 * (default .); --plan prints the counters and the files each writes, without
 * a GPU.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dns_embed.h"

static void usage(void) {
  fprintf(stderr, "usage: dns_budget [-D definitions.h] [-F fields-dir] [-O output-dir] [--plan]\n");
}

/* DT of the budget program's definitions.h (not a solver parameter); 1 when
   the file does not define it */
static long read_dt(const char *path) {
  FILE *fp = fopen(path, "r");
  long dt = 1;
  char line[1024];
  while (fp && fgets(line, sizeof line, fp)) {
    const char *s = line;
    while (*s == ' ' || *s == '\t') s++;
    char name[64], val[64];
    if (strncmp(s, "#define", 7) == 0 && sscanf(s + 7, "%63s %63s", name, val) == 2 && !strcmp(name, "DT"))
      dt = strtol(val, NULL, 10);
  }
  if (fp) fclose(fp);
  return dt;
}

int main(int argc, char **argv) {
  const char *defs = "definitions.h", *fields = "..", *out = ".";
  int plan = 0;
  for (int a = 1; a < argc; a++) {
    if (!strcmp(argv[a], "--plan")) {
      plan = 1;
    } else if (a + 1 < argc && !strcmp(argv[a], "-D")) {
      defs = argv[++a];
    } else if (a + 1 < argc && !strcmp(argv[a], "-F")) {
      fields = argv[++a];
    } else if (a + 1 < argc && !strcmp(argv[a], "-O")) {
      out = argv[++a];
    } else {
      usage();
      return 2;
    }
  }
  dns_params p;
  int rc = dns_params_from_definitions(defs, &p);
  dns_geometry g;
  if (!rc) rc = dns_geometry_of(&p, &g);
  if (rc) {
    fprintf(stderr, "dns_budget: parameters: %s (%s)\n", dns_error_string(rc), dns_last_error());
    return 1;
  }
  const long dt = read_dt(defs);
  if (dt < 1) {
    fprintf(stderr, "dns_budget: DT must be positive\n");
    return 1;
  }
  if (plan) {
    for (long t = p.TSTR; t <= p.TEND; t += dt)
      printf("%04ld budget%s\n", t, t % 200 == 0 ? " fluctuation-plane" : "");
    return 0;
  }
  const size_t nprof = (size_t)DNS_TKE_NPROF * g.nz_profile, npl = (size_t)g.nxf * g.nyf;
  double *prof = (double *)malloc(nprof * sizeof(double));
  double *ufl = (double *)malloc(npl * sizeof(double));
  double *vfl = (double *)malloc(npl * sizeof(double));
  if (!prof || !ufl || !vfl) {
    fprintf(stderr, "dns_budget: out of host memory\n");
    return 1;
  }
  int status = 0;
  for (long t = p.TSTR; t <= p.TEND && !status; t += dt) {
    const int fluct = t % 200 == 0;
    rc = dns_tke_budget_files(&p, fields, (int)t, prof, ufl, vfl);
    if (!rc) rc = dns_write_tke_budget(&p, out, (int)t, prof, fluct ? ufl : NULL, fluct ? vfl : NULL);
    if (rc) {
      fprintf(stderr, "dns_budget: snapshot %04ld: %s (%s)\n", t, dns_error_string(rc), dns_last_error());
      status = 1;
    }
  }
  free(prof);
  free(ufl);
  free(vfl);
  return status;
}
