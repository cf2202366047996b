/*
 * Reference harness — TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * Links the reference solver's own, unmodified routines (compiled from
 * DNS-solver-with-grid-embedding/src/*.c against the single-rank MPI shim and a
 * per-configuration definitions.h, see oracle/build_ref.py) and drives them in
 * exactly the order of the reference main loop
 * (DNS-solver-with-grid-embedding/src/dns-q-mgrd-all-patterns-xyc.c:1254-1375):
 *
 *   encalc2 -> wshearstr -> [statistics] -> xcomputations ->
 *   (GR-1) x {xfcomputations, tinterpolate_hrmt, derivative x2, ctfdtransfer_opt, fexchange} ->
 *   xfcomputations, tinterpolate_hrmt(GR), derivative x2, ctfdtransfer_opt(GR),
 *   ftcdtransfer (ftcdtransfer_lesfltr when FLTR is defined, as main does at
 *   :1366-1372), exchange, fexchange
 *
 * The only departure from main is the forcing switch: in constant-force mode
 * force[0] is reset to the given value after encalc2 (which still runs, so the
 * flowrate/density logs are produced), where main keeps encalc2's
 * constant-flow-rate force.
 *
 * State is read from and written to restart files in the reference layout
 * (main :1003-1163 read, :1262-1341 write): lbf-c / lbf-slf / lbf-suf hold
 * [ftemp | f] in global C order (i, j, k, a); lbf-uin / lbf-lin hold the
 * [n | p | pp] interface history (i, j, 23); force holds force[0].
 *
 * usage: ref_harness INDIR CNTR_IN OUTDIR CNTR_OUT NSTEPS cfr|const [G] [STATS_EVERY] [FIELDS] [WARMUP]
 * (INDIR "-" starts from rest instead of reading restart files; CNTR_OUT < 0
 *  skips the restart output, for timing; FIELDS = 1 also writes the
 *  reference's vel-* / den-* field files of the final state with its own
 *  vel_print, as main does at :1342; WARMUP > 0 starts the clock after that
 *  many of the NSTEPS steps, so harness_seconds covers NSTEPS - WARMUP steps)
 * The step loop time (MPI_Wtime, as main's t2-t4) is printed as
 *   "harness_seconds <s>".
 */
#include "definitions.h"
#include "fun_defs.h"

#include <unistd.h>

static void die(const char *msg, const char *arg) {
  fprintf(stderr, "ref_harness: %s %s\n", msg, arg ? arg : "");
  exit(2);
}

static DP *xcalloc(size_t n) {
  DP *p = (DP *)calloc(n, sizeof(DP));
  if (!p) die("out of memory", NULL);
  return p;
}

/* one population array with the per-rank trailing ghost column/row */
static void read_lattice(const char *path, DP *ftemp, DP *f, int nx, int ny, int nz) {
  FILE *fp = fopen(path, "rb");
  if (!fp) die("cannot open", path);
  int xd = nx + 1, yd = ny + 1;
  DP *dst[2] = {ftemp, f};
  for (int h = 0; h < 2; h++)
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++) {
        DP *p = dst[h] + ((size_t)i * yd * nz + (size_t)j * nz) * 19;
        if (fread(p, sizeof(DP), (size_t)nz * 19, fp) != (size_t)nz * 19) die("short read", path);
      }
  fclose(fp);
  /* ghost column i = nx and ghost row j = ny duplicate i = 0 / j = 0 (periodic) */
  for (int h = 0; h < 2; h++) {
    DP *a = dst[h];
    for (int j = 0; j < yd; j++) {
      int js = (j == ny) ? 0 : j;
      memcpy(a + ((size_t)nx * yd * nz + (size_t)j * nz) * 19, a + ((size_t)0 * yd * nz + (size_t)js * nz) * 19,
             sizeof(DP) * (size_t)nz * 19);
    }
    for (int i = 0; i < nx; i++)
      memcpy(a + ((size_t)i * yd * nz + (size_t)ny * nz) * 19, a + ((size_t)i * yd * nz) * 19,
             sizeof(DP) * (size_t)nz * 19);
  }
}

static void write_lattice(const char *path, const DP *ftemp, const DP *f, int nx, int ny, int nz) {
  FILE *fp = fopen(path, "wb");
  if (!fp) die("cannot create", path);
  int yd = ny + 1;
  const DP *src[2] = {ftemp, f};
  for (int h = 0; h < 2; h++)
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++) {
        const DP *p = src[h] + ((size_t)i * yd * nz + (size_t)j * nz) * 19;
        if (fwrite(p, sizeof(DP), (size_t)nz * 19, fp) != (size_t)nz * 19) die("short write", path);
      }
  fclose(fp);
}

/* interface plane: (xdc+5) x (ydc+5) x 23, logical i in [-2, xdc+2] */
static void fill_plane_halo(DP *pl, int xdc, int ydc) {
  int nx = xdc - 1, ny = ydc - 1;
  for (int i = -2; i < xdc + 3; i++)
    for (int j = -2; j < ydc + 3; j++) {
      int is = ((i % nx) + nx) % nx, js = ((j % ny) + ny) % ny;
      if (is == i && js == j) continue;
      for (int b = 0; b < 23; b++)
        Fbi(pl, i, j, 0, b, xdc, ydc, 4, 23) = Fbi(pl, is, js, 0, b, xdc, ydc, 4, 23);
    }
}

static void read_history(const char *path, DP *n, DP *p, DP *pp, int xdc, int ydc) {
  FILE *fp = fopen(path, "rb");
  if (!fp) die("cannot open", path);
  DP *dst[3] = {n, p, pp};
  for (int h = 0; h < 3; h++) {
    for (int i = 0; i < xdc - 1; i++)
      for (int j = 0; j < ydc - 1; j++)
        if (fread(&Fbi(dst[h], i, j, 0, 0, xdc, ydc, 4, 23), sizeof(DP), 23, fp) != 23) die("short read", path);
    fill_plane_halo(dst[h], xdc, ydc);
  }
  fclose(fp);
}

static void write_history(const char *path, DP *n, DP *p, DP *pp, int xdc, int ydc) {
  FILE *fp = fopen(path, "wb");
  if (!fp) die("cannot create", path);
  DP *src[3] = {n, p, pp};
  for (int h = 0; h < 3; h++)
    for (int i = 0; i < xdc - 1; i++)
      for (int j = 0; j < ydc - 1; j++)
        if (fwrite(&Fbi(src[h], i, j, 0, 0, xdc, ydc, 4, 23), sizeof(DP), 23, fp) != 23) die("short write", path);
  fclose(fp);
}

int main(int argc, char **argv) {
  if (argc < 7) die("usage: INDIR CNTR_IN OUTDIR CNTR_OUT NSTEPS cfr|const [G] [STATS_EVERY] [FIELDS] [WARMUP]", NULL);
  const char *indir = argv[1], *outdir = argv[3];
  int cin = atoi(argv[2]), cout = atoi(argv[4]);
  long nsteps = atol(argv[5]);
  int cfr = strcmp(argv[6], "cfr") == 0;
  /* strtod parses hex floats, so the force can be passed bit-exactly */
  double gconst = argc > 7 ? strtod(argv[7], NULL) : 0.0;
  long stats_every = argc > 8 ? atol(argv[8]) : 0;
  int fields = argc > 9 ? atoi(argv[9]) : 0;
  long warmup = argc > 10 ? atol(argv[10]) : 0;
  if (warmup < 0 || warmup >= nsteps) warmup = 0;

  int dims[2] = {XDIM, YDIM}, period[2] = {1, 1};
  MPI_Init(&argc, &argv);
  MPI_Cart_create(MPI_COMM_WORLD, 2, dims, period, 1, &cart_grid);
  PDATA pd;
  memset(&pd, 0, sizeof(pd));
  POINTER V;
  memset(&V, 0, sizeof(V));
  PI = 4. * atan(1.);

  int GR = gratio;
  int xdc = 1 + (xdv / XDIM), ydc = 1 + (ydv / YDIM), zdc = zdv;
  int xdf = GR * (xdc - 1) + 1, ydf = GR * (ydc - 1) + 1, zdf = zds + 1;
  int NZs = 2 * zdf + GR * (zdc - 4) + GR - 1;
  DP Reb = Rebs, ubulk = ub;
  /* relaxation rates exactly as main computes them (:447-451) */
  DP tauf = (3. / Reb) * ubulk * (NZs - 2.) + 0.5;
  DP tauc = (1. / ((double)GR)) * (3. / Reb) * ubulk * (NZs - 2.) + 0.5;
  tauf = 1. / tauf;
  tauc = 1. / tauc;

  size_t nc = (size_t)xdc * ydc * zdc, nf = (size_t)xdf * ydf * zdf, ni = (size_t)23 * (ydc + 5) * (xdc + 5);
  V.s = (int *)calloc(nc, sizeof(int));
  V.sus = (int *)calloc(nf, sizeof(int));
  V.sls = (int *)calloc(nf, sizeof(int));
  V.f = xcalloc(nc * 19);
  V.ftemp = xcalloc(nc * 19);
  V.suf = xcalloc(nf * 19);
  V.suftemp = xcalloc(nf * 19);
  V.slf = xcalloc(nf * 19);
  V.slftemp = xcalloc(nf * 19);
  V.rightbufs = xcalloc(5 * (size_t)ydc * zdc);
  V.rightbufr = xcalloc(5 * (size_t)ydc * zdc);
  V.leftbufs = xcalloc(5 * (size_t)ydc * zdc);
  V.leftbufr = xcalloc(5 * (size_t)ydc * zdc);
  V.upbufs = xcalloc(5 * (size_t)xdc * zdc);
  V.upbufr = xcalloc(5 * (size_t)xdc * zdc);
  V.dwbufs = xcalloc(5 * (size_t)xdc * zdc);
  V.dwbufr = xcalloc(5 * (size_t)xdc * zdc);
  V.urbufs = xcalloc(9 * (size_t)zdc);
  V.dlbufr = xcalloc(9 * (size_t)zdc);
  V.dlbufs = xcalloc(9 * (size_t)zdc);
  V.urbufr = xcalloc(9 * (size_t)zdc);
#define FINE_BUFS(P)                                  \
  V.P##rightbufs = xcalloc(5 * (size_t)ydf * zdf);    \
  V.P##rightbufr = xcalloc(5 * (size_t)ydf * zdf);    \
  V.P##leftbufs = xcalloc(5 * (size_t)ydf * zdf);     \
  V.P##leftbufr = xcalloc(5 * (size_t)ydf * zdf);     \
  V.P##upbufs = xcalloc(5 * (size_t)xdf * zdf);       \
  V.P##upbufr = xcalloc(5 * (size_t)xdf * zdf);       \
  V.P##dwbufs = xcalloc(5 * (size_t)xdf * zdf);       \
  V.P##dwbufr = xcalloc(5 * (size_t)xdf * zdf);       \
  V.P##urbufs = xcalloc(9 * (size_t)zdf);             \
  V.P##dlbufr = xcalloc(9 * (size_t)zdf);             \
  V.P##dlbufs = xcalloc(9 * (size_t)zdf);             \
  V.P##urbufr = xcalloc(9 * (size_t)zdf);
  FINE_BUFS(sl)
  FINE_BUFS(su)
  V.lin = xcalloc(ni);
  V.linp = xcalloc(ni);
  V.linpp = xcalloc(ni);
  V.uin = xcalloc(ni);
  V.uinp = xcalloc(ni);
  V.uinpp = xcalloc(ni);
  V.lint = xcalloc(ni * 4);
  V.uint = xcalloc(ni * 4);

  /* persistent halo channels: same buffers, peers and tags as main (:896-942);
     with one rank every peer is rank 0 */
  const int tagl = 1, tagr = 2;
#define CHANNELS(REQ, LB_S, RB_S, LB_R, RB_R, DB_S, UB_S, DB_R, UB_R, UR_S, DL_R, DL_S, UR_R, NY, NX, NZ) \
  MPI_Send_init(LB_S, 5 * NY * NZ, MPDP, 0, tagl, MPI_COMM_WORLD, &REQ[0]);                               \
  MPI_Send_init(RB_S, 5 * NY * NZ, MPDP, 0, tagr, MPI_COMM_WORLD, &REQ[1]);                               \
  MPI_Recv_init(LB_R, 5 * NY * NZ, MPDP, 0, tagr, MPI_COMM_WORLD, &REQ[2]);                               \
  MPI_Recv_init(RB_R, 5 * NY * NZ, MPDP, 0, tagl, MPI_COMM_WORLD, &REQ[3]);                               \
  MPI_Send_init(DB_S, 5 * NX * NZ, MPDP, 0, tagl, MPI_COMM_WORLD, &REQ[4]);                               \
  MPI_Send_init(UB_S, 5 * NX * NZ, MPDP, 0, tagr, MPI_COMM_WORLD, &REQ[5]);                               \
  MPI_Recv_init(DB_R, 5 * NX * NZ, MPDP, 0, tagr, MPI_COMM_WORLD, &REQ[6]);                               \
  MPI_Recv_init(UB_R, 5 * NX * NZ, MPDP, 0, tagl, MPI_COMM_WORLD, &REQ[7]);                               \
  MPI_Send_init(UR_S, 9 * NZ, MPDP, 0, tagl, MPI_COMM_WORLD, &REQ[8]);                                    \
  MPI_Recv_init(DL_R, 9 * NZ, MPDP, 0, tagl, MPI_COMM_WORLD, &REQ[9]);                                    \
  MPI_Send_init(DL_S, 9 * NZ, MPDP, 0, tagr, MPI_COMM_WORLD, &REQ[10]);                                   \
  MPI_Recv_init(UR_R, 9 * NZ, MPDP, 0, tagr, MPI_COMM_WORLD, &REQ[11]);
  CHANNELS(V.req, V.leftbufs, V.rightbufs, V.leftbufr, V.rightbufr, V.dwbufs, V.upbufs, V.dwbufr, V.upbufr,
           V.urbufs, V.dlbufr, V.dlbufs, V.urbufr, ydc, xdc, zdc)
  CHANNELS(V.slreq, V.slleftbufs, V.slrightbufs, V.slleftbufr, V.slrightbufr, V.sldwbufs, V.slupbufs,
           V.sldwbufr, V.slupbufr, V.slurbufs, V.sldlbufr, V.sldlbufs, V.slurbufr, ydf, xdf, zdf)
  CHANNELS(V.sureq, V.suleftbufs, V.surightbufs, V.suleftbufr, V.surightbufr, V.sudwbufs, V.suupbufs,
           V.sudwbufr, V.suupbufr, V.suurbufs, V.sudlbufr, V.sudlbufs, V.suurbufr, ydf, xdf, zdf)

  char fn[4096];
  int cold = strcmp(indir, "-") == 0;
  if (cold) goto cold_start;
  snprintf(fn, sizeof fn, "%s/lbf-c.%.4d", indir, cin);
  read_lattice(fn, V.ftemp, V.f, xdc - 1, ydc - 1, zdc);
  snprintf(fn, sizeof fn, "%s/lbf-slf.%.4d", indir, cin);
  read_lattice(fn, V.slftemp, V.slf, xdf - 1, ydf - 1, zdf);
  snprintf(fn, sizeof fn, "%s/lbf-suf.%.4d", indir, cin);
  read_lattice(fn, V.suftemp, V.suf, xdf - 1, ydf - 1, zdf);
  snprintf(fn, sizeof fn, "%s/force.%.4d", indir, cin);
  {
    FILE *fp = fopen(fn, "rb");
    if (!fp || fread(&V.force[0], sizeof(DP), 1, fp) != 1) die("cannot read", fn);
    fclose(fp);
  }
  snprintf(fn, sizeof fn, "%s/lbf-uin.%.4d", indir, cin);
  read_history(fn, V.uin, V.uinp, V.uinpp, xdc, ydc);
  snprintf(fn, sizeof fn, "%s/lbf-lin.%.4d", indir, cin);
  read_history(fn, V.lin, V.linp, V.linpp, xdc, ydc);

cold_start:
  V = solid_init(xdc, ydc, zdc, xdf, ydf, zdf, V);
#ifdef RSLIP
  V = slip_ridges_init(xdf, ydf, zdf, V, pd);
#endif
#ifdef PSLIP
  V = slip_posts_init(xdf, ydf, zdf, V, pd);
#endif
#ifdef SSLIP
  V = slip_spanwise_init(xdf, ydf, zdf, V, pd);
#endif

  if (cold) {
    /* INDIR "-": the reference's own cold start (mode -s, init.c: f = w at
       every non-solid node) with the interface history set to that state's
       [rho, u, fneq] = [1, 0, 0, 0, 0...] on all three levels */
    V = init(xdc, ydc, zdc, xdf, ydf, zdf, V);
    DP *lv[6] = {V.lin, V.linp, V.linpp, V.uin, V.uinp, V.uinpp};
    for (int q = 0; q < 6; q++)
      for (int i = -2; i < xdc + 3; i++)
        for (int j = -2; j < ydc + 3; j++) Fbi(lv[q], i, j, 0, 0, xdc, ydc, 4, 23) = 1.0;
    V.force[0] = gconst;
  }
  if (chdir(outdir) != 0) die("cannot enter", outdir);
  int TM = cin;
  DP Gx = 0.;
  double t4 = MPI_Wtime();
  for (long ss = 0; ss < nsteps; ss++) {
    if (ss == warmup && warmup > 0) t4 = MPI_Wtime();
    V = encalc2(xdc, ydc, zdc, xdf, ydf, zdf, GR, V, pd, TM, ss, ubulk);
    if (!cfr) V.force[0] = gconst;
    V = wshearstr(xdf, ydf, zdf, zdc, GR, V, pd, tauf, TM, ss);
    if (stats_every > 0 && ss % stats_every == 0)
      V = statistics(xdf, ydf, zdf, xdc, ydc, zdc, V, pd, (long)(TM + ss / stats_every), GR);
    V = xcomputations(xdc, ydc, zdc, GR, V, pd, Gx, tauc, ubulk);
    for (int iter = 1; iter < GR; iter++) {
      V = xfcomputations(xdf, ydf, zdf, (1. / ((double)GR)), V, pd, tauf, ubulk);
      V = tinterpolate_hrmt(xdc, ydc, zdc, V, iter, GR);
      derivative(xdc, ydc, V.uint);
      derivative(xdc, ydc, V.lint);
      V = ctfdtransfer_opt(xdc, ydc, zdc, xdf, ydf, zdf, iter, tauc, tauf, GR, V, pd);
      V = fexchange(V);
    }
    V = xfcomputations(xdf, ydf, zdf, (1. / ((double)GR)), V, pd, tauf, ubulk);
    V = tinterpolate_hrmt(xdc, ydc, zdc, V, GR, GR);
    derivative(xdc, ydc, V.uint);
    derivative(xdc, ydc, V.lint);
    V = ctfdtransfer_opt(xdc, ydc, zdc, xdf, ydf, zdf, GR, tauc, tauf, GR, V, pd);
#ifdef FLTR
    V = ftcdtransfer_lesfltr(xdf, ydf, zdf, xdc, ydc, zdc, GR, tauc, tauf, GR, V, pd);
#else
    V = ftcdtransfer(xdc, ydc, zdc, xdf, ydf, zdf, GR, tauc, tauf, GR, V, pd);
#endif
    V = exchange(V);
    V = fexchange(V);
  }
  double t2 = MPI_Wtime();
  printf("harness_seconds %.9f\n", t2 - t4);

  if (cout < 0) { /* timing run: no restart output */
    MPI_Finalize();
    return 0;
  }
  /* main writes a restart at the top of an iteration, after encalc2 has set the
     force for the state it is about to write (:1256-1306); do the same */
  V = encalc2(xdc, ydc, zdc, xdf, ydf, zdf, GR, V, pd, TM, nsteps, ubulk);
  if (!cfr) V.force[0] = gconst;
  snprintf(fn, sizeof fn, "lbf-c.%.4d", cout);
  write_lattice(fn, V.ftemp, V.f, xdc - 1, ydc - 1, zdc);
  snprintf(fn, sizeof fn, "lbf-slf.%.4d", cout);
  write_lattice(fn, V.slftemp, V.slf, xdf - 1, ydf - 1, zdf);
  snprintf(fn, sizeof fn, "lbf-suf.%.4d", cout);
  write_lattice(fn, V.suftemp, V.suf, xdf - 1, ydf - 1, zdf);
  snprintf(fn, sizeof fn, "force.%.4d", cout);
  {
    FILE *fp = fopen(fn, "wb");
    if (!fp || fwrite(&V.force[0], sizeof(DP), 1, fp) != 1) die("cannot write", fn);
    fclose(fp);
  }
  snprintf(fn, sizeof fn, "lbf-uin.%.4d", cout);
  write_history(fn, V.uin, V.uinp, V.uinpp, xdc, ydc);
  snprintf(fn, sizeof fn, "lbf-lin.%.4d", cout);
  write_history(fn, V.lin, V.linp, V.linpp, xdc, ydc);
  if (fields) V = vel_print(xdf, ydf, zdf, xdc, ydc, zdc, V, (long)cout);
  MPI_Finalize();
  return 0;
}
