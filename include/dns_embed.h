/*
 * dns_embed.h — C ABI of the B200 grid-embedded D3Q19 channel solver.
 *
 * Drop-in for the time-step path of the reference solver
 * (arstgr/DNS-solvers-with-grid-embedding, DNS-solver-with-grid-embedding/src/).
 * The reference is one monolithic C/MPI program with no library API; its
 * boundaries are the compile-time macros in src/definitions.h, the restart and
 * output files, and the routines called by main's loop.  Each entry point below
 * names the reference code it replaces.
 *
 * Conventions
 *   - Every call returns an int status: DNS_OK (0) or a negative DNS_E* code.
 *     Nothing crosses the ABI as an exception.  dns_error_string() describes a
 *     code; dns_last_error() gives the message of the last failure on the
 *     calling thread.
 *   - A handle owns all device memory of one channel.  Caller buffers are only
 *     borrowed for the duration of a call.  One host thread per handle.
 *   - Populations use the reference's D3Q19 order (src/globals.c:6-8) and the
 *     reference axes: x streamwise (i), y spanwise (j), z wall-normal (k).
 *   - The reference stores the relaxation RATE in variables named tau*; here
 *     omega_c / omega_f are rates (1 / relaxation time).
 */
#ifndef DNS_EMBED_H
#define DNS_EMBED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DNS_OK 0
#define DNS_EINVAL (-1)   /* bad argument or unsupported parameter combination */
#define DNS_ENOMEM (-2)   /* device or host allocation failed / over budget */
#define DNS_EIO (-3)      /* restart or output file missing, short or unwritable */
#define DNS_ENAN (-4)     /* NaN wall shear stress (reference aborts); batched: non-finite */
#define DNS_ETIMEOUT (-5) /* a bounded wait gave up (the request loop's deadline) */
#define DNS_ECUDA (-6)    /* CUDA runtime error */

enum dns_pattern { DNS_PATTERN_NONE = 0, DNS_PATTERN_RSLIP = 1, DNS_PATTERN_PSLIP = 2, DNS_PATTERN_SSLIP = 3 };
enum dns_forcing { DNS_FORCING_CFR = 0, DNS_FORCING_CONST = 1 };
enum dns_precision { DNS_FP64 = 0, DNS_FP32 = 1 };

/* Solver parameters.  The first block mirrors the macros of the reference's
   src/definitions.h:34-119 (same names, same meaning); XDIM/YDIM are accepted
   and ignored because one GPU holds the whole domain.  The second block holds
   run-time options that the reference sets by editing source. */
typedef struct dns_params {
  double Rebs;      /* bulk Reynolds number on the full height (definitions.h:34) */
  double ub;        /* bulk velocity, lattice units (definitions.h:35) */
  int zdv;          /* coarse wall-normal nodes incl. the two overlap planes (zdc) */
  int ydv;          /* spanwise coarse nodes */
  int xdv;          /* streamwise coarse nodes */
  int TSTR, TEND;   /* start / end in unit times (log time stamps, file counters) */
  double CFL;       /* sets utime, the number of coarse steps per unit time */
  int gratio;       /* coarse / fine grid ratio GR (>= 2) */
  int zds;          /* fine wall-normal nodes per block (zdf = zds + 1 incl. wall) */
  int gyplussize, wyplussize, gxplussize, wxplussize; /* wall pattern, fine cells */
  int pattern;      /* enum dns_pattern: RSLIP / PSLIP / SSLIP / none (definitions.h:69-71) */
  int XDIM, YDIM;   /* reference rank grid; ignored */
  long ITER;        /* fixed iteration count, < 0 when undefined (definitions.h:98) */
  /* run-time options */
  int forcing;          /* enum dns_forcing: constant flow rate (encalc2) or constant force */
  double force_const;   /* coarse-unit body force g when forcing == DNS_FORCING_CONST */
  int precision;        /* enum dns_precision */
  int device;           /* CUDA device ordinal */
  /* uniform grid of a mode -i start (definitions.h:103-109): xdu x ydu x (zdu + 2) */
  int xdu, ydu, zdu;
  /* 1 when FLTR is defined (definitions.h:87-88): the filtered fine-to-coarse
     transfer of ftcdtransfer_lesfltr.c instead of ftcdtransfer.c.  The
     reference defines it for gratio 4 (its stencil array holds gratio + 1 = 5
     planes) and it needs zds >= 7; other combinations are DNS_EINVAL. */
  int fltr;
} dns_params;

/* Derived sizes; computed on the host, no GPU needed. */
typedef struct dns_geometry {
  int nx, ny, nzc;          /* coarse nodes (xdv, ydv, zdc) */
  int nxf, nyf, zdf;        /* fine nodes per block: GR xdv, GR ydv, zds + 1 (wall incl.) */
  int gr;                   /* grid ratio */
  int nzs;                  /* NZs: wall-normal fine extent incl. the 2 wall nodes */
  int nz_profile;           /* NZ of the composite statistics profile: 2 zdf + zdc - 4 */
  int utime;                /* coarse steps per unit time */
  double omega_c, omega_f;  /* relaxation rates as the reference computes them */
  long long updates_per_step; /* xdv ydv zdc + 2 GR (GR xdv)(GR ydv) zds */
  long long device_bytes;   /* HBM the handle allocates */
} dns_geometry;

/* One coarse step's log values, computed on the pre-step state S_n exactly as
   the reference's encalc2.c:109-144 and wshearstr.c:67-166 define them. */
typedef struct dns_step_log {
  double time;      /* TM + dt * step, the reference's log time stamp */
  double force;     /* force[0] used by this step */
  double momentum;  /* normalised streamwise momentum (encalc2) */
  double denst;     /* normalised mass (density.txt) */
  double flowrate;  /* momentum (ydf-1)(NZs-2) / denst (flowrate.txt) */
  double stup, stdown, stress, pgrad; /* str-up / str-do / w-str / p-grad */
} dns_step_log;

typedef struct dns_handle dns_handle;

/* ---- parameters (host only) ------------------------------------------- */
/* Reference defaults: src/definitions.h with XDIM = YDIM = 1, CFR forcing, FP64. */
int dns_params_default(dns_params *p);
/* Parse a reference-style definitions.h ("#define NAME value" lines and the
   RSLIP/PSLIP/SSLIP/ITER switches), replacing src/definitions.h:34-119. */
int dns_params_from_definitions(const char *path, dns_params *p);
/* Sizes and rates of dns-q-mgrd-all-patterns-xyc.c:139-155,439-451. */
int dns_geometry_of(const dns_params *p, dns_geometry *g);

/* ---- lifecycle ------------------------------------------------------------ */
/* Allocate one channel on p->device (replaces main's calloc block :473-883 and
   the wall flags of solid_init.c + slip_*_init.c). */
int dns_create(const dns_params *p, dns_handle **out);
void dns_destroy(dns_handle *h);
/* Launch subsequent work on this CUDA stream (cudaStream_t passed as void*);
   NULL selects the handle's own stream. */
int dns_set_stream(dns_handle *h, void *cuda_stream);
int dns_get_geometry(const dns_handle *h, dns_geometry *g);

/* ---- state ------------------------------------------------------------------ */
/* Mode -p restart read: lbf-c, lbf-slf, lbf-suf, force, lbf-uin, lbf-lin with
   counter cntr (dns-q-mgrd-all-patterns-xyc.c:999-1163). */
int dns_load_restart(dns_handle *h, const char *dir, int cntr);
/* Restart write in the same layout (:1262-1341). */
int dns_write_restart(dns_handle *h, const char *dir, int cntr);
/* Seeded start: rho = 1, laminar profile 4 uc zeta (1 - zeta) plus Philox4x32-10
   uniform perturbations in [-amp, amp] per component, f = feq; interface
   history [rho, u, 0...] on all three levels (the state inter_init.c builds).
   Replaces mode -s (init.c), which starts from rest. */
int dns_init_seeded(dns_handle *h, uint64_t seed, double uc, double amp);
/* Mode -i start (dns-q-mgrd-all-patterns-xyc.c:978-997): read the uniform-grid
   state lbf.cntr (its first half, (xdu, ydu, zdu + 2, 19) in C order) from dir,
   interpolate it onto the coarse and both fine grids by 3-D quadratic Lagrange
   interpolation with the non-equilibrium part rescaled to each grid
   (initializer.c:303-533, sp_interpolate_qd.c), and build the interface history
   from the coarse state (inter_init.c), with levels p and pp equal to n and
   each wall's history holding its own plane's moments (the reference copies 19
   of every 23 fields into p and pp, inter_init.c:237-248, and writes the upper
   plane's density and velocity into the lower history, inter_init.c:202-205).
   DNS_EINVAL when a stencil would leave the reference's periodic halo (a
   uniform grid too short for the channel); DNS_EIO when the file is missing or
   shorter than one lattice. */
int dns_load_uniform(dns_handle *h, const char *dir, int cntr);
/* ---- turbulence statistics and kinetic-energy budget ----------------------
   The reference's offline program TKE-budget/computations (budget-no-slip-mgrd.c
   loop body :95-105: budget2D.c:13-1736, uv_fluc.c:15-49) on the device, for one
   snapshot.  prof receives DNS_TKE_NPROF profiles of NZ = 2 zdf + zdc - 4 points
   (dns_geometry.nz_profile), in the order of the three files the reference
   writes: turb-fld-2d (UAVG VAVG WAVG UTIN VTIN WTIN uw DAVG DTIN SKEWu SKEWv
   SKEWw SKEWuw SKEWp KURTu KURTv KURTw KURTuw KURTp), vort-fluc-2d (wx wy wz),
   KE-Budget-2d (Pii Puu Pvv Pww Puw Tiir Tuur Tvvr Twwr Tuwr Tiipai Tuupai
   Tvvpai Twwpai Tuwpai Paiuu Paivv Paiww Paiuw Tiis Tuus Tvvs Twws Tuws Epii
   Epuu Epvv Epww Epuw KE).  ufl / vfl (may be NULL) receive the u / v
   fluctuations of the lower fine plane k = 4, [GR xdv][GR ydv] (uv_fluc's
   ufl4 / vfl4).  Needs zds >= 5, zdv >= 7, xdv and ydv >= 4 (DNS_EINVAL). */
#define DNS_TKE_NPROF 52
/* from the handle's current state (the fields vel_print would write) */
int dns_tke_budget(dns_handle *h, double *prof, double *ufl, double *vfl);
/* from vel-c/slf/suf.cntr and den-c/slf/suf.cntr in dir (reading.c:14-226);
   runs on GPU p->device */
int dns_tke_budget_files(const dns_params *p, const char *dir, int cntr, double *prof, double *ufl, double *vfl);
/* turb-fld-2d.000.cntr, vort-fluc-2d.000.cntr, KE-Budget-2d.000.cntr and, when
   ufl / vfl are given, ufl4.cntr / vfl4.cntr (budget2D.c:1553-1641,
   uv_fluc.c:35-46), native doubles */
int dns_write_tke_budget(const dns_params *p, const char *dir, int cntr, const double *prof, const double *ufl,
                         const double *vfl);

/* Post-stream state S in reference AoS order f[i][j][k][a] of the global domain:
   level 0 coarse (xdv, ydv, zdc, 19), 1 lower fine, 2 upper fine
   ((GR xdv), (GR ydv), zdf, 19).  out must hold that many doubles. */
int dns_export_state(dns_handle *h, int level, double *aos_out);
int dns_import_state(dns_handle *h, int level, const double *aos_in);
/* Interface history [3 levels n,p,pp][2 walls lower,upper][xdv][ydv][23] of
   fields [rho, u_x, u_y, u_z, fneq_0..18], as lbf-lin / lbf-uin hold it
   (main :1078-1135).  Importing all zeros leaves the history as main's mode s
   does (it never sets it). */
int dns_export_history(dns_handle *h, double *out);
int dns_import_history(dns_handle *h, const double *in);
/* Field output as the reference's vel_print.c:15-275 (main :1342): vel-c,
   vel-slf, vel-suf (nx, ny, nz, 3) and den-c, den-slf, den-suf (nx, ny, nz),
   counter cntr, of the post-stream state; the FP64 form writes the
   reference's bytes. */
int dns_write_fields(dns_handle *h, const char *dir, int cntr);
/* Force the next step will use (encalc2 of the current state in CFR mode). */
int dns_get_force(dns_handle *h, double *force);

/* ---- the hot path ---------------------------------------------------------- */
/* Advance ncoarse coarse steps: the body of main's loop
   (dns-q-mgrd-all-patterns-xyc.c:1254-1375): encalc2, wshearstr, xcomputations,
   GR x (xfcomputations, tinterpolate_hrmt, derivative, ctfdtransfer_opt),
   ftcdtransfer, exchange/fexchange.  log (may be NULL) receives ncoarse rows.
   Returns DNS_ENAN if a wall shear stress is NaN (the reference calls
   MPI_Abort on isnan, wshearstr.c:139-143; an infinite stress is logged and
   stepping goes on, as there); the state is then left as computed. */
int dns_step(dns_handle *h, long ncoarse, dns_step_log *log);

/* ---- statistics ---------------------------------------------------------- */
/* Every `every` coarse steps (0 = off) the pre-step state is sampled on the
   device: per plane of the composite profile (statistics.c:48-146 plane order)
   FP64 sums of u, v, w, rho and their second moments are accumulated. */
int dns_set_sampling(dns_handle *h, long every);
int dns_stats_reset(dns_handle *h);
/* Accumulated profiles, out[DNS_NSTAT][nz_profile], samples in *nsamples:
   0 z/H  1 <U>  2 <V>  3 <W>  4 <rho>   (time mean of plane means)
   5 <u'u'>  6 <v'v'>  7 <w'w'>  8 <u'w'>  9 <rho'rho'>  (time mean of the
     per-sample plane variances: the reference definition, statistics.c:147-292
     with time_stat.c:161-200 averaging)
   10 <u'u'>_t  11 <v'v'>_t  12 <w'w'>_t  13 <u'w'>_t  (fluctuations about the
     time-and-plane mean). */
#define DNS_NSTAT 14
int dns_stats(dns_handle *h, double *out, long *nsamples);
/* Instantaneous plane statistics of the current state, the 9 x NZ record of
   turb-fld.000.TTT (statistics.c:303-316). */
int dns_plane_stats(dns_handle *h, double *out9xnz);

/* ---- measurement ----------------------------------------------------------- */
/* Per-kernel device time, measured with CUDA events recorded on the handle's
   stream around every launch while profiling is on (no reference counterpart;
   the reference times only the whole loop, main :1252/:1377).  Classes:
   0 coarse stream-collide, 1 interface extraction, 2 fine stream-collide,
   3 coarse-to-fine interface, 4 fine-to-coarse injection, 5 reduction finalize,
   6 statistics finalize.  Times accumulate until profiling is switched on again. */
#define DNS_NKERNEL 7
int dns_set_profiling(dns_handle *h, int on);
int dns_kernel_times(dns_handle *h, double *ms, long *launches);

/* ---- allocation-free reduction ------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
   memory — code running while a CUDA graph is being captured, hosts that give
   the library a fixed memory budget and forbid allocation after start-up, or
   pool-allocator embeddings where an extra cudaMalloc would fragment or overrun
   the pool: the constant-flow-rate reduction (encalc2's momentum and mass sums
   and the force they set) over a state the caller holds on the device in this
   library's layout — coarse fc[19][zdv][ydv][xdv], fine ff[19][2 zds][GR ydv]
   [GR xdv] with the lower block's planes k = 1..zds first, then the upper
   block's k = 0..zds-1.  The result {force, momentum, mass, unused} is written
   to out4 (4 doubles of device memory) on cuda_stream (NULL: default stream).
   Nothing is allocated: the per-block partial sums live in a 4 MiB array
   compiled into the library, which every GPU that loads the library holds
   until the process exits; a domain needing more than 262144 reduction blocks
   is rejected with DNS_EINVAL.  Only the FP64 layout is read: p->precision
   must be DNS_FP64 (DNS_EINVAL otherwise).  Every call asks the runtime for the
   array's device address on p->device (no allocation; after a cudaDeviceReset
   the new context's address is used); the first call on a device may load the
   library's device code, so make it before any stream capture.  The caller's
   current device is restored before the call returns.  All calls share the
   array, so calls that overlap on the GPU race: serialise them. */
int dns_flow_sums_static(const dns_params *p, const double *fc, const double *ff, double *out4, void *cuda_stream);

/* ---- batched FP32 engine --------------------------------------------------- */
/* No counterpart in the reference (one MPI job per channel).  Many independent
   channels of any size, wall pattern and Re_tau (one refinement ratio per
   batch) are stepped together in the FP32 deviation-storage form: each phase
   of the coarse step is one persistent kernel over a per-instance block table,
   and run() replays a captured CUDA graph of a step group.  Instances keep
   their lattice, history and statistics resident on the device until removed;
   each has its own step budget and stops when it is spent.  An instance's
   results depend only on its own parameters and tile shape, not on which
   other instances share the batch. */
typedef struct dns_batch dns_batch;

/* Tile shape of one instance: threads per row along x (8, 16, 32, 64 or 128;
   each thread updates four consecutive nodes) and row iterations per work item
   of the coarse (cw, cjb) and fine (fw, fjb) kernels. */
typedef struct dns_tile {
  int cw, cjb;
  int fw, fjb;
} dns_tile;

typedef struct dns_batch_info {
  long long steps_done;       /* coarse steps taken */
  long long remaining;        /* steps left in the budget */
  int status;                 /* DNS_OK, or DNS_ENAN after a non-finite wall shear stress */
  int slot;                   /* internal row (diagnostics) */
  double force;               /* force[0] of the next step */
  double flowrate, stress;    /* last logged values */
  long long device_bytes;     /* device memory held by the instance */
  long long updates_per_step; /* node updates per coarse step */
  dns_tile tile;              /* tile shape in use */
} dns_batch_info;

int dns_batch_create(int device, dns_batch **out);
void dns_batch_destroy(dns_batch *b);
/* Device bytes an instance of these parameters holds (FP32 form).  The
   batched engine needs xdv a multiple of 4 (DNS_EINVAL otherwise): its
   stream-collide kernels move four consecutive nodes with 16-byte accesses. */
int dns_batch_footprint(const dns_params *p, long long *bytes);
/* Tile shape an instance of these parameters gets: the batch's tuning-table
   entry for its shape if any (b may be NULL), else a fixed default. */
int dns_batch_tile_for(const dns_batch *b, const dns_params *p, dns_tile *t);
/* Tuning-table entry for every later instance of the same grid shape. */
int dns_batch_set_tile(dns_batch *b, const dns_params *shape, const dns_tile *t);
/* Time `steps` steps of each candidate tile shape on throw-away instances of
   this grid shape in a scratch batch (resident instances are untouched): as
   many copies as make about 32 M node updates a step, at most 64 and 8 GB, so
   that the GPU is as loaded as in a full batch.  The fastest goes to the
   tuning table; a candidate replaces the current best only when at least 1%
   faster.  best and ms (per step of all the copies) may be NULL. */
int dns_batch_autotune(dns_batch *b, const dns_params *shape, int steps, dns_tile *best, double *ms);
/* Add a seeded instance (the state dns_init_seeded builds) with a budget of
   `steps` coarse steps; statistics are sampled every sample_every steps of the
   instance (0: none).  tile NULL: dns_batch_tile_for.  *id receives a handle. */
int dns_batch_add(dns_batch *b, const dns_params *p, const dns_tile *tile, uint64_t seed, double uc, double amp,
                  long long steps, long long sample_every, int *id);
/* Release an instance's device memory. */
int dns_batch_remove(dns_batch *b, int id);
/* Advance every resident instance with budget left by up to nsteps coarse
   steps; *active (may be NULL) receives how many still have budget. */
int dns_batch_run(dns_batch *b, long long nsteps, int *active);
int dns_batch_info_of(dns_batch *b, int id, dns_batch_info *out);
/* The instance's statistics, as dns_stats. */
int dns_batch_stats(dns_batch *b, int id, double *out, long *nsamples);
/* Discard the instance's accumulated statistics (as dns_stats_reset), e.g.
   after a warm-up; sampling goes on at the instance's cadence. */
int dns_batch_stats_reset(dns_batch *b, int id);
/* The instance's post-stream state, as dns_export_state. */
int dns_batch_export_state(dns_batch *b, int id, int level, double *aos_out);
/* Replace one level of the instance's post-stream state, as dns_import_state
   (the interface history is kept; the next step's force is recomputed). */
int dns_batch_import_state(dns_batch *b, int id, int level, const double *aos_in);
/* Log rows [first, first + n) of the instance (rows of steps taken). */
int dns_batch_log(dns_batch *b, int id, long long first, long long n, dns_step_log *rows);
/* The batch's CUDA stream (cudaStream_t as void*): run() is ordered on it, so
   events recorded there bracket a run's device time. */
int dns_batch_stream(dns_batch *b, void **stream);

/* ---- errors -------------------------------------------------------------- */
const char *dns_error_string(int code);
const char *dns_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* DNS_EMBED_H */
