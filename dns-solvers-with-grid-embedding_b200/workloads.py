"""Parametric channel workloads for the batched and served forms.

A *channel instance* is one grid-embedded channel: coarse grid Nx (stream) x
Ny (wall-normal) x Nz (span) with a 2:1 fine level over the Ny/8 coarse cells
next to each wall, a wall pattern (streamwise ridges or square posts of a given
pitch and gas fraction) and a friction Reynolds number.  In the reference's
parameters (src/definitions.h) that is xdv = Nx, ydv = Nz, gratio = 2,
zds = 2 Ny / 8 fine planes per block and zdv = Ny - zds + 3 coarse planes, so
the fine-unit channel height is H = 2 Ny - 1 (dns-q-mgrd-all-patterns-xyc.c:155).

The flow is driven at constant flow rate (encalc2) with the reference's bulk
velocity ub = 0.0866034 (definitions.h:35); the bulk Reynolds number on the
full height follows from the target Re_tau through Dean's correlation
Re_tau = 0.175 (Re_b / 2)^(7/8), which the reference validates against.

Resolution cap.  The drawn Re_tau (uniform in [180, 395]) is kept on the
instance, but the run uses min(Re_tau, c(Ny) H / 2): a fine-grid spacing of
at most c(Ny) wall units, c = 1.75 for Ny = 32, 2.5 for Ny = 48, 2.75 for
Ny = 64.  The reference's BGK scheme diverges on these grids beyond that
(measured on B200 with this library, FP64 form = the reference's arithmetic
and FP32 batched form alike, which diverge within ~1% of the same step):
over 10000 steps, Ny = 32 ran at 2.0 wall units and diverged at 2.5
(after 1400-2700 steps), Ny = 48 ran at 3.0 and diverged at 3.5, Ny = 64 ran
at 3.0 and diverged once at 3.5; uncapped, 81 of the 96 drawn channels
diverged within 2000 steps; capped, none of them did in 3000.  The
reference's own production runs use under 2 wall units.

The quantities a solve returns (mean velocity profile, slip length, drag
reduction) are computed here on the host from the instance's on-device
statistics and log:
  - slip length b = U_s / (dU/dz)|_w per wall, with U_s and the wall gradient
    from the quadratic through the first three fine planes (z = 0.5, 1.5, 2.5
    fine units from the wall): U_s = (15 U1 - 10 U2 + 3 U3) / 8 and
    dU/dz = -2 U1 + 3 U2 - U3 (the stencil wshearstr.c:67-100 uses);
  - drag reduction DR = 100 (Cf0 - Cf) / Cf0 with Cf = tau_w / (ub^2 / 2) from
    the logged wall shear stress and flow rate (TKE-budget/postprocessing/
    CFriction.c:33-59 forms Cf the same way) and the no-slip reference
    Cf0 = 0.073 Re_b^(-1/4) (Dean) in place of that file's constant, which
    belongs to one Reynolds number.
The reference itself computes neither on the fly, so these definitions are
this project's; nothing in the reference pins them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

UB = 0.0866034
SEED, UC, AMP = 42, 0.05, 0.005  # seeded initial state: laminar profile + Philox noise
DPLUS_CAP = {32: 1.75, 48: 2.5, 64: 2.75}  # largest fine-grid spacing (wall units) per Ny


def dplus_cap(ny: int) -> float:
    return DPLUS_CAP[ny] if ny in DPLUS_CAP else (1.75 if ny <= 32 else (2.5 if ny <= 48 else 2.75))

NX_CHOICES = (64, 128, 192, 256)
NY_CHOICES = (32, 48, 64)
NZ_CHOICES = (64, 96, 128)
PITCH_CHOICES = (16, 24, 32)


def reb_from_retau(re_tau: float) -> float:
    """Bulk Reynolds number (full height) from Dean's correlation."""
    return 2.0 * (re_tau / 0.175) ** (8.0 / 7.0)


@dataclass
class Instance:
    nx: int
    ny: int  # wall-normal coarse cells
    nz: int  # spanwise
    pattern: str  # "RSLIP" ridges or "PSLIP" posts
    pitch: int  # fine cells
    gas: int  # slip width per pitch, fine cells
    re_tau: float
    seed: int = SEED
    steps: int = 2000
    arrival: float = 0.0  # seconds after the stream starts (served form)
    macros: dict = field(default_factory=dict)

    @property
    def zds(self) -> int:
        return 2 * self.ny // 8

    @property
    def gas_fraction(self) -> float:
        """Realised gas (slip) area fraction of the wall pattern."""
        g = self.gas / self.pitch
        return g if self.pattern == "RSLIP" else 1.0 - (1.0 - g) ** 2

    @property
    def height(self) -> int:
        """Fine-unit channel height H = NZs - 2 = 2 Ny - 1."""
        return 2 * self.ny - 1

    @property
    def re_tau_run(self) -> float:
        """Re_tau the run uses: the drawn value, capped at dplus_cap(ny) wall units per fine cell."""
        return min(self.re_tau, dplus_cap(self.ny) * self.height / 2.0)

    @property
    def rebs(self) -> float:
        return reb_from_retau(self.re_tau_run)

    def params(self, pkg, precision=None):
        kw = dict(xdv=self.nx, ydv=self.nz, zdv=self.ny - self.zds + 3, zds=self.zds, gratio=2, Rebs=self.rebs,
                  ub=UB, CFL=0.1, pattern=self.pattern, gyplussize=self.gas, wyplussize=self.pitch - self.gas,
                  gxplussize=self.gas, wxplussize=self.pitch - self.gas, forcing=pkg.FORCING_CFR)
        if precision is not None:
            kw["precision"] = precision
        kw.update(self.macros)
        return pkg.make_params(**kw)

    def updates_per_step(self) -> int:
        nxf, nyf = 2 * self.nx, 2 * self.nz
        return self.nx * self.nz * (self.ny - self.zds + 3) + 2 * 2 * nxf * nyf * self.zds


def _gas_width(pattern: str, pitch: int, gf: float) -> int:
    # ridges: slip width = GF pitch; posts (slip where x OR y in the gap):
    # solid post side w with (w / pitch)^2 = 1 - GF
    if pattern == "RSLIP":
        g = int(round(gf * pitch))
    else:
        g = pitch - int(round(pitch * math.sqrt(1.0 - gf)))
    return min(max(g, 1), pitch - 1)


def draw_instance(rng: np.random.Generator, seed: int, steps: int) -> Instance:
    nx = int(rng.choice(NX_CHOICES))
    ny = int(rng.choice(NY_CHOICES))
    nz = int(rng.choice(NZ_CHOICES))
    re_tau = float(rng.uniform(180.0, 395.0))
    pattern = "RSLIP" if rng.random() < 0.5 else "PSLIP"
    pitch = int(rng.choice(PITCH_CHOICES))
    gf = float(rng.uniform(0.5, 0.9))
    return Instance(nx, ny, nz, pattern, pitch, _gas_width(pattern, pitch, gf), re_tau, seed=seed, steps=steps)


def batched_instances(n: int = 96, seed: int = 4, steps: int = 2000) -> list[Instance]:
    """The batched workload: n independent channels drawn from seed."""
    rng = np.random.default_rng(seed)
    return [draw_instance(rng, SEED + q, steps) for q in range(n)]


def shard(instances: list[Instance], world: int) -> list[list[int]]:
    """Split independent channels across `world` GPUs: longest-processing-time
    first on node updates x steps (ties by index), each to the least loaded
    rank.  Deterministic, so every rank computes the same assignment without
    communicating.  Returns the instance indices of each rank, ascending."""
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(instances)), key=lambda q: (-instances[q].updates_per_step() * instances[q].steps, q))
    for q in order:
        r = min(range(world), key=lambda x: (load[x], x))
        out[r].append(q)
        load[r] += instances[q].updates_per_step() * instances[q].steps
    return [sorted(x) for x in out]


def request_stream(rate: float, n: int, seed: int = 5, budget=(1000, 10000)) -> list[Instance]:
    """The served workload: n requests with Poisson arrivals at `rate` per
    second, grids and walls drawn as in the batched workload, step budgets
    uniform in [budget[0], budget[1]]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for q in range(n):
        t += float(rng.exponential(1.0 / rate))
        inst = draw_instance(rng, SEED + q, int(rng.integers(budget[0], budget[1] + 1)))
        inst.arrival = t
        out.append(inst)
    return out


# ------------------------------------------------------------------ results
def slip_length(stats: np.ndarray, zdf: int) -> tuple[float, float]:
    """(lower, upper) slip length in fine units from the mean profile
    stats[1] (U per composite-profile plane; lower fine planes are indices
    1..zdf-1 at z = k - 1/2, the upper wall's first planes are the last ones)."""
    U = stats[1]
    nz = U.shape[0]

    def one(u1, u2, u3):
        us = (15.0 * u1 - 10.0 * u2 + 3.0 * u3) / 8.0
        g = -2.0 * u1 + 3.0 * u2 - u3
        return us / g if g != 0 else float("nan")

    low = one(U[1], U[2], U[3])
    # upper wall: profile index nz - 2 is the fluid plane next to the wall
    up = one(U[nz - 2], U[nz - 3], U[nz - 4])
    return low, up


def drag_reduction(log: np.ndarray, rebs: float, first: int = 0) -> tuple[float, float]:
    """(Cf, DR percent) from the per-step log rows [first:] (columns time,
    force, momentum, denst, flowrate, stup, stdown, stress, pgrad)."""
    rows = log[first:]
    ub = float(np.mean(rows[:, 2] / rows[:, 3]))  # momentum / mass = bulk velocity
    cf = float(np.mean(rows[:, 7])) / (0.5 * ub * ub)
    cf0 = 0.073 * rebs ** -0.25
    return cf, 100.0 * (cf0 - cf) / cf0


def solve_result(inst: Instance, stats: np.ndarray, log: np.ndarray, zdf: int) -> dict:
    """The answer to one parametric solve."""
    lo, up = slip_length(stats, zdf)
    cf, dr = drag_reduction(log, inst.rebs, first=len(log) // 2)
    return {"z": stats[0].tolist(), "U": stats[1].tolist(), "slip_length": 0.5 * (lo + up),
            "slip_length_walls": (lo, up), "cf": cf, "drag_reduction_pct": dr}


# ------------------------------------------------------------------ long-run statistics
# Profiles of the running statistics (dns_stats rows) that are time means of
# per-sample quantities, so that the mean over a window is linear in the
# accumulated sums: 1 <U> 2 <V> 3 <W> 4 <rho> 5 <u'u'> 6 <v'v'> 7 <w'w'>
# 8 <u'w'> 9 <rho'rho'> (per-sample plane moments, statistics.c:147-292,
# averaged in time as TKE-budget/postprocessing/time_stat.c:161-200 does).
LINEAR_ROWS = tuple(range(1, 10))
STAT_NAMES = {1: "U", 5: "uu", 6: "vv", 7: "ww", 8: "uw"}


def window_means(cum: list[tuple[np.ndarray, int]]) -> list[np.ndarray]:
    """Per-window means from cumulative statistics read at window boundaries.

    cum[q] = (stats, samples) as dns_stats returns them after window q
    (cum[0] at the start of the first window).  Rows LINEAR_ROWS are averages
    over all samples so far, so a window's own mean is the difference of the
    two cumulative sums over its samples; row 0 (z/H) is copied."""
    out = []
    for (a, na), (b, nb) in zip(cum[:-1], cum[1:]):
        if nb <= na:
            raise ValueError("a window without samples")
        m = np.array(b, dtype=np.float64, copy=True)
        for r in LINEAR_ROWS:
            m[r] = (b[r] * nb - a[r] * na) / (nb - na)
        out.append(m)
    return out


def batch_mean_and_error(values: list) -> tuple[np.ndarray, np.ndarray]:
    """Mean of equal-length batch means and its standard error
    std(batch means, ddof=1) / sqrt(batches)."""
    v = np.asarray(values, dtype=np.float64)
    if len(v) < 2:
        return v.mean(axis=0), np.full(v.shape[1:], np.nan)
    return v.mean(axis=0), v.std(axis=0, ddof=1) / math.sqrt(len(v))


def friction_coefficient(log: np.ndarray, nyf: int, nzs: int) -> float:
    """Cf = <tau_w> / (ub^2 / 2) over the log rows given, as
    TKE-budget/postprocessing/CFriction.c:33-59 forms it: ub is the mean of
    the logged flow rate divided by ydf (NZs - 2) with the reference's per-rank
    ydf = GR ydv + 1, and Cf the mean of w-str / (ub^2 / 2)."""
    ub = float(np.mean(log[:, 4])) / ((nyf + 1) * (nzs - 2.0))
    return float(np.mean(log[:, 7] / (0.5 * ub * ub)))


def drag_reduction_vs(cf: float, cf_noslip: float) -> float:
    """DR in percent against a no-slip run at the same bulk Reynolds number:
    100 (Cf0 - Cf) / Cf0 (CFriction.c:46-57 with a measured Cf0)."""
    return 100.0 * (cf_noslip - cf) / cf_noslip


def friction_reynolds(log: np.ndarray, nzs: int, rebs: float, ub: float = UB) -> float:
    """Re_tau = u_tau (NZs - 2) / 2 / nu with u_tau = sqrt(<p-grad>) over the
    rows and nu from the fine relaxation time (time_stat.c:95-104)."""
    tau = (3.0 / rebs) * ub * (nzs - 2.0) + 0.5
    nu = (1.0 / 6.0) * (2.0 * tau - 1.0)
    return math.sqrt(max(float(np.mean(log[:, 8])), 0.0)) * (nzs - 2.0) * 0.5 / nu


def profile_error(p: np.ndarray, ref: np.ndarray, used: slice | None = None) -> float:
    """Largest deviation of profile p from ref relative to ref's largest
    magnitude (profiles such as <u'w'> cross zero)."""
    u = slice(1, len(ref) - 1) if used is None else used
    scale = float(np.max(np.abs(ref[u])))
    return float(np.max(np.abs(p[u] - ref[u]))) / scale if scale > 0 else 0.0


def compare_runs(a: dict, ref: dict) -> dict:
    """Per-statistic error of run a against run ref (summaries from
    summarize_run), with the combined batch-means uncertainty in the same
    units and whether the error is within 1e-3 or within two standard errors."""
    out = {}
    used = slice(1, len(ref["profiles"][1]) - 1)
    for r, name in STAT_NAMES.items():
        scale = float(np.max(np.abs(ref["profiles"][r][used])))
        err = profile_error(a["profiles"][r], ref["profiles"][r], used)
        se = np.sqrt(np.square(a["stderr"][r][used]) + np.square(ref["stderr"][r][used]))
        unc = float(np.max(se)) / scale if scale > 0 else 0.0
        out[name] = {"rel_err": err, "rel_uncertainty": unc, "ok": bool(err <= 1e-3 or err <= 2.0 * unc)}
    for key in ("tau_w", "slip_length", "cf"):
        x, y = a[key], ref[key]
        err = abs(x - y) / abs(y) if y else 0.0
        se_key = key + "_stderr"
        se = math.hypot(a.get(se_key) or 0.0, ref.get(se_key) or 0.0)
        unc = se / abs(y) if y else 0.0
        ok = err <= 1e-3 or abs(x - y) <= 2.0 * se
        if key == "slip_length":  # near zero on a no-slip wall: also judged in fine units
            ok = ok or abs(x - y) <= 1e-3
        out[key] = {"value": x, "ref": y, "abs_err": abs(x - y), "rel_err": err, "rel_uncertainty": unc,
                    "ok": bool(ok)}
    return out


def summarize_run(cum: list[tuple[np.ndarray, int]], log: np.ndarray, windows: int, nyf: int, nzs: int,
                  zdf: int, rebs: float) -> dict:
    """Time averages of one run's sampled window: profiles (mean of the window
    means) with batch-means standard errors, the wall shear stress, Cf, the
    slip length and the realised Re_tau.  log holds the window's step rows."""
    wm = window_means(cum)
    prof, err = batch_mean_and_error(wm)
    rows = np.array_split(log, windows)
    tw, tw_se = batch_mean_and_error([[float(np.mean(r[:, 7]))] for r in rows])
    cf_b = [friction_coefficient(r, nyf, nzs) for r in rows]
    cf, cf_se = batch_mean_and_error([[c] for c in cf_b])
    slips = [0.5 * sum(slip_length(m, zdf)) for m in wm]
    sl, sl_se = batch_mean_and_error([[x] for x in slips])
    return {"profiles": prof, "stderr": err, "tau_w": float(tw[0]), "tau_w_stderr": float(tw_se[0]),
            "cf": float(cf[0]), "cf_stderr": float(cf_se[0]), "slip_length": float(sl[0]),
            "slip_length_stderr": float(sl_se[0]), "re_tau": friction_reynolds(log, nzs, rebs),
            "samples": int(cum[-1][1] - cum[0][1])}


def long_run(pkg, macros: dict, precision: str, warm: int, windows: int, per: int, seed: int = SEED,
             device: int = 0):
    """One channel (reference macros `macros`, constant flow rate) run long:
    `warm` steps, then `windows` windows of `per` steps with the statistics
    sampled every step.  precision "fp64": the FP64 plain form (a channel
    handle); "fp32": the FP32 deviation form of the batched engine (a batch of
    one).  Returns (cumulative statistics at the window boundaries, the
    windows' log rows, None) or (None, None, reason) when the run stopped on a
    non-finite wall shear stress."""
    p = pkg.make_params(**macros, forcing=pkg.FORCING_CFR, device=device)
    if precision == "fp64":
        with pkg.Channel(p) as ch:
            ch.init_seeded(seed, UC, AMP)
            try:
                ch.step(warm, log=False)
                ch.stats_reset()
                ch.set_sampling(1)
                cum, logs = [ch.stats()], []
                for _ in range(windows):
                    logs.append(ch.step(per, log=True))
                    cum.append(ch.stats())
            except pkg.DnsError as e:
                return None, None, str(e)
        return cum, np.concatenate(logs), None
    with pkg.Batch(device) as b:
        i = b.add(p, steps=warm + windows * per, seed=seed, uc=UC, amp=AMP, sample_every=1)
        b.run(warm)
        b.stats_reset(i)
        cum = [b.stats(i)]
        for _ in range(windows):
            b.run(per)
            cum.append(b.stats(i))
        inf = b.info(i)
        if inf.status != 0:
            return None, None, f"status {inf.status} after {inf.steps_done} steps (non-finite wall shear stress)"
        log = b.log(i, first=warm, n=windows * per)
    return cum, log, None
