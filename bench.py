"""Throughput of the grid-embedded D3Q19 channel step on B200 (MLUPS).

One "step" is one coarse time step of the channel: the coarse stream-collide,
GR fine substeps on both near-wall blocks with their coarse-to-fine interface
transfers, the fine-to-coarse injection and the flow-rate reduction.  Its work
is U = xdv ydv zdc + 2 GR (GR xdv)(GR ydv) zds node updates.

Default workload: the production channel, coarse grid 256 x 96 x 128 (stream,
wall-normal, span) with a 2:1 fine level over the 8 coarse cells next to each
wall (fine blocks 512 x 16 x 256), i.e. reference macros xdv=256, ydv=128,
zdv=83, zds=16, gratio=2; constant flow rate at Re_tau ~ 180; FP64 plain form;
seeded synthetic initial state.  The state (2.1 GB) is far larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Beside the FP64 line the same JSON carries three FP32 legs run by the
batched engine: ``fp32`` (the production channel as a batch of one),
``batched`` (96 independent channels of uneven size, wall pattern and Re_tau
drawn from a seed, 2000 steps each, against the same channels run one after
another in FP64) and ``served`` (Poisson request streams at 2, 10 and 50 per
second with step budgets of 1000-10000, admitted against a 150 GB budget:
p50/p99 latency and aggregate MLUPS, against the same requests served one at a
time by the FP64 form).

A ``budget`` object times the turbulence statistics / kinetic-energy budget of
the final state (the reference's offline TKE-budget program) on the device,
from the live state and from field files, beside the reference program itself
on one host core reading the same files.

N > 1 runs under torchrun: every rank advances its own independent channel
(replicas, weak scaling); the reported value is the whole job's updates over
the slowest rank's device time.  ``--impl reference`` times the reference's own
CPU routines (compiled from its sources, oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    # name: (macros, description)
    "c2": (dict(xdv=256, ydv=128, zdv=83, zds=16, gratio=2, Rebs=5533.0, ub=0.0866034, CFL=0.1, pattern=None),
           "channel 256x96x128 coarse, 2:1 fine blocks 512x16x256 per wall (xdv256 ydv128 zdv83 zds16 GR2), "
           "CFR Re_tau~180"),
    "c1": (dict(xdv=64, ydv=64, zdv=27, zds=8, gratio=2, Rebs=150.0 * 0.0866034 * 63, ub=0.0866034, CFL=0.1,
                pattern=None),
           "channel 64x32x64 coarse, 2:1 fine blocks 128x8x128 per wall (xdv64 ydv64 zdv27 zds8 GR2)"),
    "c3r": (dict(xdv=384, ydv=192, zdv=115, zds=16, gratio=2, Rebs=13585.0, ub=0.0866034, CFL=0.1, pattern="RSLIP",
                 gyplussize=24, wyplussize=24),
            "SHS channel 384x128x192 coarse, streamwise ridges pitch 48 GF 0.5, Re_tau~395"),
    "c3p": (dict(xdv=384, ydv=192, zdv=115, zds=16, gratio=2, Rebs=13585.0, ub=0.0866034, CFL=0.1, pattern="PSLIP",
                 gyplussize=16, wyplussize=16, gxplussize=16, wxplussize=16),
            "SHS channel 384x128x192 coarse, square posts pitch 32 GF 0.75, Re_tau~395"),
    "c3n": (dict(xdv=384, ydv=192, zdv=115, zds=16, gratio=2, Rebs=13585.0, ub=0.0866034, CFL=0.1, pattern=None),
            "channel 384x128x192 coarse with no-slip walls: the drag reference of the SHS channels, Re_tau~395"),
}
METRIC = "MLUPS (coarse-step node updates, FP64 plain form)"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str, config: str):
    """dram bytes per launch from a committed ncu summary, if one exists."""
    f = ROOT / "profiles" / f"traffic_{config}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    read every millisecond or so on a thread (nvidia-smi's 200 ms loop when
    NVML is missing).  mark() brackets the timed region on the host clock;
    the summary keeps the samples inside it (all of them if none fell inside)."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,power.draw")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int, bus_id: str | None = None):
        self.index, self.bus_id = index, bus_id
        self.rows = []  # (host time, sm MHz, max sm MHz, 4 reason flags)
        self.window = None
        self.proc = None
        self.thread = None
        self.stop = threading.Event()
        self.source = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = None
            if self.bus_id:
                try:
                    h = pynvml.nvmlDeviceGetHandleByPciBusId(self.bus_id)
                except pynvml.NVMLError:
                    h = None
            if h is None:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.thread = threading.Thread(target=self._nvml, args=(pynvml, h), daemon=True)
            self.source = "nvml"
        except Exception:
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                     "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._smi, daemon=True)
                self.source = "nvidia-smi"
            except FileNotFoundError:
                self.proc = None
        if self.thread:
            self.thread.start()
        return self

    def _nvml(self, nv, h):
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        try:
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self.stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((time.perf_counter(), float(sm), float(mx)) + tuple(bool(r & b) for b in bits))
                time.sleep(0.001)
        except Exception:
            pass

    def _smi(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7 and parts[0].replace(".", "").isdigit():
                self.rows.append((time.perf_counter(), float(parts[0]), float(parts[1]))
                                 + tuple(parts[2 + q].lower() == "active" for q in range(4)))

    def mark(self, t0: float, t1: float):
        self.window = (t0, t1)

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread and self.source == "nvml":
            self.thread.join(timeout=2)

    def summary(self):
        rows = list(self.rows)
        if self.window:
            inside = [r for r in rows if self.window[0] <= r[0] <= self.window[1]]
            rows = inside or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({self.NAMES[q] for r in rows for q in range(4) if r[3 + q]})
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows),
                "reasons": reasons, "samples": len(rows), "source": self.source}


def bus_id_of(torch, device: int):
    """PCI bus id of a CUDA device in NVML's form, or None."""
    try:
        pr = torch.cuda.get_device_properties(device)
        return f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
    except Exception:
        return None


def reference_cpu(config: str, steps: int, processes: int, timeout: float = 900.0, warmup: int = 0):
    """Time the reference's own routines (oracle/_ref/<config>/ref_harness, one
    rank per process, from rest, constant-force mode with zero force) on the host.
    Each process runs warmup + steps steps and clocks the last `steps`.
    Returns each process's step-loop seconds (its own clock), or None when the
    binary is missing or a process gave no time."""
    exe = ROOT / "oracle" / "_ref" / config / "ref_harness"
    if not exe.exists():
        return None
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for q in range(processes):
            od = Path(d) / f"p{q}"
            od.mkdir()
            procs.append(subprocess.Popen([str(exe), "-", "0", str(od), "-1", str(steps + warmup), "const", "0", "0", "0",
                                           str(warmup)],
                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        secs = []
        for pr in procs:
            out, _ = pr.communicate(timeout=timeout)
            for line in out.splitlines():
                if line.startswith("harness_seconds"):
                    secs.append(float(line.split()[1]))
    if len(secs) != processes:
        return None
    return secs


def host_parallelism(per_process_bytes: float):
    ncpu = os.cpu_count() or 1
    try:
        import psutil

        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16e9
    return max(1, min(ncpu, int(avail * 0.6 // per_process_bytes), 64))


def updates_per_step(m):
    gr = m["gratio"]
    return m["xdv"] * m["ydv"] * m["zdv"] + 2 * gr * (gr * m["xdv"]) * (gr * m["ydv"]) * m["zds"]


def arm_config(args, world: int) -> dict:
    """The workload description both arms print (same keys, same values)."""
    m, desc = CONFIGS[args.config]
    U = updates_per_step(m)
    state = U * 2 * 19 * 8  # both ping-pong copies of every population, FP64
    return {"workload": args.config, "description": desc, "updates_per_step": U,
            "l2": (f"state {state / 1e9:.1f} GB of populations >> 126 MB L2 (no flush needed)"
                   if state > 8 * 126e6 else f"state {state / 1e9:.2f} GB: not enough to defeat L2"),
            "parallelism": f"replicas x{world}"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    m, desc = CONFIGS[args.config]
    U = updates_per_step(m)
    # about 2.3 GB of AoS arrays per process at the default config
    per_proc = 19 * 8 * 2.2 * (U + 2 * (m["gratio"] * m["xdv"]) * (m["gratio"] * m["ydv"]))
    nproc = host_parallelism(per_proc)
    # the reference spends about 2.3 s per c2 step per process: K and W are
    # capped so that the run stays within a few minutes
    steps = max(1, min(args.steps, 40))
    warm = max(0, min(args.warmup, 5))
    secs = reference_cpu(args.config, steps, nproc, warmup=warm)
    line = {"impl": "reference", "metric": METRIC, "unit": "MLUPS", "n_gpus": world, "steps": steps,
            "warmup": warm, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference cold start from rest)", "config": arm_config(args, world)}
    if secs is None:
        line["unavailable"] = "compiled reference binary missing (oracle/_ref not built)"
        print(json.dumps(line), flush=True)
        return 0
    mlups = U * steps * len(secs) / max(secs) / 1e6
    line.update({"value": mlups, "ms_per_step": 1e3 * max(secs) / steps})
    line["cpu_baseline"] = {"value": mlups, "unit": "MLUPS", "cores": len(secs), "kind": "reference",
                            "sample": f"{len(secs)} concurrent single-rank reference processes x {steps} coarse "
                                      f"steps of {args.config} after {warm} untimed ones (own step-loop clock, "
                                      f"main's t2-t4)"}
    line["e2e"] = {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)
    return 0


def timed_batch_run(torch, b, n):
    """Device time (ms) of b.run(n), CUDA events on the batch's stream."""
    s = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    b.run(n)
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def max_over_ranks(torch, dist, x: float, group=None) -> float:
    """The largest x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend(group) == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(torch, dist, x: float, group=None) -> float:
    if dist is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend(group) == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def fp64_reference_run(pkg, torch, inst, steps, sample_every, device=0):
    """One drawn channel alone in the FP64 plain form for `steps` steps with
    its statistics sampled: (device ms, statistics) or (device ms, None) when
    it stopped on a NaN wall shear stress."""
    p = inst.params(pkg, precision=pkg.FP64)
    p.device = device
    with pkg.Channel(p) as ch:
        st = torch.cuda.Stream()
        ch.set_stream(st.cuda_stream)
        ch.init_seeded(inst.seed, 0.05, 0.005)
        ch.set_sampling(sample_every)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        try:
            ch.step(steps, log=False)
            ok = True
        except pkg.DnsError:
            ok = False
        e1.record(st)
        torch.cuda.synchronize()
        stats = ch.stats()[0] if ok else None
    return e0.elapsed_time(e1), stats


def bench_batched(pkg, torch, args, peak, rank=0, world=1, dist=None, device=0):
    """Config 4: n channels of uneven size / pattern / Re_tau in one batch per
    GPU; with N GPUs each rank takes its shard (workloads.shard), the value is
    all ranks' node updates over the slowest rank's device time.  Every
    instance is then run alone in the FP64 plain form for the same steps and
    its statistics compared with the batch's (per instance: the largest
    deviation of each profile relative to the profile's scale)."""
    W = importlib.import_module(PKG + ".workloads")
    everything = W.batched_instances(args.c4_instances, steps=args.c4_steps)
    mine = W.shard(everything, world)[rank]
    insts = [everything[q] for q in mine]
    every = 20
    b = pkg.Batch(device)
    tuned = {}
    if args.autotune:
        # the engine's tuner on each distinct grid shape; admissions of that
        # shape then take the tuned tile
        t0 = time.perf_counter()
        for x in insts:
            p = x.params(pkg)
            p.device = device
            key = (p.xdv, p.ydv, p.zdv, p.zds, p.gratio)
            if key not in tuned:
                tuned[key] = b.autotune(p, steps=5)
        tune_s = time.perf_counter() - t0
    ids = []
    for x in insts:
        p = x.params(pkg)
        p.device = device
        ids.append(b.add(p, steps=x.steps, seed=x.seed, sample_every=every))
    U = sum_over_ranks(torch, dist, sum(x.updates_per_step() for x in insts))
    held = sum(b.info(i).device_bytes for i in ids)
    b.run(args.warmup)
    before = [b.info(i).steps_done for i in ids]
    if dist is not None:
        dist.barrier()
    ms = max_over_ranks(torch, dist, timed_batch_run(torch, b, args.c4_steps - args.warmup))
    steps = args.c4_steps - args.warmup
    # work actually done: an instance that stops (non-finite wall shear stress) does no more
    done = [b.info(i).steps_done - s0 for i, s0 in zip(ids, before)]
    work = sum_over_ranks(torch, dist, sum(x.updates_per_step() * d for x, d in zip(insts, done)))
    value = work / (ms * 1e-3) / 1e6
    failed = int(sum_over_ranks(torch, dist, sum(1 for i in ids if b.info(i).status != 0)))
    stats32 = [b.stats(i)[0] if b.info(i).status == 0 else None for i in ids]
    b.close()
    tiles = ({"tuned_shapes": len(tuned), "tuning_seconds": tune_s,
              "tiles": {"x".join(map(str, k)): list(v[0]) for k, v in tuned.items()}} if tuned else "default")
    if args.no_c4_reference:
        return {"value": value, "unit": "MLUPS", "instances": len(everything), "gpus": world, "steps": steps,
                "ms_per_step": ms / steps, "updates_per_step": U, "failed_instances": failed,
                "whole_step_hbm_frac": (work * 152 / (ms * 1e-3) / 1e9) / peak, "tile": tiles}
    # the same channels one after another in FP64 (device time of each whole
    # run), every rank its own shard, and the per-instance comparison
    seq_ms, errs, f64_failed = 0.0, {name: [] for name in W.STAT_NAMES.values()}, 0
    for x, s32 in zip(insts, stats32):
        t, s64 = fp64_reference_run(pkg, torch, x, args.c4_steps, every, device=device)
        seq_ms += t
        if s64 is None:
            f64_failed += 1
            continue
        if s32 is None:
            continue
        for r, name in W.STAT_NAMES.items():
            errs[name].append(W.profile_error(s32[r], s64[r]))
    seq_ms = max_over_ranks(torch, dist, seq_ms)
    v64 = U * args.c4_steps / (seq_ms * 1e-3) / 1e6
    compared = int(sum_over_ranks(torch, dist, len(errs["U"])))
    per_stat = {name: {"max_rel_err": max_over_ranks(torch, dist, max(e) if e else 0.0),
                       "median_rel_err": float(np.median(e)) if e else None} for name, e in errs.items()}
    return {
        "value": value, "unit": "MLUPS", "dtype": "f32 (deviation storage, FP64 reductions)",
        "instances": len(everything), "gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
        "updates_per_step": U, "device_bytes": held, "failed_instances": failed,
        "whole_step_hbm_frac": (work * 152 / (ms * 1e-3) / 1e9) / peak, "tile": tiles,
        "re_tau_drawn_range": [min(x.re_tau for x in insts), max(x.re_tau for x in insts)],
        "re_tau_run_range": [min(x.re_tau_run for x in insts), max(x.re_tau_run for x in insts)],
        "gas_fraction_range": [min(x.gas_fraction for x in insts), max(x.gas_fraction for x in insts)],
        "fp64_sequential": {"value": v64, "unit": "MLUPS", "ms_all": seq_ms,
                            "how": f"each channel alone in the FP64 plain form for all {args.c4_steps} steps "
                                   "(device time of each run, summed)", "failed_instances": f64_failed},
        "over_fp64_sequential": value / v64,
        "fp32_vs_fp64_per_instance": {
            "instances_compared": compared, "statistics_sampled_every": every,
            "note": "per instance and statistic: max over the profile of |FP32 - FP64| / max |FP64| after "
                    f"{args.c4_steps} steps from the same seeded state, both sampled every {every} steps",
            **per_stat},
        "workload": "96 channels drawn from seed 4: Nx {64,128,192,256}, Ny {32,48,64} (Ny/8 coarse cells "
                    "embedded 2:1 per wall), Nz {64,96,128}, Re_tau U[180,395], ridges or posts, pitch "
                    "{16,24,32} fine cells, gas fraction U[0.5,0.9]; the run's Re_tau capped at 1.75 / 2.5 / "
                    "2.75 wall units per fine cell for Ny 32 / 48 / 64 (the BGK scheme diverges beyond that on "
                    "these grids, in FP64 as in FP32)",
    }


def bench_served(pkg, torch, args, peak):
    """Config 5: Poisson request streams served by continuous batching, and
    the first requests of each stream served one at a time by the FP64 plain
    form (a measured run, not a model)."""
    W = importlib.import_module(PKG + ".workloads")
    S = importlib.import_module(PKG + ".serve")
    out = {"budget_bytes": 150e9, "requests_per_rate": args.c5_requests, "group_steps": 32,
           "note": "latency = completion - arrival on the host clock. The drawn Re_tau is capped on these grids "
                   "(the BGK scheme diverges beyond about 3 wall units per fine cell), so the physics results are "
                   "at re_tau_run, not the drawn value; drag reduction is against Dean's no-slip correlation at "
                   "the run's Re_b after a short budget from a near-laminar start, not a converged turbulent DR. "
                   "Admission: first come first served while the footprint fits the HBM budget and the resident "
                   "requests do at most max_resident_updates_per_step node updates a step (the GPU is saturated "
                   "by one production-size channel; beyond that, more residents only share it).",
           "max_resident_updates_per_step": 64e6, "rates": {}}
    for rate in args.c5_rates:
        reqs = W.request_stream(rate, args.c5_requests, seed=7)
        srv = S.Server(pkg, hbm_budget=150e9, group=32, sample_every=20)
        t0 = time.perf_counter()
        recs = srv.run(reqs)
        span = time.perf_counter() - t0
        srv.batch.close()
        lat = S.latency_summary(recs)
        mlups = srv.updates / span / 1e6
        ok = [r for r in recs if r.status == 0]
        entry = {
            **lat, "aggregate_mlups": mlups, "hbm_frac": mlups * 1e6 * 152 / 1e9 / peak, "makespan_s": span,
            "peak_resident_bytes": srv.peak_used,
            "re_tau_drawn_median": float(np.median([r.inst.re_tau for r in recs])),
            "re_tau_run_median": float(np.median([r.inst.re_tau_run for r in recs])),
            "slip_length_median": float(np.median([r.result["slip_length"] for r in ok])) if ok else None,
            "drag_reduction_vs_dean_pct_median": float(np.median([r.result["drag_reduction_pct"] for r in ok]))
            if ok else None,
        }
        # the first requests of the same stream, alone: served by the batched
        # FP32 loop and one at a time by the FP64 plain form (both measured)
        k = min(args.c5_fp64_requests, len(reqs))
        if k > 0:
            first = sorted(reqs, key=lambda r: r.arrival)[:k]
            srv_k = S.Server(pkg, hbm_budget=150e9, group=32, sample_every=20)
            t0 = time.perf_counter()
            r32 = srv_k.run(first)
            span32 = time.perf_counter() - t0
            srv_k.batch.close()
            t0 = time.perf_counter()
            r64 = S.serve_one_at_a_time(pkg, first, sample_every=20)
            span64 = time.perf_counter() - t0
            work = sum(r.inst.steps * r.inst.updates_per_step() for r in r64 if r.status == 0)
            in_full = S.latency_summary(sorted(recs, key=lambda r: r.arrival)[:k])
            entry["first_requests"] = {
                "requests": k,
                "subset": f"the first {k} arrivals of this stream, served alone (measured)",
                "fp32_served": {**S.latency_summary(r32), "makespan_s": span32,
                                "aggregate_mlups": srv_k.updates / span32 / 1e6},
                "fp64_one_at_a_time": {**S.latency_summary(r64), "makespan_s": span64,
                                       "aggregate_mlups": work / span64 / 1e6},
                "fp32_in_the_full_stream": {"p50_s": in_full["p50_s"], "p99_s": in_full["p99_s"]}}
        out["rates"][str(rate)] = entry
    return out


PKG = "dns-solvers-with-grid-embedding_b200"


def bench_longrun(pkg, args):
    """BASELINE configs 2 and 3 run long: warm-up, then sampled steps whose
    statistics are time-averaged on the device in FP64 (every step); FP64 plain
    form against the FP32 deviation form, per statistic, with batch-means
    standard errors; config 3 with a no-slip companion run for the drag
    reduction.  Errors are relative to each profile's largest magnitude."""
    W = importlib.import_module(PKG + ".workloads")
    warm, windows = args.longrun_warmup, args.longrun_windows
    out = {"warmup_steps": warm, "sampled_steps": {"c2": args.longrun_steps, "c3": args.longrun_c3_steps},
           "windows": windows, "sample_every": 1,
           "note": "errors: max over the profile of |FP32 - FP64| / max |FP64| (statistics); rel_uncertainty: "
                   "the two runs' batch-means standard errors combined, same units; ok: error <= 1e-3 or "
                   "within two standard errors. Config 3 (Re_tau 395 on 255 fine cells, fine relaxation time "
                   "0.5049) samples 15,000 steps: run 10,000 + 20,000, its FP64 no-slip companion reached a NaN "
                   "wall shear stress at step 28,194 (the FP32 run did not), as the reference's BGK scheme does "
                   "this close to tau = 1/2.", "cases": {}}
    summaries = {}
    for name in args.longrun_cases:
        m, desc = CONFIGS[name]
        per = (args.longrun_c3_steps if name.startswith("c3") else args.longrun_steps) // windows
        g = pkg.geometry(pkg.make_params(**m))
        case = {"description": desc}
        t0 = time.perf_counter()
        runs = {}
        for prec in ("fp64", "fp32"):
            cum, log, err = W.long_run(pkg, m, prec, warm, windows, per)
            if err:
                case[prec] = {"diverged": err}
                continue
            s = W.summarize_run(cum, log, windows, g.nyf, g.nzs, g.zdf, m["Rebs"])
            runs[prec] = s
            case[prec] = {"tau_w": s["tau_w"], "tau_w_stderr": s["tau_w_stderr"], "cf": s["cf"],
                          "cf_stderr": s["cf_stderr"], "slip_length": s["slip_length"],
                          "slip_length_stderr": s["slip_length_stderr"], "re_tau_realised": s["re_tau"],
                          "samples": s["samples"],
                          "u_centre": float(s["profiles"][1][len(s["profiles"][1]) // 2]),
                          "uu_max": float(np.max(s["profiles"][5])), "uw_absmax": float(np.max(np.abs(s["profiles"][8])))}
        if "fp64" in runs and "fp32" in runs:
            case["fp32_vs_fp64"] = W.compare_runs(runs["fp32"], runs["fp64"])
        case["seconds"] = time.perf_counter() - t0
        summaries[name] = runs
        out["cases"][name] = case
    # drag reduction of the patterned walls against the no-slip companion
    for name in args.longrun_cases:
        if name in ("c3r", "c3p") and "c3n" in summaries:
            dr = {}
            for prec in ("fp64", "fp32"):
                if prec in summaries[name] and prec in summaries["c3n"]:
                    dr[prec] = W.drag_reduction_vs(summaries[name][prec]["cf"], summaries["c3n"][prec]["cf"])
            if "fp64" in dr and "fp32" in dr:
                dr["abs_err_pct_points"] = abs(dr["fp32"] - dr["fp64"])
            out["cases"][name]["drag_reduction_pct_vs_noslip"] = dr
    return out


def bench_budget(pkg, ch, p, config: str):
    """The turbulence statistics / kinetic-energy budget of one snapshot of the
    channel's current state: on the device from the live state and from the
    field files, and the reference's own offline program (TKE-budget/
    computations, compiled under the single-rank shim) on the same files on
    one host core.  Wall-clock seconds of whole calls (file reads included
    where files are read); the largest profile deviation from the reference's
    output, relative to each profile's magnitude."""
    import numpy as np

    cntr = int(CONFIGS[config][0].get("TSTR", 0))
    g = pkg.geometry(p)
    out = {"workload": f"{config} fields ({g.nx}x{g.ny}x{g.nzc} coarse, 2 x {g.nxf}x{g.nyf}x{g.zdf} fine)",
           "profiles": len(pkg.TKE_NAMES), "nz": g.nz_profile}
    ch.tke_budget()
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        prof = ch.tke_budget()
    out["gpu_ms_live"] = 1e3 * (time.perf_counter() - t0) / reps
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        ch.write_fields(d, cntr)
        pkg.tke_budget_files(p, d, cntr)
        t0 = time.perf_counter()
        files = pkg.tke_budget_files(p, d, cntr)
        out["gpu_ms_files"] = 1e3 * (time.perf_counter() - t0)
        exe = ROOT / "oracle" / "_ref" / config / "tke_budget"
        if exe.exists():
            (d / "tke").mkdir()
            t0 = time.perf_counter()
            subprocess.run([str(exe)], cwd=d / "tke", check=True, capture_output=True)
            secs = time.perf_counter() - t0
            ref = np.concatenate([np.fromfile(d / "tke" / f"{n}.000.{cntr:04d}").reshape(k, -1)
                                  for n, k in pkg.TKE_FILES])
            scale = np.maximum(np.max(np.abs(ref), axis=1, keepdims=True), 1e-300)
            out["cpu_baseline"] = {"value": 1e3 * secs, "unit": "ms", "cores": 1, "kind": "reference",
                                   "sample": "one snapshot, reading the same files"}
            out["speedup_files_vs_cpu"] = 1e3 * secs / out["gpu_ms_files"]
            dev = np.maximum(np.max(np.abs(prof - ref) / scale, axis=1), np.max(np.abs(files - ref) / scale, axis=1))
            out["max_rel_dev_vs_reference"] = float(np.max(dev))
            out["worst_profile"] = pkg.TKE_NAMES[int(np.argmax(dev))]
    return out


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    pkg = importlib.import_module(PKG)
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    m, desc = CONFIGS[args.config]
    p = pkg.make_params(**m, forcing=pkg.FORCING_CFR, device=local_rank)
    geom = pkg.geometry(p)
    U = geom.updates_per_step
    ch = pkg.Channel(p)
    stream = torch.cuda.Stream()
    ch.set_stream(stream.cuda_stream)
    ch.init_seeded(42 + rank, 0.05, 0.005)
    ch.step(args.warmup, log=False)
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- timed region: K coarse steps, state resident in HBM
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank, bus_id_of(torch, local_rank)) as clk:
        time.sleep(0.2)  # let the sampler start before the timed region
        barrier()
        t_host0 = time.perf_counter()
        start.record(stream)
        log = ch.step(args.steps, log=True)
        end.record(stream)
        barrier()
        clk.mark(t_host0, time.perf_counter())
    ms = start.elapsed_time(end)
    # ---- per-kernel device time: the same steps again with CUDA events around
    # every launch on the library's stream (recording them slows the step a
    # little, so it is kept out of the timed region above)
    prof_steps = min(args.steps, 400)
    ch.set_profiling(True)
    ch.step(prof_steps, log=False)
    kt = ch.kernel_times()
    ch.set_profiling(False)
    ms_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = U * args.steps * world / (ms_max * 1e-3) / 1e6

    # ---- end to end through the C ABI with pinned host buffers: import the
    # state, K steps with the per-step log read back, export the state
    shapes = [(geom.nx, geom.ny, geom.nzc, 19), (geom.nxf, geom.nyf, geom.zdf, 19), (geom.nxf, geom.nyf, geom.zdf, 19)]
    host = [torch.empty(s, dtype=torch.float64, pin_memory=True).numpy() for s in shapes]
    for lv in range(3):
        host[lv][...] = ch.export_state(lv)
    state_bytes = sum(h.nbytes for h in host)
    barrier()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for lv in range(3):
        ch.import_state(lv, host[lv])
    ch.step(args.steps, log=True)
    for lv in range(3):
        lib_out = host[lv]
        pkg.lib().dns_export_state(ch.h, lv, lib_out.ctypes.data)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    e2e_ms = max(e0.elapsed_time(e1), 1e3 * t_e2e)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = U * args.steps * world / (e2e_ms * 1e-3) / 1e6

    # ---- batched channels sharded over the GPUs (every rank takes part)
    batched_multi = None
    if world > 1 and not args.no_batched:
        ch.close()
        peak_, _ = measured_peak()
        batched_multi = bench_batched(pkg, torch, args, peak_, rank=rank, world=world, dist=dist,
                                      device=local_rank)

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    # ---- roofline of the dominant kernel (fine stream-collide, both blocks)
    fine_ms, fine_n = kt["fine"]
    fine_nodes = 2 * geom.nxf * geom.nyf * p.zds
    bytes_per_launch = fine_nodes * 2 * 19 * 8
    achieved = bytes_per_launch / (fine_ms / fine_n * 1e-3) / 1e9 if fine_n else None
    peak, peak_kind = measured_peak()
    # launches per step: coarse, extract, GR x (fine + 2 interface), inject, finalize
    launches = args.steps * (4 + 3 * geom.gr)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (Philox-seeded laminar profile + noise)",
        "config": arm_config(args, world),
        "roofline": {"bound": "hbm", "kernel": "fine_kernel", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "traffic": traffic_from_profiles("fine_kernel", args.config)},
        "kernel_ms_per_step": {k: (v[0] / prof_steps) for k, v in kt.items()},
        "whole_step_hbm_frac": (U * args.steps * 304 / (ms_max * 1e-3) / 1e9) / peak,
        "e2e": {"value": e2e, "unit": "MLUPS", "h2d_bytes_per_step": state_bytes / args.steps,
                "d2h_bytes_per_step": (state_bytes + 72 * args.steps) / args.steps,
                "note": "import state from pinned host, K steps with per-step log read-back, export state"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "log_tail": {"force": float(log[-1, 1]), "flowrate": float(log[-1, 4]), "stress": float(log[-1, 7])},
    }
    if world == 1 and not args.no_budget:
        line["budget"] = bench_budget(pkg, ch, p, args.config)
    if world == 1 and args.longrun_cases:
        ch.close()
        line["longrun"] = bench_longrun(pkg, args)
    # ---- the FP32 deviation-storage form on the same workload (same GPU):
    # the single-channel handle (dns_create with FP32 precision), and the same
    # channel as a batch of one in the batched engine
    if not args.no_fp32:
        ch.close()  # (idempotent)
        p32 = pkg.make_params(**m, forcing=pkg.FORCING_CFR, device=local_rank)
        p32.precision = pkg.FP32
        n32 = max(128, -(-args.steps // 32) * 32)
        with pkg.Channel(p32) as c32:
            s32 = torch.cuda.Stream()
            c32.set_stream(s32.cuda_stream)
            c32.init_seeded(42 + rank, 0.05, 0.005)
            c32.step(args.warmup, log=False)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s32)
            c32.step(n32, log=True)
            e1.record(s32)
            barrier()
            ms32 = max_over_ranks(torch, dist, e0.elapsed_time(e1))
            c32.set_profiling(True)
            c32.step(min(n32, 400), log=False)
            kt32 = c32.kernel_times()
            c32.set_profiling(False)
        v32 = U * n32 * world / (ms32 * 1e-3) / 1e6
        line["fp32"] = {"value": v32, "unit": "MLUPS", "steps": n32, "ms_per_step": ms32 / n32,
                        "dtype": "f32 (deviation storage, FP64 reductions)", "engine": "single channel (dns_step)",
                        "over_fp64": v32 / value,
                        "whole_step_hbm_frac": (U * n32 * 152 / (ms32 * 1e-3) / 1e9) / peak,
                        "kernel_ms_per_step": {k: v[0] / min(n32, 400) for k, v in kt32.items()}}
        b1 = pkg.Batch(local_rank)
        p1 = pkg.make_params(**m, forcing=pkg.FORCING_CFR, device=local_rank)
        tile32 = b1.autotune(p1, steps=5)[0] if args.autotune else None
        b1.add(p1, steps=10 ** 9, seed=42 + rank)
        b1.run(args.warmup)
        # the batched engine replays 32-step graphs and single-step graphs for
        # the rest: timed over whole groups (at least 128 steps) so that the
        # figure is the replayed step's, not the single-step graphs'
        msb = max_over_ranks(torch, dist, timed_batch_run(torch, b1, n32))
        b1.close()
        vb = U * n32 * world / (msb * 1e-3) / 1e6
        line["fp32"]["batch_of_one"] = {"value": vb, "unit": "MLUPS", "steps": n32, "ms_per_step": msb / n32,
                                        "engine": "batched, one instance", "tile": tile32 if tile32 else "default",
                                        "over_fp64": vb / value,
                                        "whole_step_hbm_frac": (U * n32 * 152 / (msb * 1e-3) / 1e9) / peak}
    if world == 1 and not args.no_batched:
        line["batched"] = bench_batched(pkg, torch, args, peak)
    if batched_multi is not None:
        line["batched"] = batched_multi
        line["batched"]["whole_step_hbm_frac"] /= world  # of N GPUs' bandwidth
    if "batched" in line:
        line["batched"]["over_fp64_plain"] = line["batched"]["value"] / value
    if world == 1 and not args.no_served:
        line["served"] = bench_served(pkg, torch, args, peak)
    if world == 1 and not args.no_cpu_baseline:
        m_ = CONFIGS[args.config][0]
        secs = reference_cpu(args.config, args.cpu_steps, 1)
        if secs:
            line["cpu_baseline"] = {"value": U * args.cpu_steps / secs[0] / 1e6, "unit": "MLUPS", "cores": 1,
                                    "kind": "reference",
                                    "sample": f"{args.cpu_steps} coarse steps of {args.config}, one single-rank "
                                              "reference process (its own routines, own step-loop clock)"}
        else:
            line["cpu_baseline"] = None
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c2")
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-budget", action="store_true")
    ap.add_argument("--autotune", action=argparse.BooleanOptionalAction, default=False,
                    help="autotune the tiles of the FP32 and batched legs (the engine's own tuner, "
                         "per grid shape) before timing them")
    ap.add_argument("--c4-instances", type=int, default=96)
    ap.add_argument("--c4-steps", type=int, default=2000)
    ap.add_argument("--no-c4-reference", action="store_true",
                    help="skip the batched channels' FP64 runs (throughput only)")
    ap.add_argument("--c5-requests", type=int, default=100)
    ap.add_argument("--c5-fp64-requests", type=int, default=24,
                    help="first requests of each stream served alone by the FP32 loop and one at a time in FP64")
    ap.add_argument("--c5-rates", type=float, nargs="+", default=[10.0])
    # the default run keeps to a few minutes: config 2's long run (about 40 s);
    # config 3's three cases (about 75 s each) with --longrun-cases c2 c3n c3r c3p
    ap.add_argument("--longrun-cases", nargs="*", default=["c2"],
                    help="channels run long for the FP32-vs-FP64 statistics (none: skip; config 3: c3n c3r c3p, "
                         "c3n being the no-slip companion of the drag reduction)")
    ap.add_argument("--longrun-warmup", type=int, default=10000)
    ap.add_argument("--longrun-steps", type=int, default=20000, help="sampled steps after the warm-up")
    ap.add_argument("--longrun-c3-steps", type=int, default=15000,
                    help="sampled steps of the config-3 cases (the no-slip companion at Re_tau 395 reaches a NaN "
                         "wall stress at step 28,194 in FP64)")
    ap.add_argument("--longrun-windows", type=int, default=10, help="windows for the batch-means errors")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
