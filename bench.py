#!/usr/bin/env python3
"""Benchmark: batched multi-GNSS acquisition cells/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload acq_multi_24mhz|acq_l1ca_12mhz|acq_long_48mhz|track_24mhz|
                                refine_12mhz|mix_24mhz|ingest_raw32_24mhz|
                                search_batch_24mhz|l6_csk_24mhz] [--worklist -1|0|1]

Besides the default acquisition workload: acq_l1ca_12mhz is the plain 12 MHz
GPS L1 C/A search (32 PRNs x 41 bins x 5 x 4 ms), acq_long_48mhz the weak-signal
long coherent search (48 MHz, GPS L5-Q and QZSS L6D, 10 ms coherent =
480 000-point FFTs x 20 sums, 401 bins of 50 Hz), track_24mhz times the batched
tracking correlators (channel-epochs/s) and refine_12mhz the grid search plus
Gauss-Newton refinement of 64 signals (signals/s, with the refinement's cost
against the grid and its agreement with the FP64 oracle), mix_24mhz the
carrier wipe-off of a device-resident IF buffer (samples/s, HBM bound).

A step is one full search of the workload: every PRN of every signal group x
every Doppler bin x every code offset, accumulated over all non-coherent sums,
plus the per-PRN peak / C/N0 / fine-Doppler reduction. A cell is one
(PRN, Doppler bin, code offset) of the final grid.

Default workload acq_multi_24mhz: 24 MHz complex IQ, 3-bit, GPS L1 C/A (32
PRNs, 21 bins, 20 x 1 ms), Galileo E1-B (36 PRNs, 81 bins, 5 x 4 ms, BOC(1,1)),
BeiDou B1I (63 PRNs, 21 bins, 20 x 1 ms), GPS L5-I (32 PRNs, 21 bins, 20 x 1 ms),
FFT length 2N - 343.9 M cells per step. Seeded synthetic IF (see
pocketsdr_b200/synth.py); each rank searches its own IF block (weak scaling,
no collective on the data path).

Timing: W warm-up steps; then K steps, each bracketed by CUDA events on the
launch stream, with an L2 flush (a 512 MB write) between steps outside the
events; barrier + synchronize around the timed region; the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "acq cells/s (PRN x Doppler x code-offset) on 1 B200, batched vs plain, same peaks"
UNIT = "cells/s"
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # 148 SM x 128 FP32 lanes x FMA at 1965 MHz


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def emit(line: dict) -> None:
    """Prints the one JSON result line; a CPU baseline names the host's CPU."""
    if isinstance(line.get("cpu_baseline"), dict):
        line["cpu_baseline"].setdefault("cpu_model", _cpu_model())
    print(json.dumps(line), flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="acq_multi_24mhz")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--prn-limit", type=int, default=None,
                    help="fewer PRNs per group (profiling runs)")
    ap.add_argument("--scaling", choices=("weak", "strong"), default="weak",
                    help="weak: one IF block per rank; strong: PRNs dealt over ranks")
    ap.add_argument("--t-sum", type=float, default=20e-3,
                    help="non-coherent time per group (s)")
    ap.add_argument("--worklist", type=int, choices=(-1, 0, 1), default=0,
                    help="consumer launches: 0 per group (default), 1 one work-list launch, "
                         "-1 the work list where the plan allows it")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thr = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def rd():
            for line in self.proc.stdout:
                self.rows.append([x.strip() for x in line.split(",")])
        self.thr = threading.Thread(target=rd, daemon=True)
        self.thr.start()

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thr:
            self.thr.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for nm, v in zip(names, r[4:8]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def make_workload(name: str, seed: int, prn_limit=None, t_sum=20e-3):
    from pocketsdr_b200 import synth
    if name == "acq_multi_24mhz":
        return synth.acq_multi_24mhz(seed=seed, prn_limit=prn_limit, t_sum=t_sum)
    if name == "acq_l1ca_12mhz":
        return synth.acq_l1ca_12mhz(seed=seed)
    if name == "acq_long_48mhz":
        return synth.acq_long_48mhz(seed=seed, prn_limit=prn_limit)
    raise SystemExit(f"unknown workload {name}")


def workload_code_ffts(wl, g):
    """Conjugated code DFTs [n_prn, L] of group g of a workload."""
    from pocketsdr_b200 import synth
    if getattr(wl, "name", "") == "acq_long_48mhz":
        return synth.long_code_ffts(g)
    return synth.group_code_ffts(g)


def cons_flops(groups) -> float:
    """Algorithmic FLOPs of the consumer kernels of one step: per (PRN, bin,
    sum) an L-point inverse FFT (5 L log2 L), the code product with scaling
    (8 L) and the power accumulation (3 Nmax)."""
    f = 0.0
    for g in groups:
        per = 5 * g.L * math.log2(g.L) + 8 * g.L + 3 * g.Nmax
        f += len(g.prns) * len(g.fds) * g.n_sum * per
    return f


def cons_hbm_bytes(groups) -> float:
    """Unique HBM bytes of the consumer kernels of one step: forward spectra
    (8 L per bin and sum), code DFTs (8 L per PRN), grid written once
    (4 Nmax per PRN and bin)."""
    b = 0.0
    for g in groups:
        b += 8 * g.L * len(g.fds) * g.n_sum + 8 * g.L * len(g.prns) + 4 * g.Nmax * len(g.prns) * len(g.fds)
    return b


def load_traffic() -> dict:
    """ncu dram bytes per consumer launch, from profiles/cons_kernel_traffic.txt
    (`<workload> <bytes_per_launch>` lines), if recorded."""
    path = os.path.join(ROOT, "profiles", "cons_kernel_traffic.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            p = line.split()
            if len(p) == 2 and not line.startswith("#"):
                try:
                    out[p[0]] = float(p[1])
                except ValueError:
                    pass
    return out


# ---------------------------------------------------------------------------
def cpu_reference_rate(wl, max_threads: int | None = None, budget_prn: int | None = None,
                       max_bins: int | None = None, variants: dict | None = None):
    """Reference CPU throughput (cells/s) of the whole workload on this host,
    estimated from a bounded sample: for each group, up to `threads` PRN
    searches (every sum, the reference's own sdr_search_code built from
    source, or the oracle restatement when that build is absent) run in
    parallel threads, over every Doppler bin or the first `max_bins` (the
    search cost is the same per bin); core-seconds per PRN scale to the full
    bin and PRN sets, spread over all cores.

    With `variants` (a dict) two more rates are filled in: "single_thread"
    (one PRN search per group timed alone on one thread, scaled to the whole
    workload) and "no_sleep" (the all-core rate without sdr_search_code's 1 ms
    CPU release after every 22nd bin: the sleeps a full search makes, times
    the measured cost of the reference's own sdr_sleep_msec(1), taken off the
    core-seconds; the restatement does not sleep)."""
    import concurrent.futures as cf
    from oracle import oracle
    from pocketsdr_b200 import synth
    R = oracle.best()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    threads = min(cores, max_threads or cores)
    total_core_s, total_cells, sample_desc = 0.0, 0, []
    single_s, sleeps = 0.0, 0
    for g in wl.groups:
        n = min(len(g.prns), threads, budget_prn or threads)
        if getattr(wl, "name", "") == "acq_long_48mhz":
            cfs = [synth.long_replica_fft(g.sig, p, g.fs, g.T, g.L) for p in g.prns[:n]]
        else:
            cfs = [synth.tiled_code_fft(g.sig, p, g.fs, g.tile, g.N, g.L - g.N) for p in g.prns[:n]]
        buf = wl.bufs[g.buf]
        nb = min(len(g.fds), max_bins or len(g.fds))
        fds = np.ascontiguousarray(g.fds[:nb])

        def one(c):
            P = np.zeros((nb, g.L), np.float32)
            t0 = time.perf_counter()
            for s in range(g.n_sum):
                R.search_code(c, buf, (s * g.N) % len(buf), g.L, g.fs, g.fi, fds, P, g.T)
            R.corr_max(P, g.L, g.Nmax, nb, g.T)
            return (time.perf_counter() - t0) * len(g.fds) / nb
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            per = list(ex.map(one, cfs))
        wall = time.perf_counter() - t0
        core_s_per_prn = sum(per) / n
        total_core_s += core_s_per_prn * len(g.prns)
        total_cells += len(g.prns) * len(g.fds) * g.Nmax
        if variants is not None:
            single_s += one(cfs[0]) * len(g.prns)
            sleeps += g.n_sum * (len(g.fds) // 22) * len(g.prns)
        sample_desc.append(f"{g.sig}:{n}/{len(g.prns)} PRN" +
                           (f" x {nb}/{len(g.fds)} bins" if nb < len(g.fds) else "") +
                           f" ({wall:.1f}s)")
    rate = total_cells / (total_core_s / threads)
    if variants is not None:
        sleep_s = R.sleep_cost() if hasattr(R, "sleep_cost") else 0.0
        variants["single_thread"] = total_cells / single_s
        variants["no_sleep"] = total_cells / ((total_core_s - sleeps * sleep_s) / threads)
        variants["sleeps"] = {"count": sleeps, "ms_each": sleep_s * 1e3}
    return rate, threads, R.kind, "; ".join(sample_desc) + \
        f"; full PRN (and bin) sets extrapolated from core-seconds per PRN over {threads} threads"


def cpu_reference_full(wl, gpu_res=None, grid_groups=(), max_threads: int | None = None):
    """The reference's own search path over the WHOLE workload on this host's
    cores (oracle.search_groups: for every (group, PRN) sdr_search_code over
    every sum with its 1 ms CPU release every 22 bins, then sdr_corr_max and
    sdr_fine_dop, one PRN search per thread); for each group index in
    grid_groups the grid of its first visible satellite's PRN is kept."""
    from oracle import oracle
    keep = {}
    for gi in grid_groups:
        g = wl.groups[gi]
        vis = [s.prn for s in wl.sats if s.sig == g.sig and s.prn in g.prns]
        keep[gi] = g.prns.index(vis[0]) if vis else 0
    return oracle.search_groups(wl.groups, wl.bufs, [workload_code_ffts(wl, g) for g in wl.groups],
                                gpu_res=gpu_res, keep=keep, max_threads=max_threads)


def acq_parity(wl, gpu_res, ref, grids_gpu=None) -> dict:
    """Per-PRN GPU results against the reference's (cpu_reference_full) on
    the same IF: peak (Doppler bin, code offset) identical, C/N0 difference,
    fine Doppler difference; a differing peak whose cell holds, in the
    reference's own grid, a value within 1e-5 of the reference maximum is an
    FP32 tie (a replica tiled from a shorter periodic code has equal maxima
    one code period apart). With grids_gpu ({g: GPU grid of the PRN row the
    reference kept}), the largest grid difference per cell over
    max(|P_ref|, mean P_ref)."""
    r = ref["res"]
    same = (gpu_res["bin"] == r["bin"]) & (gpu_res["offset"] == r["offset"])
    tie = ~same & (np.abs(r["at_gpu"] - r["pmax"]) <= 1e-5 * r["pmax"])
    # a replica tiled from a shorter periodic code (the 12 MHz L1 C/A search:
    # 1 ms x 4) makes the grid periodic in the offset: its equal maxima lie
    # one code period apart, in the same Doppler bin
    period = np.concatenate([np.full(len(g.prns), g.N // g.tile if g.tile > 1 else 0)
                             for g in wl.groups])
    same_mod = tie & (gpu_res["bin"] == r["bin"]) & (period > 0) & \
        (gpu_res["offset"] % np.maximum(period, 1) == r["offset"] % np.maximum(period, 1))
    d_cn0 = np.abs(gpu_res["cn0"].astype(np.float64) - r["cn0"])
    d_fd = np.abs(gpu_res["fd"] - r["fd"])
    out = {"peaks_match": f"{int(same.sum())}/{len(r)}",
           "peaks_tied": int(tie.sum()),
           "tied_same_bin_offset_mod_code_period": int(same_mod.sum()),
           "peaks_differ": int((~same & ~tie).sum()),
           "cn0_max_diff_db": float(d_cn0[same | tie].max()) if (same | tie).any() else None,
           "fine_dop_max_diff_hz": float(d_fd[same].max()) if same.any() else None,
           "reference": f"{ref['kind']} build: sdr_search_code x sums + sdr_corr_max + "
                        f"sdr_fine_dop per PRN on the same IF, {ref['cores']} threads"}
    if grids_gpu:
        errs = {}
        for gi, (pi, Pr) in ref["grids"].items():
            Pg = grids_gpu.get(gi)
            if Pg is None:
                continue
            floor = float(Pr.mean(dtype=np.float64))
            e = np.abs(Pg.astype(np.float64) - Pr) / np.maximum(np.abs(Pr), floor)
            errs[f"{wl.groups[gi].sig}:{wl.groups[gi].prns[pi]}"] = float(e.max())
        out["grid_max_rel_err"] = max(errs.values()) if errs else None
        out["grid_prns"] = errs
    return out


def _bin_budget(wl):
    """Doppler bins per sampled PRN search on the CPU: all of them, except for
    the 480 000-point searches (401 bins x 20 sums would take minutes per PRN)."""
    return 2 if getattr(wl, "name", "") == "acq_long_48mhz" else None


# ---------------------------------------------------------------------------
def _reference_other(args):
    """The reference arm of the non-acquisition workloads: their reference
    CPU paths (the same functions as their cpu_baseline legs), one JSON line
    in each workload's metric and unit; refinement has no reference
    counterpart."""
    w = args.workload
    if w == "refine_12mhz":
        return {"impl": "reference", "unavailable": "the reference has no delay / Doppler "
                "refinement after its grid search (its finest estimate is sdr_fine_dop); "
                "refine_12mhz's cpu_baseline times the reference grid plus the FP64 oracle"}
    vals, desc, cores, kind, metric, unit, cfg = [], "", 0, "", "", "", {}
    # the arithmetic type of each workload's GPU arm, named the same here
    dtype = {"track_24mhz": "int8", "mix_24mhz": "u8/i8"}.get(w, "f32")
    for k in range(args.warmup + args.steps):
        if w == "track_24mhz":
            from pocketsdr_b200 import synth
            wl = synth.track_24mhz(seed=5)
            specs_list = []
            for e in range(20):
                sp = wl.jobs_at(e * 1e-3, [0] * len(wl.channels))
                for s_, c in zip(sp, [c for c in wl.channels
                                      if abs(round(e * 1e-3 / c.T) * c.T - e * 1e-3) < 1e-9]):
                    s_["ch"] = wl.channels.index(c)
                specs_list.append(sp)
            rate, cores, kind, desc = cpu_track_rate(wl, specs_list, synth.track_banks(wl))
            metric, unit = TRACK_METRIC, "channel-epochs/s"
            cfg = {"workload": w, "channels": len(wl.channels), "antennas": len(wl.bufs),
                   "taps": 44, "epochs_per_step": TRACK_EPOCHS_PER_STEP,
                   "l2": "flushed between timed steps (512 MB write outside the events)"}
            per_step = 100 * sum(len(sp) for sp in specs_list) / len(specs_list)   # 100 ms
        elif w == "ingest_raw32_24mhz":
            raw = np.random.default_rng(3).integers(0, 256, 24000 * 4 * 200, dtype=np.uint8)
            rate, cores, kind, desc = cpu_ingest_rate(ingest_config(24000), raw, 1000)
            metric, unit, cfg = INGEST_METRIC, "samples/s", {"workload": w}
            per_step = 2400000                                                     # 100 ms
        elif w == "l6_csk_24mhz":
            fs, fi, T, N, Lc, sats, buf, pos, cfs = _l6_workload(7)
            rate, cores, kind, desc = cpu_l6_rate(fs, fi, N, Lc, sats, buf, pos, cfs, 20)
            metric, unit, cfg = L6_METRIC, "channel-epochs/s", {"workload": w, "channels": 10}
            per_step = 250 * len(sats)                                             # 1 s
        elif w == "mix_24mhz":
            buf = np.random.default_rng(8).integers(0, 256, MIX_N, dtype=np.uint8)
            rate, cores, kind, desc = cpu_mix_rate(buf, 24e6, 2.0e6 + 1234.5, 0.3, 64_000_000)
            metric, unit, cfg = MIX_METRIC, "samples/s", dict(MIX_CFG)
            per_step = MIX_N
        elif w == "search_batch_24mhz":
            wl = make_workload("acq_multi_24mhz", 2)
            ref = cpu_reference_full(wl)
            n_srch = sum(len(g.prns) for g in wl.groups)
            rate, cores, kind = n_srch / ref["wall_s"], ref["cores"], ref["kind"]
            desc = f"all {n_srch} channel searches in every step, one per thread"
            metric, unit, cfg = SRCH_METRIC, "searches/s", {"workload": w, "channels": 163}
            per_step = 163                                                         # one call
        else:
            return None
        if k >= args.warmup:
            vals.append(rate)
    v = statistics.median(vals)
    return {"metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step / v * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": unit, "cores": cores, "kind": kind, "sample": desc},
            "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference(args):
    """The reference arm: the reference's own C search (oracle/_ref build of
    src/sdr_func.c, PocketFFT, AVX2, its 1 ms sleep every 22 bins included) on
    the host's cores. Acquisition workloads run WHOLE in every step (every
    PRN, bin and sum, one PRN search per thread), timed by wall clock; only
    the 480 000-point long search samples 2 of its 401 bins per PRN (the
    whole search takes minutes of all cores per step)."""
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    if args.workload not in ("acq_multi_24mhz", "acq_l1ca_12mhz", "acq_long_48mhz"):
        line = _reference_other(args)
        if line is None:
            raise SystemExit(f"unknown workload {args.workload}")
        emit(line)
        return 0
    wl = make_workload(args.workload, 2, args.prn_limit, args.t_sum)
    walls, desc, cores, kind = [], "", 0, ""
    for k in range(args.warmup + args.steps):
        if args.workload == "acq_long_48mhz":
            rate, cores, kind, desc = cpu_reference_rate(wl, budget_prn=4, max_bins=_bin_budget(wl))
            wall = wl.cells / rate
        else:
            ref = cpu_reference_full(wl)
            wall, cores, kind = ref["wall_s"], ref["cores"], ref["kind"]
            desc = (f"the whole workload in every step ({sum(len(g.prns) for g in wl.groups)} PRN "
                    f"searches, every bin and sum), one PRN search per thread over {cores} threads")
        if k >= args.warmup:
            walls.append(wall)
    v = wl.cells * len(walls) / sum(walls)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sum(walls) / len(walls) * 1e3,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": acq_config(wl, wl.groups, args.gpus, False, wl.cells),
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "timing": "wall clock per step on the host (perf_counter), steps summed"}
    emit(line)
    return 0


def acq_config(wl, groups, world: int, strong: bool, job_cells: int) -> dict:
    """The workload's config dict, the same in both arms' lines."""
    return {"workload": wl.name, "cells_per_step": job_cells,
            "groups": [f"{g.sig}:{len(g.prns)}prn x {len(g.fds)}bin x {g.Nmax}off x "
                       f"{g.n_sum}sum L={g.L}" for g in groups],
            "l2": "GPU arm: flushed between timed steps (512 MB write outside the events)",
            "parallelism": (f"PRNs dealt over {world} ranks, results all-gathered once"
                            if strong else f"replica x{world} (one IF block per rank)")}


def acq_measure(args, name: str, steps: int, warmup: int, dist, rank: int, world: int,
                local: int, cpu_leg: bool) -> dict:
    """One acquisition workload on this rank's GPU: the device-resident rate
    (K steps between CUDA events, L2 flushed between steps), the end-to-end
    rate through the public API (host IF in, host results out, CUDA graph
    replay), the consumer kernel's roofline and, with cpu_leg (rank 0, one
    GPU), the reference's CPU path over the whole workload on the same IF:
    its rate (cpu_baseline) and the per-PRN parity of the GPU results."""
    import torch
    from pocketsdr_b200 import acquire
    from pocketsdr_b200 import dist as D
    strong = args.scaling == "strong" and world > 1
    # weak: every rank searches its own IF block; strong: one IF block, the
    # PRNs of every group dealt over the ranks
    wl = make_workload(name, 2 + (0 if strong else rank), args.prn_limit, args.t_sum)
    full_groups = wl.groups
    shard_index = None
    if strong:
        wl.groups, shard_index = D.shard_groups(full_groups, rank, world)
    cfs = [workload_code_ffts(wl, g) for g in wl.groups]
    plan = acquire.AcqPlan(wl.groups, cfs)
    worklist = plan.set_worklist(args.worklist)
    cells = plan.cells
    job_cells = sum(len(g.prns) * len(g.fds) * g.Nmax for g in full_groups) if strong \
        else cells * world
    st = torch.cuda.Stream()          # every launch of ours and every event on it
    torch.cuda.set_stream(st)
    bufs_d = [torch.from_numpy(b).cuda() for b in wl.bufs]
    lens = [len(b) for b in wl.bufs]
    res_d = torch.empty(plan.n_res * acquire.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def step(graph=False):
        plan.run_device([b.data_ptr() for b in bufs_d], lens, wl.ix, res_d.data_ptr(), st.cuda_stream,
                        graph=graph)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    plan.profile(True)
    plan.profile_get()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    clk = ClockSampler(local)
    clk.start()
    torch.cuda.synchronize()
    for k in range(steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        step()
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    if dist:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    prof_all = plan.profile_get()
    prof_g = {k: v for k, v in prof_all.items() if k[0] != "span"}
    # launches of different groups overlap on the plan's streams: a kernel
    # family's time per step is its span (earliest start .. latest end)
    prof = {k: (prof_all[("span", k)][0],
                sum(v[1] for (g, kk), v in prof_g.items() if kk == k))
            for k in ("fwd", "cons", "peak")}
    plan.profile(False)
    total_ms = D.max_over_ranks(sum(step_ms), dist)
    value = job_cells * steps / (total_ms / 1e3)

    # the other consumer launch mode on the same plan and buffers, for comparison
    alt = None
    if plan.set_worklist(0 if worklist else -1) != worklist:   # the other mode, if any
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        a_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(steps)]
        for k in range(steps):
            flush.fill_(k & 0xFF)
            a_ev[k][0].record(st)
            step()
            a_ev[k][1].record(st)
        torch.cuda.synchronize()
        a_ms = D.max_over_ranks(sum(a.elapsed_time(b) for a, b in a_ev), dist)
        alt = {"launch": "per-group streams" if worklist else "work list",
               "value": job_cells * steps / (a_ms / 1e3), "ms_per_step": a_ms / steps}
        plan.set_worklist(args.worklist)

    # ---- end to end through the public API: host IF -> device -> results -> host
    bufs_h = [torch.from_numpy(b).pin_memory() for b in wl.bufs]
    res_h = torch.empty(res_d.numel(), dtype=torch.uint8).pin_memory()
    h2d = sum(b.numel() for b in bufs_h)
    d2h = res_h.numel()

    def e2e_step():
        for bh, bd in zip(bufs_h, bufs_d):
            bd.copy_(bh, non_blocking=True)
        step(graph=True)      # the captured launch sequence, one graph launch
        res_h.copy_(res_d, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
    for k in range(steps):
        flush.fill_((k + 1) & 0xFF)
        e2e_ev[k][0].record(st)
        e2e_step()
        e2e_ev[k][1].record(st)
    torch.cuda.synchronize()
    e2e_ms = D.max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev), dist)
    e2e_value = job_cells * steps / (e2e_ms / 1e3)
    res = np.frombuffer(res_h.numpy().tobytes(), dtype=acquire.RESULT_DTYPE)
    if strong:   # the per-PRN results of every rank, once (32 B per PRN)
        res = np.concatenate(D.gather_results(res, shard_index, full_groups, world, dist))

    # ---- roofline of the dominant kernel (consumer: code product + inverse FFT + power)
    cons_ms, cons_n = prof["cons"]
    flops_step = cons_flops(wl.groups)
    achieved = flops_step * steps / (cons_ms / 1e3) / 1e12 if cons_ms > 0 else None
    hbm_b = cons_hbm_bytes(wl.groups)
    traffic = load_traffic().get(name)
    roofline = {
        "kernel": "cons_kernel (code product + inverse FFT + |y|^2 accumulate)",
        "bound": "fp32", "achieved": achieved, "unit": "TFLOP/s",
        **_fp32_roofline(achieved),
        "flops_per_step": flops_step,
        "traffic": traffic,
        "traffic_source": ("ncu dram bytes read + written per consumer launch, measured on the "
                           "full workload and averaged over the consumer launches of one step "
                           "(profiles/cons_kernel_traffic.txt)" if traffic else None),
        "time_basis": "span of the concurrent consumer launches per step (CUDA events)",
        "span_ms_per_step": cons_ms / steps,
        "launches": cons_n,
        "share_of_step": cons_ms / sum(step_ms) if sum(step_ms) else None,
        "hbm": {"algorithmic_bytes_per_step": hbm_b,
                "achieved_gbs": hbm_b * steps / (cons_ms / 1e3) / 1e9 if cons_ms else None,
                "peak_gbs": _measured_hbm(), "frac": None},
    }
    if roofline["hbm"]["achieved_gbs"] and roofline["hbm"]["peak_gbs"]:
        roofline["hbm"]["frac"] = roofline["hbm"]["achieved_gbs"] / roofline["hbm"]["peak_gbs"]

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
            "scaling": "strong" if strong else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": acq_config(wl, full_groups, world, strong, job_cells // (1 if strong else world)),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "launch": "CUDA graph replay (sdrg_acq_run_graph)",
                    "graph_captures": plan.graph_captures()},
            "gpu_launches": sum(n for _, n in prof.values()),
            "kernel_ms_per_step": {(("all" if worklist and k != "peak" else wl.groups[g].sig)
                                    + f".{k}"): v[0] / steps
                                   for (g, k), v in prof_g.items() if v[1] > 0},
            "consumer_launch": ("work list: one forward launch for every group, one persistent "
                                "consumer launch (clusters of 8 where they fit, else 2) over every "
                                "group's (PRN, bin) tasks, a drain launch, each group's peaks"
                                if worklist else
                                "per group: forward, consumer and peak launches on concurrent "
                                "streams"),
            "roofline": roofline, "clocks": clocks,
            "detected": int(sum(1 for r in res if r["cn0"] >= 38.0))}
    if alt:
        line["other_launch_mode"] = alt
    if cpu_leg:
        if name == "acq_long_48mhz":
            # 480 000-point searches: a sample of the bins (the whole workload
            # takes several minutes of all cores); no per-PRN parity here
            var = {}
            rate, cores, kind, desc = cpu_reference_rate(wl, max_bins=_bin_budget(wl), variants=var)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                    "sample": desc, "single_thread": var["single_thread"],
                                    "no_sleep": var["no_sleep"], "sleeps": var["sleeps"]}
        else:
            ref = cpu_reference_full(wl, gpu_res=res, grid_groups=range(len(wl.groups)))
            grids_gpu = {gi: plan.grid(gi)[pi] for gi, (pi, _) in ref["grids"].items()}
            rate = wl.cells / ref["wall_s"]
            var = {}
            cpu_reference_rate(wl, budget_prn=1, variants=var)
            sleep_s = var["sleeps"]["ms_each"] / 1e3
            busy = ref["wall_s"] * ref["cores"] - var["sleeps"]["count"] * sleep_s
            line["cpu_baseline"] = {
                "value": rate, "unit": UNIT, "cores": ref["cores"], "kind": ref["kind"],
                "sample": f"the whole workload once ({sum(len(g.prns) for g in wl.groups)} PRN "
                          f"searches, every bin and sum) over {ref['cores']} threads: "
                          f"{ref['wall_s']:.2f} s wall",
                "single_thread": var["single_thread"],
                "no_sleep": wl.cells / (busy / ref["cores"]) if busy > 0 else None,
                "sleeps": var["sleeps"]}
            line["parity"] = acq_parity(wl, res, ref, grids_gpu)
    plan.close()
    return line, wl


def run_ours(args):
    import torch
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    from pocketsdr_b200 import dist as D
    dist = D.init(backend="nccl", device=torch.device("cuda", local))
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    line, wl = acq_measure(args, args.workload, args.steps, args.warmup, dist, rank, world,
                           local, cpu_leg)
    if rank == 0 and world == 1:
        cf = cufft_pipeline_rate(wl)
        if cf:
            cons_ms = line["roofline"]["span_ms_per_step"]
            line["cufft_comparison"] = {
                "cells_per_s": cf[0], "ms_per_step": cf[1], "ours_over_cufft": line["value"] / cf[0],
                "cufft_inverse_only_ms": cf[2],
                "ours_consumer_span_ms": cons_ms,
                "what": "timing only: torch.fft (cuFFT) forward FFTs of the blocks, code "
                        "product, inverse FFTs, |y|^2 summed over the sums, per-PRN max; "
                        "random data of the same shapes, FP32"}
    if args.workload == "acq_multi_24mhz" and world == 1 and args.prn_limit is None:
        # the plain 12 MHz GPS L1 C/A search (32 PRNs x 41 bins x 5 x 4 ms)
        # beside the headline, with its own CPU leg and parity
        sub, _ = acq_measure(args, "acq_l1ca_12mhz", max(args.steps, 20), max(args.warmup, 3),
                             dist, rank, world, local, cpu_leg)
        keep = ("value", "unit", "ms_per_step", "steps", "config", "e2e", "gpu_launches",
                "roofline", "clocks", "detected", "cpu_baseline", "parity")
        line["extra"] = {"acq_l1ca_12mhz": {k: sub[k] for k in keep if k in sub}}
        # refinement after the grid (64 signals at 12 MHz): its cost against
        # the plain grid search and its agreement with the FP64 oracle
        rf = refine_measure(args, 10, 3, with_oracle=cpu_leg, with_cpu=False)
        keep = ("value", "unit", "ms_per_step", "grid_ms", "refine_ms", "cost_vs_grid", "e2e",
                "config", "vs_fp64_oracle", "vs_truth", "clocks", "roofline")
        line["extra"]["refine_12mhz"] = {k: rf[k] for k in keep if k in rf}
        # the tracking correlator batch (256 channels x 44 taps, 100 ms steps)
        tr = track_measure(args, 3, 3, cpu_leg)
        keep = ("value", "unit", "ms_per_step", "steps", "config", "e2e", "gpu_launches",
                "tap_samples_per_s", "clocks", "cpu_baseline")
        line["extra"]["track_24mhz"] = {k: tr[k] for k in keep if k in tr}
        # the weak-signal long coherent search at full size (480 000-point
        # transforms, 42 PRNs x 401 bins x 20 sums; 1.6 s per step)
        lg, _ = acq_measure(args, "acq_long_48mhz", 2, 3, dist, rank, world, local, cpu_leg)
        keep = ("value", "unit", "ms_per_step", "steps", "config", "e2e", "gpu_launches",
                "roofline", "clocks", "cpu_baseline")
        line["extra"]["acq_long_48mhz"] = {k: lg[k] for k in keep if k in lg}
    if rank == 0:
        emit(line)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cufft_pipeline_rate(wl, reps: int = 3):
    """Timing comparison only, never the product path: the same search shapes
    through torch.fft (cuFFT) and torch elementwise kernels on random data -
    forward FFT of every (bin, sum) block, code product, inverse FFT, |y|^2 of
    the Nmax kept offsets summed over the sums, per-PRN maximum. Returns
    (cells/s, ms per search, ms of the search's inverse transforms alone), or
    None when the spectra would exceed 4 GB."""
    import torch
    dev = torch.device("cuda")
    if sum(len(g.fds) * g.n_sum * g.L * 8 for g in wl.groups) > (4 << 30):
        return None
    gen = torch.Generator(device=dev)
    gen.manual_seed(11)
    work = [(g, torch.randn((len(g.fds) * g.n_sum, g.L), dtype=torch.complex64, device=dev,
                            generator=gen),
             torch.randn((len(g.prns), g.L), dtype=torch.complex64, device=dev, generator=gen))
            for g in wl.groups]

    def search():
        peaks = []
        for g, x, c in work:
            nb, ns, L, Nmax = len(g.fds), g.n_sum, g.L, g.Nmax
            X = torch.fft.fft(x).view(nb, ns, L)
            pc = max(1, (1 << 30) // (nb * L * 8))          # PRNs per batch: ~1 GB of products
            for p0 in range(0, len(g.prns), pc):
                cc = c[p0:p0 + pc]
                P = None
                for s_ in range(ns):
                    Y = torch.fft.ifft(X[:, s_][None] * cc[:, None])
                    pw = torch.view_as_real(Y[..., :Nmax]).square().sum(-1)
                    P = pw if P is None else P.add_(pw)
                peaks.append(P.flatten(1).max(1))
        return peaks

    search()
    torch.cuda.synchronize()
    a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a_.record()
    for _ in range(reps):
        search()
    b_.record()
    torch.cuda.synchronize()
    ms = a_.elapsed_time(b_) / reps
    cells = sum(len(g.prns) * len(g.fds) * g.Nmax for g in wl.groups)
    # the inverse transforms alone: as many as the search makes, same lengths
    inv_ms = 0.0
    for g, x, c in work:
        n_inv = len(g.prns) * len(g.fds) * g.n_sum
        bt = max(1, min(n_inv, (1 << 30) // (g.L * 8)))
        Z = torch.randn((bt, g.L), dtype=torch.complex64, device=dev, generator=gen)
        torch.fft.ifft(Z)
        a_.record()
        done = 0
        while done < n_inv:
            k = min(bt, n_inv - done)
            torch.fft.ifft(Z[:k])
            done += k
        b_.record()
        torch.cuda.synchronize()
        inv_ms += a_.elapsed_time(b_)
        del Z
    del work
    torch.cuda.empty_cache()
    return cells / (ms / 1e3), ms, inv_ms


_FP32_PEAK = None


def _measured_fp32():
    """FP32 CUDA-core peak measured in this run: cuBLAS SGEMM of 8192^3 with
    TF32 off (every product an FP32 FMA), best of 5 after a warm-up - for FP32
    kernels what the cuBLAS bf16 figure is for tensor-core ones. TFLOP/s, or
    None when it cannot be measured."""
    global _FP32_PEAK
    if _FP32_PEAK is not None:
        return _FP32_PEAK
    import torch
    mm = torch.backends.cuda.matmul
    prev = getattr(mm, "fp32_precision", None)
    prev_tf32 = mm.allow_tf32
    try:
        if prev is not None:
            mm.fp32_precision = "ieee"
        mm.allow_tf32 = False
        n = 8192
        a = torch.randn(n, n, device="cuda", dtype=torch.float32)
        b = torch.randn(n, n, device="cuda", dtype=torch.float32)
        c = a @ b
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            c = a @ b
            e1.record()
            e1.synchronize()
            best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12)
        del a, b, c
        torch.cuda.empty_cache()
        _FP32_PEAK = best
    except Exception:
        _FP32_PEAK = None
    finally:
        if prev is not None:
            mm.fp32_precision = prev
        mm.allow_tf32 = prev_tf32
    return _FP32_PEAK


def _fp32_roofline(achieved):
    """peak, frac and their source for an FP32 kernel: the SGEMM figure of
    this run, else the nominal FMA rate; both reported."""
    meas = _measured_fp32()
    peak = meas or FP32_NOMINAL_TFLOPS
    src = ("measured in this run: cuBLAS SGEMM 8192^3, FP32 CUDA cores (TF32 off), best of 5"
           if meas else "nominal FP32 FMA rate at max clock (148 SM x 128 lanes x 2 x 1965 MHz)")
    return {"peak": peak, "frac": achieved / peak if achieved else None, "peak_source": src,
            "peak_nominal": FP32_NOMINAL_TFLOPS,
            "frac_nominal": achieved / FP32_NOMINAL_TFLOPS if achieved else None}


def _measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


TRACK_METRIC = "tracking correlator channel-epochs/s (mix + 44-tap corr_std per channel code period)"


def _track_setup(args, rank):
    import torch
    from pocketsdr_b200 import synth
    wl = synth.track_24mhz(seed=5 + rank)
    uniq = {}
    banks = synth.track_banks(wl)
    ptrs = []
    for c, bk in zip(wl.channels, banks):
        key = (c.sig, c.prn)
        if key not in uniq:
            uniq[key] = torch.from_numpy(bk).cuda()
        ptrs.append(uniq[key].data_ptr())
    return wl, uniq, ptrs


def cpu_track_rate(wl, specs_list, banks_host, max_jobs=6000, min_s=2.0):
    """Reference CPU rate (jobs/s): sdr_mix_carr + sdr_corr_std per job (the
    reference's own C build), driven from C over a pthread pool on every host
    core (oracle TrackRun), repeated until at least min_s has passed. Without
    that driver, the restatement's calls from a Python thread pool."""
    import concurrent.futures as cf
    from oracle import oracle
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    jobs = [s for specs in specs_list for s in specs][:max_jobs]
    if oracle.track_run_available():
        tr = oracle.TrackRun(wl.bufs, jobs, banks_host)
        tr.run(cores)                      # warm: page in the banks and buffers
        n, t0 = 0, time.perf_counter()
        while True:
            tr.run(cores)
            n += len(jobs)
            dt = time.perf_counter() - t0
            if dt >= min_s:
                break
        return n / dt, cores, tr.kind, (f"{len(jobs)} channel-epochs of the same stream, "
                                        f"{n // len(jobs)} passes, C pthread driver")
    R = oracle.best()
    jobs = jobs[:600]

    def one(s):
        IQ = R.mix_carr(wl.bufs[s["buf"]], s["ix"], s["N"], s["fs"], s["fc"], s["phi"])
        R.corr_std(IQ, banks_host[s["ch"]], s["coff"], s["pos"], False)
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        list(ex.map(one, jobs))
    dt = time.perf_counter() - t0
    return len(jobs) / dt, cores, R.kind, f"{len(jobs)} channel-epochs of the same stream"


TRACK_EPOCHS_PER_STEP = 100   # one step = 100 ms of the stream


def track_measure(args, steps: int, warmup: int, cpu_leg: bool) -> dict:
    """Tracking-correlator workload: every step is 100 ms of the 24 MHz
    8-antenna stream, 100 consecutive 1 ms epochs; each epoch is one batch
    (sdrg_corr_batch) of a correlator job per channel whose code period
    starts there (L1CA/L5I every ms, E1B every 4 ms). Open-loop trajectories,
    so the epochs' jobs are known in advance; still one batch per epoch, as a
    receiver closing its loops each epoch would run them. With cpu_leg, the
    reference's own mix + corr_std per job on the host's cores beside."""
    import torch
    from pocketsdr_b200 import synth, track
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    wl, uniq, ptrs = _track_setup(args, rank)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    bufs_d = [torch.from_numpy(b).cuda() for b in wl.bufs]
    lens = [len(b) for b in wl.bufs]
    E = TRACK_EPOCHS_PER_STEP
    n_ep = (warmup + steps) * E
    specs_list = []
    for e in range(n_ep):
        sp = wl.jobs_at(e * 1e-3, ptrs)
        for s, c in zip(sp, [c for c in wl.channels if abs(round(e * 1e-3 / c.T) * c.T - e * 1e-3) < 1e-9]):
            s["ch"] = wl.channels.index(c)
        specs_list.append(sp)
    jobs_list = [track.make_jobs(sp) for sp in specs_list]
    max_j = max(len(s) for s in specs_list)
    per_ep = max_j * track.SDR_MAX_CORR * 2          # floats of one epoch's correlations
    corr = torch.empty(E * per_ep, dtype=torch.float32, device="cuda")
    Cb = torch.empty(E * max_j * 4, dtype=torch.float32, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    ptr_b = [b.data_ptr() for b in bufs_d]

    def step(k):
        for i in range(E):
            track.corr_batch(jobs_list[k * E + i], ptr_b, lens, corr.data_ptr() + 4 * i * per_ep,
                             Cb.data_ptr() + 16 * i * max_j, st.cuda_stream)

    for k in range(warmup):
        step(k)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    clk = ClockSampler(local)
    clk.start()
    for k in range(steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        step(warmup + k)
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    timed = [specs_list[e] for e in range(warmup * E, n_ep)]
    n_jobs = sum(len(sp) for sp in timed)
    value = n_jobs / (ms / 1e3)
    taps = sum(len(s["pos"]) * s["N"] for sp in timed for s in sp)

    # end to end: the step's 100 ms of IF (every antenna) from pinned host
    # memory into the device buffers, the batches, every correlation back
    bufs_h = [torch.from_numpy(b).pin_memory() for b in wl.bufs]
    corr_h = torch.empty(corr.numel(), dtype=torch.float32).pin_memory()
    h2d = sum(b.numel() for b in bufs_h)
    d2h = corr_h.numel() * 4

    def e2e_step(k):
        for bh, bd in zip(bufs_h, bufs_d):
            bd.copy_(bh, non_blocking=True)
        step(k)
        corr_h.copy_(corr, non_blocking=True)

    e2e_step(0)
    torch.cuda.synchronize()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
    for k in range(steps):
        flush.fill_((k + 1) & 0xFF)
        e2e_ev[k][0].record(st)
        e2e_step(warmup + k)
        e2e_ev[k][1].record(st)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev)

    line = {"metric": TRACK_METRIC, "value": value, "unit": "channel-epochs/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic",
            "config": {"workload": "track_24mhz", "channels": len(wl.channels),
                       "antennas": len(wl.bufs), "taps": 44, "epochs_per_step": E,
                       "l2": "flushed between timed steps (512 MB write outside the events)"},
            "e2e": {"value": n_jobs / (e2e_ms / 1e3), "unit": "channel-epochs/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "tap_samples_per_s": taps / (ms / 1e3), "clocks": clocks,
            "gpu_launches": 3 * E * steps}
    if cpu_leg:
        banks_host = synth.track_banks(wl)
        rate, cores, kind, desc = cpu_track_rate(wl, specs_list, banks_host)
        line["cpu_baseline"] = {"value": rate, "unit": "channel-epochs/s", "cores": cores,
                                "kind": kind, "sample": desc}
    return line


def run_track(args):
    rank, world, _ = dist_info()
    line = track_measure(args, args.steps, args.warmup,
                         rank == 0 and world == 1 and not args.no_cpu_baseline)
    if rank == 0:
        emit(line)
    return 0


REFINE_METRIC = ("refined signals/s: grid search + 5 Gauss-Newton steps of (tau, fd, phi), "
                 "10 ms coherent x 4 blocks")
REFINE_FLOPS_PER_SAMPLE = 60   # mode-1 sums: sincos ~20, mixing 4, code 3, 11 accumulators ~33


def _fp64_refine(wl, th0, models):
    """The FP64 oracle's Gauss-Newton from th0 for every signal, threads over
    signals (the C oracle releases the GIL). Returns (theta [n, 3], wall s,
    threads)."""
    import concurrent.futures as cf
    from oracle.oracle import Restatement
    from pocketsdr_b200 import codes, synth
    orc = Restatement()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    def one(i):
        s = wl.sats[i]
        th, _, _ = orc.refine_gn(codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig),
                                 synth.CARRIER[s.sig], wl.fi, th0[i], wl.buf, wl.iq, wl.fs,
                                 wl.ix0, wl.Nb, wl.K, models)
        return th
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        out = np.array(list(ex.map(one, range(len(wl.sats)))))
    return out, time.perf_counter() - t0, cores


def refine_measure(args, steps: int, warmup: int, with_oracle: bool = True,
                   with_cpu: bool = True) -> dict:
    """Differentiable-refinement workload: 64 GPS L1 C/A + Galileo E1-B
    signals at 12 MHz (C/N0 30-45 dB-Hz, off-grid delay and Doppler). A step
    is the plain grid search (10 ms / 8 ms coherent, +-5 kHz) of all 64 PRNs
    followed by 5 Gauss-Newton steps from its peaks; the line reports both
    parts, their cost ratio and the refinement's agreement with the FP64
    oracle and with the truth (with_oracle) and, with with_cpu, the CPU
    baseline (reference grid + FP64 oracle Gauss-Newton)."""
    import torch
    from pocketsdr_b200 import acquire, codes, synth
    from pocketsdr_b200.refine import RefinePlan, RefineSpec
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    wl = synth.refine_12mhz(seed=4 + rank)
    n = len(wl.sats)
    models = [1] * 5
    acq = acquire.AcqPlan(wl.groups, [synth.periodic_code_ffts(g) for g in wl.groups])
    specs = [RefineSpec(codes.gen_code(s.sig, s.prn), synth.code_rate(s.sig), wl.fi,
                        synth.CARRIER[s.sig]) for s in wl.sats]
    plan = RefinePlan(specs, wl.fs, wl.iq, wl.Nb, wl.K)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    buf_d = torch.from_numpy(wl.buf).cuda()
    res_d = torch.empty(n * acquire.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    theta = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    rate = torch.zeros(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def grid():
        acq.run_device([buf_d.data_ptr()], [buf_d.numel()], [0], res_d.data_ptr(), st.cuda_stream)

    def refine():
        plan.from_peaks(res_d, 0, wl.ix0, theta, rate)
        plan.gn(buf_d, wl.ix0, theta, rate, models, info=False)

    for _ in range(warmup):
        grid()
        refine()
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    clk = ClockSampler(local)
    clk.start()
    for k in range(steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        grid()
        ev[k][1].record(st)
        refine()
        ev[k][2].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    grid_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / steps
    ref_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / steps
    # the sums kernel alone (mode 1), for its roofline
    s_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    flush.fill_(1)
    s_ev[0].record(st)
    for _ in range(10):
        plan.sums(buf_d, wl.ix0, theta, rate, mode=1)
    s_ev[1].record(st)
    torch.cuda.synchronize()
    sums_ms = s_ev[0].elapsed_time(s_ev[1]) / 10
    step_ms = grid_ms + ref_ms
    value = n / (step_ms / 1e3)

    # end to end: host IF -> device, grid + refinement, theta -> host
    buf_h = torch.from_numpy(wl.buf).pin_memory()
    th_h = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
    for k in range(steps):
        flush.fill_((k + 1) & 0xFF)
        e2e_ev[k][0].record(st)
        buf_d.copy_(buf_h, non_blocking=True)
        grid()
        refine()
        th_h.copy_(theta, non_blocking=True)
        e2e_ev[k][1].record(st)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev) / steps

    # parity with the FP64 oracle from the same starting peaks, and the truth
    res = np.frombuffer(res_d.cpu().numpy().tobytes(), dtype=acquire.RESULT_DTYPE)
    plan.from_peaks(res_d, 0, wl.ix0, theta, rate)
    th0 = theta.cpu().numpy()
    plan.gn(buf_d, wl.ix0, theta, rate, models, info=False)
    th = theta.cpu().numpy()
    line_extra = {}
    if rank == 0 and with_oracle:
        th_ref, cpu_gn_s, cores = _fp64_refine(wl, th0, models)
        div = np.array([2.0 if s.sig == "E1B" else 1.0 for s in wl.sats])
        rn = np.array([synth.code_rate(s.sig) for s in wl.sats])
        T = np.array([codes.code_cyc(s.sig) for s in wl.sats])
        tau_t = np.array([s.tau for s in wl.sats])
        fd_t = np.array([s.doppler for s in wl.sats])
        e_tau = ((th[:, 0] - tau_t + T / 2) % T - T / 2) * rn / div
        e0_tau = ((th0[:, 0] - tau_t + T / 2) % T - T / 2) * rn / div
        line_extra["vs_fp64_oracle"] = {
            "max_dtau_chip": float(np.max(np.abs(th[:, 0] - th_ref[:, 0]) * rn / div)),
            "max_dfd_hz": float(np.max(np.abs(th[:, 1] - th_ref[:, 1]))),
            "bar": "0.01 chip, 5 Hz"}
        # truth statistics over the signals the grid acquired (peak within
        # one chip and one 10 ms Doppler bin of the truth)
        ok = (np.abs(e0_tau) < 1.0) & (np.abs(th0[:, 1] - fd_t) < 50.0)
        line_extra["vs_truth"] = {
            "acquired": int(ok.sum()),
            "rms_dtau_chip": float(np.sqrt(np.mean(e_tau[ok] ** 2))),
            "rms_dfd_hz": float(np.sqrt(np.mean((th[ok, 1] - fd_t[ok]) ** 2))),
            "within_5hz": int(np.sum(np.abs(th[ok, 1] - fd_t[ok]) < 5.0)),
            "start_rms_dtau_chip": float(np.sqrt(np.mean(e0_tau[ok] ** 2))),
            "start_rms_dfd_hz": float(np.sqrt(np.mean((th0[ok, 1] - fd_t[ok]) ** 2)))}
        if world == 1 and with_cpu:
            class _W:   # the grid's groups / buffers in cpu_reference_rate's shape
                groups, bufs = wl.groups, [wl.buf]
            rate_c, cores_c, kind, desc = cpu_reference_rate(_W, budget_prn=4)
            cells = sum(len(g.prns) * len(g.fds) * g.Nmax for g in wl.groups)
            cpu_grid_s = cells / rate_c          # both legs use every host core
            cpu_s = cpu_grid_s + cpu_gn_s
            line_extra["cpu_baseline"] = {
                "value": n / cpu_s, "unit": "signals/s", "cores": cores_c,
                "kind": kind + " grid + port FP64 Gauss-Newton",
                "sample": desc + f"; Gauss-Newton: all {n} signals x 5 steps in the FP64 oracle "
                                 f"({cpu_gn_s:.1f} s on {cores} threads)",
                "grid_s": cpu_grid_s, "gn_s": cpu_gn_s}
    samples = n * wl.K * wl.Nb
    achieved = REFINE_FLOPS_PER_SAMPLE * samples / (sums_ms / 1e3) / 1e12
    line = {"metric": REFINE_METRIC, "value": value, "unit": "signals/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "refine_12mhz", "signals": n, "coherent_ms": 10, "blocks": wl.K,
                       "gn_steps": len(models), "model": "coherent (one real amplitude)",
                       "grid": [f"{g.sig}:{len(g.prns)}prn x {len(g.fds)}bin x {g.Nmax}off x "
                                f"{g.n_sum}sum L={g.L}" for g in wl.groups],
                       "l2": "flushed between timed steps (512 MB write outside the events)"},
            "grid_ms": grid_ms, "refine_ms": ref_ms, "cost_vs_grid": step_ms / grid_ms,
            "sums_kernel_ms": sums_ms,
            "e2e": {"value": n / (e2e_ms / 1e3), "unit": "signals/s",
                    "h2d_bytes_per_step": int(buf_h.numel()), "d2h_bytes_per_step": n * 24},
            "gpu_launches": None,
            "roofline": {"kernel": "refine_sums_kernel<1> (per-sample model, derivatives, 11 sums)",
                         "bound": "fp32", "achieved": achieved, "unit": "TFLOP/s",
                         **_fp32_roofline(achieved),
                         "flops_per_sample": REFINE_FLOPS_PER_SAMPLE, "samples": samples,
                         "traffic": None},
            "clocks": clocks, "detected": int(np.sum(res["cn0"] >= 30.0))}
    line.update(line_extra)
    acq.profile(True)
    acq.profile_get()
    grid()
    torch.cuda.synchronize()
    line["gpu_launches"] = (sum(v[1] for k, v in acq.profile_get().items() if k[0] != "span")
                            + 1 + 2 * len(models)) * steps
    acq.profile(False)
    plan.close()
    acq.close()
    return line


def run_refine(args):
    rank, _, _ = dist_info()
    line = refine_measure(args, args.steps, args.warmup, with_oracle=not args.no_cpu_baseline,
                          with_cpu=not args.no_cpu_baseline)
    if rank == 0:
        emit(line)
    return 0


MIX_METRIC = ("carrier wipe-off samples/s (sdr_mix_carr on a device-resident 24 MHz complex "
              "IF buffer: 4 s = 96 M packed samples per step)")
MIX_N = 96_000_000
MIX_IX = 12345          # window start: not 16-byte aligned, and the window wraps the buffer end
MIX_CFG = {"workload": "mix_24mhz", "samples_per_step": MIX_N, "ix": MIX_IX,
           "window": "starts at an unaligned offset and wraps the circular buffer's end",
           "l2": "flushed between timed steps (512 MB write outside the events); the 288 MB of "
                 "traffic per step exceeds L2 anyway"}


def cpu_mix_rate(buf, fs, fc, phi, n_samples):
    """Reference CPU rate (samples/s): the reference's own sdr_mix_carr over
    consecutive windows of the buffer, one window per host thread at a time,
    n_samples in all."""
    import concurrent.futures as cf
    from oracle import oracle
    R = oracle.best()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    W = 1_000_000
    n_win = max(cores, n_samples // W)

    def one(k):
        ix = (k * W) % (len(buf) - W)
        return R.mix_carr(buf, ix, W, fs, fc, phi + 0.01 * k).shape[0]
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        done = sum(ex.map(one, range(n_win)))
    wall = time.perf_counter() - t0
    return done / wall, cores, R.kind, (f"{n_win} windows of {W} samples over {cores} threads "
                                        f"({wall:.1f}s)")


def run_mix(args):
    """Carrier wipe-off (the mixing stage of every search and tracking
    epoch): one step mixes a 4 s window (96 M samples) of a 24 MHz complex
    3-bit IF buffer resident on the device (sdrg_mix_carr; bit-identical to
    sdr_mix_carr). HBM bound: 1 byte read, 2 bytes written per sample."""
    import ctypes as C
    import torch
    from pocketsdr_b200._lib import lib
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    rng = np.random.default_rng(8 + rank)
    buf = rng.integers(0, 256, MIX_N, dtype=np.uint8)
    fs, fc, phi = 24e6, 2.0e6 + 1234.5, 0.3
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    d_buf = torch.from_numpy(buf).cuda()
    d_out = torch.empty(2 * MIX_N, dtype=torch.int8, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def step():
        if lib.sdrg_mix_carr(C.c_void_p(d_buf.data_ptr()), MIX_N, MIX_IX, MIX_N, fs, fc, phi,
                             C.c_void_p(d_out.data_ptr()), C.c_void_p(st.cuda_stream)):
            raise RuntimeError("sdrg_mix_carr failed")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clk = ClockSampler(local)
    clk.start()
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        step()
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    from pocketsdr_b200 import dist as D
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    value = MIX_N / (ms / 1e3) * world
    # end to end: IF from pinned host memory, mixed samples back to the host
    buf_h = torch.from_numpy(buf).pin_memory()
    out_h = torch.empty(2 * MIX_N, dtype=torch.int8).pin_memory()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    for k in range(args.steps):
        e2e_ev[k][0].record(st)
        d_buf.copy_(buf_h, non_blocking=True)
        step()
        out_h.copy_(d_out, non_blocking=True)
        e2e_ev[k][1].record(st)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev) / args.steps
    bytes_step = 3 * MIX_N
    achieved = bytes_step / (ms / 1e3) / 1e9
    peak = _measured_hbm()
    line = {"metric": MIX_METRIC, "value": value, "unit": "samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/i8",
            "data": "synthetic", "config": dict(MIX_CFG),
            "e2e": {"value": MIX_N / (e2e_ms / 1e3) * world, "unit": "samples/s",
                    "h2d_bytes_per_step": MIX_N, "d2h_bytes_per_step": 2 * MIX_N},
            "gpu_launches": args.steps,
            "roofline": {"kernel": "mix_kernel (carrier wipe-off, one dp2a per sample)",
                         "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "peak_source": ("MEASURED_PEAKS.json" if os.path.exists(
                             os.path.join(ROOT, "MEASURED_PEAKS.json")) else "fallback 6650 GB/s"),
                         "algorithmic_bytes_per_step": bytes_step, "traffic": None},
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, kind, desc = cpu_mix_rate(buf, fs, fc, phi, 64_000_000)
        line["cpu_baseline"] = {"value": rate, "unit": "samples/s", "cores": cores, "kind": kind,
                                "sample": desc}
    if rank == 0:
        emit(line)
    return 0


INGEST_METRIC = ("IF ingest samples/s (Pocket SDR FE 8CH RAW32 at 24 MHz -> 8 RF + 2 array "
                 "cpx8 buffers, fs/4 mixing, LPF, beam-forming)")


def ingest_config(N):
    """The receiver setup of the ingest workload: RF channels 1-4 3-bit real
    (fs/4 real-to-complex) with the receiver's automatic LPF (cutoff
    0.9 * fs/4, src/sdr_rcv.c:538-545), 5-8 2-bit complex, and two array
    channels over channels 1-4 (Q8 weights of amplitude 64 = 256 / 4
    antennas, steering phases of a seeded beam)."""
    fs = 24e6
    rng = np.random.default_rng(11)
    ph = rng.uniform(0, 2 * np.pi, (2, 4))
    w = np.zeros((2, 8, 2), np.int16)
    w[:, :4, 0] = np.floor(64 * np.cos(ph) + 0.5)
    w[:, :4, 1] = np.floor(64 * np.sin(ph) + 0.5)
    return dict(fmt=6, N=N, fs=fs, IQ=[1, 1, 1, 1, 2, 2, 2, 2], bits=[3, 3, 3, 3, 2, 2, 2, 2],
                off=(0.0, 0.0), scale=(1.0, 1.0), lpf_fc=[0.9 * 0.5 * fs * 0.5] * 4 + [0.0] * 4,
                w=w, arch_on=[1, 1])


def cpu_ingest_rate(cfg_block, raw, n_blocks):
    """Reference CPU rate (samples/s): the reference's own write_buff (with its
    LPFs and array combine) over 1 ms blocks, one independent receiver per
    host thread, all host threads."""
    import concurrent.futures as cf
    from oracle import oracle
    chk = oracle.Ingest()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    N = cfg_block["N"]
    blocks = [raw[j * N * 4:(j + 1) * N * 4] for j in range(len(raw) // (N * 4))]

    def one(_):
        rcv = chk.receiver(**cfg_block)
        t0 = time.perf_counter()
        for j in range(n_blocks):
            rcv.write(blocks[j % len(blocks)], j)
        return time.perf_counter() - t0
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        per = list(ex.map(one, range(cores)))
    wall = time.perf_counter() - t0
    rate = cores * n_blocks * N / wall
    return rate, cores, chk.kind, (f"{n_blocks} blocks of {N} samples per thread, {cores} "
                                   f"independent receivers in parallel ({wall:.1f}s; mean "
                                   f"{statistics.mean(per) / n_blocks * 1e6:.0f} us per block)")


def run_ingest(args):
    """IF ingest workload: a step is 100 ms of 24 MHz RAW32 front-end data
    (100 receiver blocks of 1 ms, one call: the LPF history and fs/4 phase
    carry over exactly as block by block) into 8 RF + 2 array IF buffers."""
    import torch
    from pocketsdr_b200 import ingest
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    blk = 24000                     # the receiver's block (1 ms)
    K = 100                         # blocks per step
    cfg = ingest_config(blk * K)
    rng = np.random.default_rng(3 + rank)
    n_steps = args.warmup + args.steps
    NR = 16                         # raw blocks rotated through (16 x 9.6 MB)
    raw = rng.integers(0, 256, blk * K * 4 * NR, dtype=np.uint8)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    ing = ingest.Ingest(cfg["fmt"], cfg["N"], cfg["fs"], IQ=cfg["IQ"], bits=cfg["bits"],
                        lut_off=cfg["off"], lut_scale=cfg["scale"], lpf_fc=cfg["lpf_fc"],
                        w=cfg["w"], arch_on=cfg["arch_on"])
    raw_d = torch.from_numpy(raw).cuda()
    nbuf = ing.n_rf + ing.narch
    slots = 8                                   # IF buffers of 8 calls (800 ms) per channel
    bufs = [torch.zeros(cfg["N"] * slots, dtype=torch.uint8, device="cuda") for _ in range(nbuf)]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    step_bytes = cfg["N"] * 4

    def step(k, raw_src):
        j = k % (raw_src.numel() // step_bytes)
        ing.run(raw_src[j * step_bytes:(j + 1) * step_bytes], k * K, bufs,
                cfg["N"] * (k % slots), st.cuda_stream)

    for k in range(args.warmup):
        step(k, raw_d)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clk = ClockSampler(local)
    clk.start()
    reps = 200                                  # calls per timed step (a long enough region
                                                # for the clock sampler)
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        for r in range(reps):
            step(args.warmup + k * reps + r, raw_d)
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev) / (reps * args.steps)   # one call
    value = cfg["N"] / (ms / 1e3)
    # algorithmic bytes per sample: 4 raw + 8 RF + 2 array bytes
    bps = 4 + ing.n_rf + ing.narch
    achieved = bps * cfg["N"] / (ms / 1e3) / 1e9

    # end to end: raw bytes from pinned host memory, ingest, every buffer back
    raw_h = torch.from_numpy(raw[:step_bytes]).pin_memory()
    out_h = [torch.empty(cfg["N"], dtype=torch.uint8).pin_memory() for _ in range(nbuf)]
    raw_e = torch.empty(step_bytes * 2, dtype=torch.uint8, device="cuda")

    def e2e_step(k):
        raw_e[(k % 2) * step_bytes:(k % 2 + 1) * step_bytes].copy_(raw_h, non_blocking=True)
        step(k, raw_e)
        base = cfg["N"] * (k % slots)
        for b, o in zip(bufs, out_h):
            o.copy_(b[base:base + cfg["N"]], non_blocking=True)

    e2e_step(0)
    torch.cuda.synchronize()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_((k + 1) & 0xFF)
        e2e_ev[k][0].record(st)
        e2e_step(args.warmup + k)
        e2e_ev[k][1].record(st)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev) / args.steps
    line = {"metric": INGEST_METRIC, "value": value, "unit": "samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded random raw bytes: every 2/3-bit code equally likely)",
            "config": {"workload": "ingest_raw32_24mhz", "samples_per_step": cfg["N"],
                       "rf_channels": ing.n_rf, "array_channels": ing.narch, "lpf_channels": 4,
                       "timing": f"each timed step = {reps} back-to-back calls, averaged",
                       "l2": "flushed between timed steps (512 MB write outside the events); "
                             "calls rotate over 16 raw blocks (154 MB) and 8 output slots "
                             "(192 MB), more than L2"},
            "e2e": {"value": cfg["N"] / (e2e_ms / 1e3), "unit": "samples/s",
                    "h2d_bytes_per_step": step_bytes, "d2h_bytes_per_step": nbuf * cfg["N"]},
            "gpu_launches": reps * args.steps,
            "roofline": {"kernel": "ingest_kernel (unpack + fs/4 mix + LPF + array combine)",
                         "bound": "hbm", "achieved": achieved, "peak": _measured_hbm(),
                         "unit": "GB/s", "frac": achieved / _measured_hbm(),
                         "bytes_per_sample": bps, "traffic": None},
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = dict(cfg, N=blk)
        rate, cores, kind, desc = cpu_ingest_rate(cb, raw, 1000)
        line["cpu_baseline"] = {"value": rate, "unit": "samples/s", "cores": cores, "kind": kind,
                                "sample": desc}
    if rank == 0:
        emit(line)
    ing.close()
    return 0


SRCH_METRIC = ("channel searches/s: every idle channel of the multi-GNSS setup (163 channels, "
               "sdr_t_acq 20 ms) through one batched search call")


def run_search_batch(args):
    """Batched search scheduling: a step is one sdrg_search_batch call that
    searches every channel of the acq_multi_24mhz signal set (GPS L1 C/A 32,
    Galileo E1-B 36, BeiDou B1I 63, GPS L5-I 32; sdr_t_acq = 20 ms, so 20 /
    5 / 20 / 20 code periods) from its chips: grouping, plan and code DFTs on
    the device, search, decisions back on the host. Timed with CUDA events on
    the call's stream around the whole (synchronous) call, so host work
    inside it counts."""
    import torch
    from pocketsdr_b200 import codes, schedule
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    wl = make_workload("acq_multi_24mhz", 2 + rank)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    bufs_d = [torch.from_numpy(b).cuda() for b in wl.bufs]
    setups, reqs = [], []
    for i, g in enumerate(wl.groups):
        # the receiver's codes live on the device (uploaded once, not per call)
        chips = torch.from_numpy(np.stack([codes.gen_code(g.sig, p) for p in g.prns])).cuda()
        setups.append(schedule.Setup(chips, g.T, g.fs, g.fi, max_dop=5000.0, buf=g.buf, N=g.N))
        reqs += [schedule.Request(i, k) for k in range(len(g.prns))]
    t_acq, thres = 20e-3, 38.0
    for _ in range(args.warmup):
        schedule.search(setups, reqs, bufs_d, 0, t_acq, thres)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clk = ClockSampler(local)
    clk.start()
    res = None
    for k in range(args.steps):
        ev[k][0].record(st)
        res = schedule.search(setups, reqs, bufs_d, 0, t_acq, thres)
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    n = len(reqs)
    line = {"metric": SRCH_METRIC, "value": n / (ms / 1e3), "unit": "searches/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "search_batch_24mhz", "channels": n,
                                            "t_acq_s": t_acq, "thres_cn0": thres,
                                            "includes": "grouping, plan build, device code DFTs, "
                                                        "search, decisions to host"},
            "e2e": {"value": n / (ms / 1e3), "unit": "searches/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": n * 40,
                    "note": "the call is already end to end from the caller's view (device IF "
                            "buffers, host results)"},
            # per call and signal group: code DFT (forward + combine), forward
            # FFT, consumer, peak (partial + final)
            "gpu_launches": 6 * len(setups) * args.steps,
            "found": int(res["found"].sum()), "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = cpu_reference_full(wl)
        line["cpu_baseline"] = {"value": n / ref["wall_s"], "unit": "searches/s",
                                "cores": ref["cores"], "kind": ref["kind"],
                                "sample": f"all {n} channel searches once, one per thread"}
    if rank == 0:
        emit(line)
    return 0


L6_METRIC = ("L6 CSK channel-epochs/s (QZSS L6D, 24 MHz: mix + 96 000-point FFT correlation "
             "+ CSK decode per channel per 4 ms code period)")


def _l6_workload(seed, n_ch=10):
    """10 QZSS L6D channels (PRN 193-202) in a 24 MHz complex
    IF of 0.2 s, each keyed by its own code shift; per channel its code bank
    DFT (bank i % 10) and tap set (P, E, L, noise + 9 taps of 0.25 chip)."""
    from pocketsdr_b200 import codes, synth
    fs, fi, T = 24e6, 2.0e6, 4e-3
    N = int(fs * T)
    Lc = codes.SIGNALS["L6D"][0]
    rng = np.random.default_rng(seed)
    prns = list(codes.PRN_SETS["L6D"])[:n_ch]
    sats = [synth.Sat("L6D", p, 2.0 * float(rng.integers(0, 256)), float(rng.uniform(-3000, 3000)),
                      float(rng.uniform(0, 1)), 45.0) for p in prns]
    buf = synth.gen_if(int(0.2 * fs), fs, {"L6D": fi}, sats, iq=True, bits=3, seed=seed)
    sc = N / (Lc / 2)
    pos = np.array([0.0, -0.5 * sc, 0.5 * sc, -120.0] + list(np.arange(-4, 5) * 0.25 * sc))
    cfs = [codes.gen_code_fft(codes.gen_code("L6D", s.prn), T, -(i % 10) / fs / 10, fs, N, 0)
           for i, s in enumerate(sats)]
    return fs, fi, T, N, Lc, sats, buf, pos, cfs


def cpu_l6_rate(fs, fi, N, Lc, sats, buf, pos, cfs, n_epochs):
    """Reference CPU rate: sdr_mix_carr + sdr_corr_fft (reference build) and
    the reference channel's CSK per channel-epoch, one thread per channel."""
    import concurrent.futures as cf
    from oracle import oracle
    R = oracle.best()
    chk = oracle.Channel() if os.path.exists(oracle.CH_SO) else oracle.Restatement()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    def one(i):
        t0 = time.perf_counter()
        for e in range(n_epochs):
            ix = (e * N) % len(buf)
            IQ = R.mix_carr(buf, ix, N, fs, fi + sats[i].doppler, 0.0)
            chk.csk(R.corr_fft(IQ, cfs[i]), Lc, pos)
        return time.perf_counter() - t0
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=min(cores, len(sats))) as ex:
        list(ex.map(one, range(len(sats))))
    wall = time.perf_counter() - t0
    return (len(sats) * n_epochs / wall, min(cores, len(sats)), R.kind,
            f"{n_epochs} epochs x {len(sats)} channels, one thread per channel ({wall:.1f}s)")


def run_l6(args):
    """QZSS L6 CSK tracking: a step is 250 epochs (1 s) of 10 L6D channels,
    one sdrg_l6_csk_batch call per 4 ms epoch."""
    import torch
    from pocketsdr_b200 import track
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    fs, fi, T, N, Lc, sats, buf, pos, cfs = _l6_workload(7 + rank)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    d = torch.from_numpy(buf).cuda()
    cfd = [torch.from_numpy(c).cuda() for c in cfs]
    E = 250                                     # 1 s of stream per step

    def specs(e):
        ix = (e * N) % len(buf)
        return [dict(buf=0, ix=ix, N=N, fs=fs, fc=fi + s.doppler, phi=0.0, code_fft=cfd[i],
                     len_code=Lc, pos=pos) for i, s in enumerate(sats)]
    epochs = [specs(e) for e in range(E)]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    outs = [(torch.empty(len(sats), dtype=torch.uint8, device="cuda"),
             torch.empty((len(sats), 107), dtype=torch.complex64, device="cuda"),
             torch.empty((len(sats), N), dtype=torch.complex64, device="cuda")) for _ in range(4)]

    # the job arrays of every epoch are built before timing (a C host fills
    # its job array in place); the timed loop is one library call per epoch
    batches = [track.L6Batch(epochs[e], [d.data_ptr()], [len(buf)], outs[e % 4]) for e in range(E)]

    def step():
        for bt in batches:
            bt.run(st.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clk = ClockSampler(local)
    clk.start()
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        step()
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    n = E * len(sats)
    line = {"metric": L6_METRIC, "value": n / (ms / 1e3), "unit": "channel-epochs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "l6_csk_24mhz", "channels": len(sats),
                                            "epochs_per_step": E, "N": N, "taps": len(pos),
                                            "l2": "flushed between timed steps"},
            "e2e": {"value": n / (ms / 1e3), "unit": "channel-epochs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0,
                    "note": "device IF; results stay on the device (the tracking loop's next "
                            "step reads them there)"},
            "gpu_launches": 5 * E * args.steps,   # per epoch: code gather, code permutation,
                                                  # forward FFT, consumer, CSK decode (batched)
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, kind, desc = cpu_l6_rate(fs, fi, N, Lc, sats, buf, pos, cfs, 20)
        line["cpu_baseline"] = {"value": rate, "unit": "channel-epochs/s", "cores": cores,
                                "kind": kind, "sample": desc}
    if rank == 0:
        emit(line)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "search_batch_24mhz":
        return run_search_batch(args)
    if args.workload == "l6_csk_24mhz":
        return run_l6(args)
    if args.workload == "ingest_raw32_24mhz":
        return run_ingest(args)
    if args.workload == "mix_24mhz":
        return run_mix(args)
    if args.workload == "track_24mhz":
        return run_track(args)
    if args.workload == "refine_12mhz":
        return run_refine(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
