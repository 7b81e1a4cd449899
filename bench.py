"""Benchmark of the per-tile halo-finding path (run_tile) on B200.

Workload (default): single periodic tile, nmesh = 384^3 Float32, box 768 Mpc/h
(alatt 2), 2LPT, Eisenstein-Hu no-wiggle P(k) normalised to sigma8 = 0.808
(Om 0.315, Ob 0.049, OL 0.685, h 0.674, ns 0.965), 20 top-hat filters
Rf = 1.5 * 20^(i/19) Mpc/h, nbuff = 32, rmax2rs = 0, ioutshear = 1 (33-field
records), collapse table = the reference's 50 x 20 x 20 make_table output
(tests/golden/HomelTab_julia.dat), seed 7.  A "step" is one full run_tile of
that tile: noise, fields, filter bank + peaks, shells, records.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--plain]
  python bench.py --serve      # the serving stream: 200 requests, Poisson arrivals
  python bench.py --lightcone  # 4 lightcone tiles of 384^3 (run_multitile) + merge_catalog
  python bench.py --shells     # batched shell analysis: 10^6 peaks on a 512^3 power-law field
  python bench.py --table      # collapse-table generation (make_table, RK4) on the GPU
  python bench.py --split      # run_multitile_split, 8 tiles of nmesh 192 (--split-n 128..384)
Under torchrun each rank runs independent tiles on its own GPU (run_tile
does not shard: replicas) with its own seed; the job value is the tiles of
all ranks over the slowest rank's device time.

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "peakpatch.jl_b200"))

N_DEFAULT = 384
BOX_PER_CELL = 2.0
FILTERS = [1.5 * 20.0 ** (i / 19.0) for i in range(20)]
SEED = 7
METRIC = "tiles/s"


def tile_config(n: int):
    import peakpatch_b200 as pp
    return pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=BOX_PER_CELL * n,
                             nbuff=32, z_out=0.0, z_max=0.0, ievol=0, ilpt=2, ioutshear=1, wsmooth=1, rmax2rs=0.0)


def workload_name(n: int) -> str:
    return f"run_tile nmesh={n}^3 box={BOX_PER_CELL * n:g}Mpc/h 2LPT 20 top-hat filters ioutshear=1"


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as td
            td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.td = td
            self.pg = True

    def barrier(self):
        if self.pg:
            self.td.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.td.destroy_process_group()


# ---------------------------------------------------------------------------
# clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (a C++/OpenMP restatement of the reference's CPU
# run_tile) on a bounded sample of the same workload
# ---------------------------------------------------------------------------
def config_dict(n: int, world: int, path: str = "optimised") -> dict:
    """The workload's config, the same in both arms."""
    ws = 92 * n ** 3   # fields 8 x 4 B, spectra about 7 x 4 B, records 32 B per cell
    return {"workload": workload_name(n), "nmesh": n, "boxsize": BOX_PER_CELL * n, "filters": 20, "nbuff": 32,
            "ilpt": 2, "ioutshear": 1, "seed": SEED, "path": path,
            "l2": f"inputs larger than L2: each tile rewrites its fields ({4 * n ** 3 / 1e6:.0f} MB each), spectra "
                  f"and records, about {ws / 1e9:.2f} GB against 126 MB of L2",
            "parallelism": f"replicas x{world}"}


class CpuTile:
    """The oracle's run_tile on one tile: fields and the 20-filter peak search
    at full size once, then the shell analysis timed on random samples of the
    tile's peaks and extrapolated to all of them.  Two shell figures: the
    reference's own loop (every peak gathers its whole shell list), and the
    same loop stopping once the shells the later phases read are in (the
    truncation the GPU path uses; the same results)."""

    def __init__(self, n: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        from peakpatch_b200 import powerspec
        oracle.build()
        self.ora = oracle
        self.cores = os.cpu_count() or 1
        oracle.set_threads(self.cores)
        k, P = powerspec.eh_table()
        self.T = oracle.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
        cfg = tile_config(n)
        ocfg = oracle.Config(**{f: getattr(cfg, f) for f in oracle.Config.__dataclass_fields__})
        filters = [(i + 1, 1.686, R) for i, R in enumerate(FILTERS)]
        self.tm = {}
        self.st = oracle.run_tile_stages(ocfg, SEED, k, P, filters, self.T, peak_sample=np.arange(0), timings=self.tm)
        self.npk = len(self.st["peaks"]["ipp"])
        self.n = n
        self.rng = np.random.default_rng(0)
        self.pp = {False: [], True: []}    # per-peak seconds of each timed sub-batch, by truncation
        self.peaks = {False: 0, True: 0}
        self.secs = {False: 0.0, True: 0.0}
        self.est = {False: None, True: None}

    def _run(self, size: int, truncate: bool) -> float:
        st = self.st
        sub = np.sort(self.rng.choice(self.npk, size=min(self.npk, max(1, size)), replace=False))
        t0 = time.perf_counter()
        self.ora.analyse_peaks(st["fields"], st["peaks"]["ipp"][sub], st["Rf"][sub], st["ir2min"][sub],
                               st["ZZon"][sub], st["fcrit"], st["alatt"], st["shells"], self.T, nbuff=32,
                               truncate=truncate)
        return time.perf_counter() - t0, len(sub)

    def sample(self, budget_s: float, truncate: bool, parts: int = 4):
        """Times `parts` random sub-batches of about budget_s seconds in all."""
        if self.npk == 0:
            return
        if self.est[truncate] is None:   # per-peak cost from a small probe (not counted)
            dt, k = self._run(max(64, 8 * self.cores), truncate)
            self.est[truncate] = dt / k
        size = int(budget_s / parts / max(self.est[truncate], 1e-7))
        for _ in range(parts):
            dt, k = self._run(size, truncate)
            self.pp[truncate].append(dt / k)
            self.peaks[truncate] += k
            self.secs[truncate] += dt

    def reset_samples(self):
        self.pp = {False: [], True: []}
        self.peaks = {False: 0, True: 0}
        self.secs = {False: 0.0, True: 0.0}

    def figure(self, truncate: bool) -> dict:
        v = self.pp[truncate]
        mean = statistics.fmean(v)
        se = statistics.stdev(v) / np.sqrt(len(v)) / mean if len(v) > 1 else None
        shells_s = mean * self.npk
        tile_s = self.tm["fields_s"] + self.tm["peaks_s"] + shells_s
        return {"tiles_per_s": 1.0 / tile_s, "tile_s": tile_s, "shells_s_extrapolated": shells_s,
                "sampled_peaks": self.peaks[truncate], "sampled_s": self.secs[truncate],
                "rel_std_error": se}

    def baseline(self) -> dict:
        full, trunc = self.figure(False), self.figure(True)
        return {"value": full["tiles_per_s"], "unit": METRIC, "cores": self.cores, "kind": "port",
                "sample": (f"{workload_name(self.n)}: the oracle (C++/OpenMP + threaded pocketfft) runs the fields "
                           f"and the 20-filter peak search at full size ({self.tm['fields_s'] + self.tm['peaks_s']:.1f}"
                           f" s), then analyse_peak on {full['sampled_peaks']} random peaks of {self.npk} "
                           f"({full['sampled_s']:.1f} s, whole shell lists as the reference), extrapolated to all "
                           f"peaks (relative standard error {full['rel_std_error'] or 0:.3f})"),
                "stages_s": {"fields": self.tm["fields_s"], "peaks": self.tm["peaks_s"],
                             "shells_extrapolated": full["shells_s_extrapolated"]},
                "npeaks": self.npk,
                "truncated_shells": {**trunc, "note": "the same oracle loop stopping each peak's gather once the "
                                                      "shells its later phases read are in (the GPU's truncation; "
                                                      "identical results): separates the algorithmic gain from "
                                                      "the kernels'"}}


def cpu_baseline(n: int, budget_s: float = 20.0):
    c = CpuTile(n)
    c.sample(0.75 * budget_s, False)
    c.sample(0.25 * budget_s, True)
    return c.baseline()


def run_reference(args, dist: Dist):
    """The reference arm: the oracle's CPU run_tile on the host cores, each
    step a bounded sample of the tile (fields and peaks are timed once at
    full size; every step times the shell analysis of fresh random peaks)."""
    if dist.rank != 0:
        return
    n = args.n
    c = CpuTile(n)
    per_step = max(1.0, min(6.0, args.cpu_budget / 4))
    for _ in range(args.warmup):
        c.sample(0.5, False, parts=1)
        c.sample(0.2, True, parts=1)
    c.reset_samples()   # warm-up samples do not count
    vals, walls = [], []
    for _ in range(args.steps):
        k0 = len(c.pp[False])
        t0 = time.perf_counter()
        c.sample(0.75 * per_step, False, parts=2)
        c.sample(0.25 * per_step, True, parts=1)
        walls.append(time.perf_counter() - t0)
        step_pp = statistics.fmean(c.pp[False][k0:])
        vals.append(1.0 / (c.tm["fields_s"] + c.tm["peaks_s"] + step_pp * c.npk))
    base = c.baseline()
    v = base["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.fmean(walls),
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 shell sums", "data": "synthetic",
            "config": config_dict(n, args.gpus),
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "step_values": vals, "stages_s": base["stages_s"], "truncated_shells": base["truncated_shells"],
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "tile_s_extrapolated": 1.0 / v,
            "note": "each timed step runs a sample of the tile (ms_per_step is its wall time); value is the tile "
                    "rate extrapolated from all steps' samples with the full-size fields and peak search"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def run_ours(args, dist: Dist):
    import peakpatch_b200 as pp
    from peakpatch_b200 import powerspec
    n = args.n
    gpu = dist.local
    ctx = pp.Context(gpu)
    _apply_options(ctx, args)
    k, P = powerspec.eh_table()
    T = pp.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
    ctx.set_pk_table(k, P)
    ctx.set_collapse_table(T)
    cfg = tile_config(n)
    seed0 = SEED + 1000 * dist.rank
    cap = 4_000_000
    dev_out = ctx.alloc_device(cap * 33 * 4)
    host_out = ctx.alloc_host(cap * 33 * 4)
    for w in range(args.warmup):
        ctx.run_tile_into(cfg, seed0, FILTERS, dev_out, cap, plain=args.plain)
    # ---- device-resident throughput (value) ----
    dist.barrier()
    ctx.synchronize()
    clocks = ClockSampler(gpu)
    clocks.start()
    l0 = ctx.launch_count()
    ctx.event_record(0)
    shell_ms, shell_visits, npk_tot, nh_tot, stage = 0.0, 0, 0, 0, None
    gather_ms = 0.0
    for s in range(args.steps):
        cnt, rmax, npk, dms = ctx.run_tile_into(cfg, seed0, FILTERS, dev_out, cap, plain=args.plain)
        st = ctx.shell_stats()
        last_shell_stats = st
        shell_ms += st["ms"]
        gather_ms += st["kernel_ms"]["gather"]
        shell_visits += st["visits"]
        npk_tot += npk
        nh_tot += cnt
        stage = ctx.stage_ms()
    ctx.event_record(1)
    ctx.synchronize()
    launches = ctx.launch_count() - l0
    dev_ms = ctx.event_elapsed(0, 1)
    clk = clocks.stop()
    # ---- end to end through the public API with host output (e2e) ----
    dist.barrier()
    ctx.synchronize()
    t0 = time.perf_counter()
    ctx.event_record(2)
    h2d = d2h = 0
    for s in range(args.steps):
        cnt, rmax, npk, dms = ctx.run_tile_into(cfg, seed0, FILTERS, host_out, cap, plain=args.plain)
        d2h += cnt * 33 * 4 + 64
        h2d += len(FILTERS) * 8 + 4 * len(FILTERS)
    ctx.event_record(3)
    ctx.synchronize()
    e2e_ms = ctx.event_elapsed(2, 3)
    wall_e2e = time.perf_counter() - t0
    dist.barrier()
    dev_ms_max = dist.max(dev_ms)
    e2e_ms_max = dist.max(max(e2e_ms, wall_e2e * 1000.0))
    tiles = dist.sum(float(args.steps))
    value = tiles / (dev_ms_max / 1000.0)
    e2e = tiles / (e2e_ms_max / 1000.0)
    # roofline of the dominant own kernel (the shell gather): algorithmic
    # bytes = in-bounds cell visits x 32 B packed record (delta, deltaT,
    # psi1 x3, psi2 x3 as Float32)
    bytes_alg = shell_visits * 32
    achieved = bytes_alg / (gather_ms / 1000.0) / 1e9 if gather_ms > 0 else 0.0
    peaks = _measured_peaks()
    extra = {}
    if dist.rank == 0 and not args.plain and not args.no_extras:
        extra["plain_path"] = _plain_compare(ctx, cfg, seed0, dev_out, cap, value / max(1, dist.world))
        extra["serving_burst"] = _serving_burst(ctx)
    line = None
    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, compensated-f32 shell sums, f64 collapse walk",
            "data": "synthetic (seeded Threefry noise, EH P(k))",
            "config": config_dict(n, dist.world, "plain" if args.plain else "optimised"),
            "peaks_per_s": npk_tot / (dev_ms / 1000.0), "halos_per_tile": nh_tot / args.steps,
            "peaks_per_tile": npk_tot / args.steps,
            "stage_ms_last_step": stage,
            "shell_stats_last_step": last_shell_stats,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "gpu_launches": int(launches),
            "roofline": {"kernel": "gather_kernel (shell sums)", "bound": "hbm",
                         "achieved": achieved, "peak": peaks[0], "unit": "GB/s",
                         "frac": achieved / peaks[0] if peaks[0] else None,
                         "traffic": gather_traffic(last_shell_stats["visits"], last_shell_stats["pool_rows"]),
                         "traffic_model": "dram read 2.35 B per cell visit + dram write 218 B per profile row "
                                          "(ncu capture of the 384^3 launch)",
                         "peak_source": peaks[1],
                         "alg_bytes_per_launch": bytes_alg / max(1, args.steps),
                         "kernel_ms_per_launch": gather_ms / max(1, args.steps),
                         "shell_stage_ms_per_step": shell_ms / max(1, args.steps)},
            "clocks": clk,
            "graphs": ctx.graph_stats(),
            "autotune": ctx.tune_entries(),
        }
        line.update(extra)
    ctx.free_device(dev_out)
    ctx.free_host(host_out)
    ctx.close()
    return line


# DRAM traffic of the gather kernel: reads per cell visit (records the L2
# does not hold) and writes per profile row (the 24-double rows of the pool
# and the staging slots that reach DRAM), from the ncu capture of one launch
# on the 384^3 benchmark tile (dram__bytes_read.sum 1.94 GB and
# dram__bytes_write.sum 6.11 GB for 824,483,046 visits and 27,993,492 rows;
# the 256^3 tile's launch, 0.403 + 1.30 GB for 179,268,416 visits and
# 6,073,951 rows, is within 3 % of the same model)
GATHER_DRAM_READ_PER_VISIT = 1.94e9 / 824_483_046
GATHER_DRAM_WRITE_PER_ROW = 6.11e9 / 27_993_492


def gather_traffic(visits: float, rows: float) -> float:
    return GATHER_DRAM_READ_PER_VISIT * visits + GATHER_DRAM_WRITE_PER_ROW * rows


def _plain_compare(ctx, cfg, seed, dev_out, cap, opt_tiles_per_s):
    """The plain GPU path (full spheres, FP64 shell sums, unbatched
    transforms) on the same tile: one warm-up and one timed run."""
    ctx.run_tile_into(cfg, seed, FILTERS, dev_out, cap, plain=True)
    ctx.synchronize()
    ctx.event_record(4)
    cnt, rmax, npk, dms = ctx.run_tile_into(cfg, seed, FILTERS, dev_out, cap, plain=True)
    ctx.event_record(5)
    ctx.synchronize()
    ms = ctx.event_elapsed(4, 5)
    return {"tiles_per_s": 1000.0 / ms, "ms_per_tile": ms, "halos": cnt, "peaks": npk,
            "optimised_over_plain": opt_tiles_per_s * ms / 1000.0}


SERVE_SIZES = (128, 192, 256, 384)


def _serving_request(rng):
    import peakpatch_b200 as pp
    n = int(rng.choice(SERVE_SIZES))
    ievol = int(rng.integers(0, 2))
    s8 = float(rng.uniform(0.75, 0.85))
    box = BOX_PER_CELL * n
    cfg = pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=box, nbuff=32,
                            z_out=0.0, z_max=4.6 if ievol else 0.0, ievol=ievol, ilpt=2, ioutshear=1, wsmooth=1,
                            rmax2rs=0.0, cenx=-box / 2 if ievol else 0.0, ceny=-box / 2 if ievol else 0.0,
                            cenz=-box / 2 if ievol else 0.0)
    return cfg, int(rng.integers(1, 2**31)), (s8 / 0.808) ** 2


def _warm_request(n, ievol):
    import peakpatch_b200 as pp
    box = BOX_PER_CELL * n
    return pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=box, nbuff=32,
                             z_out=0.0, z_max=4.6 if ievol else 0.0, ievol=ievol, ilpt=2, ioutshear=1, wsmooth=1,
                             rmax2rs=0.0, cenx=-box / 2 if ievol else 0.0, ceny=-box / 2 if ievol else 0.0,
                             cenz=-box / 2 if ievol else 0.0)


def _serving_burst(ctx, nreq=24, slots=4):
    """nreq mixed requests (nmesh in {128,192,256,384}, random seeds,
    sigma8 in 0.75-0.85, ievol 0/1) submitted at once to the serving loop,
    against the same requests run one after another through run_tile.  Both
    arms are warm: before timing, the synchronous slot and every serving slot
    have run each grid size and walk class once (plans, buffers, graphs and
    the shell-stage tuning exist, as in a service that has been running)."""
    rng = np.random.default_rng(123)
    reqs = [_serving_request(rng) for _ in range(nreq)]
    warm = [_warm_request(n, ievol) for n in SERVE_SIZES for ievol in (0, 1, 1)]
    for cfg in warm:
        ctx.run_tile_arrays(cfg, 1000, FILTERS)
    t0 = time.perf_counter()
    for cfg, seed, sc in reqs:
        ctx.run_tile_arrays(cfg, seed, FILTERS, pk_scale=sc)
    seq_s = time.perf_counter() - t0
    ctx.serve_config(slots)
    for cfg in warm:
        for t in [ctx.submit(cfg, 1000 + s, FILTERS) for s in range(slots)]:
            ctx.wait(t)
    ctx.serve_stats_reset()
    t0 = time.perf_counter()
    tickets = [ctx.submit(cfg, seed, FILTERS, pk_scale=sc) for cfg, seed, sc in reqs]
    for t in tickets:
        ctx.wait(t)
    served_s = time.perf_counter() - t0
    st = ctx.serve_stats()
    return {"requests": nreq, "slots": slots, "sizes": list(SERVE_SIZES),
            "served_tiles_per_s": nreq / served_s, "sequential_tiles_per_s": nreq / seq_s,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "hbm_in_use_gb": st["hbm_in_use"] / 1e9}


def run_serve(args, dist: Dist):
    """The serving stream: 200 requests with Poisson arrivals (mean 4/s),
    nmesh uniform in {128,192,256,384}^3, random seeds, sigma8 uniform in
    0.75-0.85, ievol in {0,1}; latency from arrival to result."""
    import peakpatch_b200 as pp
    from peakpatch_b200 import powerspec
    if dist.rank != 0:
        return None
    ctx = pp.Context(dist.local)
    _apply_options(ctx, args)
    k, P = powerspec.eh_table()
    ctx.set_pk_table(k, P)
    ctx.set_collapse_table(pp.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat")))
    ctx.serve_config(args.slots)
    rng = np.random.default_rng(2026)
    reqs = [_serving_request(rng) for _ in range(args.requests)]
    gaps = rng.exponential(1.0 / args.rate, size=args.requests)
    # warm-up (not timed): every slot once for every grid size and both
    # ievol classes, so that cuFFT plans, graphs and the shell-stage tuning
    # of each kind of request exist before the stream starts
    # (ievol 0, 1, 1: the collapse walks of a lightcone batch set the walk
    # class the tuner keys the next batch of the slot on)
    for n in SERVE_SIZES:
        for ievol in (0, 1, 1):
            cfg = _warm_request(n, ievol)
            for t in [ctx.submit(cfg, 1000 + s, FILTERS) for s in range(args.slots)]:
                ctx.wait(t)
    ctx.serve_stats_reset()
    tuned_warm = len(ctx.tune_entries())
    done = []
    lock = threading.Lock()
    tickets = []

    def collector():
        while True:
            with lock:
                if len(done) == len(reqs):
                    return
                pending = [t for t in tickets if t not in done]
            for t in pending:
                if ctx.wait(t, timeout_ms=5) is not None:
                    with lock:
                        done.append(t)
            time.sleep(0.001)

    th = threading.Thread(target=collector)
    t0 = time.perf_counter()
    th.start()
    tnext = t0
    for (cfg, seed, sc), g in zip(reqs, gaps):
        tnext += g
        dt = tnext - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        t = ctx.submit(cfg, seed, FILTERS, pk_scale=sc)
        with lock:
            tickets.append(t)
    th.join()
    wall = time.perf_counter() - t0
    st = ctx.serve_stats()
    tuned_end = len(ctx.tune_entries())
    ctx.close()
    return {"metric": "tiles/s (served stream)", "value": st["tiles_per_s"], "unit": "tiles/s", "n_gpus": 1,
            "steps": args.requests, "warmup": len(SERVE_SIZES) * 3 * args.slots, "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "dtype": "f32 fields, compensated-f32 shell sums",
            "config": {"workload": "serving stream: Poisson arrivals, nmesh in {128,192,256,384}^3, sigma8 0.75-0.85, "
                                   "ievol 0/1", "requests": args.requests, "rate_per_s": args.rate,
                       "slots": args.slots},
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "failed": st["failed"], "wall_s": wall,
            "peaks_per_s": st["peaks_done"] / wall, "hbm_in_use_gb": st["hbm_in_use"] / 1e9,
            "tuned_kinds": {"after_warmup": tuned_warm, "at_end": tuned_end}}


def run_lightcone(args, dist: Dist):
    """Lightcone multi-tile: run_multitile with nmesh = 384, nbuff = 32
    (nsub = 320, full grid N = 704, alatt 2 Mpc/h), ievol = 1, z_out = 0,
    z_max = 4.6, observer at the corner of the 2^3 cores
    (cen = -N_core alatt / 2 = -640 Mpc/h); the 4 tiles of the (it, jt, 1)
    layer of ntile = 2, then merge_catalog.  A step is the whole chain.
    Under torchrun the tiles are shared round-robin between the ranks (each
    computes the global fields), rank 0 gathers the records in tile order and
    merges them."""
    import peakpatch_b200 as pp
    from peakpatch_b200 import distributed as D
    from peakpatch_b200 import powerspec
    n, nbuff, ntile = 384, 32, 2
    alatt = BOX_PER_CELL
    ncore = (n - 2 * nbuff) * ntile
    cen = -ncore * alatt / 2
    cfg = pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=alatt * n,
                            nbuff=nbuff, z_out=0.0, z_max=4.6, ievol=1, ilpt=2, ioutshear=1, wsmooth=1,
                            rmax2rs=0.0, cenx=cen, ceny=cen, cenz=cen)
    tiles = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (2, 2, 1)]
    mine = D.shard_tiles(tiles, dist.rank, dist.world)
    dcore = (n - 2 * nbuff) * alatt
    ctx = pp.Context(dist.local)
    _apply_options(ctx, args)
    k, P = powerspec.eh_table()
    ctx.set_pk_table(k, P)
    ctx.set_collapse_table(pp.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat")))
    empty = np.zeros((0, 33), np.float32)

    def chain():
        """this rank's tiles, then (rank 0) the gather and merge; returns
        (device s of run_multitile, device s of merge_catalog, catalogue)"""
        ctx.event_record(6)
        rec, rmax, npk = ctx.run_multitile_arrays(cfg, SEED, FILTERS, ntile, tiles=mine) if mine else (empty, 0.0, 0)
        ctx.event_record(7)
        ctx.synchronize()
        t_mt = ctx.event_elapsed(6, 7) / 1000.0
        full = rec
        if dist.world > 1:
            parts = dict(zip(mine, D.split_by_tile(rec, mine, ntile, dcore)))
            full = D.gather_tile_records(parts, tiles, 33)
        t_mg, merged = 0.0, None
        if dist.rank == 0:
            ctx.event_record(8)
            merged = ctx.merge_catalog(full)
            ctx.event_record(9)
            ctx.synchronize()
            t_mg = ctx.event_elapsed(8, 9) / 1000.0
        return t_mt, t_mg, full, merged, npk

    for _ in range(max(1, args.warmup)):
        chain()
    t_mt, t_mg, w_all = [], [], []
    for _ in range(args.steps):
        dist.barrier()
        t0 = time.perf_counter()
        a, b, full, merged, npk = chain()
        dist.barrier()
        w_all.append(time.perf_counter() - t0)
        t_mt.append(dist.max(a))
        t_mg.append(b)
    stage = ctx.stage_ms()
    sh = ctx.shell_stats()
    npk_all = dist.sum(float(npk))
    ctx.close()
    if dist.rank != 0:
        return None
    tm, tg = statistics.median(t_mt), statistics.median(t_mg)
    return {"metric": "tiles/s (lightcone chain)", "value": len(tiles) / (tm + tg), "unit": "tiles/s",
            "n_gpus": dist.world, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": 1000 * (tm + tg),
            "higher_is_better": True, "scaling": "strong" if dist.world > 1 else "weak", "vs_baseline": None,
            "data": "synthetic", "dtype": "f32 fields, compensated-f32 shell sums",
            "config": {"workload": "run_multitile lightcone: 4 tiles of 384^3 (nbuff 32, N = 704), ievol 1, "
                                   "z_max 4.6, observer at the core corner, then merge_catalog",
                       "tiles": tiles, "seed": SEED,
                       "parallelism": f"tiles round-robin over {dist.world} ranks" if dist.world > 1 else "1 GPU"},
            "multitile_ms": 1000 * tm, "merge_ms": 1000 * tg, "stage_ms_rank0": stage,
            "shell_kernel_ms_rank0": sh["kernel_ms"], "peaks": int(npk_all), "halos": len(full),
            "halos_after_merge": len(merged), "wall_ms_per_step": 1000 * statistics.median(w_all),
            "note": "device time (CUDA events on the library stream): the slowest rank's run_multitile plus "
                    "rank 0's merge_catalog; records copied to host inside it; the record gather between "
                    "ranks is in wall_ms_per_step only"}


# the multi-resolution sweep of the reference (run_multitile_split, GPU,
# RTX A5000): per-tile wall time and halo count at nmesh 128..384
SPLIT_PUBLISHED = {128: (0.818, 4982), 192: (2.550, 20467), 256: (6.667, 54057), 320: (12.312, 112271),
                   384: (20.605, 198049)}


def run_split_bench(args, dist: Dist):
    """run_multitile_split on the reference's GPU scaling-sweep workload:
    ntile 2 (8 tiles), nbuff 8, nmesh = --split-n (N = 2 (nmesh - 16) + 16,
    isolated boxes (2 nmesh)^3), boxsize = N * 226.67/68 Mpc/h (as the
    sweep sets it: the driver's cell is boxsize / nmesh), ilpt 2, ioutshear 0,
    the automatic coarse grid, P(k) = 1e4 k^-1.5 tabulated at 200
    log-spaced k in [1e-4, 10], filters 8 / 5 / 3 Mpc/h, the collapse table of
    make_table for (Om 0.31, Ob 0.049, OL 0.69, h 0.68), seed 42.  A step is
    the whole run: coarse phase, then per tile the split fields, peaks,
    shells and records, copied to the host.  Under torchrun the tiles are
    shared round-robin between the ranks (the reference's devices= dispatch)
    and rank 0 gathers the records."""
    import peakpatch_b200 as pp
    from peakpatch_b200 import distributed as D
    nm, nbuff, ntile = args.split_n, 8, 2
    nsub = nm - 2 * nbuff
    N = nsub * ntile + 2 * nbuff
    box = N * 226.67 / 68.0
    cfg = pp.PipelineConfig(Omx=0.261, OmB=0.049, Omvac=0.69, h=0.68, n=nm, boxsize=box, nbuff=nbuff,
                            z_out=0.0, z_max=0.0, ievol=0, ilpt=2, ioutshear=0, wsmooth=1, rmax2rs=0.0)
    rf = [8.0, 5.0, 3.0]
    tiles = [(it, jt, kt) for kt in (1, 2) for jt in (1, 2) for it in (1, 2)]
    mine = D.shard_tiles(tiles, dist.rank, dist.world)
    ctx = pp.Context(dist.local)
    _apply_options(ctx, args)
    k = 10.0 ** np.linspace(-4, 1, 200)
    ctx.set_pk_table(k, 1e4 * k ** -1.5)
    ctx.make_table(0.31, 0.049, 0.69, 0.68, install=1)
    from peakpatch_b200 import multires
    M = multires.coarse_grid_size(nm, nbuff, ntile)
    empty = np.zeros((0, 11), np.float32)

    def run():
        ctx.event_record(6)
        rec, _, npk = ctx.run_multitile_split_arrays(cfg, 42, rf, ntile, tiles=mine) if mine else (empty, 0.0, 0)
        ctx.event_record(7)
        ctx.synchronize()
        return ctx.event_elapsed(6, 7) / 1000.0, rec, npk

    for _ in range(max(1, args.warmup)):
        run()
    t_dev, t_wall = [], []
    for _ in range(args.steps):
        dist.barrier()
        t0 = time.perf_counter()
        a, rec, npk = run()
        dist.barrier()
        t_wall.append(dist.max(time.perf_counter() - t0))
        t_dev.append(dist.max(a))
    stage = ctx.stage_ms()
    full = rec
    if dist.world > 1:   # rank 0 gathers the last run's records in tile order
        dcore = nsub * (box / nm)
        parts = dict(zip(mine, D.split_by_tile(rec, mine, ntile, dcore)))
        full = D.gather_tile_records(parts, tiles, 11)
    npk_all = dist.sum(float(npk))
    ctx.close()
    if dist.rank != 0:
        return None
    nh = len(full)
    td, tw = statistics.median(t_dev), statistics.median(t_wall)
    pub = SPLIT_PUBLISHED.get(nm)
    line = {"metric": "tiles/s (run_multitile_split)", "value": len(tiles) / td, "unit": "tiles/s",
            "n_gpus": dist.world, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": 1000 * td,
            "higher_is_better": True, "scaling": "strong" if dist.world > 1 else "weak",
            "vs_baseline": (len(tiles) / td) / (1.0 / pub[0]) if pub else None, "data": "synthetic",
            "dtype": "f32 fields, compensated-f32 shell sums",
            "config": {"workload": f"run_multitile_split, ntile 2, nmesh {nm} (N {N}, coarse grid {M}^3, isolated "
                                   f"boxes {2 * nm}^3), nbuff 8, boxsize {box:.2f} Mpc/h, ilpt 2, ioutshear 0, "
                                   "P(k) = 1e4 k^-1.5, filters 8/5/3 Mpc/h, seed 42",
                       "parallelism": f"tiles round-robin over {dist.world} ranks" if dist.world > 1 else "1 GPU"},
            "e2e": {"value": len(tiles) / tw, "unit": "tiles/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(nh) * 11 * 4},
            "halos": int(nh), "peaks": int(npk_all), "stage_ms_rank0_last_run": stage,
            "note": "value: device time (CUDA events on the library stream) of the slowest rank's run; e2e: wall "
                    "clock of the Python call, records copied to the host (the records gather between ranks "
                    "follows the timed runs)"}
    if pub:
        line["reference_published"] = {"per_tile_s": pub[0], "tiles_per_s": 1.0 / pub[0], "halos": pub[1],
                                       "hardware": "RTX A5000 (the reference's GPU scaling sweep)"}
    return line


def _threefry2x64_20(k0, k1, c0, c1):
    """Threefry-2x64 with 20 rounds (Salmon et al., SC'11; Random123), on
    uint64 numpy arrays."""
    rot = (16, 42, 12, 31, 16, 32, 24, 21)
    M = np.uint64(0xFFFFFFFFFFFFFFFF)
    k0, k1 = np.uint64(k0), np.uint64(k1)
    ks = (k0, k1, k0 ^ k1 ^ np.uint64(0x1BD11BDAA9FC1A22))
    x0 = (c0 + ks[0]) & M
    x1 = (c1 + ks[1]) & M
    for r in range(20):
        x0 = (x0 + x1) & M
        x1 = ((x1 << np.uint64(rot[r % 8])) | (x1 >> np.uint64(64 - rot[r % 8]))) & M
        x1 ^= x0
        if r % 4 == 3:
            j = r // 4 + 1
            x0 = (x0 + ks[j % 3]) & M
            x1 = (x1 + ks[(j + 1) % 3] + np.uint64(j)) & M
    return x0, x1


def _resampled_table(T, nodes=(1000, 10, 10)):
    """The collapse table trilinearly resampled (in double precision) onto a
    finer node grid over the same (log F, e, p/e) ranges."""
    nx, ny, nz = nodes
    d = T.data.astype(np.float64)            # (nz, ny, nx) C order
    def axis(lo, hi, m, mt):
        x = np.linspace(0.0, mt - 1.0, m)
        i = np.minimum(np.floor(x).astype(int), mt - 2)
        return i, x - i
    ix, wx = axis(T.X1, T.X2, nx, d.shape[2])
    iy, wy = axis(T.Y1, T.Y2, ny, d.shape[1])
    iz, wz = axis(T.Z1, T.Z2, nz, d.shape[0])
    out = np.zeros((nz, ny, nx))
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = ((wz if dz else 1 - wz)[:, None, None] * (wy if dy else 1 - wy)[None, :, None] *
                     (wx if dx else 1 - wx)[None, None, :])
                out += w * d[(iz + dz)[:, None, None], (iy + dy)[None, :, None], (ix + dx)[None, None, :]]
    return out


def run_shells_bench(args, dist: Dist):
    """Batched shell analysis in isolation: a 512^3 Gaussian random field with
    P(k) = A k^-2.5 (seed 3; A set so that the cell rms of delta is 1), 2LPT
    displacements and the Laplacian; 10^6 peak cells uniform over the grid
    (Threefry-2x64-20, key (3, 0), counters 2^32 + i); per-peak shell limit
    R_p = clip(exp(ln 8 + 0.6 g), 2, 40) cells (g normal, numpy seed 3),
    Rf = R_p alatt (alatt 2 Mpc/h), ir2min = min(floor((1.75 R_p)^2),
    floor((40/alatt - 1)^2)); collapse table in Float64 on 1000 x 10 x 10
    nodes (the reference's 50 x 20 x 20 table resampled).  Times the shell
    stage on device-resident fields: the optimised path (adaptive
    truncation, compensated FP32 sums) and the plain path (full spheres to
    R_p, FP64 sums)."""
    import peakpatch_b200 as pp
    if dist.rank != 0:
        return None
    n, alatt, npk = args.shells_n, 2.0, args.shells_peaks
    ctx = pp.Context(dist.local)
    _apply_options(ctx, args)
    kk = np.logspace(-5, 2, 500)
    ctx.set_pk_table(kk, kk ** -2.5)
    cfg = pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=alatt * n, nbuff=32,
                            z_out=0.0, z_max=0.0, ievol=0, ilpt=2, ioutshear=1, wsmooth=1, rmax2rs=0.0)
    probe = ctx.generate_fields(cfg, 3)["delta"]
    scale = 1.0 / float(np.mean(probe.astype(np.float64) ** 2))
    del probe
    f = ctx.generate_fields(cfg, 3, pk_scale=scale)
    sigma = float(np.sqrt(np.mean(f["delta"].astype(np.float64) ** 2)))
    x0, _ = _threefry2x64_20(3, 0, np.uint64(2 ** 32) + np.arange(npk, dtype=np.uint64), np.zeros(npk, np.uint64))
    ipp = (x0 % np.uint64(n ** 3)).astype(np.int64) + 1
    g = np.random.default_rng(3).standard_normal(npk)
    R = np.clip(np.exp(np.log(8.0) + 0.6 * g), 2.0, 40.0)
    Rf = R * alatt
    ir2 = np.minimum(np.floor((1.75 * R) ** 2), np.floor((40.0 / alatt - 1) ** 2)).astype(np.int64)
    r2lim = np.floor(R ** 2).astype(np.int32)
    T = pp.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
    ctx.set_collapse_table_f64(_resampled_table(T), (T.X1, T.X2, T.Y1, T.Y2, T.Z1, T.Z2))
    out = {}
    for name, plain in (("optimised", False), ("plain", True)):
        # warm-up on the whole batch: tables, pool, and the autotuner's
        # timing of the order bricks and collapse widths for this batch
        ctx.analyse_peaks(f, ipp, Rf, ir2, 1.0, 1.686, alatt, 40, plain=plain, r2lim=r2lim)
        ctx.analyse_peaks(f, ipp, Rf, ir2, 1.0, 1.686, alatt, 40, plain=plain, r2lim=r2lim)
        st = ctx.shell_stats()
        km = st["kernel_ms"]
        gather_s = km["gather"] / 1000.0
        out[name] = {"shell_stage_ms": st["ms"], "kernel_ms": km, "visits": st["visits"], "pool_rows": st["pool_rows"],
                     "peaks_per_s": npk / (st["ms"] / 1000.0), "batches": st["batches"],
                     "gather_GBps": st["visits"] * 32 / gather_s / 1e9 if gather_s > 0 else None,
                     "halos": None}
    peaks = _measured_peaks()
    opt = out["optimised"]
    tune = ctx.tune_entries()
    ctx.close()
    return {"metric": "shell peaks/s (batched shell analysis)", "value": opt["peaks_per_s"], "unit": "peaks/s",
            "n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic", "dtype": "compensated-f32 shell sums, f64 collapse walk and table",
            "config": {"workload": f"{npk} peaks on a {n}^3 power-law (k^-2.5) field, R_p lognormal 2-40 cells, "
                                   "FP64 1000x10x10 table", "nmesh": n, "peaks": npk, "sigma_cell": sigma,
                       "pk_scale": scale},
            "optimised": opt, "plain": out["plain"], "autotune": tune,
            "roofline": {"kernel": "gather_kernel (compensated)", "bound": "hbm", "achieved": opt["gather_GBps"],
                         "peak": peaks[0], "unit": "GB/s", "frac": (opt["gather_GBps"] or 0) / peaks[0],
                         "traffic": gather_traffic(opt["visits"], opt["pool_rows"]), "peak_source": peaks[1],
                         "traffic_model": "dram read 2.35 B per cell visit + dram write 218 B per profile row "
                                          "(ncu capture of the 384^3 tile's launch)"},
            "optimised_over_plain": out["plain"]["shell_stage_ms"] / opt["shell_stage_ms"],
            "roofline_plain_gather": {"bound": "hbm", "achieved": out["plain"]["gather_GBps"], "peak": peaks[0],
                                      "frac": (out["plain"]["gather_GBps"] or 0) / peaks[0], "unit": "GB/s",
                                      "alg_bytes": out["plain"]["visits"] * 32}}


def run_table_bench(args, dist: Dist):
    """Collapse-table generation: make_table with the RK4 solver and the
    default 50 x 20 x 20 grid (log10 F in [log10 1.5, log10 8], e_v in
    [0, 0.5], p_v/e_v in [-1, 1]) for the Planck 2018 cosmology of the tile
    benchmark, on the GPU (one FP64 integration per node), beside the same
    table computed by the oracle on every host core."""
    import peakpatch_b200 as pp
    if dist.rank != 0:
        return None
    cosmo = (0.315, 0.049, 0.685, 0.674)
    ctx = pp.Context(dist.local)
    for _ in range(max(1, args.warmup)):
        ctx.make_table(*cosmo)
    ms, steps = [], 0
    for _ in range(args.steps):
        ctx.make_table(*cosmo)
        st = ctx.table_stats()
        ms.append(st["ms"])
        steps = st["rk4_steps"]
    ctx.close()
    t = statistics.median(ms)
    line = {"metric": "collapse tables/s (make_table, RK4, 50x20x20)", "value": 1000.0 / t, "unit": "tables/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "dtype": "f64", "config": {"workload": "make_table RK4, default CollapseTableParams and EllipsoidParams, "
                                                   "Om 0.315 Ob 0.049 OL 0.685 h 0.674", "nodes": 20000},
            "rk4_steps_per_table": steps, "rk4_steps_per_s": steps / (t / 1000.0)}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.build()
        cores = os.cpu_count() or 1
        oracle.set_threads(cores)
        t0 = time.perf_counter()
        oracle.make_table(*cosmo)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "tables/s", "cores": cores, "kind": "port",
                                "sample": "the whole 50x20x20 table, oracle C++/OpenMP (one node per task)"}
    return line


def _default_extras(args, dist: Dist) -> dict:
    """The batched shell kernel of 10^6 peaks on a 512^3 field, a shortened
    serving stream (60 Poisson requests at 4/s), the 128^3 tile (config 1,
    with its CPU figure) and the lightcone chain (config 4), run after the
    tile benchmark in the default invocation so that one line carries their
    numbers."""
    out = {}
    c1 = argparse.Namespace(**vars(args))
    c1.n, c1.steps, c1.warmup, c1.plain = 128, 20, 3, False
    l1 = run_ours(c1, dist)
    cb1 = cpu_baseline(128, budget_s=3.0)
    out["config1"] = {"metric": METRIC, "value": l1["value"], "unit": METRIC, "config": l1["config"],
                      "e2e": l1["e2e"], "roofline_frac": l1["roofline"]["frac"],
                      "halos_per_tile": l1.get("halos_per_tile"),
                      "cpu_baseline": {k: cb1[k] for k in ("value", "unit", "cores", "kind", "sample")}}
    c4 = argparse.Namespace(**vars(args))
    c4.steps, c4.warmup = 3, 3
    l4 = run_lightcone(c4, dist)
    out["config4_lightcone"] = {k: l4[k] for k in ("metric", "value", "unit", "config", "ms_per_step") if k in l4}
    out["config4_lightcone"].update({k: l4[k] for k in ("multitile_ms", "merge_ms", "halos", "halos_after_merge")
                                     if k in l4})
    a = argparse.Namespace(**vars(args))
    sh = run_shells_bench(a, dist)
    out["shells_batched"] = {k: sh[k] for k in ("metric", "value", "unit", "config", "roofline",
                                                "optimised_over_plain")}
    out["shells_batched"]["kernel_ms"] = sh["optimised"]["kernel_ms"]
    out["shells_batched"]["visits"] = sh["optimised"]["visits"]
    out["shells_batched"]["plain_peaks_per_s"] = sh["plain"]["peaks_per_s"]
    a.requests, a.rate = 60, 4.0
    sv = run_serve(a, dist)
    out["serving_stream"] = {k: sv[k] for k in ("metric", "value", "unit", "config", "p50_ms", "p99_ms", "failed",
                                                "wall_s", "peaks_per_s")}
    return out


def _apply_options(ctx, args):
    import peakpatch_b200 as pp
    ctx.set_option(pp.OPT_GRAPHS, 0 if getattr(args, "no_graphs", False) else 1)
    ctx.set_option(pp.OPT_AUTOTUNE, 0 if getattr(args, "no_autotune", False) else 1)
    if getattr(args, "collapse", 0):
        ctx.set_option(pp.OPT_COLLAPSE_THREADS, args.collapse)
    if getattr(args, "gather_ring", -1) >= 0:
        ctx.set_option(pp.OPT_GATHER_RING, args.gather_ring)
    if getattr(args, "gather_tex", -2) >= -1:
        ctx.set_option(pp.OPT_GATHER_TEX, args.gather_tex)
    if getattr(args, "collapse_order", -1) >= 0:
        ctx.set_option(pp.OPT_COLLAPSE_ORDER, args.collapse_order)


def _measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-path and serving-burst comparisons")
    ap.add_argument("--serve", action="store_true", help="run the serving stream instead of the tile benchmark")
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--lightcone", action="store_true", help="run the lightcone multi-tile chain instead")
    ap.add_argument("--shells", action="store_true", help="run the batched shell analysis instead")
    ap.add_argument("--shells-n", type=int, default=512)
    ap.add_argument("--shells-peaks", type=int, default=1_000_000)
    ap.add_argument("--table", action="store_true", help="run the collapse-table generation instead")
    ap.add_argument("--split", action="store_true", help="run the multi-resolution run_multitile_split instead")
    ap.add_argument("--split-n", type=int, default=192, help="nmesh of the --split workload")
    ap.add_argument("--no-graphs", action="store_true", help="launch kernels one by one instead of as CUDA graphs")
    ap.add_argument("--no-autotune", action="store_true", help="default shell-stage choices, no autotuning")
    ap.add_argument("--gather-tex", type=int, default=-2,
                    help="gather record loads: 1 texture pipe, 0 256-bit loads, -1 the tuner's choice (default: library)")
    ap.add_argument("--gather-ring", type=int, default=-1,
                    help="1: gather records through TMA-staged shared-memory rings, 0: plain loads (default: library)")
    ap.add_argument("--collapse-order", type=int, default=-1,
                    help="1: collapse peaks by descending crossing shell, 0: in gather-list order (default: library)")
    ap.add_argument("--collapse", type=int, default=0,
                    help="fix the collapse kernel (PPB_OPT_COLLAPSE_THREADS: 1, 2, 4, 8; 0 the tuner's choice)")
    args = ap.parse_args()
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, dist)
            return
        if args.shells:
            line = run_shells_bench(args, dist)
            if line is not None:
                print(json.dumps(line), flush=True)
            return
        if args.table:
            line = run_table_bench(args, dist)
            if line is not None:
                print(json.dumps(line), flush=True)
            return
        if args.split:
            line = run_split_bench(args, dist)
            if line is not None:
                print(json.dumps(line), flush=True)
            return
        if args.lightcone:
            line = run_lightcone(args, dist)
            if line is not None:
                print(json.dumps(line), flush=True)
            return
        if args.serve:
            line = run_serve(args, dist)
            if line is not None:
                print(json.dumps(line), flush=True)
            return
        line = run_ours(args, dist)
        if dist.rank == 0 and line is not None and dist.world == 1 and not args.no_extras and not args.plain:
            line.update(_default_extras(args, dist))
        if dist.rank == 0 and line is not None:
            if dist.world == 1 and not args.no_cpu_baseline:
                cb = cpu_baseline(args.n, budget_s=args.cpu_budget)
                line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                           "stages_s", "truncated_shells")}
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
