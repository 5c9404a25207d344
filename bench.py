#!/usr/bin/env python3
"""Benchmark of the SCMF polymer Monte Carlo hot path (move -> grid -> field).

Metric: MC bead-moves/s (beads x sweeps / time) on one B200.  A step is one MC
sweep of the large single system: 1.6M AB diblock chains of N=32 (51.2M
beads), f_A=0.3, 128^3 cells, chiN=25, kappaN=50, Philox seed 7, FP32 SoA
coordinates (614 MB, larger than L2, so no flush is needed), uint32 counts,
FP32 omega.  Inputs are synthetic (random-walk chains).  Beside it the line
carries the batched and served forms (256-system mix; Poisson request stream),
the roofline of the dominant kernel, an end-to-end number through the C ABI
with host buffers, and the CPU oracle (OpenMP) on this host's cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank runs its own replica (the path is one system per
GPU; replicas only), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MC bead-moves/s on 1 B200, batched/served vs plain; p50/p99 request latency"
UNIT = "bead-moves/s"
WORKLOAD = "large single system: 1.6M AB diblocks N=32 (51.2M beads), f_A=0.3, 128^3 cells, chiN=25, kappaN=50, seed 7"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["replicas", "sharded"], default="replicas",
                    help="N GPUs: a replica of the large system per rank (default), or the large system's "
                         "chains split over the ranks with an NCCL sum of the counts per sweep")
    ap.add_argument("--forms", choices=["all", "plain", "blend", "batched", "served"], default="all")
    ap.add_argument("--batched-sweeps", type=int, default=100)
    ap.add_argument("--served-requests", type=int, default=20000)
    ap.add_argument("--capacity-requests", type=int, default=3000)
    ap.add_argument("--served-rate", type=float, default=200.0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML in a thread."""
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
               0x100: "display_clock_setting"}

    def __init__(self, local_index: int):
        self.samples, self.reasons = [], 0
        self._stop = threading.Event()
        self._t = None
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = local_index
            if vis:
                parts = [p for p in vis.split(",") if p.strip()]
                if local_index < len(parts) and parts[local_index].strip().isdigit():
                    idx = int(parts[local_index])
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report nothing rather than guess
            self._nv = None
            self.error = str(e)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    nv.nvmlDeviceGetCurrentClocksThrottleReasons
                self.reasons |= get(self._h)
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        if self._nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self) -> dict:
        if self._t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        self._stop.set()
        self._t.join()
        reasons = [n for b, n in self.REASONS.items() if self.reasons & b]
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------- helpers
def workload_config(spec) -> dict:
    """The workload every arm of the bench runs (both arms print the same dict)."""
    return {"workload": WORKLOAD, "beads": spec.n_beads, "cells": spec.n_cells,
            "l2": "inputs larger than L2 (614 MB coordinates), no flush"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(key: str):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(key)
    except Exception:
        return None


def oracle_cpu_rate(spec, seconds: float, threads: int, warm: int = 1):
    """Bead-moves/s of the OpenMP oracle on this host: full sweeps of `spec`."""
    from oracle.oracle import OracleSystem, set_threads
    set_threads(threads)
    o = OracleSystem(spec)
    o.init_coords()
    o.reset_density()
    o.update_omega()
    o.step(warm)
    n, t0 = 0, time.perf_counter()
    while True:
        o.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return spec.n_beads * n / el, n, el


# ------------------------------------------------------------ reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import OracleSystem, set_threads
    from new_arch_b200.spec import large_system
    threads = os.cpu_count() or 1
    set_threads(threads)
    spec = large_system(seed=7)
    o = OracleSystem(spec)
    o.init_coords()
    o.reset_density()
    o.update_omega()
    # each step is one full sweep of the 51.2M-bead system; if the host is so
    # slow that K+W sweeps would exceed ~3 minutes, steps become bounded samples
    t0 = time.perf_counter()
    o.step(1)
    per = time.perf_counter() - t0
    budget = 180.0
    sweeps_per_step = 1
    sample = "one full sweep of the 51.2M-bead system per step"
    if per * (args.steps + args.warmup) > budget:
        sample = "first sweeps only (host too slow for K full sweeps)"
    for _ in range(max(0, args.warmup - 1)):
        o.step(1)
    done, t0 = 0, time.perf_counter()
    for _ in range(args.steps):
        o.step(sweeps_per_step)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    value = spec.n_beads * done / el
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * el / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(spec), "run": {"parallelism": f"{threads} host threads", "sweeps_timed": done},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import new_arch_b200 as nb
    from new_arch_b200.spec import batched_mix, large_system, served_request

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from new_arch_b200.replicas import gather_ints, reduce_max, replica_seed, whole_job_rate

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(v: float) -> float:
        return reduce_max(v, dist, "cuda")

    # ---- plain large system: the headline step (one replica per rank).  The K
    # sweeps are timed as the library runs them (scmf_step_async: one CUDA
    # graph replay per sweep) between CUDA events on the system's stream; a
    # second pass of K sweeps launch by launch, each launch between events,
    # gives the per-kernel times of the roofline and the phases.
    stream = torch.cuda.Stream()
    spec = large_system(seed=replica_seed(7, rank))
    s = nb.System(spec, stream=stream.cuda_stream)
    s.init_coords()
    s.step(args.warmup)  # also captures the sweep's graph
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    s.synchronize()
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.step_async(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    ms_total = ev0.elapsed_time(ev1)
    ms_move, ms_field, ms_profiled = s.step_profiled(args.steps)
    clocks = sampler.stop()
    barrier()
    ms_total = allmax(ms_total)
    st = s.stats()
    accept_ratio = st["last_accepts"] / spec.n_beads
    beads_all = gather_ints(spec.n_beads, dist, "cuda")
    value = whole_job_rate(beads_all, args.steps, ms_total / 1e3)
    peak, peak_kind = measured_peaks()
    # move+grid kernel per launch: read and write x, y, z (counts change only for
    # accepted moves that leave their cell, ~1 % of beads here: not counted)
    alg_bytes = 24 * spec.n_beads
    achieved = alg_bytes / (ms_move / args.steps / 1e3) / 1e9
    traffic = profiled_traffic("sweep_large_system")
    field_bytes = 8 * spec.n_types * spec.n_cells                           # read counts, write omega
    field_gbs = field_bytes / (ms_field / args.steps / 1e3) / 1e9

    # ---- end to end through the C ABI with host buffers
    xyz = s.coords()
    pinned = torch.empty(xyz.size, dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = xyz.reshape(-1)
    host_in = pinned.numpy()
    import ctypes
    stat_bytes = ctypes.sizeof(nb._lib.Stats)
    stats_host = torch.empty(stat_bytes * args.steps, dtype=torch.uint8, pin_memory=True)
    counts_host = torch.empty(spec.n_types * spec.n_cells, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    barrier()
    t0 = time.perf_counter()
    s.set_coords(host_in)
    for k in range(args.steps):
        s.step_stats_async(1, stats_host.data_ptr() + k * stat_bytes)
    s.synchronize()
    cnt = s.counts(out=counts_host)
    e2e_s = allmax(time.perf_counter() - t0)
    last = nb.System.stats_at(stats_host.data_ptr() + (args.steps - 1) * stat_bytes)
    assert last["step"] == st["step"] + args.steps and last["error_word"] == 0, last
    e2e = {"value": whole_job_rate(beads_all, args.steps, e2e_s), "unit": UNIT,
           "h2d_bytes_per_step": xyz.nbytes / args.steps,
           "d2h_bytes_per_step": (stat_bytes * args.steps + cnt.nbytes) / args.steps,
           "how": "wall clock around scmf_set_coords(pinned host xyz) + K x scmf_step_stats_async(1) (each sweep's "
                  "statistics copied to pinned host memory) + scmf_synchronize + scmf_get_counts (into pinned memory)"}
    s.close()
    del pinned

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (random-walk chains)",
            "config": workload_config(spec),
            "run": {"parallelism": f"replicas x{world}" if world > 1 else "single GPU", "sweeps_timed": args.steps},
            "clocks": clocks, "e2e": e2e, "gpu_launches": 2 * args.steps,
            "accept_ratio": accept_ratio,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "kernel": "k_sweep_lean<move+grid>",
                         "alg_bytes_per_launch": alg_bytes,
                         "traffic": traffic.get("dram_bytes_per_launch") if traffic else None,
                         "ms_per_launch": ms_move / args.steps},
            "phases": {"move_grid_ms": ms_move / args.steps, "field_ms": ms_field / args.steps,
                       "field_gbs": field_gbs, "field_frac": field_gbs / peak,
                       "profiled_ms_per_step": ms_profiled / args.steps,
                       "timing": "value: K graph-replayed sweeps between CUDA events on the system's stream; "
                                 "phases: K more sweeps launch by launch, each launch between events"}}

    # ---- the blend (largest single-GPU configuration), batched vs plain on the
    # same 256-system mix, and the served stream (rank-local)
    if args.forms in ("all", "blend"):
        line["configs"] = {"blend": run_blend(nb, args, peak)}
    if args.forms in ("all", "batched"):
        line["batched"] = run_batched(nb, batched_mix, args, torch, peak)
    if args.forms in ("all", "served"):
        line["served"] = run_served(nb, served_request, args)
        line["served_capacity"] = run_capacity(nb, served_request, args)

    # ---- CPU oracle on this host (rank 0, N=1 only)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, el = oracle_cpu_rate(spec, args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n} full sweeps of the 51.2M-bead system in {el:.1f} s (OpenMP oracle)"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_blend(nb, args, peak):
    """The homopolymer blend with a diblock compatibiliser (2M chains: A and B
    homopolymers of N=64 and 10 % AB diblocks of N=32, 121.6M beads,
    256x256x64 cells, chiN=15 at N_ref=64, kappaN=40, seed 11): device-timed
    sweeps with the per-phase HBM fractions."""
    import torch
    from new_arch_b200.spec import blend_system
    spec = blend_system(seed=11)
    K = args.steps
    stream = torch.cuda.Stream()
    with nb.System(spec, stream=stream.cuda_stream) as s:
        s.init_coords()
        s.step(args.warmup)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.step_async(K)  # graph replay, as for the large system
        ev1.record(stream)
        ev1.synchronize()
        ms_total = ev0.elapsed_time(ev1)
        ms_move, ms_field, _ = s.step_profiled(K)
        st = s.stats()
    move_gbs = 24 * spec.n_beads / (ms_move / K / 1e3) / 1e9
    field_gbs = 8 * spec.n_types * spec.n_cells / (ms_field / K / 1e3) / 1e9
    return {"workload": "blend: 50% A-homopolymer N=64, 40% B-homopolymer N=64, 10% AB diblock N=32; 2M chains "
                        "(121.6M beads), 256x256x64 cells, chiN=15 (N_ref=64), kappaN=40, seed 11",
            "beads": spec.n_beads, "cells": spec.n_cells, "sweeps_timed": K,
            "bead_moves_per_s": spec.n_beads * K / (ms_total / 1e3), "ms_per_step": ms_total / K,
            "move_ms": ms_move / K, "field_ms": ms_field / K,
            "move_gbs": move_gbs, "move_frac": move_gbs / peak, "field_gbs": field_gbs, "field_frac": field_gbs / peak,
            "accept_ratio": st["last_accepts"] / spec.n_beads}


def run_batched(nb, batched_mix, args, torch, peak):
    specs = batched_mix(256)
    st = torch.cuda.Stream()
    systems = [nb.System(sp, stream=st.cuda_stream) for sp in specs]
    for x in systems:
        x.init_coords()
    beads = sum(sp.n_beads for sp in specs)
    K = args.batched_sweeps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # plain engine: one system at a time, each with its own graph-launched sweeps
    for x in systems:
        x.step_async(1)
    torch.cuda.synchronize()
    e0.record(st)
    for x in systems:
        x.step_async(K)
    e1.record(st)
    e1.synchronize()
    plain_ms = e0.elapsed_time(e1)
    b = nb.Batch(systems, stream=st.cuda_stream)
    tune = b.autotune(2)
    trials = b.tune_trials()
    b.step_async(1)
    torch.cuda.synchronize()
    e0.record(st)
    b.step_async(K)
    e1.record(st)
    e1.synchronize()
    batched_ms = e0.elapsed_time(e1)
    # per-phase device time of the batched sweeps (launch by launch, no graph)
    pm, pf, _ = b.step_profiled(10)
    cells_all = sum(sp.n_cells * sp.n_types for sp in specs)
    b.close()
    for x in systems:
        x.close()
    plain = beads * K / (plain_ms / 1e3)
    batched = beads * K / (batched_ms / 1e3)

    def move_launches(lengths):
        # one register-kernel launch per tile kind: chains filling warps exactly, chains across warps
        kinds = {32 % ((n + 1) // 2) != 0 for n in lengths}
        return len(kinds)
    per_sys = sum(1 + move_launches([a.length for a in sp.archs]) for sp in specs)
    per_batch = 1 + move_launches([a.length for sp in specs for a in sp.archs])
    return {"workload": "256 diblock systems, edges {16..64}^3, N {16..64}, 100 sweeps each", "beads": beads,
            "sweeps": K, "plain_bead_moves_per_s": plain, "batched_bead_moves_per_s": batched,
            "batched_over_plain": batched / plain, "tune": tune, "gpu_launches_batched": per_batch * K,
            "gpu_launches_plain": per_sys * K,
            "move_frac": 24 * beads / (pm / 10 / 1e3) / 1e9 / peak,
            "field_frac": 8 * cells_all / (pf / 10 / 1e3) / 1e9 / peak,
            "phase_ms": {"move": pm / 10, "field": pf / 10},
            "tune_trials": [{"beads_per_tile": t["beads_per_tile"], "threads_move": t["threads_move"],
                             "persistent_ctas": t["persistent_ctas"], "cells_per_tile": t["cells_per_tile"],
                             "ms": round(t["ms"], 3)} for t in trials]}


def run_served(nb, served_request, args):
    from new_arch_b200.server import Server
    rng = np.random.default_rng(4242)
    n = args.served_requests
    reqs = [served_request(rng, seed=50_000 + i) for i in range(n)]
    gaps = rng.exponential(1.0 / args.served_rate, n)
    arrive = np.cumsum(gaps)
    done = []
    with Server(150 * 10**9) as srv:
        t0 = time.perf_counter()
        for i, (sp, k) in enumerate(reqs):
            now = time.perf_counter() - t0
            if arrive[i] > now:
                time.sleep(arrive[i] - now)
            srv.submit(sp, k, want_counts=False)
            done += srv.poll(256, 0)
        while len(done) < n:
            done += srv.poll(256, 200)
        wall = time.perf_counter() - t0
    lat = np.array([r["t_done"] - r["t_submit"] for r in done])
    ok = sum(1 for r in done if r["status"] == 0)
    moves = sum(r["n_beads"] * r["n_sweeps"] for r in done)
    span = max(r["t_done"] for r in done) - min(r["t_submit"] for r in done)
    return {"workload": f"Poisson {args.served_rate:g}/s, {n} requests, edges log-U[16,128], K {{50,100,500}}, 150 GB budget",
            "requests": n, "ok": ok, "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "bead_moves_per_s": moves / span,
            "offered_bead_moves_per_s": moves / float(arrive[-1]), "wall_s": wall}


def run_capacity(nb, served_request, args):
    """Capacity of the served form: requests drawn as in the served stream, all
    submitted at once (an offered rate far above what the GPU sustains), so
    the bead-moves/s over the makespan is the largest the server sustains."""
    from new_arch_b200.server import Server
    rng = np.random.default_rng(777)
    n = args.capacity_requests
    reqs = [served_request(rng, seed=80_000 + i) for i in range(n)]
    done = []
    with Server(150 * 10**9) as srv:
        t0 = time.perf_counter()
        for sp, k in reqs:
            srv.submit(sp, k, want_counts=False)
        while len(done) < n:
            done += srv.poll(256, 200)
        wall = time.perf_counter() - t0
    lat = np.array([r["t_done"] - r["t_submit"] for r in done])
    moves = sum(r["n_beads"] * r["n_sweeps"] for r in done)
    span = max(r["t_done"] for r in done) - min(r["t_submit"] for r in done)
    return {"workload": f"{n} requests as in the served stream, all submitted at t=0", "requests": n,
            "ok": sum(1 for r in done if r["status"] == 0), "bead_moves_per_s": moves / span, "makespan_s": span,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "wall_s": wall}


def run_sharded(args):
    """The large system as chain shards over the ranks (strong scaling): per
    sweep each rank moves its chains, the counts are summed with one NCCL
    all-reduce, and every rank computes the field of the sum."""
    import datetime
    import torch
    from new_arch_b200.shard import ShardedSystem
    from new_arch_b200.spec import large_system
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from new_arch_b200.replicas import reduce_max
    spec = large_system(seed=7)
    sh = ShardedSystem(spec)
    sh.init_coords()
    sh.step(args.warmup)
    st = sh.stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    e0.record(st)
    sh.step(args.steps)
    e1.record(st)
    e1.synchronize()
    clocks = sampler.stop()
    ms = reduce_max(e0.elapsed_time(e1), dist, "cuda")
    cnt = sh.counts()
    assert int(cnt.sum()) == spec.n_beads
    sh.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": spec.n_beads * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (random-walk chains)",
                "config": workload_config(spec),
                "run": {"parallelism": f"chain shards x{world}, NCCL all-reduce of the counts per sweep",
                        "sweeps_timed": args.steps},
                "clocks": clocks, "gpu_launches": 2 * args.steps * 1, "mode": "sharded"}
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "sharded":
        return run_sharded(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
