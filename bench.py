#!/usr/bin/env python3
"""Benchmark: elements ranked per second on one B200 (and weak-scaled over N).

Workload (default): weighted list ranking of n = 2^28 elements, uint64
indices, uint32 weights uniform in [0, 2^16), the list order a seeded random
permutation; exact uint64 ranks.  Inputs are generated on the device by the
library's seeded generators (no dataset exists for this path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload list|list_local|forest_rrt|forest_cat]

One JSON line on rank 0.  `value` is device-timed whole-job throughput with
inputs resident in HBM; `e2e` is the same metric through the host-buffer API
call (host->device copy of the inputs and device->host copy of root and rank
inside the timed region).  Under torchrun every rank ranks its own instance
(replicas, no data-path collective): scaling is weak.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "elements ranked/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    # name: (description, n, kind, layout/kind arg, weights)
    "list": ("weighted list ranking, random permutation order, n=2^28, uint32 weights in [0,2^16)", 1 << 28,
             "list", 0, True),
    "list_local": ("weighted list ranking, runs of 64 consecutive indices in random run order, n=2^28, "
                   "uint32 weights in [0,2^16)", 1 << 28, "list", 1, True),
    "list20": ("list ranking, random permutation order, n=2^20, unit weights", 1 << 20, "list", 0, False),
    "forest_rrt": ("tree rooting, 64 random recursive trees, n=2^26 vertices", 1 << 26, "forest", 0, False),
    "forest_cat": ("tree rooting, 64 caterpillars (spine 2^19, uniform leaves), n=2^26 vertices", 1 << 26, "forest",
                   1, False),
}

# Algorithmic bytes per unit (HBM roofline, integer work): stream-read succ
# (8 B) + weights (4 B) + stream-write root and rank (16 B) + one random 32 B
# sector for the dependent successor load.  Forest: 8 B parent + 16 B outputs
# + 2 tour elements x (32 B random sector + 16 B streamed tour state).
B_ALG = {"list": lambda w: 8 + (4 if w else 0) + 16 + 32, "forest": lambda w: 8 + 16 + 2 * (32 + 16)}
# The chase kernel's own algorithmic bytes per element it visits: the
# dependent 16 B record read lands in one random 32 B sector, and the 16 B
# stamp it writes back.
B_CHASE = 32 + 16
# Random-access roofline, stated as 32 B sectors touched x 32 B / peak: the
# sectors the ranking pipeline touches per level-0 list element.  prepare:
# succ 8 B (1/4 sector) + weight 4 B (1/8) + record write 16 B (1/2); chase:
# the record's random sector read + its stamp written back (1 + 1);
# propagate: record read (1/2) + the ruler result's random sector (1) + root
# and rank writes (1/2).  Deeper levels add ~2% and are left out.
SECTORS_LIST = {True: 0.25 + 0.125 + 0.5 + 2 + 2, False: 0.25 + 0.5 + 2 + 2}
# The same count for the write-free level 0 (the default from 2^25 elements):
# prepare as above; chase: the record's random sector read + the 16 B log
# entry (1 + 1/2); resolve: log read + resolved entry written (1/2 + 1/2; its
# ruler lookups hit L1 for the most part and are left out); partition: read +
# write (1/2 + 1/2); place: read (1/2) + root and rank writes (1/2).
SECTORS_LIST_LOG = {True: 0.25 + 0.125 + 0.5 + 1.5 + 1 + 1 + 1, False: 0.25 + 0.5 + 1.5 + 1 + 1 + 1}
# DRAM bytes the write-free pipeline's kernels move, measured by ncu on a
# weighted 2^25-element list (dram__bytes_read.sum + dram__bytes_write.sum;
# profiles/write_free_level0_list25_ncu.md): per element for the streaming
# kernels, per record read for the chase.  Scaled to a run, they give the
# traffic the pipeline really moves (the measured form of "sectors touched").
DRAM_PER_ELEM_LOG = {"prepare": (402.7e6 + 480.9e6) / 2**25, "resolve": (554.3e6 + 480.4e6) / 2**25,
                     "partition": (537.1e6 + 480.8e6) / 2**25, "place": (537.0e6 + 480.8e6) / 2**25}
# DRAM bytes the level-0 chase moves per record it reads, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of the level-0 k_chase launch
# on a 2^25-element list: 3.924 GB + 1.036 GB over 2^25 + 2 797 812 record
# reads, every element once plus each chain's closing ruler record; traffic
# grows in proportion): profiles/chase_propagate_prepare_list25_ncu.md
CHASE_DRAM_BYTES_PER_VISIT = (3.924e9 + 1.036e9) / (33_554_432 + 2_797_812)
# The same for the write-free chase (k_chase_log), which reads each record
# and appends a 16 B log entry: 3.901 GB read + 0.560 GB written over 2^25 +
# 1 048 211 record reads (profiles/write_free_level0_list25_ncu.md)
CHASE_LOG_DRAM_BYTES_PER_VISIT = (3.900669e9 + 0.560097e9) / (33_554_432 + 1_048_211)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    if PEAKS_FILE.exists():
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_backend() -> str:
    """nccl on GPUs; gloo where there are none (the host-side multi-rank
    tests), or when KASCADE_BENCH_BACKEND says so."""
    import torch

    return os.environ.get("KASCADE_BENCH_BACKEND") or ("nccl" if torch.cuda.is_available() else "gloo")


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        if dist_backend() == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device(f"cuda:{local}"))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job(n_per_rank: int, t_ms_local: float, steps: int, world: int) -> tuple[float, float]:
    """(ms per step, whole-job elements/s): the slowest rank's time, every
    rank's elements (each rank ranks its own replica)."""
    t_ms = max_over_ranks(t_ms_local, world)
    ms_per_step = t_ms / steps
    return ms_per_step, n_per_rank * world / (ms_per_step / 1000.0)


def cpu_reference_time(n_sample: int, wl: str, reps: int = 1) -> tuple[float, str, str]:
    """The reference's own GatherChase (oracle/_ref, built from the reference
    source) when present, else the oracle restatement; one host core."""
    import numpy as np

    import oracle

    _, _, kind, arg, weighted = WORKLOADS[wl]
    if kind == "list":
        succ = oracle.gen_list(n_sample, 0xC1, arg)
        rank = (oracle.gen_weights(n_sample, 0xC1 + 1, 16).astype(np.int64) if weighted
                else np.ones(n_sample, np.int64))
        rank[succ == np.arange(n_sample, dtype=np.uint64)] = 0
    else:
        succ = oracle.gen_forest(n_sample, 0xC2, arg, 64, n_sample // 128)
        rank = np.where(succ == np.arange(n_sample, dtype=np.uint64), 0, 1).astype(np.int64)
    use_ref = oracle.has_ref()
    best = float("inf")
    for _ in range(reps):
        s, r = succ.copy(), rank.copy()
        t0 = time.perf_counter()
        if use_ref:
            oracle.ref_local_pointer_chasing(s, r)
        else:
            oracle.local_pointer_chasing(s, r)
        best = min(best, time.perf_counter() - t0)
    return n_sample / best, ("reference" if use_ref else "port"), (
        f"{n_sample}-element instance of the same generator, GatherChase "
        f"(lib/kascade/local_pointer_chasing.cpp{' compiled from the reference source' if use_ref else ' restated'}),"
        f" best of {reps}")


def calibrate(local: int) -> None:
    """Random 16 B access rate of the device (the chase's ceiling)."""
    import ctypes

    import kascade_b200 as kb

    ctx = kb.Context(local)
    out = {}
    names = ["independent_read", "independent_read_write", "dependent_read", "dependent_read_write",
             "dependent_32B_full_write", "dependent_64B_full_write", "dependent_64B_16B_write", "dependent_32B_read"]
    for mode, nm in enumerate(names):
        for bps in (8, 16):
            v = ctypes.c_double(0)
            kb._lib.check(kb.lib.kascade_calibrate_random_access(ctx.handle, 1 << 28, mode, bps, ctypes.byref(v)),
                          "calibrate", ctx.handle)
            out[f"{nm}@{bps}blk"] = round(v.value, 2)
    print(json.dumps({"calibration": "G random record accesses/s, 2^28 records of 16 B (modes 0-3), 32 B or "
                                     "64 B (modes 4-7; 16 B of each read, the whole record or 16 B written back)",
                      **out}), flush=True)
    ctx.close()


def measure_batched(kb, ctx, dev, steps: int = 3) -> dict:
    """4096 independent instances (sizes log-uniform in
    [2^6, 2^22] rescaled to sum to 2^28; 70% weighted lists, 30% random
    recursive forests) ranked by one kascade_rank_batch call, against plain
    per-instance calls on the same instances."""
    import numpy as np
    import torch

    sizes, kinds = kb.batch_sizes(4096, 0xC3, lo_log2=6, hi_log2=22, total=1 << 28)
    inputs, w = kb.gen_batch(sizes, kinds, seed=0xC3, device=dev)
    segs = kb.make_segments(sizes, kinds)
    total = int(sizes.sum())
    root = torch.empty(total, dtype=torch.int64, device=dev)
    rk = torch.empty(total, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(2):
        kb.rank_batch(inputs, segs, w, root_out=root, rank_out=rk, ctx=ctx)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        kb.rank_batch(inputs, segs, w, root_out=root, rank_out=rk, ctx=ctx)
    e1.record(stream)
    torch.cuda.synchronize()
    tb = e0.elapsed_time(e1) / steps / 1000.0
    # plain per-instance launches of the same instances (one call each)
    root2 = torch.empty_like(root)
    rk2 = torch.empty_like(rk)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    torch.cuda.synchronize()
    p0 = time.perf_counter()
    p_ev0, p_ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p_ev0.record(stream)
    for i in range(len(sizes)):
        a, b = int(offs[i]), int(offs[i + 1])
        if kinds[i] == kb.SEG_LIST:
            kb.rank_list(inputs[a:b], w[a:b], root_out=root2[a:b], rank_out=rk2[a:b], ctx=ctx)
        else:
            kb.root_forest(inputs[a:b], root_out=root2[a:b], depth_out=rk2[a:b], ctx=ctx)
    p_ev1.record(stream)
    torch.cuda.synchronize()
    tp = max(p_ev0.elapsed_time(p_ev1) / 1000.0, time.perf_counter() - p0)
    same = bool(torch.equal(root, root2) and torch.equal(rk, rk2))
    # the same batch captured once as a CUDA graph and replayed
    graph = None
    try:
        plan = kb.BatchPlan(inputs, segs, w, root_out=root2, rank_out=rk2)
        plan.launch()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(steps):
            plan.launch()
        g1.record(stream)
        torch.cuda.synchronize()
        tg = g0.elapsed_time(g1) / steps / 1000.0
        graph = {"ms_per_batch": round(tg * 1e3, 3), "elements_per_s": total / tg,
                 "speedup_vs_plain": round(tp / tg, 2),
                 "results_equal": bool(torch.equal(root, root2) and torch.equal(rk, rk2))}
        plan.close()
    except kb.KascadeError as e:  # a batch the device-driven recursion cannot hold
        graph = {"unavailable": str(e)}
    return {"workload": "4096 instances, sizes log-uniform in [2^6,2^22] rescaled to sum 2^28, 70% weighted lists / "
                        "30% random recursive forests, one kascade_rank_batch call",
            "instances": len(sizes), "elements": total, "ms_per_batch": round(tb * 1e3, 3),
            "req_per_s": round(len(sizes) / tb, 1), "elements_per_s": total / tb,
            "plain_per_instance_ms": round(tp * 1e3, 1), "plain_elements_per_s": total / tp,
            "speedup_vs_plain": round(tp / tb, 2), "results_equal_plain": same, "graph_replay": graph}


def measure_served(kb, dev, n_requests: int = 1000, rate: float = 20000.0, **server_kw) -> dict:
    """Poisson arrivals (mean 20k req/s) of sizes
    log-uniform in [2^8, 2^24], 70% weighted lists / 30% random recursive
    forests, served under a 40 GB HBM budget with device-resident inputs;
    p50 / p99 latency and throughput, against plain per-request calls."""
    import numpy as np
    import torch

    rng = np.random.default_rng(0xC4)
    sizes = np.floor(2.0 ** rng.uniform(8, 24, n_requests)).astype(np.int64)
    kinds = np.where(rng.random(n_requests) < 0.7, kb.SEG_LIST, kb.SEG_FOREST)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    inputs, w = kb.gen_batch(sizes, kinds, seed=0xC4, device=dev)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    torch.cuda.synchronize()
    kw = dict(hbm_budget=40 << 30, small_max=1 << 20, small_batch_elements=1 << 23)
    kw.update(server_kw)
    srv = kb.Server(device=dev.index or 0, **kw)
    # warm the lanes once
    wid = srv.submit(int(kinds[0]), inputs[0:int(sizes[0])], w[0:int(sizes[0])] if kinds[0] == kb.SEG_LIST else None)
    srv.wait(wid, 60.0)
    srv.release(wid)
    srv.reset_stats()
    import queue
    import threading

    ids = [None] * n_requests
    done_q: "queue.Queue" = queue.Queue()
    check_at = {0, n_requests // 2, n_requests - 1}
    # destinations for the spot checks, allocated before the run: an
    # allocation inside it could synchronise the device and stall the lanes
    checks = {i: (torch.empty(int(sizes[i]), dtype=torch.int64, device=dev),
                  torch.empty(int(sizes[i]), dtype=torch.int64, device=dev)) for i in check_at}
    torch.cuda.synchronize()
    errors = []

    def collector():
        # waits in submission order and releases each result once read, so
        # the budget holds only requests in flight
        for i in range(n_requests):
            rid = done_q.get()
            try:
                srv.wait(rid, 300.0)
                if i in check_at:
                    r_dev, k_dev = srv.result_device(rid)
                    checks[i][0].copy_(r_dev.view(torch.int64))
                    checks[i][1].copy_(k_dev.view(torch.int64))
                srv.release(rid)
            except Exception as e:  # noqa: BLE001
                errors.append(e)

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for i in range(n_requests):
        delay = t0 + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        a, b = int(offs[i]), int(offs[i + 1])
        ids[i] = srv.submit(int(kinds[i]), inputs[a:b], w[a:b] if kinds[i] == kb.SEG_LIST else None)
        done_q.put(ids[i])
    th.join(timeout=600.0)
    if th.is_alive() or errors:
        raise RuntimeError(f"served run did not complete: {errors[:1]}")
    st = srv.stats()
    srv.close()
    # spot-check three results against plain calls
    ok = True
    for i, (r_dev, k_dev) in checks.items():
        a, b = int(offs[i]), int(offs[i + 1])
        if kinds[i] == kb.SEG_LIST:
            r_p, k_p = kb.rank_list(inputs[a:b], w[a:b])
        else:
            r_p, k_p = kb.root_forest(inputs[a:b])
        ok &= bool(torch.equal(r_dev, r_p) and torch.equal(k_dev, k_p))
    # plain per-request calls of the same requests, back to back
    ctx = kb.Context(dev.index or 0)
    root = torch.empty(int(sizes.max()), dtype=torch.int64, device=dev)
    rk = torch.empty_like(root)
    torch.cuda.synchronize()
    p0 = time.perf_counter()
    for i in range(n_requests):
        a, b = int(offs[i]), int(offs[i + 1])
        n = b - a
        if kinds[i] == kb.SEG_LIST:
            kb.rank_list(inputs[a:b], w[a:b], root_out=root[:n], rank_out=rk[:n], ctx=ctx)
        else:
            kb.root_forest(inputs[a:b], root_out=root[:n], depth_out=rk[:n], ctx=ctx)
    torch.cuda.synchronize()
    tp = time.perf_counter() - p0
    ctx.close()
    total = int(sizes.sum())
    return {"workload": f"{n_requests} requests, Poisson arrivals at {rate:.0f}/s, sizes log-uniform in [2^8,2^24], "
                        "70% weighted lists / 30% random recursive forests, 40 GB admission budget, device-resident "
                        "inputs",
            "requests": n_requests, "elements": total, "req_per_s": round(st["requests_per_s"], 1),
            "elements_per_s": st["elements_per_s"], "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
            "p50_ms_le_2^20": round(st["p50_small_ms"], 3), "p99_ms_le_2^20": round(st["p99_small_ms"], 3),
            "requests_le_2^20": int(st["completed_small"]), "batches": int(st["batches"]),
            "plain_elements_per_s": total / tp, "plain_req_per_s": round(n_requests / tp, 1),
            "throughput_vs_plain": round(st["elements_per_s"] / (total / tp), 2), "spot_check_equal": ok,
            "lanes": {k: st[k] for k in ("lane_batches", "lane_elements", "lane_busy_ms", "lane_max_batch_ms",
                                         "partition_sms", "partition_batches")}}


def run_reference(args, world, rank):
    if rank != 0:
        return
    wl = args.workload
    n_sample = args.cpu_sample
    for _ in range(args.warmup):
        cpu_reference_time(n_sample // 4, wl)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, kind, sample = cpu_reference_time(n_sample, wl)
        vals.append(v)
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "elements/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOADS[wl][0], "n": WORKLOADS[wl][1], "sample_n": n_sample,
                   "parallelism": "one host core (GatherChase is sequential)"},
        "cpu_baseline": {"value": v, "unit": "elements/s", "cores": 1, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's MPI binary cannot be built here (no MPI, no network for its FetchContent "
                "dependencies); its GatherChase source compiles standalone and is what runs",
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="list")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample", type=int, default=1 << 24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--spacing", type=int, default=0)
    ap.add_argument("--chains", type=int, default=0)
    ap.add_argument("--block", type=int, default=0, help="chase block size override (128, 256 or 512)")
    ap.add_argument("--n", type=int, default=0, help="override the workload size (profiling runs)")
    ap.add_argument("--level0-mode", type=int, default=0, help="0 auto, 1 stamping chase, 2 write-free chase")
    ap.add_argument("--calibrate", action="store_true",
                    help="measure the random 16 B access rate of this GPU (2^28 records) and exit")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world, rank, local = dist_setup()
    if args.calibrate:
        calibrate(local)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    import numpy as np
    import torch

    import kascade_b200 as kb

    desc, n, kind, arg, weighted = WORKLOADS[args.workload]
    if args.n:
        n = args.n
        desc = f"{desc} [size overridden: n={n}]"
    dev = torch.device(f"cuda:{local}")
    ctx = kb.Context(local)
    stream = torch.cuda.current_stream(dev)
    seed = 0xC1 + 1000 * rank
    tuning = kb.GpuTuning(profile=True, ruler_spacing=args.spacing, chains_per_thread=args.chains,
                          block_size=args.block,
                          level0_mode=args.level0_mode)
    if kind == "list":
        inp = kb.gen_list(n, seed, arg, device=dev)
        w = kb.gen_weights(n, seed + 1, 16, device=dev) if weighted else None
        root = torch.empty(n, dtype=torch.int64, device=dev)
        rk = torch.empty(n, dtype=torch.int64, device=dev)
        ctx.reserve(kb.lib.kascade_scratch_bytes_rank_list(n))

        def step():
            kb.rank_list(inp, w, tuning=tuning, root_out=root, rank_out=rk, ctx=ctx)
    else:
        blocks = 64
        spine = (n // blocks) // 2 if arg == 1 else 0
        inp = kb.gen_forest(n, seed, arg, blocks, spine, device=dev)
        w = None
        root = torch.empty(n, dtype=torch.int64, device=dev)
        rk = torch.empty(n, dtype=torch.int64, device=dev)
        ctx.reserve(kb.lib.kascade_scratch_bytes_root_forest(n))

        def step():
            kb.root_forest(inp, tuning=tuning, root_out=root, depth_out=rk, ctx=ctx)

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ctx.reset_kernel_times()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms_per_step, value = whole_job(n, ev0.elapsed_time(ev1), args.steps, world)
    ktimes = ctx.kernel_times()
    launches = sum(c for (_, c) in ktimes.values())
    step_kernel_ms = {k: v[0] / args.steps for k, v in ktimes.items()}
    dominant = max(ktimes, key=lambda k: ktimes[k][0]) if ktimes else None
    levels = ctx.levels()
    write_free = "place" in ktimes  # level 0 ran the write-free chase

    hbm, hbm_src = peaks()
    b_alg = B_ALG[kind](weighted)
    pipe_gbs = n * b_alg / (ms_per_step / 1000.0) / 1e9
    roofline = None
    if dominant:
        d_ms, d_cnt = ktimes[dominant]
        per_launch_s = d_ms / d_cnt / 1000.0
        if dominant == "chase":
            # elements visited by the level-0 chase launch (every non-ruler
            # element plus each ruler's own start record)
            units = levels[0] if levels else n
            per_launch_units = units * (1 if kind == "list" else 1)
            launches_per_step = d_cnt / args.steps
            # deeper-level chases are far smaller; attribute bytes of all
            # levels, divided over the chase launches of one step
            total_units = sum(levels[:-1]) if len(levels) > 1 else units
            per_launch_bytes = B_CHASE * total_units / launches_per_step
            per_visit = CHASE_LOG_DRAM_BYTES_PER_VISIT if write_free else CHASE_DRAM_BYTES_PER_VISIT
            traffic = per_visit * total_units / launches_per_step if per_visit else None
            second = "16 B log entry" if write_free else "16 B stamp"
            bytes_note = (f"{B_CHASE} B per element visited (one random 32 B sector for the 16 B record + {second}) "
                          f"x {total_units} elements over {launches_per_step:.0f} chase launches per step")
        else:
            per_launch_bytes = n * b_alg / (d_cnt / args.steps)
            traffic = None
            bytes_note = f"{b_alg} B/element x n per step, over this kernel's launches"
        ach = per_launch_bytes / per_launch_s / 1e9
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(ach / hbm, 4), "peak_source": f"{hbm_src} (MEASURED_PEAKS.json hbm_gbs)"
                    if hbm_src == "measured" else "fallback 6.65 TB/s",
                    "traffic": round(traffic) if traffic else None,
                    "traffic_note": ("ncu dram bytes per visited element on a 2^25 list, scaled by the visits per "
                                     "launch" if traffic else None),
                    "algorithmic_bytes": bytes_note}
    pipeline = {"b_alg_per_elem": b_alg, "achieved_gbs": round(pipe_gbs, 1), "frac": round(pipe_gbs / hbm, 4)}
    random_access = None
    if kind == "list":
        sectors = (SECTORS_LIST_LOG if write_free else SECTORS_LIST)[bool(weighted)]
        floor_ms = n * 32 * sectors / (hbm * 1e9) * 1000.0
        # the fewer-sector design (stamping level 0) as a conservative floor
        sectors_min = min(SECTORS_LIST[bool(weighted)], SECTORS_LIST_LOG[bool(weighted)])
        floor_min_ms = n * 32 * sectors_min / (hbm * 1e9) * 1000.0
        random_access = {"level0": "write-free" if write_free else "stamping",
                         "sectors_per_element": sectors, "bytes_per_element": 32 * sectors,
                         "floor_ms": round(floor_ms, 3), "frac": round(floor_ms / ms_per_step, 4),
                         "sectors_min_design": sectors_min, "frac_min_design": round(floor_min_ms / ms_per_step, 4),
                         "peak_gbs": hbm}
        if write_free and weighted:
            # measured traffic of the level-0 kernels (deeper levels, ~2%, left out)
            visits = sum(levels[:2]) if len(levels) > 1 else n
            dram = n * sum(DRAM_PER_ELEM_LOG.values()) + visits * CHASE_LOG_DRAM_BYTES_PER_VISIT
            random_access["measured"] = {
                "bytes_per_element": round(dram / n, 1), "sectors_per_element": round(dram / n / 32, 2),
                "achieved_gbs": round(dram / (ms_per_step / 1000.0) / 1e9, 1),
                "frac": round(dram / (ms_per_step / 1000.0) / 1e9 / hbm, 4),
                "source": "ncu DRAM bytes per kernel on a 2^25 list, scaled by elements and chase visits"}

    # end-to-end through the host-buffer API (pinned host memory)
    e2e = None
    if args.e2e_steps > 0:
        pin_in = torch.empty(n, dtype=torch.int64, pin_memory=True)
        pin_in.copy_(inp.cpu())
        pin_w = None
        if w is not None:
            pin_w = torch.empty(n, dtype=torch.int32, pin_memory=True)
            pin_w.copy_(w.cpu())
        pin_root = torch.empty(n, dtype=torch.int64, pin_memory=True)
        pin_rank = torch.empty(n, dtype=torch.int64, pin_memory=True)
        o = kb.GpuTuning(ruler_spacing=args.spacing, chains_per_thread=args.chains, block_size=args.block,
                         level0_mode=args.level0_mode).to_opts()
        import ctypes

        def e2e_step():
            if kind == "list":
                st = kb.lib.kascade_rank_list_host(ctx.handle, pin_in.data_ptr(),
                                                   pin_w.data_ptr() if pin_w is not None else None, n,
                                                   pin_root.data_ptr(), pin_rank.data_ptr(), ctypes.byref(o),
                                                   stream.cuda_stream)
            else:
                st = kb.lib.kascade_root_forest_host(ctx.handle, pin_in.data_ptr(), n, pin_root.data_ptr(),
                                                     pin_rank.data_ptr(), ctypes.byref(o), stream.cuda_stream)
            kb._lib.check(st, "host-buffer call", ctx.handle)

        # two warm-up calls: the first grows the context's arena by the device
        # copies of the host buffers, the second folds it into one block
        for _ in range(2):
            e2e_step()
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        te = max_over_ranks(e0.elapsed_time(e1), world) / args.e2e_steps
        # correctness spot check of the host result against the device result
        ok = bool(np.array_equal(pin_rank[:4096].numpy(), rk[:4096].cpu().numpy()))
        h2d = n * 8 + (n * 4 if w is not None else 0)
        e2e = {"value": n * world / (te / 1000.0), "unit": "elements/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": 16 * n, "ms_per_step": round(te, 3), "host_matches_device": ok}

    secondary = {}
    if not args.no_secondary and kind == "list" and args.workload == "list" and world == 1:
        # the locality-biased layout of the same configuration
        inp2 = kb.gen_list(n, seed, 1, device=dev)
        tun2 = kb.GpuTuning(ruler_spacing=args.spacing, chains_per_thread=args.chains, block_size=args.block,
                            level0_mode=args.level0_mode)
        for _ in range(2):
            kb.rank_list(inp2, w, tuning=tun2, root_out=root, rank_out=rk, ctx=ctx)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(3):
            kb.rank_list(inp2, w, tuning=tun2, root_out=root, rank_out=rk, ctx=ctx)
        a1.record(stream)
        torch.cuda.synchronize()
        tl = a0.elapsed_time(a1) / 3
        secondary["list_local"] = {"workload": WORKLOADS["list_local"][0], "value": n / (tl / 1000.0),
                                   "ms_per_step": round(tl, 3),
                                   "pipeline_frac": round(n * b_alg / (tl / 1000.0) / 1e9 / hbm, 4)}
        del inp2

    batched = served = None
    if world == 1 and not args.no_secondary and args.workload == "list" and not args.n:
        del inp
        torch.cuda.empty_cache()
        batched = measure_batched(kb, ctx, dev)
        torch.cuda.empty_cache()
        served = measure_served(kb, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kd, sample = cpu_reference_time(args.cpu_sample, args.workload)
        cpu = {"value": v, "unit": "elements/s", "cores": 1, "kind": kd, "sample": sample}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded device generator)",
            "config": {"workload": desc, "n": n, "global_elements": n * world,
                       "parallelism": f"replicas x{world} (independent instances, no collective)",
                       "l2": "inputs larger than L2 (16 B records x n = %.1f GiB)" % (16 * n / 2**30),
                       "ruler_spacing": args.spacing or "auto", "levels": levels},
            "roofline": roofline, "pipeline_roofline": pipeline, "random_access_roofline": random_access,
            "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clk, "gpu_launches": launches,
            "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(step_kernel_ms.items())},
            "secondary": secondary or None, "batched": batched, "served": served,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
