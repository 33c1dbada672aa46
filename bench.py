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
# The chase kernel's algorithmic bytes per element it visits: the one random
# 32 B sector its dependent 16 B record read lands in.  The implementation
# also writes 16 B per visit (the log entry of the write-free chase, or the
# stamp of the stamping chase); that figure is reported beside it.
B_CHASE = 32
B_CHASE_IMPL = 32 + 16
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
# DRAM bytes the write-free pipeline's kernels move, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on a weighted 2^25-element
# list: per element for the streaming kernels, per record read for the chase.
# Scaled to a run, they give the traffic the pipeline really moves (the
# measured form of "sectors touched").
NCU_LIST_N = 1 << 25
DRAM_PER_ELEM_LOG = {"prepare": (402.7e6 + 480.9e6) / NCU_LIST_N, "resolve": (554.3e6 + 480.4e6) / NCU_LIST_N,
                     "partition": (537.1e6 + 480.8e6) / NCU_LIST_N, "place": (537.0e6 + 480.8e6) / NCU_LIST_N}
# DRAM bytes the level-0 stamping chase moves per record it reads (ncu on a
# 2^25-element list: 3.924 GB read + 1.036 GB written over 2^25 + 2 797 812
# record reads, every element once plus each chain's closing ruler record).
CHASE_NCU_VISITS = NCU_LIST_N + 2_797_812
CHASE_DRAM_BYTES_PER_VISIT = (3.924e9 + 1.036e9) / CHASE_NCU_VISITS
# The same for the write-free chase (k_chase_log), which reads each record
# and appends a 16 B log entry: 3.901 GB read + 0.560 GB written over 2^25 +
# 1 048 211 record reads.
CHASE_LOG_NCU_VISITS = NCU_LIST_N + 1_048_211
CHASE_LOG_DRAM_BYTES_PER_VISIT = (3.900669e9 + 0.560097e9) / CHASE_LOG_NCU_VISITS


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


def cpu_inputs(wl: str, n: int, seed: int):
    """The workload's seeded input built on the host cores (bit-identical to
    the device generators): (succ or parent, rank array in the reference's
    in-place form: distance to the successor, 0 at roots)."""
    import numpy as np

    import oracle

    _, _, kind, arg, weighted = WORKLOADS[wl]
    if kind == "list":
        succ = oracle.cpu_gen_list(n, seed, arg)
        rank = (oracle.cpu_gen_weights(n, seed + 1, 16).astype(np.int64) if weighted else np.ones(n, np.int64))
    else:
        succ = oracle.cpu_gen_forest(n, seed, arg, 64, (n // 64) // 2 if arg == 1 else 0)
        rank = np.ones(n, np.int64)
    rank[succ == np.arange(n, dtype=np.uint64)] = 0
    return succ, rank


def cpu_time(variant: str, succ, rank, threads: int = 0):
    """Seconds of one in-place CPU ranking of (succ, rank) on copies, and the
    result.  Variants: the reference's own GatherChase (oracle/_ref, compiled
    from lib/kascade/local_pointer_chasing.cpp; its restatement when absent;
    one core), and the multi-core restatements of the sparse ruling set and
    of pointer doubling over `threads` host threads (0 = all)."""
    import oracle

    s, r = succ.copy(), rank.copy()
    t0 = time.perf_counter()
    if variant == "gather_chase":
        if oracle.has_ref():
            oracle.ref_local_pointer_chasing(s, r)
        else:
            oracle.local_pointer_chasing(s, r)
    elif variant == "sparse_ruling_set":
        oracle.cpu_sparse_ruling_set(s, r, spacing=32, threads=threads)
    else:
        oracle.cpu_pointer_doubling(s, r, threads=threads)
    return time.perf_counter() - t0, s, r


def cpu_variant_meta(variant: str, threads: int) -> tuple[str, int, str]:
    """(kind, cores, description) of a CPU variant."""
    import oracle

    if variant == "gather_chase":
        return (("reference" if oracle.has_ref() else "port"), 1,
                "GatherChase, lib/kascade/local_pointer_chasing.cpp " +
                ("compiled from the reference source" if oracle.has_ref() else "restated") + ", 1 core")
    t = threads or oracle.cpu_threads()
    name = {"sparse_ruling_set": "sparse ruling set (post-invert chase from rulers and leaves, recursion, pull "
                                 "propagation)", "pointer_doubling": "synchronous pointer doubling"}[variant]
    return "port", t, f"multi-core CPU restatement of the reference's {name}, {t} threads"


def cpu_baseline(wl: str, n: int, seed: int, full=None, sample_n: int = 1 << 24, check=None) -> dict:
    """The best of the reference's CPU variants on the host cores: the
    multi-core sparse ruling set on the full workload (`full` = its host
    arrays, else generated here), the sequential GatherChase and multi-core
    pointer doubling on a `sample_n`-element instance of the same generator.
    `check` = (root, rank) host arrays of the GPU result of the full
    workload, compared with the CPU ruling set's result."""
    import numpy as np

    _, _, kind, _, _ = WORKLOADS[wl]
    variants = {}
    if kind == "list":
        succ, rank = full if full is not None else cpu_inputs(wl, n, seed)
        dt, s, r = cpu_time("sparse_ruling_set", succ, rank)
        k, c, d = cpu_variant_meta("sparse_ruling_set", 0)
        variants["sparse_ruling_set"] = {"value": n / dt, "seconds": round(dt, 3), "n": n, "kind": k, "cores": c,
                                         "what": d}
        if check is not None:
            variants["sparse_ruling_set"]["equals_gpu_result"] = bool(
                np.array_equal(s, check[0]) and np.array_equal(r.view(np.uint64), check[1]))
        del s, r, succ, rank
    m = min(sample_n, n)
    succ, rank = cpu_inputs(wl, m, seed)
    for v in ("gather_chase", "pointer_doubling"):
        dt, _, _ = cpu_time(v, succ, rank)
        k, c, d = cpu_variant_meta(v, 0)
        variants[v] = {"value": m / dt, "seconds": round(dt, 3), "n": m, "kind": k, "cores": c, "what": d}
    best = max(variants, key=lambda v: variants[v]["value"])
    b = variants[best]
    return {"value": b["value"], "unit": "elements/s" if kind == "list" else "vertices/s", "cores": b["cores"],
            "kind": b["kind"], "best": best,
            "sample": f"{b['what']}, on a {b['n']}-element instance of the same seeded generator"
                      + (" (the full workload)" if b["n"] == n else ""),
            "same_config": b["n"] == n, "variants": variants}


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


def measure_served(kb, dev, n_requests: int = 1000, rate: float = 20000.0, batched_rate: float | None = None,
                   **server_kw) -> dict:
    """Poisson arrivals (mean 20k req/s) of sizes
    log-uniform in [2^8, 2^24], 70% weighted lists / 30% random recursive
    forests, served under a 40 GB HBM budget with device-resident inputs;
    p50 / p99 latency and throughput, against plain per-request calls.  Every
    served result is copied (device to device) into a result store before its
    release and compared, on the device, with a plain call on the same input
    after the run.  `batched_rate`: the batched form's elements/s on this
    GPU, the served form's ceiling."""
    import numpy as np
    import torch

    rng = np.random.default_rng(0xC4)
    sizes = np.floor(2.0 ** rng.uniform(8, 24, n_requests)).astype(np.int64)
    kinds = np.where(rng.random(n_requests) < 0.7, kb.SEG_LIST, kb.SEG_FOREST)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    inputs, w = kb.gen_batch(sizes, kinds, seed=0xC4, device=dev)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    total = int(sizes.sum())
    # the result store, allocated before the run: an allocation inside it
    # could synchronise the device and stall the lanes
    store_root = torch.empty(total, dtype=torch.int64, device=dev)
    store_rank = torch.empty(total, dtype=torch.int64, device=dev)
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
    copy_stream = torch.cuda.Stream(dev, priority=0)
    errors = []

    def collector():
        # waits in submission order, copies each result into the store and
        # releases it once the copy is done, so the budget holds only
        # requests in flight
        with torch.cuda.stream(copy_stream):
            for i in range(n_requests):
                rid = done_q.get()
                try:
                    srv.wait(rid, 300.0)
                    r_dev, k_dev = srv.result_device(rid)
                    a, b = int(offs[i]), int(offs[i + 1])
                    store_root[a:b].copy_(r_dev.view(torch.int64), non_blocking=True)
                    store_rank[a:b].copy_(k_dev.view(torch.int64), non_blocking=True)
                    copy_stream.synchronize()
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
    # plain per-request calls of the same requests, back to back
    ctx = kb.Context(dev.index or 0)
    root = torch.empty(int(sizes.max()), dtype=torch.int64, device=dev)
    rk = torch.empty_like(root)

    def plain(i):
        a, b = int(offs[i]), int(offs[i + 1])
        n = b - a
        if kinds[i] == kb.SEG_LIST:
            kb.rank_list(inputs[a:b], w[a:b], root_out=root[:n], rank_out=rk[:n], ctx=ctx)
        else:
            kb.root_forest(inputs[a:b], root_out=root[:n], depth_out=rk[:n], ctx=ctx)
        return a, b

    torch.cuda.synchronize()
    p0 = time.perf_counter()
    for i in range(n_requests):
        plain(i)
    torch.cuda.synchronize()
    tp = time.perf_counter() - p0
    # every served result against its plain call, compared on the device
    equal = 0
    for i in range(n_requests):
        a, b = plain(i)
        equal += bool(torch.equal(store_root[a:b], root[:b - a]) and torch.equal(store_rank[a:b], rk[:b - a]))
    ctx.close()
    del store_root, store_rank, inputs, w
    served_rate = st["elements_per_s"]
    plain_rate = total / tp
    out = {"workload": f"{n_requests} requests, Poisson arrivals at {rate:.0f}/s, sizes log-uniform in [2^8,2^24], "
                       "70% weighted lists / 30% random recursive forests, 40 GB admission budget, device-resident "
                       "inputs",
           "requests": n_requests, "elements": total, "req_per_s": round(st["requests_per_s"], 1),
           "elements_per_s": served_rate, "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
           "p50_ms_le_2^20": round(st["p50_small_ms"], 3), "p99_ms_le_2^20": round(st["p99_small_ms"], 3),
           "requests_le_2^20": int(st["completed_small"]), "batches": int(st["batches"]),
           "plain_elements_per_s": plain_rate, "plain_req_per_s": round(n_requests / tp, 1),
           "throughput_vs_plain": round(served_rate / plain_rate, 2),
           "results_checked": n_requests, "results_equal_plain": equal,
           "lanes": {k: st[k] for k in ("lane_batches", "lane_elements", "lane_busy_ms", "lane_max_batch_ms",
                                        "partition_sms", "partition_batches")}}
    if batched_rate:
        # the whole GPU's batched rate bounds what serving can reach: this
        # mix's ceiling against plain calls, and the share of it reached
        out["ceiling_vs_plain"] = round(batched_rate / plain_rate, 2)
        out["frac_of_batched_rate"] = round(served_rate / batched_rate, 3)
    return out


def run_reference(args, world, rank):
    """The reference's CPU path on the host cores: each step one in-place
    ranking of the full workload by the multi-core sparse ruling set (the
    reference's own MPI binary cannot be built here), the sequential
    GatherChase (the reference's own source, oracle/_ref) and multi-core
    pointer doubling measured once on a 2^24-element sample; the value is the
    best of the three.  Tree-rooting workloads have no ruling-set leg (the
    reference's ruling set takes lists only)."""
    if rank != 0:
        return
    import oracle

    wl = args.workload
    desc, n, kind, _, _ = WORKLOADS[wl]
    if args.n:
        n = args.n
    seed = 0xC1
    succ, rk = cpu_inputs(wl, n, seed)
    steps_variant = "sparse_ruling_set" if kind == "list" else "pointer_doubling"
    if kind != "list":
        succ, rk = cpu_inputs(wl, min(n, args.cpu_sample), seed)
    m = succ.size
    for _ in range(args.warmup):
        cpu_time(steps_variant, succ, rk)
    times = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dt, _, _ = cpu_time(steps_variant, succ, rk)
        times.append(dt)
    wall = time.perf_counter() - t0
    variants = {}
    k, c, d = cpu_variant_meta(steps_variant, 0)
    variants[steps_variant] = {"value": m / statistics.median(times), "n": m, "kind": k, "cores": c, "what": d,
                               "steps": args.steps}
    del succ, rk
    succ, rk = cpu_inputs(wl, min(n, args.cpu_sample), seed)
    for v in ("gather_chase", "pointer_doubling"):
        if v in variants:
            continue
        dt, _, _ = cpu_time(v, succ, rk)
        k, c, d = cpu_variant_meta(v, 0)
        variants[v] = {"value": succ.size / dt, "n": int(succ.size), "kind": k, "cores": c, "what": d}
    best = max(variants, key=lambda v: variants[v]["value"])
    b = variants[best]
    unit = "elements/s"
    secondary = {}
    if kind == "list" and not args.no_secondary and not args.n:
        # tree rooting (the forests of the rooting workload): the reference's
        # GatherRank chase on one core and multi-core pointer doubling
        for fw in ("forest_rrt", "forest_cat"):
            fs, fr = cpu_inputs(fw, args.cpu_sample, seed)
            fv = {}
            for v in ("gather_chase", "pointer_doubling"):
                dt, _, _ = cpu_time(v, fs, fr)
                k, c, d = cpu_variant_meta(v, 0)
                fv[v] = {"value": fs.size / dt, "n": int(fs.size), "kind": k, "cores": c, "what": d}
            fb = max(fv, key=lambda v: fv[v]["value"])
            secondary[fw] = {"workload": WORKLOADS[fw][0], "value": fv[fb]["value"], "unit": "vertices/s",
                             "best": fb, "variants": fv}
    out = {
        "impl": "reference", "metric": METRIC, "value": b["value"], "unit": unit, "n_gpus": args.gpus,
        # ms_per_step: the full workload at the reported rate (the median
        # ranking time when the ruling set is best); wall_ms_per_step adds the
        # fresh copies of the inputs each in-place step ranks
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000.0 * n / b["value"], 3),
        "wall_ms_per_step": round(1000.0 * wall / max(args.steps, 1), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": desc, "n": n, "sample_n": b["n"],
                   "parallelism": f"{b['cores']} host thread(s), {oracle.cpu_threads()} available"},
        "cpu_baseline": {"value": b["value"], "unit": unit, "cores": b["cores"], "kind": b["kind"],
                         "sample": f"{b['what']}, {b['n']}-element instance of the same seeded generator"
                                   + (" (the full workload)" if b["n"] == n else ""),
                         "same_config": b["n"] == n, "best": best, "variants": variants},
        "e2e": {"value": b["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "secondary": secondary or None,
        "note": "the reference's MPI binary cannot be built here (no MPI, no network for its FetchContent "
                "dependencies, GCC 13); its GatherChase source compiles standalone (oracle/_ref) and its "
                "sparse ruling set and pointer doubling run as multi-core CPU restatements",
    }
    print(json.dumps(out), flush=True)


def measure_device(kb, ctx, dev, wl: str, n: int, tuning, steps: int, warmup: int, world: int, seed: int,
                   clocks: bool = False) -> dict:
    """Device-timed ranking of one workload with inputs resident in HBM: CUDA
    events on the launching stream around `steps` calls (barrier and
    synchronize on both sides), kernel times from the library's own events,
    the dominant kernel's roofline."""
    import torch

    desc, _, kind, arg, weighted = WORKLOADS[wl]
    stream = torch.cuda.current_stream(dev)
    if kind == "list":
        inp = kb.gen_list(n, seed, arg, device=dev)
        w = kb.gen_weights(n, seed + 1, 16, device=dev) if weighted else None
        ctx.reserve(kb.lib.kascade_scratch_bytes_rank_list(n))
    else:
        spine = (n // 64) // 2 if arg == 1 else 0
        inp = kb.gen_forest(n, seed, arg, 64, spine, device=dev)
        w = None
        ctx.reserve(kb.lib.kascade_scratch_bytes_root_forest(n))
    root = torch.empty(n, dtype=torch.int64, device=dev)
    rk = torch.empty(n, dtype=torch.int64, device=dev)

    def step():
        if kind == "list":
            kb.rank_list(inp, w, tuning=tuning, root_out=root, rank_out=rk, ctx=ctx)
        else:
            kb.root_forest(inp, tuning=tuning, root_out=root, depth_out=rk, ctx=ctx)

    torch.cuda.synchronize()
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ctx.reset_kernel_times()
    sampler = ClockSampler(dev.index or 0) if clocks else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = sampler.stop() if sampler else None
    ms_per_step, value = whole_job(n, ev0.elapsed_time(ev1), steps, world)
    ktimes = ctx.kernel_times()
    levels = ctx.levels()
    hbm, hbm_src = peaks()
    b_alg = B_ALG[kind](weighted)
    pipe_gbs = n * b_alg / (ms_per_step / 1000.0) / 1e9
    return {"desc": desc, "n": n, "kind": kind, "weighted": weighted, "inp": inp, "w": w, "root": root, "rank": rk,
            "ms_per_step": ms_per_step, "value": value, "ktimes": ktimes, "levels": levels, "clocks": clk,
            "launches": sum(c for (_, c) in ktimes.values()),
            "kernels_ms_per_step": {k: round(v[0] / steps, 4) for k, v in sorted(ktimes.items())},
            "roofline": kernel_roofline(ktimes, levels, steps, kind, n, weighted, hbm, hbm_src),
            "pipeline": {"b_alg_per_elem": b_alg, "achieved_gbs": round(pipe_gbs, 1),
                         "frac": round(pipe_gbs / hbm, 4), "peak_gbs": hbm, "peak_source": hbm_src},
            "write_free": "place" in ktimes}


def kernel_roofline(ktimes, levels, steps, kind, n, weighted, hbm, hbm_src) -> dict | None:
    """Roofline of the step's dominant kernel.  For the chase: one random
    32 B sector per element visited (all levels' visits, over the chase
    launches of one step); the 16 B log entry or stamp the implementation
    writes per visit is reported beside it.  `traffic`: ncu DRAM bytes per
    visit from a 2^25-element capture, scaled to the visits per launch."""
    if not ktimes:
        return None
    dominant = max(ktimes, key=lambda k: ktimes[k][0])
    d_ms, d_cnt = ktimes[dominant]
    per_launch_s = d_ms / d_cnt / 1000.0
    launches_per_step = d_cnt / steps
    write_free = "place" in ktimes
    out = {"bound": "hbm", "kernel": dominant, "peak": hbm, "unit": "GB/s",
           "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if hbm_src == "measured"
                           else "fallback 6.65 TB/s"), "ms_per_launch": round(per_launch_s * 1e3, 4),
           "launches_per_step": round(launches_per_step, 2)}
    if dominant == "chase":
        units = levels[0] if levels else n
        total_units = sum(levels[:-1]) if len(levels) > 1 else units
        per_launch_units = total_units / launches_per_step
        ach = B_CHASE * per_launch_units / per_launch_s / 1e9
        impl = B_CHASE_IMPL * per_launch_units / per_launch_s / 1e9
        per_visit = CHASE_LOG_DRAM_BYTES_PER_VISIT if write_free else CHASE_DRAM_BYTES_PER_VISIT
        ncu_visits = CHASE_LOG_NCU_VISITS if write_free else CHASE_NCU_VISITS
        out.update({"achieved": round(ach, 1), "frac": round(ach / hbm, 4),
                    "algorithmic_bytes": f"{B_CHASE} B per element visited (one random 32 B sector) x "
                                         f"{per_launch_units:.0f} visits per launch",
                    "implementation_bytes": {"bytes_per_visit": B_CHASE_IMPL,
                                             "what": "the random sector + the 16 B " +
                                                     ("log entry" if write_free else "stamp") + " per visit",
                                             "achieved": round(impl, 1), "frac": round(impl / hbm, 4)},
                    "traffic": round(per_visit * per_launch_units),
                    "traffic_note": f"ncu dram bytes per visit ({per_visit:.1f} B) of the level-0 "
                                    f"{'write-free' if write_free else 'stamping'} chase on a 2^25-element list "
                                    f"({ncu_visits} visits), scaled to this launch's visits",
                    "traffic_scale": round(per_launch_units / ncu_visits, 4)})
    else:
        b_alg = B_ALG[kind](weighted)
        per_launch_bytes = n * b_alg / launches_per_step
        ach = per_launch_bytes / per_launch_s / 1e9
        out.update({"achieved": round(ach, 1), "frac": round(ach / hbm, 4), "traffic": None,
                    "algorithmic_bytes": f"{b_alg} B per unit x n per step, over this kernel's launches"})
    return out


def random_access_roofline(r: dict, hbm: float) -> dict | None:
    """The north-star form: sectors touched x 32 B / peak, with the sectors
    the pipeline that ran touches per list element."""
    if r["kind"] != "list":
        return None
    n, weighted, write_free, levels = r["n"], r["weighted"], r["write_free"], r["levels"]
    ms = r["ms_per_step"]
    sectors = (SECTORS_LIST_LOG if write_free else SECTORS_LIST)[bool(weighted)]
    floor_ms = n * 32 * sectors / (hbm * 1e9) * 1000.0
    sectors_min = min(SECTORS_LIST[bool(weighted)], SECTORS_LIST_LOG[bool(weighted)])
    floor_min_ms = n * 32 * sectors_min / (hbm * 1e9) * 1000.0
    out = {"level0": "write-free" if write_free else "stamping", "sectors_per_element": sectors,
           "bytes_per_element": 32 * sectors, "floor_ms": round(floor_ms, 3), "frac": round(floor_ms / ms, 4),
           "sectors_min_design": sectors_min, "frac_min_design": round(floor_min_ms / ms, 4), "peak_gbs": hbm}
    if write_free and weighted:
        visits = sum(levels[:2]) if len(levels) > 1 else n
        dram = n * sum(DRAM_PER_ELEM_LOG.values()) + visits * CHASE_LOG_DRAM_BYTES_PER_VISIT
        out["measured"] = {"bytes_per_element": round(dram / n, 1), "sectors_per_element": round(dram / n / 32, 2),
                           "achieved_gbs": round(dram / (ms / 1000.0) / 1e9, 1),
                           "frac": round(dram / (ms / 1000.0) / 1e9 / hbm, 4),
                           "source": "ncu DRAM bytes per kernel on a 2^25 list, scaled by elements and chase visits"}
    return out


def summary(r: dict) -> dict:
    """The figures of one workload for the JSON line."""
    return {"workload": r["desc"], "n": r["n"], "value": r["value"],
            "unit": "elements/s" if r["kind"] == "list" else "vertices/s", "ms_per_step": round(r["ms_per_step"], 4),
            "pipeline_frac": r["pipeline"]["frac"], "b_alg_per_unit": r["pipeline"]["b_alg_per_elem"],
            "roofline": r["roofline"], "levels": r["levels"], "kernels_ms_per_step": r["kernels_ms_per_step"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="list")
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--e2e-contexts", type=int, default=2,
                    help="contexts (and streams) the pipelined host-buffer calls take turns on")
    ap.add_argument("--cpu-sample", type=int, default=1 << 24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--spacing", type=int, default=0)
    ap.add_argument("--chains", type=int, default=0)
    ap.add_argument("--block", type=int, default=0, help="chase block size override (128, 256 or 512)")
    ap.add_argument("--n", "--elements", dest="n", type=int, default=0,
                    help="override the workload size (profiling runs)")
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

    import ctypes

    import numpy as np
    import torch

    import kascade_b200 as kb

    desc, n, kind, arg, weighted = WORKLOADS[args.workload]
    if args.n:
        n = args.n
    dev = torch.device(f"cuda:{local}")
    ctx = kb.Context(local)
    stream = torch.cuda.current_stream(dev)
    seed = 0xC1 + 1000 * rank
    tune = dict(ruler_spacing=args.spacing, chains_per_thread=args.chains, block_size=args.block,
                level0_mode=args.level0_mode)
    tuning = kb.GpuTuning(profile=True, **tune)
    main_r = measure_device(kb, ctx, dev, args.workload, n, tuning, args.steps, args.warmup, world, seed,
                            clocks=True)
    if args.n:
        main_r["desc"] = f"{main_r['desc']} [size overridden: n={n}]"
    inp, w, root, rk = main_r["inp"], main_r["w"], main_r["root"], main_r["rank"]
    hbm, _ = peaks()

    # end-to-end through the host-buffer API (pinned host memory): K steps,
    # each with its own copy-in, ranking and copy-out inside the timed region.
    # Serial: one context, each call complete before the next.  Pipelined (the
    # reported value): async host-buffer calls taking turns over a ring of
    # contexts and streams, a context synced before its next call, so one
    # step's copy-out overlaps the next steps' copy-in and ranking.
    e2e = None
    if args.e2e_steps > 0:
        pin_in = torch.empty(n, dtype=torch.int64, pin_memory=True)
        pin_in.copy_(inp.cpu())
        pin_w = None
        if w is not None:
            pin_w = torch.empty(n, dtype=torch.int32, pin_memory=True)
            pin_w.copy_(w.cpu())
        outs = [(torch.empty(n, dtype=torch.int64, pin_memory=True), torch.empty(n, dtype=torch.int64, pin_memory=True))]
        o_sync = kb.GpuTuning(**tune).to_opts()
        o_async = kb.GpuTuning(**tune).to_opts()
        o_async.async_ = 1
        ctxs, strs = [ctx], [stream]

        def e2e_call(i, o):
            c, s_, (r_, k_) = ctxs[i], strs[i], outs[i]
            if kind == "list":
                st = kb.lib.kascade_rank_list_host(c.handle, pin_in.data_ptr(),
                                                   pin_w.data_ptr() if pin_w is not None else None, n,
                                                   r_.data_ptr(), k_.data_ptr(), ctypes.byref(o), s_.cuda_stream)
            else:
                st = kb.lib.kascade_root_forest_host(c.handle, pin_in.data_ptr(), n, r_.data_ptr(), k_.data_ptr(),
                                                     ctypes.byref(o), s_.cuda_stream)
            kb._lib.check(st, "host-buffer call", c.handle)

        def e2e_sync(i):
            kb._lib.check(kb.lib.kascade_ctx_sync(ctxs[i].handle, strs[i].cuda_stream), "kascade_ctx_sync",
                          ctxs[i].handle)

        def matches(i):
            return bool(torch.equal(outs[i][1], rk.cpu()) and torch.equal(outs[i][0], root.cpu()))

        # two warm-up calls: the first grows the context's arena by the device
        # copies of the host buffers, the second folds it into one block
        for _ in range(2):
            e2e_call(0, o_sync)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            e2e_call(0, o_sync)
        e1.record(stream)
        torch.cuda.synchronize()
        te_serial = max_over_ranks(e0.elapsed_time(e1), world) / args.e2e_steps
        ok = matches(0)
        h2d = n * 8 + (n * 4 if w is not None else 0)
        unit_e = "elements/s" if kind == "list" else "vertices/s"
        e2e = {"value": n * world / (te_serial / 1000.0), "unit": unit_e, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": 16 * n, "ms_per_step": round(te_serial, 3), "host_matches_device": ok,
               "mode": "serial: one context, each host-buffer call complete before the next"}
        R = max(1, args.e2e_contexts)
        # set-up of the extra contexts on every rank first; the ranks agree on
        # its outcome before any of them enters a collective of the timed part
        setup_err = None
        try:
            for i in range(1, R):
                ctxs.append(kb.Context(dev.index or 0))
                strs.append(torch.cuda.Stream(dev))
                outs.append((torch.empty(n, dtype=torch.int64, pin_memory=True),
                             torch.empty(n, dtype=torch.int64, pin_memory=True)))
                for _ in range(2):
                    e2e_call(i, o_sync)
        except (RuntimeError, kb.KascadeError) as ex:  # e.g. no room for a second set of pinned buffers
            setup_err = str(ex)[:200]
        if max_over_ranks(1.0 if setup_err else 0.0, world) > 0.0:
            e2e["pipelined_error"] = setup_err or "set-up failed on another rank"
        else:
            barrier(world)
            torch.cuda.synchronize()
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            g0.record(stream)
            for i in range(1, R):
                strs[i].wait_event(g0)
            pending = [False] * R
            for k in range(args.e2e_steps):
                i = k % R
                if pending[i]:
                    e2e_sync(i)
                e2e_call(i, o_async)
                pending[i] = True
            for i in range(R):
                if pending[i]:
                    e2e_sync(i)
            for i in range(1, R):
                tail = torch.cuda.Event()
                tail.record(strs[i])
                stream.wait_event(tail)
            g1.record(stream)
            torch.cuda.synchronize()
            te = max_over_ranks(g0.elapsed_time(g1), world) / args.e2e_steps
            serial = {k: e2e[k] for k in ("value", "ms_per_step", "mode")}
            e2e.update(value=n * world / (te / 1000.0), ms_per_step=round(te, 3),
                       host_matches_device=ok and all(matches(i) for i in range(R)), serial=serial,
                       mode=f"pipelined: async host-buffer calls taking turns over {R} contexts and streams "
                            "(a step's copy-out overlaps the next steps' copy-in and ranking)")
        for c in ctxs[1:]:
            c.close()
        del pin_in, pin_w, outs

    # CPU baseline on the same seeded input (host copy of the device arrays),
    # its full-size ruling-set result compared with the GPU result
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        succ_h = inp.cpu().numpy().view(np.uint64)
        rank_h = (w.cpu().numpy().view(np.uint32).astype(np.int64) if w is not None
                  else np.ones(n, np.int64))
        rank_h[succ_h == np.arange(n, dtype=np.uint64)] = 0
        check = (root.cpu().numpy().view(np.uint64), rk.cpu().numpy().view(np.uint64))
        cpu = cpu_baseline(args.workload, n, seed, full=(succ_h, rank_h) if kind == "list" else None,
                           sample_n=args.cpu_sample, check=check if kind == "list" else None)
        del succ_h, rank_h, check

    secondary = {}
    batched = served = None
    full_default = world == 1 and not args.no_secondary and args.workload == "list" and not args.n
    del inp, w, root, rk
    main_r.update(inp=None, w=None, root=None, rank=None)
    torch.cuda.empty_cache()
    if full_default:
        # the locality-biased layout of the same configuration, the 2^20 unit
        # list of the reference's own small case, and the 2^26-vertex forests
        for wl2, steps2 in (("list_local", args.steps), ("list20", 5 * args.steps), ("forest_rrt", args.steps),
                            ("forest_cat", args.steps)):
            try:
                r2 = measure_device(kb, ctx, dev, wl2, WORKLOADS[wl2][1], kb.GpuTuning(profile=True, **tune),
                                    steps2, args.warmup, world, seed)
                secondary[wl2] = summary(r2)
                secondary[wl2]["steps"] = steps2
                del r2
            except kb.KascadeError as e:  # reported in the line, the other workloads still run
                secondary[wl2] = {"workload": WORKLOADS[wl2][0], "error": str(e)}
            torch.cuda.empty_cache()
        batched = measure_batched(kb, ctx, dev)
        torch.cuda.empty_cache()
        served = measure_served(kb, dev, batched_rate=batched["elements_per_s"])

    if rank == 0:
        out = {
            "metric": METRIC, "value": main_r["value"], "unit": "elements/s" if kind == "list" else "vertices/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(main_r["ms_per_step"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded device generator)",
            "config": {"workload": main_r["desc"], "n": n, "global_elements": n * world,
                       "parallelism": f"replicas x{world} (independent instances, no collective)",
                       "l2": "inputs larger than L2 (16 B records x n = %.1f GiB)" % (16 * n / 2**30),
                       "ruler_spacing": args.spacing or "auto", "levels": main_r["levels"]},
            "roofline": main_r["roofline"], "pipeline_roofline": main_r["pipeline"],
            "random_access_roofline": random_access_roofline(main_r, hbm),
            "cpu_baseline": cpu, "e2e": e2e, "clocks": main_r["clocks"], "gpu_launches": main_r["launches"],
            "kernels_ms_per_step": main_r["kernels_ms_per_step"],
            "secondary": secondary or None, "batched": batched, "served": served,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
