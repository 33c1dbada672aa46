"""Per-size-class autotuner for the ranker's launch parameters.

For each size class it times batches made only of instances of that class
(sizes log-uniform inside the class, 70% weighted random lists / 30% random
recursive forests, the batched workload's mix) and picks

  1. the mean ruler spacing (ruler density), then, at that spacing,
  2. the chains in flight per chase thread and the chase block size,
  3. the ruler spacing for calls that rank one instance on their own (up to
     32 of the class's instances, one call each),

by measured elements/s.  The table it returns is what `load_tuning` installs
in a context; `write_header` turns it into the library's built-in defaults
(kascade_b200/csrc/tuned_classes.h), so every context starts tuned.

    python -m kascade_b200.autotune --json tuning.json --header kascade_b200/csrc/tuned_classes.h
"""
from __future__ import annotations

import argparse
import json
import math
import statistics
from pathlib import Path

import numpy as np

# class upper bounds (elements; ranking records for forests are 2 per vertex)
CLASS_MAX = (1 << 10, 1 << 13, 1 << 16, 1 << 19, 1 << 22, 1 << 25, 1 << 27, (1 << 64) - 1)
SPACINGS = (4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128)
CHAINS = (1, 2, 4)
BLOCKS = (128, 256, 512)


def class_sizes(k: int, total: int, seed: int):
    """Instance sizes inside class k (log-uniform over (lower bound, upper
    bound]) summing to about `total`, and their kinds."""
    lo = 64 if k == 0 else CLASS_MAX[k - 1] + 1
    hi = CLASS_MAX[k] if k + 1 < len(CLASS_MAX) else 1 << 28
    rng = np.random.default_rng(seed)
    sizes = []
    acc = 0
    while acc < total:
        sz = int(2.0 ** rng.uniform(math.log2(lo), math.log2(hi)))
        sz = max(lo, min(hi, sz))
        sizes.append(sz)
        acc += sz
    sizes = np.array(sizes, np.int64)
    kinds = np.where(rng.random(len(sizes)) < 0.7, 0, 1)
    return sizes, kinds


def _time_ms(fn, reps: int) -> float:
    import torch

    fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return statistics.median(out)


def tune(device: int = 0, total: int = 1 << 24, reps: int = 3, log=print) -> dict:
    import torch

    from . import api as kb

    dev = torch.device(f"cuda:{device}")
    ctx = kb.Context(device)
    classes = []
    for k, cmax in enumerate(CLASS_MAX):
        # the three largest classes: a few instances each (up to 2^25, 2^27, 2^28 elements)
        scale = {len(CLASS_MAX) - 3: 4, len(CLASS_MAX) - 2: 8, len(CLASS_MAX) - 1: 24}.get(k, 1)
        sizes, kinds = class_sizes(k, scale * total, 0xA7 + k)
        kinds = np.where(kinds == 0, kb.SEG_LIST, kb.SEG_FOREST)
        inp, w = kb.gen_batch(sizes, kinds, seed=0x7E + k, device=dev)
        segs = kb.make_segments(sizes, kinds)
        n = int(sizes.sum())
        root = torch.empty(n, dtype=torch.int64, device=dev)
        rank = torch.empty(n, dtype=torch.int64, device=dev)
        ref_root, ref_rank = kb.rank_batch(inp, segs, w, ctx=ctx)
        ref_root, ref_rank = ref_root.clone(), ref_rank.clone()

        def run(t):
            kb.rank_batch(inp, segs, w, tuning=t, root_out=root, rank_out=rank, ctx=ctx)

        best = None
        for sp in SPACINGS:
            ms = _time_ms(lambda: run(kb.GpuTuning(ruler_spacing=sp)), reps)
            if best is None or ms < best[0]:
                best = (ms, sp)
        spacing = best[1]
        best = None
        for c in CHAINS:
            for b in BLOCKS:
                t = kb.GpuTuning(ruler_spacing=spacing, chains_per_thread=c, block_size=b)
                ms = _time_ms(lambda: run(t), reps)
                if best is None or ms < best[0]:
                    best = (ms, c, b)
        ms, chains, block = best
        run(kb.GpuTuning(ruler_spacing=spacing, chains_per_thread=chains, block_size=block))
        torch.cuda.synchronize()
        if not (torch.equal(root, ref_root) and torch.equal(rank, ref_rank)):
            raise RuntimeError(f"class {k}: tuned parameters change the results")
        # one instance per call: up to 32 of the class's instances, back to back
        offs = np.concatenate([[0], np.cumsum(sizes)])
        picks = list(range(min(32, len(sizes))))

        def run_single(t):
            for i in picks:
                a, b_ = int(offs[i]), int(offs[i + 1])
                if kinds[i] == kb.SEG_LIST:
                    kb.rank_list(inp[a:b_], w[a:b_], tuning=t, root_out=root[a:b_], rank_out=rank[a:b_], ctx=ctx)
                else:
                    kb.root_forest(inp[a:b_], tuning=t, root_out=root[a:b_], depth_out=rank[a:b_], ctx=ctx)

        best_single = None
        for sp in SPACINGS:
            t = kb.GpuTuning(ruler_spacing=sp, chains_per_thread=chains, block_size=block)
            ms1 = _time_ms(lambda: run_single(t), reps)
            if best_single is None or ms1 < best_single[0]:
                best_single = (ms1, sp)
        n_single = int(offs[len(picks)])
        entry = {"max": int(min(cmax, (1 << 64) - 1)), "spacing": spacing, "chains": chains, "block": block,
                 "spacing_single": best_single[1], "instances": int(len(sizes)), "elements": n, "ms": round(ms, 4),
                 "elements_per_s": n / (ms / 1000.0), "single_calls": len(picks),
                 "single_elements_per_s": n_single / (best_single[0] / 1000.0)}
        log(json.dumps(entry))
        classes.append(entry)
        del inp, w, root, rank, ref_root, ref_rank
        torch.cuda.empty_cache()
    ctx.close()
    return {"gpu": torch.cuda.get_device_name(dev), "total_elements_per_class": total, "reps": reps,
            "classes": classes}


def write_header(table: dict, path) -> None:
    cls = table["classes"]

    def arr(key, fmt):
        return "{" + ", ".join(fmt(c[key]) for c in cls) + "}"

    def max_fmt(v):
        return "~0ull" if v >= (1 << 64) - 1 else f"{v}ull"

    text = f"""// Size-class table: mean ruler spacing, chains per thread and chase block
// size for instances of at most KS_TUNED_MAX[i] elements.  Written by
// kascade_b200/autotune.py from measurements on the GPU named below; the
// library starts every context with it.
#pragma once
#define KS_TUNED_GPU "{table['gpu']}"
#define KS_TUNED_COUNT {len(cls)}
#define KS_TUNED_MAX {arr('max', max_fmt)}
#define KS_TUNED_SPACING {arr('spacing', lambda v: f'{v}u')}
#define KS_TUNED_SPACING_SINGLE {arr('spacing_single', lambda v: f'{v}u')}
#define KS_TUNED_CHAINS {arr('chains', lambda v: f'{v}u')}
#define KS_TUNED_BLOCK {arr('block', lambda v: f'{v}u')}
"""
    Path(path).write_text(text)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--total", type=int, default=1 << 24, help="elements per class batch")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--json", default=None, help="write the table here")
    ap.add_argument("--header", default=None, help="write the library defaults header here")
    args = ap.parse_args()
    table = tune(args.device, args.total, args.reps)
    if args.json:
        Path(args.json).write_text(json.dumps(table, indent=1) + "\n")
    if args.header:
        write_header(table, args.header)
    print(json.dumps(table))


if __name__ == "__main__":
    main()
