"""One rank of the two-rank host-side check of bench.py's multi-GPU logic
(launched by tests/test_bench_dist.py under torch.distributed.run, gloo)."""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import bench  # noqa: E402


def main() -> None:
    world, rank, _ = bench.dist_setup()
    # every rank takes the same collective steps: barrier, then the max
    bench.barrier(world)
    t_local = 10.0 * (rank + 1)  # rank 1 is the slower one
    ms, value = bench.whole_job(1000, t_local, 5, world)
    # one file per rank (the ranks share stdout, where lines can interleave)
    out = Path(os.environ["KASCADE_DIST_OUT"]) / f"rank{rank}.json"
    out.write_text(json.dumps({"rank": rank, "world": world, "ms_per_step": ms, "value": value,
                               "backend": bench.dist_backend()}))
    bench.barrier(world)
    import torch.distributed as dist

    dist.destroy_process_group()


if __name__ == "__main__":
    os.environ.setdefault("KASCADE_BENCH_BACKEND", "gloo")
    main()
