"""One rank of the two-rank gloo check of the sharded ranking protocol
(launched by tests/test_shard.py under torch.distributed.run): rank r holds
its index range of one seeded weighted list, runs kascade_b200.shard's
protocol with the CPU stand-in for the device work, and saves its outputs."""
from __future__ import annotations

import datetime
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import oracle  # noqa: E402
from shard_cpu_ops import CpuShardOps  # noqa: E402


def main() -> None:
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    from kascade_b200 import shard

    r, world = dist.get_rank(), dist.get_world_size()
    n = 30_011
    succ = oracle.gen_list(n, 0x5A, 0)
    w = oracle.gen_weights(n, 0x5B, 16)
    lo, hi = (0, 12_345) if r == 0 else (12_345, n)
    root, rank, info = shard.rank_list_sharded(torch.from_numpy(succ[lo:hi].view(np.int64).copy()),
                                               torch.from_numpy(w[lo:hi].view(np.int32).copy()),
                                               ops=CpuShardOps(), spacing=8)
    out = Path(os.environ["KASCADE_SHARD_OUT"])
    np.savez(out / f"rank{r}.npz", root=root.numpy(), rank=rank.numpy())
    if r == 0:
        (out / "n.txt").write_text(str(n))
    assert world == 2 and info["rounds"] >= 1
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
