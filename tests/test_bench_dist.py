"""bench.py's multi-rank path on the host: two gloo ranks launched the way the
driver launches the GPU bench (torch.distributed.run, 127.0.0.1)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, timeout=240, extra_env=None):
    env = dict(os.environ, KASCADE_BENCH_BACKEND="gloo", CUDA_VISIBLE_DEVICES="", **(extra_env or {}))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port())] + args
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def _json_lines(text):
    out = []
    for line in text.splitlines():
        line = line.strip()
        if line.startswith("{"):
            try:
                out.append(json.loads(line))
            except json.JSONDecodeError:
                pass
    return out


def test_whole_job_takes_the_slowest_rank_and_every_ranks_elements(tmp_path):
    res = _torchrun([str(ROOT / "tests" / "dist_helper.py")], extra_env={"KASCADE_DIST_OUT": str(tmp_path)})
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in (0, 1)]
    assert sorted(d["rank"] for d in lines) == [0, 1]
    for d in lines:
        assert d["world"] == 2 and d["backend"] == "gloo"
        # max over ranks: rank 1 took 20 ms for 5 steps
        assert d["ms_per_step"] == pytest.approx(4.0)
        # 1000 elements per rank, two ranks, 4 ms per step
        assert d["value"] == pytest.approx(2 * 1000 / 0.004)


def test_reference_arm_prints_one_line_from_rank_zero(oracle_mod):
    res = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
                     "--cpu-sample", "65536", "--elements", "1048576"])
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [d for d in _json_lines(res.stdout) if d.get("impl") == "reference"]
    assert len(lines) == 1
    d = lines[0]
    assert d["n_gpus"] == 2 and d["value"] > 0 and d["unit"] == "elements/s"
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    # the multi-core ruling set ran on the whole (here reduced) list
    v = d["cpu_baseline"]["variants"]
    assert set(v) == {"sparse_ruling_set", "gather_chase", "pointer_doubling"}
    assert v["sparse_ruling_set"]["n"] == 1048576 and v["sparse_ruling_set"]["cores"] >= 1
