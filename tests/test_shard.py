"""The sharded ranking protocol (kascade_b200/shard.py) on the CPU: shards
in one process and two gloo ranks, each shard's device work done by the CPU
stand-in (tests/shard_cpu_ops.py); results bit-exact against the reference's
GatherChase (oracle/_ref) on the whole list."""
from __future__ import annotations

import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]


def _expected(oracle_mod, succ, w):
    rank = w.astype(np.int64) if w is not None else np.ones(succ.size, np.int64)
    rank[succ == np.arange(succ.size, dtype=np.uint64)] = 0
    s = succ.copy()
    if oracle_mod.has_ref():
        oracle_mod.ref_local_pointer_chasing(s, rank)
    else:
        oracle_mod.local_pointer_chasing(s, rank)
    return s, rank


def _split(n, parts, seed):
    cuts = np.sort(np.random.default_rng(seed).choice(np.arange(0, n + 1), parts - 1))
    return np.concatenate([[0], cuts, [n]])


def _many_lists(n, k, seed):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    succ = np.empty(n, np.uint64)
    for seg in np.split(perm, np.sort(rng.choice(np.arange(1, n), k, replace=False))):
        succ[seg[:-1]] = seg[1:]
        succ[seg[-1]] = seg[-1]
    return succ


def _run_local(kb_shard, ops_cls, succ, w, bounds, **kw):
    shards = [(torch.from_numpy(succ[a:b].view(np.int64).copy()),
               None if w is None else torch.from_numpy(w[a:b].view(np.int32).copy()))
              for a, b in zip(bounds, bounds[1:])]
    out = kb_shard.rank_list_sharded_local(shards, ops_factory=lambda i, s: ops_cls(), **kw)
    root = np.concatenate([o[0].numpy() for o in out]).view(np.uint64)
    rank = np.concatenate([o[1].numpy() for o in out])
    return root, rank, out[0][2]


@pytest.fixture(scope="module")
def shard_mod():
    from kascade_b200 import shard

    return shard


@pytest.fixture(scope="module")
def cpu_ops():
    sys.path.insert(0, str(ROOT / "tests"))
    from shard_cpu_ops import CpuShardOps

    return CpuShardOps


@pytest.mark.parametrize("parts", [1, 2, 3, 5])
def test_sharded_protocol_in_one_process(oracle_mod, shard_mod, cpu_ops, parts):
    cases = [("random", oracle_mod.gen_list(20_000, 3, 0), None),
             ("weighted", oracle_mod.gen_list(15_000, 4, 0), oracle_mod.gen_weights(15_000, 5, 16)),
             ("runs", oracle_mod.gen_list(12_800, 6, 1), None),
             ("many", _many_lists(10_000, 700, 7), None)]
    for name, succ, w in cases:
        exp_root, exp_rank = _expected(oracle_mod, succ, w)
        root, rank, info = _run_local(shard_mod, cpu_ops, succ, w, _split(succ.size, parts, parts), spacing=8)
        np.testing.assert_array_equal(root, exp_root, err_msg=name)
        np.testing.assert_array_equal(rank, exp_rank, err_msg=name)
        assert info["rulers"] >= 1 and info["offsets"][-1] == succ.size


def test_sharded_protocol_reports_errors_on_every_shard(oracle_mod, shard_mod, cpu_ops):
    succ = np.roll(np.arange(3000, dtype=np.uint64), 1)  # one rootless cycle
    with pytest.raises(shard_mod.KascadeError) as e:
        _run_local(shard_mod, cpu_ops, succ, None, _split(succ.size, 3, 1), spacing=8)
    assert e.value.name == "CYCLE"
    bad = oracle_mod.gen_list(3000, 9, 0)
    bad[5] = 10**6
    with pytest.raises(shard_mod.KascadeError) as e:
        _run_local(shard_mod, cpu_ops, bad, None, _split(bad.size, 2, 2), spacing=8)
    assert e.value.name == "OUT_OF_RANGE"


def test_distribution_mirrors_the_reference(shard_mod):
    d = shard_mod.Distribution([3, 0, 5])
    assert d.offsets == [0, 3, 3, 8] and d.counts() == [3, 0, 5]
    assert [d.get_owner(i) for i in range(8)] == [0, 0, 0, 2, 2, 2, 2, 2]
    assert d.is_local(4, 2) and not d.is_local(4, 0)
    assert d.get_local_idx(4, 2) == 1 and d.get_global_idx(1, 2) == 4 and d.get_global_size() == 8


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_protocol_on_two_gloo_ranks(oracle_mod, tmp_path):
    """Two processes, one shard each, exchanging over gloo: the same results
    as the reference's GatherChase on the whole list."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", KASCADE_SHARD_OUT=str(tmp_path))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "tests" / "shard_dist_helper.py")]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=240)
    assert res.returncode == 0, res.stderr[-3000:]
    n = int((tmp_path / "n.txt").read_text())
    succ = oracle_mod.gen_list(n, 0x5A, 0)
    w = oracle_mod.gen_weights(n, 0x5B, 16)
    exp_root, exp_rank = _expected(oracle_mod, succ, w)
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in (0, 1)]
    root = np.concatenate([p["root"] for p in parts]).view(np.uint64)
    rank = np.concatenate([p["rank"] for p in parts])
    np.testing.assert_array_equal(root, exp_root)
    np.testing.assert_array_equal(rank, exp_rank)
