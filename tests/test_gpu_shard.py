"""The sharded ranking's device work (kascade_shard_* kernels through the C
ABI) with several shards in one process on one GPU: every shard's chase,
fix-up, sub-list and propagation run in the library's kernels, the exchanges
in memory.  Results bit-exact against the oracle on the whole list."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shard_mod():
    from kascade_b200 import shard

    return shard


def _split(n, parts, seed):
    cuts = np.sort(np.random.default_rng(seed).choice(np.arange(0, n + 1), parts - 1))
    return np.concatenate([[0], cuts, [n]])


def _run(shard_mod, succ, w, bounds, **kw):
    shards = [(torch.from_numpy(succ[a:b].view(np.int64).copy()).cuda(),
               None if w is None else torch.from_numpy(w[a:b].view(np.int32).copy()).cuda())
              for a, b in zip(bounds, bounds[1:])]
    out = shard_mod.rank_list_sharded_local(shards, **kw)
    root = np.concatenate([o[0].cpu().numpy() for o in out]).view(np.uint64)
    rank = np.concatenate([o[1].cpu().numpy() for o in out]).view(np.uint64)
    return root, rank, out[0][2]


def _many_lists(n, k, seed):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    succ = np.empty(n, np.uint64)
    for seg in np.split(perm, np.sort(rng.choice(np.arange(1, n), k, replace=False))):
        succ[seg[:-1]] = seg[1:]
        succ[seg[-1]] = seg[-1]
    return succ


@pytest.mark.parametrize("parts", [1, 2, 4, 7])
def test_sharded_kernels_exact(oracle_mod, shard_mod, parts):
    cases = [("random", oracle_mod.gen_list(1 << 18, 0x51, 0), oracle_mod.gen_weights(1 << 18, 0x52, 16)),
             ("runs", oracle_mod.gen_list(200_000, 0x53, 1), None),
             ("many", _many_lists(150_000, 3000, 0x54), None),
             ("all roots", np.arange(5000, dtype=np.uint64), None)]
    for name, succ, w in cases:
        exp_root, exp_rank = oracle_mod.rank_list(succ, w)
        for spacing in (4, 16):
            root, rank, info = _run(shard_mod, succ, w, _split(succ.size, parts, parts + spacing), spacing=spacing)
            np.testing.assert_array_equal(root, exp_root, err_msg=f"{name} spacing {spacing}")
            np.testing.assert_array_equal(rank, exp_rank, err_msg=f"{name} spacing {spacing}")
            assert info["offsets"][-1] == succ.size


def test_sharded_kernels_report_errors(oracle_mod, shard_mod):
    ring = np.roll(np.arange(50_000, dtype=np.uint64), 1)  # one rootless cycle
    with pytest.raises(shard_mod.KascadeError) as e:
        _run(shard_mod, ring, None, _split(ring.size, 3, 1))
    assert e.value.name == "CYCLE"
    bad = oracle_mod.gen_list(40_000, 0x55, 0)
    bad[77] = 10**7
    with pytest.raises(shard_mod.KascadeError) as e:
        _run(shard_mod, bad, None, _split(bad.size, 2, 2))
    assert e.value.name == "OUT_OF_RANGE"
    two = oracle_mod.gen_list(40_000, 0x56, 0)
    two[100] = two[200]  # an element with two predecessors
    with pytest.raises(shard_mod.KascadeError) as e:
        _run(shard_mod, two, None, _split(two.size, 4, 3))
    assert e.value.name in ("NOT_A_LIST", "CYCLE")
    # the library still works afterwards
    succ = oracle_mod.gen_list(30_000, 0x57, 0)
    root, rank, _ = _run(shard_mod, succ, None, _split(succ.size, 3, 4))
    exp_root, exp_rank = oracle_mod.rank_list(succ)
    np.testing.assert_array_equal(root, exp_root)
    np.testing.assert_array_equal(rank, exp_rank)
