"""Full-size runs (BASELINE configs 1 and 2) checked through the local
conditions that determine the answer uniquely, so no CPU oracle is needed:
  lists : rank[root] = 0, rank[x] = w[x] + rank[succ[x]], root[x] = root[succ[x]]
  trees : depth[root] = 0, depth[v] = 1 + depth[parent[v]], root[v] = root[parent[v]]
plus, for the single list, that the ranks of a unit-weight list are a
permutation of 0..n-1."""
from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kb():
    import kascade_b200

    return kascade_b200


def _check_list(succ, w, root, rank):
    n = succ.numel()
    idx = torch.arange(n, device=succ.device, dtype=torch.int64)
    is_root = succ == idx
    assert int(is_root.sum()) >= 1
    assert bool((rank[is_root] == 0).all())
    assert bool((root[is_root] == idx[is_root]).all())
    nr = ~is_root
    wv = w.to(torch.int64) & 0xFFFFFFFF if w is not None else torch.ones_like(succ)
    assert bool((rank[nr] == wv[nr] + rank[succ[nr]]).all())
    assert bool((root[nr] == root[succ[nr]]).all())


@pytest.mark.parametrize("layout", [0, 1])
def test_list_2_28_weighted(kb, layout):
    n = 1 << 28
    succ = kb.gen_list(n, 0xC1, layout)
    w = kb.gen_weights(n, 0xC2, 16)
    root, rank = kb.rank_list(succ, w)
    _check_list(succ, w, root, rank)
    assert int((root == root[0]).sum()) == n  # one list


def test_list_2_28_unit_is_permutation(kb):
    n = 1 << 28
    succ = kb.gen_list(n, 0xC3, 0)
    root, rank = kb.rank_list(succ)
    _check_list(succ, None, root, rank)
    counts = torch.bincount(rank, minlength=n)
    assert bool((counts == 1).all())


@pytest.mark.parametrize("kind,blocks,spine", [(0, 64, 0), (1, 64, 1 << 19)])
def test_forest_2_26(kb, kind, blocks, spine):
    n = 1 << 26
    par = kb.gen_forest(n, 0xC4, kind, blocks, spine)
    root, depth = kb.root_forest(par)
    idx = torch.arange(n, device=par.device, dtype=torch.int64)
    is_root = par == idx
    assert int(is_root.sum()) == blocks
    assert bool((depth[is_root] == 0).all()) and bool((root[is_root] == idx[is_root]).all())
    nr = ~is_root
    assert bool((depth[nr] == 1 + depth[par[nr]]).all())
    assert bool((root[nr] == root[par[nr]]).all())
    if kind == 1:
        assert int(depth.max()) >= spine - 1


def test_many_lists_2_26(kb):
    """About 2^20 lists over 2^26 elements on the default (write-free) path:
    every list head before its first ruler walks to it, in every window."""
    n = 1 << 26
    g = torch.Generator(device="cuda")
    g.manual_seed(0xC5)
    perm = torch.randperm(n, device="cuda", generator=g)
    tail = torch.rand(n, device="cuda", generator=g) < (1.0 / 64)
    tail[-1] = True
    nxt = torch.roll(perm, -1)
    succ = torch.where(tail, perm, nxt)
    succ_by_elem = torch.empty_like(succ)
    succ_by_elem[perm] = succ
    w = kb.gen_weights(n, 0xC6, 16)
    root, rank = kb.rank_list(succ_by_elem, w)
    _check_list(succ_by_elem, w, root, rank)
    assert int((succ_by_elem == torch.arange(n, device="cuda")).sum()) == int(tail.sum())


def test_batch_2_25_write_free_equals_stamping(kb):
    """A batch of 2^25 records (lists and forests) on its default write-free
    level 0 gives exactly the stamping level 0's results."""
    sizes, kinds = kb.batch_sizes(512, 0xC7, lo_log2=8, hi_log2=21, total=(1 << 25) + 4097)
    inputs, w = kb.gen_batch(sizes, kinds, seed=0xC8)
    segs = kb.make_segments(sizes, kinds)
    ctx = kb.Context()
    root, rank = kb.rank_batch(inputs, segs, w, ctx=ctx, tuning=kb.GpuTuning(profile=True))
    assert "place" in ctx.kernel_times()  # the write-free path ran
    root_s, rank_s = kb.rank_batch(inputs, segs, w, tuning=kb.GpuTuning(level0_mode=1))
    assert torch.equal(root, root_s) and torch.equal(rank, rank_s)
    ctx.close()
