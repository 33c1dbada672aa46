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
