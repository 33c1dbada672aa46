"""Device-side result statistics (the bench's compute_stats) against the
oracle's restatement, on rankings and rootings the library produced."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import dev64, host_u64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kb():
    import kascade_b200

    return kascade_b200


def _check(kb, oracle_mod, root, rank):
    for level in (kb.STATS_BASIC, kb.STATS_REDUCED_EXTENSIVE, kb.STATS_EXTENSIVE):
        figs, trees = kb.compute_stats(root, rank, level)
        exp, exp_trees = oracle_mod.compute_stats(host_u64(root), host_u64(rank), level)
        for k, v in exp.items():
            if isinstance(v, float):
                assert figs[k] == pytest.approx(v, rel=1e-12, abs=0.0), k
            else:
                assert figs[k] == v, k
        assert [tuple(int(x) for x in t) for t in trees] == exp_trees


def test_stats_of_a_forest(kb, oracle_mod):
    par = kb.gen_forest(1 << 18, 0x51, kb.FOREST_RRT, 64)
    root, depth = kb.root_forest(par)
    _check(kb, oracle_mod, root, depth)


def test_stats_of_many_lists_and_one_list(kb, oracle_mod):
    # one list: every element has the same root (the warp-aggregated path)
    succ = kb.gen_list(1 << 20, 0x52)
    w = kb.gen_weights(1 << 20, 0x53, 16)
    root, rank = kb.rank_list(succ, w)
    _check(kb, oracle_mod, root, rank)
    # many lists of uneven length, including single-element ones
    rng = np.random.default_rng(7)
    n = 200_000
    perm = rng.permutation(n)
    cuts = np.sort(rng.choice(np.arange(1, n), 5000, replace=False))
    succ_h = np.empty(n, np.uint64)
    for seg in np.split(perm, cuts):
        succ_h[seg[:-1]] = seg[1:]
        succ_h[seg[-1]] = seg[-1]
    root, rank = kb.rank_list(dev64(succ_h))
    _check(kb, oracle_mod, root, rank)


def test_stats_of_signed_in_place_ranks(kb, oracle_mod):
    """Ranks from the in-place signed-weight path: negative distances and
    negative root ranks (roots keep their input rank), so every tree's ranks
    are negative.  Expected values come from the statement-by-statement
    transcription of bench/detail/stats.cpp (a tree's max_rank starts at 0)."""
    rng = np.random.default_rng(0x5A)
    n = 60_000
    perm = rng.permutation(n)
    cuts = np.sort(rng.choice(np.arange(1, n), 300, replace=False))
    succ_h = np.empty(n, np.uint64)
    for seg in np.split(perm, cuts):
        succ_h[seg[:-1]] = seg[1:]
        succ_h[seg[-1]] = seg[-1]
    rank_h = rng.integers(-1000, 0, n).astype(np.int64)
    s, r = dev64(succ_h), dev64(rank_h)
    kb.sparse_ruling_set(kb.SparseRulingSetConfig(), s, r)
    root_h, rk_h = host_u64(s), r.cpu().numpy()
    assert rk_h.max() < 0
    for level in (kb.STATS_BASIC, kb.STATS_REDUCED_EXTENSIVE, kb.STATS_EXTENSIVE):
        figs, trees = kb.compute_stats(s, r, level)
        exp, exp_trees = oracle_mod.compute_stats_transcribed(root_h, rk_h, level)
        for k, v in exp.items():
            if isinstance(v, float):
                assert figs[k] == pytest.approx(v, rel=1e-12, abs=0.0), k
            else:
                assert figs[k] == v, k
        assert [tuple(int(x) for x in t) for t in trees] == exp_trees
    assert exp_trees and all(t[2] == 0 for t in exp_trees)


def test_stats_edge_cases(kb, oracle_mod):
    # every element its own tree: no non-trivial trees
    idx = dev64(np.arange(1000, dtype=np.uint64))
    zero = dev64(np.zeros(1000, np.uint64))
    _check(kb, oracle_mod, idx, zero)
    figs, trees = kb.compute_stats(idx, zero, kb.STATS_NONE)
    assert figs["num_trees"] == 0 and trees.shape[0] == 0
    # a root out of range is reported
    bad = dev64(np.array([0, 7, 1], np.uint64))
    with pytest.raises(kb.KascadeError) as e:
        kb.compute_stats(bad, dev64(np.zeros(3, np.uint64)))
    assert e.value.name == "OUT_OF_RANGE"
