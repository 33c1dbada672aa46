"""The CPU oracle against the reference's own code and known answers."""
from __future__ import annotations

import numpy as np
import pytest


def test_oracle_matches_golden(oracle_mod, golden_cases):
    """Golden outputs were produced by the reference's GatherChase."""
    for name, c in golden_cases.items():
        if "w" in c:
            root, rank = oracle_mod.rank_list(c["succ"], c["w"])
        else:
            root, rank = oracle_mod.rank_list(c["succ"])
        np.testing.assert_array_equal(root, c["root"], err_msg=name)
        np.testing.assert_array_equal(rank.view(np.int64), c["rank"], err_msg=name)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_reference_chase(oracle_mod, seed):
    if not oracle_mod.has_ref():
        pytest.skip("oracle/_ref not built (reference source tree absent)")
    inputs = [
        oracle_mod.gen_list(20000, seed, 0),
        oracle_mod.gen_list(20000, seed, 1),
        oracle_mod.gen_forest(30000, seed, 0, 5),
        oracle_mod.gen_forest(30000, seed, 1, 4, 3000),
    ]
    for succ in inputs:
        r1, k1 = oracle_mod.root_forest(succ)
        r2, k2 = oracle_mod.ref_gather_rank(succ)
        np.testing.assert_array_equal(r1, r2)
        np.testing.assert_array_equal(k1.view(np.int64), k2)


def test_pointer_doubling_oracle_agrees(oracle_mod, golden_cases):
    for name, c in golden_cases.items():
        s = c["succ"].copy()
        r = (c["w"].astype(np.int64) if "w" in c else np.ones(s.size, np.int64))
        r[s == np.arange(s.size, dtype=np.uint64)] = 0
        rounds = oracle_mod.pointer_doubling(s, r)
        assert rounds >= 0, name
        np.testing.assert_array_equal(s, c["root"], err_msg=name)
        np.testing.assert_array_equal(r, c["rank"], err_msg=name)


def test_pack_kat(oracle_mod, kat):
    p = kat["pack_works"]
    sp, rp = oracle_mod.pack(np.array(p["succ"]), np.array(p["rank"]), np.array(p["active"]))
    assert sp.tolist() == p["packed_succ"]
    assert rp.tolist() == p["packed_rank"]
    succ = np.array(p["succ"], np.uint64)
    rank = np.array(p["rank"], np.int64)
    oracle_mod.unpack(np.array(p["ranked_packed_succ"]), np.array(p["ranked_packed_rank"]),
                      np.array(p["active"]), succ, rank)
    assert succ.tolist() == p["unpacked_succ"]
    assert rank.tolist() == p["unpacked_rank"]
    s = kat["pack_sanity"]
    n = len(s["succ"])
    sp, rp = oracle_mod.pack(np.array(s["succ"]), np.array(s["rank"]), np.arange(n))
    assert sp.tolist() == s["succ"] and rp.tolist() == s["rank"]


def test_euler_tour_kat(oracle_mod, kat):
    e = kat["euler_tour_small"]
    ts, tw, es, ed, up = oracle_mod.euler_tour(np.array(e["parent"], np.uint64))
    assert ts.tolist() == e["tour_succ"]
    s = np.array(e["parent"], np.uint64)
    r = np.where(s == np.arange(s.size, dtype=np.uint64), 0, 1).astype(np.int64)
    oracle_mod.rank_via_euler_tour(s, r)
    assert s.tolist() == e["root"] and r.tolist() == e["depth"]


@pytest.mark.parametrize("kind,blocks,spine", [(0, 3, 0), (1, 2, 50), (0, 1, 0)])
def test_euler_tour_is_one_list_per_tree(oracle_mod, kind, blocks, spine):
    parent = oracle_mod.gen_forest(700, 9, kind, blocks, spine)
    ts, tw, es, ed, up = oracle_mod.euler_tour(parent)
    m = ts.size
    roots = int((parent == np.arange(700, dtype=np.uint64)).sum())
    assert m == 2 * (700 - roots) + roots
    assert oracle_mod.is_list(ts)
    # ranking the tour with the chase gives the depths at up edges
    s, r = oracle_mod.root_forest(parent)
    ts2 = ts.copy()
    tw2 = tw.copy()
    oracle_mod.local_pointer_chasing(ts2, tw2)
    for e in np.nonzero(up)[0]:
        assert tw2[e] == int(r[es[e]])


def test_generators_are_valid(oracle_mod):
    for layout in (0, 1, 2):
        succ = oracle_mod.gen_list(5000, 3, layout)
        assert oracle_mod.is_list(succ)
        assert int((succ == np.arange(5000, dtype=np.uint64)).sum()) == 1
        root, rank = oracle_mod.rank_list(succ)
        assert sorted(rank.tolist()) == list(range(5000))
    parent = oracle_mod.gen_forest(6400, 4, 0, 64)
    assert int((parent == np.arange(6400, dtype=np.uint64)).sum()) == 64
    cat = oracle_mod.gen_forest(6000, 4, 1, 3, 1000)
    root, depth = oracle_mod.root_forest(cat)
    assert int(depth.max()) in (999, 1000)


def test_generator_fixture_is_stable(oracle_mod, golden_cases):
    """The generators behind the golden inputs have not drifted."""
    np.testing.assert_array_equal(oracle_mod.gen_list(1000, 0xC0, 0), golden_cases["list_random_1000"]["succ"])
    np.testing.assert_array_equal(oracle_mod.gen_weights(3000, 12, 16), golden_cases["list_weighted_3000"]["w"])
    np.testing.assert_array_equal(oracle_mod.gen_forest(6000, 22, 1, 3, 1500), golden_cases["forest_cat_6000"]["succ"])


def test_oracle_detects_cycle(oracle_mod):
    succ = np.array([1, 2, 0, 3], np.uint64)  # 0->1->2->0, 3 root
    with pytest.raises(ValueError):
        oracle_mod.rank_list(succ)


def test_stats_restatement_small(oracle_mod):
    """compute_stats restated with numpy against a direct loop on a tiny case."""
    root = np.array([0, 0, 2, 0, 4, 4, 6], np.uint64)
    rank = np.array([0, 3, 0, 1, 0, 2, 0], np.int64)
    figs, trees = oracle_mod.compute_stats(root, rank, 4)
    assert figs["num_trees"] == 4 and figs["max_rank"] == 3
    assert figs["avg_rank"] == pytest.approx(6 / 7)
    assert figs["ext_num_trees"] == 4 and figs["num_nontrivial_trees"] == 2
    assert figs["nontrivial_size_sum"] == 5 and figs["nontrivial_rank_sum"] == 6
    assert figs["max_size"] == 3
    assert figs["avg_size"] == pytest.approx((5 + 2) / 4)
    assert figs["nontrivial_avg_size"] == pytest.approx(5 / 2)
    assert figs["nontrivial_avg_rank"] == pytest.approx(6 / 5)
    assert trees == [(0, 3, 3, 4), (4, 2, 2, 2)]
    assert oracle_mod.compute_stats_transcribed(root, rank, 4) == (figs, trees)


@pytest.mark.parametrize("lo,hi", [(-1000, 1000), (-1000, -1), (0, 1 << 40)])
def test_stats_restatement_equals_transcription(oracle_mod, lo, hi):
    """The numpy restatement equals the statement-by-statement transcription
    of stats.cpp, signed and all-negative ranks included (a tree of negative
    ranks reports max_rank 0; a negative rank sum averages as unsigned)."""
    rng = np.random.default_rng(lo & 0xFFFF)
    n = 3000
    root = rng.integers(0, 200, n).astype(np.uint64)
    root[:200] = np.arange(200, dtype=np.uint64)
    rank = rng.integers(lo, hi, n).astype(np.int64)
    for level in (1, 2, 3, 4):
        a = oracle_mod.compute_stats(root, rank, level)
        b = oracle_mod.compute_stats_transcribed(root, rank, level)
        assert a[0].keys() == b[0].keys()
        for k in b[0]:
            assert a[0][k] == b[0][k], (level, k)
        assert a[1] == b[1]
    if hi <= 0:
        figs, trees = oracle_mod.compute_stats_transcribed(root, rank, 4)
        assert all(t[2] == 0 for t in trees)
        assert figs["avg_rank"] > 1e15


def _tour_forests():
    """Forests of a few dozen vertices: several roots, isolated roots,
    vertices of degree 3 and more, a star, a path, and random forests."""
    rng = np.random.default_rng(0xE7)
    out = [np.array([0], np.uint64),
           np.array([0, 1, 2], np.uint64),                      # three isolated roots
           np.array([0, 0, 0, 0, 0, 0], np.uint64),             # a star
           np.array([1, 2, 3, 4, 4], np.uint64),                # a path ending in root 4
           np.array([3, 3, 3, 3, 2, 2, 6, 6, 9, 9, 0, 6, 11], np.uint64)]  # two trees, an isolated root, deg >= 3
    for n in (20, 37, 64):
        par = np.arange(n, dtype=np.uint64)
        for v in range(1, n):
            if rng.random() < 0.85:
                par[v] = rng.integers(0, v)
        perm = rng.permutation(n)  # relabel: parents no longer below their children
        relabel = np.empty(n, np.uint64)
        relabel[perm] = np.arange(n, dtype=np.uint64)
        p2 = np.empty(n, np.uint64)
        p2[relabel] = relabel[par]
        out.append(p2)
    return out


def test_euler_tour_restatement_equals_transcription(oracle_mod):
    """The C restatement's reference-numbered tour equals the statement-by-
    statement transcription of reverse_rooted_tree + make_graph +
    compute_euler_tour_impl on forests with several roots, isolated roots
    and high degrees."""
    forests = _tour_forests()
    for n in (200, 1000):
        forests.append(oracle_mod.gen_forest(n, n, 0, 7))
        forests.append(oracle_mod.gen_forest(n, n + 1, 1, 3, n // 10))
    for par in forests:
        ts, tw, _, _, up = oracle_mod.euler_tour(par)
        t2, w2, up2 = oracle_mod.euler_tour_transcribed(par)
        np.testing.assert_array_equal(ts, t2, err_msg=str(par[:20]))
        np.testing.assert_array_equal(tw, w2)
        np.testing.assert_array_equal(up, up2)


def test_high_degree_variant_builds_the_same_tour_on_one_rank(oracle_mod):
    """The resolve_high_degree_tag construction, transcribed for one rank
    (no remote parent, so no proxy; its two edges per vertex sent in the
    other order), gives the same CSR graph and so the same tour as the plain
    construction: compute_euler_tour and rank_via_euler_tour accept the flag
    with unchanged results."""
    forests = _tour_forests()
    forests.append(np.zeros(40, np.uint64))  # a star
    for n in (200, 1000):
        forests.append(oracle_mod.gen_forest(n, n + 7, 0, 5))
    for par in forests:
        a = oracle_mod.euler_tour_transcribed(par)
        b = oracle_mod.euler_tour_transcribed(par, high_degree=True)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
