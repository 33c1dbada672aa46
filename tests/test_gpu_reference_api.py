"""The reference-shaped in-place calls, pack/unpack known answers, is_list,
the initial state, error statuses, and the AbstractAlgorithm-style plug-in."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gpu_util import DEEP, dev64, host_i64, host_u64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kb():
    import kascade_b200

    return kascade_b200


def _signed_case(oracle_mod, n=120_000, seed=3):
    succ = oracle_mod.gen_list(n, seed, 0)
    rng = np.random.default_rng(seed)
    rank = rng.integers(-1000, 1000, n).astype(np.int64)
    roots = succ == np.arange(n, dtype=np.uint64)
    rank[roots] = 0
    return succ, rank


@pytest.mark.parametrize("fn", ["sparse_ruling_set", "pointer_doubling", "rank_on_root", "async_pointer_doubling",
                                "rma_pointer_doubling", "local_pointer_chasing"])
def test_in_place_signed_weights(kb, oracle_mod, fn):
    succ, rank = _signed_case(oracle_mod)
    s_o, r_o = succ.copy(), rank.copy()
    oracle_mod.local_pointer_chasing(s_o, r_o)
    s, r = dev64(succ), dev64(rank)
    f = getattr(kb, fn)
    if fn == "sparse_ruling_set":
        f(kb.SparseRulingSetConfig(gpu=kb.GpuTuning(**DEEP)), s, r)
    elif fn == "pointer_doubling":
        f(kb.PointerDoublingConfig(), s, r)
    elif fn in ("async_pointer_doubling", "rma_pointer_doubling"):
        f(None, s, r)
    else:
        f(s, r)
    np.testing.assert_array_equal(host_u64(s), s_o)
    np.testing.assert_array_equal(host_i64(r), r_o)


def test_roots_keep_input_rank(kb, oracle_mod):
    """GatherChase leaves roots untouched even when their rank is nonzero."""
    n = 50_000
    succ = oracle_mod.gen_list(n, 12, 1)
    rank = np.ones(n, np.int64)
    rank[succ == np.arange(n, dtype=np.uint64)] = 5
    if oracle_mod.has_ref():
        s_o, r_o = succ.copy(), rank.copy()
        oracle_mod.ref_local_pointer_chasing(s_o, r_o)
    else:
        s_o, r_o = succ.copy(), rank.copy()
        oracle_mod.local_pointer_chasing(s_o, r_o)
    for name in ("sparse_ruling_set", "rank_on_root"):
        s, r = dev64(succ), dev64(rank)
        if name == "sparse_ruling_set":
            kb.sparse_ruling_set(kb.SparseRulingSetConfig(), s, r)
        else:
            kb.rank_on_root(s, r)
        np.testing.assert_array_equal(host_u64(s), s_o)
        np.testing.assert_array_equal(host_i64(r), r_o)


def test_set_initial_ranking_state(kb, oracle_mod):
    par = oracle_mod.gen_forest(10_000, 2, 0, 9)
    root, rank = kb.set_initial_ranking_state(dev64(par))
    np.testing.assert_array_equal(host_u64(root), par)
    exp = np.where(par == np.arange(par.size, dtype=np.uint64), 0, 1)
    np.testing.assert_array_equal(host_i64(rank), exp)


def test_is_list(kb, oracle_mod):
    assert kb.is_list(dev64(oracle_mod.gen_list(100_000, 1, 0)))
    assert not kb.is_list(dev64(oracle_mod.gen_forest(100_000, 1, 0, 3)))
    assert kb.is_list(dev64(np.arange(10, dtype=np.uint64)))


def test_pack_unpack_kat(kb, kat):
    p = kat["pack_works"]
    sp, rp = kb.pack(dev64(np.array(p["succ"])), dev64(np.array(p["rank"])), dev64(np.array(p["active"])))
    assert host_u64(sp).tolist() == p["packed_succ"]
    assert host_i64(rp).tolist() == p["packed_rank"]
    s, r = dev64(np.array(p["succ"])), dev64(np.array(p["rank"]))
    kb.unpack(dev64(np.array(p["ranked_packed_succ"])), dev64(np.array(p["ranked_packed_rank"])), s, r,
              dev64(np.array(p["active"])))
    assert host_u64(s).tolist() == p["unpacked_succ"]
    assert host_i64(r).tolist() == p["unpacked_rank"]
    q = kat["pack_sanity"]
    n = len(q["succ"])
    sp, rp = kb.pack(dev64(np.array(q["succ"])), dev64(np.array(q["rank"])), dev64(np.arange(n)))
    assert host_u64(sp).tolist() == q["succ"] and host_i64(rp).tolist() == q["rank"]


def test_pack_then_rank_then_unpack(kb, oracle_mod):
    """Rank a packed sub-list and unpack: the reference's recursion step."""
    n = 40_000
    succ = oracle_mod.gen_list(n, 21, 0)
    root_o, rank_o = oracle_mod.rank_list(succ)
    # the elements at even list positions form a sub-list when we contract:
    # simplest closed sub-list is the whole list
    active = np.arange(n, dtype=np.uint64)
    rank_in = np.where(succ == np.arange(n, dtype=np.uint64), 0, 1).astype(np.int64)
    sp, rp = kb.pack(dev64(succ), dev64(rank_in), dev64(active))
    kb.sparse_ruling_set(kb.SparseRulingSetConfig(), sp, rp)
    s, r = dev64(succ), dev64(rank_in)
    kb.unpack(sp, rp, s, r, dev64(active))
    np.testing.assert_array_equal(host_u64(s), root_o)
    np.testing.assert_array_equal(host_u64(r), rank_o)


def test_error_statuses(kb):
    # successor out of range
    bad = dev64(np.array([1, 5, 2], np.uint64))
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_list(bad)
    assert e.value.name == "OUT_OF_RANGE"
    with pytest.raises(kb.KascadeError) as e:
        kb.root_forest(bad)
    assert e.value.name == "OUT_OF_RANGE"
    # rootless cycles, small (base case) and large (ruling set / doubling)
    for n in (10, 100_000):
        cyc = dev64(((np.arange(n) + 1) % n).astype(np.uint64))
        for alg in (kb.Algorithm.SparseRulingSet, kb.Algorithm.PointerDoubling):
            with pytest.raises(kb.KascadeError) as e:
                kb.rank_list(cyc, algorithm=alg)
            assert e.value.name == "CYCLE"
    # the same on the write-free level 0
    cyc = dev64(((np.arange(100_000) + 1) % 100_000).astype(np.uint64))
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_list(cyc, tuning=kb.GpuTuning(level0_mode=2, base_case_size=64))
    assert e.value.name == "CYCLE"
    # a tail leading into a rootless cycle (not a list): the write-free chase
    # stops at its hop cap and the stamping chase reports the input
    rho = np.arange(1, 3001, dtype=np.uint64)
    rho[-1] = 1000
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_list(dev64(rho), tuning=kb.GpuTuning(level0_mode=2, base_case_size=16, ruler_spacing=4,
                                                      max_chain=64))
    assert e.value.name in ("NOT_A_LIST", "CYCLE")
    # a tree given to the list-only ranker with validation on
    tree = dev64(np.array([0, 0, 0, 1], np.uint64))
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_list(tree, tuning=kb.GpuTuning(validate=True))
    assert e.value.name == "NOT_A_LIST"
    # the context stays usable after errors
    root, rank = kb.rank_list(dev64(np.array([1, 1], np.uint64)))
    assert host_i64(rank).tolist() == [1, 0]


def test_plugin_matches_golden(kb, golden_cases):
    for alg in (kb.Algorithm.SparseRulingSet, kb.Algorithm.PointerDoubling, kb.Algorithm.GatherChase):
        for name, c in golden_cases.items():
            if "w" in c or (alg == kb.Algorithm.SparseRulingSet and c["kind"][0] == "forest"):
                continue
            plug = kb.B200Ranking(alg)
            plug.ingest(c["succ"])
            plug.run()
            np.testing.assert_array_equal(plug.get_root_array(), c["root"], err_msg=name)
            np.testing.assert_array_equal(plug.get_rank_array(), c["rank"], err_msg=name)
    for name in ("forest_rrt_5000", "forest_cat_6000", "forest_star_2000"):
        c = golden_cases[name]
        plug = kb.B200Ranking(kb.Algorithm.EulerTour)
        plug.ingest(c["succ"])
        plug.run()
        np.testing.assert_array_equal(plug.get_root_array(), c["root"], err_msg=name)
        np.testing.assert_array_equal(plug.get_rank_array(), c["rank"], err_msg=name)


def test_streams_and_async(kb, oracle_mod):
    n = 500_000
    succ_h = oracle_mod.gen_list(n, 77, 0)
    root_o, rank_o = oracle_mod.rank_list(succ_h)
    ctx = kb.Context()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    succ = dev64(succ_h)
    torch.cuda.synchronize()
    outs = []
    for st in (s1, s2, s1):
        with torch.cuda.stream(st):
            root, rank = kb.rank_list(succ, tuning=kb.GpuTuning(async_=True), ctx=ctx)
            ctx.sync(st)
            outs.append((root, rank))
    torch.cuda.synchronize()
    for root, rank in outs:
        np.testing.assert_array_equal(host_u64(root), root_o)
        np.testing.assert_array_equal(host_u64(rank), rank_o)
    ctx.close()
