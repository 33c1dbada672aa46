"""Batched ranking of many lists and forests in one call, instance by
instance against the oracle (bit-exact)."""
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


def _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank):
    inp = host_u64(inputs)
    wh = w.cpu().numpy().view(np.uint32) if w is not None else None
    r_all, k_all = host_u64(root), host_u64(rank)
    off = 0
    for i, (sz, kd) in enumerate(zip(sizes, kinds)):
        sz = int(sz)
        sl = slice(off, off + sz)
        if kd == kb.SEG_LIST:
            r_o, k_o = oracle_mod.rank_list(inp[sl], None if wh is None else wh[sl])
        else:
            r_o, k_o = oracle_mod.root_forest(inp[sl])
        np.testing.assert_array_equal(r_all[sl], r_o, err_msg=f"instance {i} kind {kd} size {sz}")
        np.testing.assert_array_equal(k_all[sl], k_o, err_msg=f"instance {i} kind {kd} size {sz}")
        off += sz


@pytest.mark.parametrize("tuning", [{}, DEEP, dict(base_case_size=64), dict(ruler_spacing=5),
                                    # the write-free level 0 (the default from 2^25 records), forced
                                    dict(level0_mode=2), dict(DEEP, level0_mode=2)])
@pytest.mark.parametrize("weighted", [False, True])
def test_batch_mixed(kb, oracle_mod, tuning, weighted):
    sizes, kinds = kb.batch_sizes(300, seed=7, lo_log2=0, hi_log2=14)
    inputs, w = kb.gen_batch(sizes, kinds, seed=0xC3)
    segs = kb.make_segments(sizes, kinds)
    root, rank = kb.rank_batch(inputs, segs, w if weighted else None, tuning=kb.GpuTuning(**tuning))
    _check(kb, oracle_mod, inputs, w if weighted else None, sizes, kinds, root, rank)


@pytest.mark.parametrize("level0_mode", [0, 1, 2])
def test_batch_large_instances(kb, oracle_mod, level0_mode):
    sizes = np.array([1 << 20, 64, 3000, 1 << 19, 1, 2, 70000], np.int64)
    kinds = np.array([0, 1, 0, 1, 1, 0, 0])
    inputs, w = kb.gen_batch(sizes, kinds, seed=11)
    segs = kb.make_segments(sizes, kinds)
    root, rank = kb.rank_batch(inputs, segs, w, tuning=kb.GpuTuning(level0_mode=level0_mode))
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)


def test_batch_write_free_overflow_and_profile(kb, oracle_mod):
    """A batch on the write-free level 0: its kernels run (profile names), and
    an all-roots batch, whose levels outgrow the device-driven capacities, is
    ranked again on the host-driven path with the same exact results."""
    sizes, kinds = kb.batch_sizes(64, seed=41, lo_log2=10, hi_log2=18)
    inputs, w = kb.gen_batch(sizes, kinds, seed=43)
    ctx = kb.Context()
    root, rank = kb.rank_batch(inputs, kb.make_segments(sizes, kinds), w, ctx=ctx,
                               tuning=kb.GpuTuning(level0_mode=2, profile=True))
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    times = ctx.kernel_times()
    assert "resolve" in times and "place" in times
    sizes = np.full(40, 50_000, np.int64)
    kinds = np.zeros(40, np.int64)
    inputs = torch.cat([torch.arange(50_000, dtype=torch.int64, device="cuda") for _ in range(40)])
    root, rank = kb.rank_batch(inputs, kb.make_segments(sizes, kinds), None, ctx=ctx,
                               tuning=kb.GpuTuning(level0_mode=2))
    _check(kb, oracle_mod, inputs, None, sizes, kinds, root, rank)
    ctx.close()


def test_batch_device_levels_and_fallback(kb, oracle_mod):
    """The batch recursion keeps level sizes on the device; a batch whose
    levels outgrow their capacities (every element a root) is ranked again on
    the host-driven path, with the same exact results."""
    # normal: a batch big enough for several device-driven levels
    sizes, kinds = kb.batch_sizes(64, seed=21, lo_log2=12, hi_log2=19)
    inputs, w = kb.gen_batch(sizes, kinds, seed=23)
    ctx = kb.Context()
    root, rank = kb.rank_batch(inputs, kb.make_segments(sizes, kinds), w, ctx=ctx)
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    # all roots: level 1 is as large as level 0
    sizes = np.full(40, 50_000, np.int64)
    kinds = np.zeros(40, np.int64)
    inputs = torch.cat([torch.arange(50_000, dtype=torch.int64, device="cuda") for _ in range(40)])
    root, rank = kb.rank_batch(inputs, kb.make_segments(sizes, kinds), None, ctx=ctx)
    _check(kb, oracle_mod, inputs, None, sizes, kinds, root, rank)
    ctx.close()


def test_batch_plan_graph_replay(kb, oracle_mod):
    """A batch captured as a CUDA graph: replays give the plain call's exact
    results, also after the inputs' contents change in place."""
    sizes, kinds = kb.batch_sizes(200, seed=31, lo_log2=6, hi_log2=16)
    inputs, w = kb.gen_batch(sizes, kinds, seed=33)
    segs = kb.make_segments(sizes, kinds)
    plan = kb.BatchPlan(inputs, segs, w)
    for _ in range(2):
        root, rank = plan.launch()
        torch.cuda.synchronize()
        _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    # new contents, same shape
    inputs2, w2 = kb.gen_batch(sizes, kinds, seed=35)
    inputs.copy_(inputs2)
    w.copy_(w2)
    root, rank = plan.launch()
    torch.cuda.synchronize()
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    r_p, k_p = kb.rank_batch(inputs, segs, w)
    assert torch.equal(root, r_p) and torch.equal(rank, k_p)
    plan.close()
    # a batch that needs the host-driven recursion cannot be planned
    sizes = np.full(40, 50_000, np.int64)
    kinds = np.zeros(40, np.int64)
    roots = torch.cat([torch.arange(50_000, dtype=torch.int64, device="cuda") for _ in range(40)])
    with pytest.raises(kb.KascadeError) as e:
        kb.BatchPlan(roots, kb.make_segments(sizes, kinds))
    assert e.value.name == "UNSUPPORTED"


def test_batch_plan_write_free(kb, oracle_mod):
    """A plan over the write-free level 0 (the path of batches from 2^25
    records, forced here): the captured graph holds the read-only chase, the
    partition passes, the place step and the head walk, and its replays give
    the oracle's results, also after the inputs change in place."""
    sizes, kinds = kb.batch_sizes(120, seed=51, lo_log2=6, hi_log2=17)
    inputs, w = kb.gen_batch(sizes, kinds, seed=53)
    segs = kb.make_segments(sizes, kinds)
    plan = kb.BatchPlan(inputs, segs, w, tuning=kb.GpuTuning(level0_mode=2))
    for _ in range(2):
        root, rank = plan.launch()
        torch.cuda.synchronize()
        _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    inputs2, w2 = kb.gen_batch(sizes, kinds, seed=55)
    inputs.copy_(inputs2)
    w.copy_(w2)
    root, rank = plan.launch()
    torch.cuda.synchronize()
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    plan.close()


def test_batch_only_lists_and_only_forests(kb, oracle_mod):
    for kind in (0, 1):
        sizes = np.array([5000, 1, 7, 20000, 333], np.int64)
        kinds = np.full(sizes.size, kind)
        inputs, w = kb.gen_batch(sizes, kinds, seed=13 + kind)
        root, rank = kb.rank_batch(inputs, kb.make_segments(sizes, kinds), w)
        _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)


def test_class_launch_parameters_keep_results(kb, oracle_mod):
    """Every chains / block choice the autotuner may install gives the same
    ranks; a batch takes them from the class holding most of its elements."""
    sizes, kinds = kb.batch_sizes(300, seed=8, lo_log2=4, hi_log2=15)
    inputs, w = kb.gen_batch(sizes, kinds, seed=29)
    segs = kb.make_segments(sizes, kinds)
    ctx = kb.Context()
    kb.set_size_classes(ctx, [1 << 9, 1 << 12, 1 << 40], [4, 8, 24])
    assert kb.get_class_launch(ctx) == ([2, 2, 2], [256, 256, 256], [4, 8, 24])
    for chains, block in ((1, 128), (2, 512), (4, 256), (4, 512)):
        kb.set_class_launch(ctx, [chains] * 3, [block] * 3)
        assert kb.get_class_launch(ctx)[:2] == ([chains] * 3, [block] * 3)
        root, rank = kb.rank_batch(inputs, segs, w, ctx=ctx)
        _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    with pytest.raises(kb.KascadeError):
        kb.set_class_launch(ctx, [3, 2, 2], [256, 256, 256])
    with pytest.raises(kb.KascadeError):
        kb.set_class_launch(ctx, [2, 2], [256, 256])
    ctx.close()


def test_autotune_table_loads(kb):
    from kascade_b200 import autotune

    table = {"gpu": "test", "classes": [{"max": 1 << 10, "spacing": 6, "chains": 1, "block": 128, "spacing_single": 16},
                                        {"max": (1 << 64) - 1, "spacing": 40, "chains": 4, "block": 512,
                                         "spacing_single": 48}]}
    ctx = kb.Context()
    kb.load_tuning(ctx, table)
    assert kb.get_size_classes(ctx) == ([1 << 10, (1 << 64) - 1], [6, 40])
    assert kb.get_class_launch(ctx) == ([1, 4], [128, 512], [16, 48])
    ctx.close()
    sizes, kinds = autotune.class_sizes(2, 1 << 16, 1)
    assert sizes.min() > autotune.CLASS_MAX[1] and sizes.max() <= autotune.CLASS_MAX[2]


def test_batch_size_classes_and_errors(kb, oracle_mod):
    ctx = kb.Context()
    kb.set_size_classes(ctx, [1 << 8, 1 << 12, 1 << 40], [4, 9, 40])
    ms, sp = kb.get_size_classes(ctx)
    assert sp == [4, 9, 40] and ms[-1] == (1 << 64) - 1
    sizes, kinds = kb.batch_sizes(100, seed=3, lo_log2=2, hi_log2=13)
    inputs, w = kb.gen_batch(sizes, kinds, seed=17)
    root, rank = kb.rank_batch(inputs, kb.make_segments(sizes, kinds), w, ctx=ctx)
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    # an instance-local index out of its instance
    bad = inputs.clone()
    bad[0] = int(sizes[0]) + 5
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_batch(bad, kb.make_segments(sizes, kinds), w, ctx=ctx)
    assert e.value.name == "OUT_OF_RANGE"
    # a segment table that does not tile the input
    segs = kb.make_segments(sizes, kinds)
    segs[1].offset += 1
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_batch(inputs, segs, w, ctx=ctx)
    assert e.value.name == "INVALID_ARG"
    ctx.close()


def test_batch_write_free_errors(kb, oracle_mod):
    """Invalid instances in a batch on the write-free level 0: an out-of-range
    successor, and a forest whose parents close a rootless cycle, report
    their error status; a valid batch afterwards is exact."""
    sizes = np.array([5000, 3000, 20000, 64], np.int64)
    kinds = np.array([kb.SEG_LIST, kb.SEG_FOREST, kb.SEG_LIST, kb.SEG_FOREST])
    inputs, w = kb.gen_batch(sizes, kinds, seed=61)
    segs = kb.make_segments(sizes, kinds)
    t = kb.GpuTuning(level0_mode=2)
    ctx = kb.Context()
    bad = inputs.clone()
    bad[10] = int(sizes[0]) + 3
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_batch(bad, segs, w, tuning=t, ctx=ctx)
    assert e.value.name == "OUT_OF_RANGE"
    cyc = inputs.clone()
    off = int(sizes[0])  # the first forest
    cyc[off + 0], cyc[off + 1], cyc[off + 2] = 1, 2, 0
    with pytest.raises(kb.KascadeError) as e:
        kb.rank_batch(cyc, segs, w, tuning=t, ctx=ctx)
    assert e.value.name in ("CYCLE", "NOT_A_LIST")
    root, rank = kb.rank_batch(inputs, segs, w, tuning=t, ctx=ctx)
    _check(kb, oracle_mod, inputs, w, sizes, kinds, root, rank)
    ctx.close()


def test_batch_4096_instances_full_size_against_reference_chase(kb, oracle_mod):
    """The batched workload at full size (4096 instances, sizes log-uniform in
    [2^6, 2^22], sum 2^28, 70% weighted lists / 30% random recursive forests)
    in one call, every instance against the reference's own GatherChase
    (oracle/_ref, one core): the instances are shifted into one global index
    space by their offsets and ranked by one chase (lists with their weights,
    forests with unit weights, as the reference's GatherRank does)."""
    sizes, kinds = kb.batch_sizes(4096, 0xC3, lo_log2=6, hi_log2=22, total=1 << 28)
    inputs, w = kb.gen_batch(sizes, kinds, seed=0xC3)
    segs = kb.make_segments(sizes, kinds)
    root, rank = kb.rank_batch(inputs, segs, w)
    dev = inputs.device
    sz = torch.from_numpy(np.asarray(sizes, np.int64)).to(dev)
    starts = torch.cumsum(sz, 0) - sz
    seg = torch.repeat_interleave(torch.arange(len(sizes), device=dev), sz)
    off = starts[seg]
    is_list = torch.from_numpy(np.asarray(kinds) == kb.SEG_LIST).to(dev)[seg]
    del seg
    g_succ = inputs + off
    g_rank = torch.where(is_list, w.to(torch.int64) & 0xFFFFFFFF, torch.ones_like(inputs))
    g_rank[g_succ == torch.arange(g_succ.numel(), device=dev)] = 0
    del is_list
    s_h = g_succ.cpu().numpy().view(np.uint64).copy()
    r_h = g_rank.cpu().numpy().copy()
    del g_succ, g_rank
    if oracle_mod.has_ref():
        oracle_mod.ref_local_pointer_chasing(s_h, r_h)
    else:
        oracle_mod.local_pointer_chasing(s_h, r_h)
    exp_root = torch.from_numpy(s_h.view(np.int64)).to(dev) - off
    exp_rank = torch.from_numpy(r_h).to(dev)
    bad = (exp_root != root) | (exp_rank != rank)
    assert not bool(bad.any()), f"{int(bad.sum())} elements differ, first at {int(bad.nonzero()[0])}"


def _shaped_forests(rng):
    """Forests that exercise every element of a batch's leaf-contracted tour:
    isolated roots, stars (a root whose every child is a leaf), paths (no
    leaf but the last vertex), caterpillars, two-vertex trees, several trees
    in one forest, and random trees with vertices relabelled so that parents
    are not below their children."""
    out = [np.array([0], np.uint64), np.array([0, 1, 2, 3], np.uint64), np.zeros(50, np.uint64),
           np.array([1, 1], np.uint64), np.array([0, 0, 2, 2, 4, 4], np.uint64)]
    path = np.arange(1, 801, dtype=np.uint64)
    path[-1] = 799
    out.append(path)
    spine = 300
    cat = np.empty(spine * 3, np.uint64)
    cat[:spine] = np.arange(-1, spine - 1) % spine
    cat[0] = 0
    cat[spine:] = rng.integers(0, spine, 2 * spine)
    out.append(cat)
    for n in (33, 257, 4000):
        par = np.arange(n, dtype=np.uint64)
        for v in range(1, n):
            if rng.random() < 0.97:
                par[v] = rng.integers(0, v)
        perm = rng.permutation(n)
        relabel = np.empty(n, np.uint64)
        relabel[perm] = np.arange(n, dtype=np.uint64)
        p2 = np.empty(n, np.uint64)
        p2[relabel] = relabel[par]
        out.append(p2)
    return out


@pytest.mark.parametrize("tuning", [{}, DEEP, dict(level0_mode=1), dict(level0_mode=2), dict(DEEP, level0_mode=2),
                                    dict(ruler_spacing=3, level0_mode=2), dict(base_case_size=1 << 16)])
def test_batch_forest_shapes(kb, oracle_mod, tuning):
    """Hand-shaped forests between lists in one batch, every tuning path
    (single-CTA base case, stamping and write-free level 0, deep recursion):
    depths and roots equal the oracle's, leaves included."""
    rng = np.random.default_rng(0xF0)
    parts, kinds = [], []
    for f in _shaped_forests(rng):
        lst = oracle_mod.gen_list(int(rng.integers(1, 500)), int(rng.integers(1 << 30)), 0)
        parts += [lst, f]
        kinds += [kb.SEG_LIST, kb.SEG_FOREST]
    sizes = np.array([p.size for p in parts], np.int64)
    kinds = np.array(kinds)
    inputs = dev64(np.concatenate(parts))
    segs = kb.make_segments(sizes, kinds)
    for _ in range(2):  # a second call on the same context reuses its scratch
        root, rank = kb.rank_batch(inputs, segs, None, tuning=kb.GpuTuning(**tuning))
        _check(kb, oracle_mod, inputs, None, sizes, kinds, root, rank)
