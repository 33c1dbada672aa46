"""List ranking on the GPU against the oracle and the reference's own outputs
(golden fixtures), bit-exact."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gpu_util import DEEP, SPARSE, dev32, dev64, host_i64, host_u64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kb():
    import kascade_b200

    return kascade_b200


TUNINGS = {"default": {}, "deep": DEEP, "sparse": SPARSE, "chains1": dict(DEEP, chains_per_thread=1),
           "chains4": dict(DEEP, chains_per_thread=4),
           # the write-free level 0 (log, radix partition by element, dense placement), forced at small sizes
           "log": dict(DEEP, level0_mode=2), "log_sparse": dict(SPARSE, level0_mode=2),
           "log_chains1": dict(DEEP, level0_mode=2, chains_per_thread=1),
           "log_chains4": dict(DEEP, level0_mode=2, chains_per_thread=4),
           # a hop cap so small that level 0 always falls back to the stamping chase
           "log_fallback": dict(DEEP, level0_mode=2, max_chain=2),
           # chase block sizes the autotuner may pick
           "block128": dict(DEEP, block_size=128), "block512_chains4": dict(DEEP, block_size=512, chains_per_thread=4),
           "log_block512": dict(DEEP, level0_mode=2, block_size=512)}


@pytest.mark.parametrize("tuning", list(TUNINGS))
def test_golden_lists_ruling_set(kb, golden_cases, tuning):
    t = kb.GpuTuning(**TUNINGS[tuning])
    for name, c in golden_cases.items():
        if c["kind"][0] != "list":
            continue
        succ = dev64(c["succ"])
        w = dev32(c["w"]) if "w" in c else None
        root, rank = kb.rank_list(succ, w, tuning=t)
        np.testing.assert_array_equal(host_u64(root), c["root"], err_msg=name)
        np.testing.assert_array_equal(host_i64(rank), c["rank"], err_msg=name)


@pytest.mark.parametrize("alg", ["PointerDoubling", "GatherChase", "AsyncPointerDoubling", "RMAPointerDoubling"])
def test_golden_all_cases_pointer_doubling(kb, golden_cases, alg):
    """The doubling family accepts forests of trees too (GatherChase contract)."""
    for tuning in ({}, {"base_case_size": 16}):
        t = kb.GpuTuning(**tuning)
        for name, c in golden_cases.items():
            succ = dev64(c["succ"])
            w = dev32(c["w"]) if "w" in c else None
            root, rank = kb.rank_list(succ, w, tuning=t, algorithm=kb.Algorithm[alg])
            np.testing.assert_array_equal(host_u64(root), c["root"], err_msg=name)
            np.testing.assert_array_equal(host_i64(rank), c["rank"], err_msg=name)


@pytest.mark.parametrize("n", [8191, 8192, 8193, 65536, 1 << 20])
@pytest.mark.parametrize("layout", [0, 1, 2])
@pytest.mark.parametrize("weighted", [False, True])
def test_generated_lists_vs_oracle(kb, oracle_mod, n, layout, weighted):
    succ_h = oracle_mod.gen_list(n, 0xC0 + n, layout)
    w_h = oracle_mod.gen_weights(n, 0xC1, 16) if weighted else None
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    succ = kb.gen_list(n, 0xC0 + n, layout)
    np.testing.assert_array_equal(host_u64(succ), succ_h)  # device generator == host generator
    w = kb.gen_weights(n, 0xC1, 16) if weighted else None
    if weighted:
        np.testing.assert_array_equal(w.cpu().numpy().view(np.uint32), w_h)
    for mode in (1, 2):
        root, rank = kb.rank_list(succ, w, tuning=kb.GpuTuning(level0_mode=mode))
        np.testing.assert_array_equal(host_u64(root), root_o)
        np.testing.assert_array_equal(host_u64(rank), rank_o)


@pytest.mark.parametrize("layout", [0, 1])
def test_write_free_above_2_22(kb, oracle_mod, layout):
    """The write-free level 0 at a size with several output windows."""
    n = (1 << 22) + 12345
    succ_h = oracle_mod.gen_list(n, 0xD0, layout)
    w_h = oracle_mod.gen_weights(n, 0xD1, 16)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    ctx = kb.Context()
    root, rank = kb.rank_list(dev64(succ_h), dev32(w_h), tuning=kb.GpuTuning(profile=True, level0_mode=2), ctx=ctx)
    np.testing.assert_array_equal(host_u64(root), root_o)
    np.testing.assert_array_equal(host_u64(rank), rank_o)
    times = ctx.kernel_times()
    assert "resolve" in times and "partition" in times and "place" in times
    # the recursion ran on the device: its level sizes come back with the status
    levels = ctx.levels()
    assert levels[0] == n and len(levels) >= 3
    assert all(a > b for a, b in zip(levels, levels[1:]))
    ctx.close()


def test_write_free_many_lists_several_windows(kb, oracle_mod):
    """The write-free level 0 on 30 000 lists over three 2^20-element output
    windows (the last one partial): thousands of list heads ahead of their
    first ruler, spread over many sub-windows, walk to their first reached
    element."""
    rng = np.random.default_rng(0xE1)
    n = 2 * (1 << 20) + 777
    order = rng.permutation(n).astype(np.uint64)
    cuts = np.sort(rng.choice(np.arange(1, n), size=30_000 - 1, replace=False))
    succ_h = np.empty(n, np.uint64)
    for seg in np.split(order, cuts):
        succ_h[seg[:-1]] = seg[1:]
        succ_h[seg[-1]] = seg[-1]
    w_h = rng.integers(0, 1 << 16, n).astype(np.uint32)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    for tuning in (dict(level0_mode=2), dict(level0_mode=2, ruler_spacing=200)):
        root, rank = kb.rank_list(dev64(succ_h), dev32(w_h), tuning=kb.GpuTuning(**tuning))
        np.testing.assert_array_equal(host_u64(root), root_o)
        np.testing.assert_array_equal(host_u64(rank), rank_o)


@pytest.mark.parametrize("spacing", [16, 48, 2000])
@pytest.mark.parametrize("lists", [1, 3000])
def test_write_free_spacings_and_list_counts(kb, oracle_mod, spacing, lists):
    """The write-free level 0 from dense to very sparse rulers: at spacing
    2000 the few rulers are all taken at once and every chain is long (the
    longest ~15 000 hops); with 3000 lists most lists hold no ruler but their
    root, so their heads are walked after the place step.  Results stay
    exact, and a second call on the same input agrees."""
    rng = np.random.default_rng(spacing * 7 + lists)
    n = (1 << 22) + 5
    order = rng.permutation(n).astype(np.uint64)
    cuts = np.sort(rng.choice(np.arange(1, n), size=lists - 1, replace=False))
    succ_h = np.empty(n, np.uint64)
    for seg in np.split(order, cuts):
        succ_h[seg[:-1]] = seg[1:]
        succ_h[seg[-1]] = seg[-1]
    w_h = rng.integers(0, 1 << 16, n).astype(np.uint32)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    tuning = kb.GpuTuning(level0_mode=2, ruler_spacing=spacing)
    for _ in range(2):
        root, rank = kb.rank_list(dev64(succ_h), dev32(w_h), tuning=tuning)
        np.testing.assert_array_equal(host_u64(root), root_o)
        np.testing.assert_array_equal(host_u64(rank), rank_o)


@pytest.mark.parametrize("offset", [(0, 0), (1, 0), (0, 1), (1, 3)])
def test_input_alignment(kb, oracle_mod, offset):
    """Inputs that start 16 B aligned take the bulk-copy prepare for their full
    tiles and the plain one for the tail; shifted inputs take the plain one."""
    import torch

    n = 148 * 2048 * 2 + 777
    succ_h = oracle_mod.gen_list(n, 0xA1, 0)
    w_h = oracle_mod.gen_weights(n, 0xA2, 16)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    so, wo = offset
    sbuf = torch.empty(n + so, dtype=torch.int64, device="cuda")
    sbuf[so:] = dev64(succ_h)
    wbuf = torch.empty(n + wo, dtype=torch.int32, device="cuda")
    wbuf[wo:] = dev32(w_h)
    for w in (wbuf[wo:], None):
        root, rank = kb.rank_list(sbuf[so:], w)
        if w is None:
            ro, ko = oracle_mod.rank_list(succ_h)
        else:
            ro, ko = root_o, rank_o
        np.testing.assert_array_equal(host_u64(root), ro)
        np.testing.assert_array_equal(host_u64(rank), ko)


def test_device_levels_overflow_rerun(kb, oracle_mod):
    """Every element a root: the first level is as large as the list, more
    than the device-driven recursion holds; the call reranks on the
    host-driven path and the result is exact."""
    n = 300_000
    succ_h = np.arange(n, dtype=np.uint64)
    succ_h[1::2] = np.arange(0, n, 2, dtype=np.uint64)  # pairs: odd -> even, evens are roots
    root, rank = kb.rank_list(dev64(succ_h))
    r_o, k_o = oracle_mod.rank_list(succ_h)
    np.testing.assert_array_equal(host_u64(root), r_o)
    np.testing.assert_array_equal(host_u64(rank), k_o)


@pytest.mark.parametrize("parts", [2, 37, 1000, 20000])
def test_many_lists(kb, oracle_mod, parts):
    rng = np.random.default_rng(parts)
    n = 200_000
    order = rng.permutation(n).astype(np.uint64)
    cuts = np.sort(rng.choice(np.arange(1, n), size=parts - 1, replace=False))
    succ_h = np.empty(n, np.uint64)
    for seg in np.split(order, cuts):
        succ_h[seg[:-1]] = seg[1:]
        succ_h[seg[-1]] = seg[-1]
    w_h = rng.integers(0, 1 << 16, n).astype(np.uint32)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    for tuning in ({}, DEEP, SPARSE, dict(DEEP, level0_mode=2), dict(level0_mode=2, base_case_size=64)):
        root, rank = kb.rank_list(dev64(succ_h), dev32(w_h), tuning=kb.GpuTuning(**tuning))
        np.testing.assert_array_equal(host_u64(root), root_o)
        np.testing.assert_array_equal(host_u64(rank), rank_o)


def test_edge_sizes(kb, oracle_mod):
    for succ_h in (np.array([0], np.uint64), np.array([1, 1], np.uint64), np.array([0, 0], np.uint64),
                   np.arange(50_000, dtype=np.uint64),  # all roots
                   np.minimum(np.arange(1, 30_001), 29_999).astype(np.uint64),  # path 0 -> 1 -> ...
                   np.maximum(np.arange(-1, 29_999), 0).astype(np.uint64)):  # path n-1 -> ... -> 0
        root_o, rank_o = oracle_mod.rank_list(succ_h)
        for tuning in ({}, DEEP, dict(DEEP, level0_mode=2)):
            root, rank = kb.rank_list(dev64(succ_h), tuning=kb.GpuTuning(**tuning))
            np.testing.assert_array_equal(host_u64(root), root_o)
            np.testing.assert_array_equal(host_u64(rank), rank_o)
    empty = torch.empty(0, dtype=torch.int64, device="cuda")
    root, rank = kb.rank_list(empty)
    assert root.numel() == 0 and rank.numel() == 0


def test_zero_and_max_weights(kb, oracle_mod):
    n = 100_000
    succ_h = oracle_mod.gen_list(n, 7, 0)
    for w_h in (np.zeros(n, np.uint32), np.full(n, 0xFFFFFFFF, np.uint32)):
        root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
        for tuning in ({}, DEEP, dict(DEEP, level0_mode=2)):
            root, rank = kb.rank_list(dev64(succ_h), dev32(w_h), tuning=kb.GpuTuning(**tuning))
            np.testing.assert_array_equal(host_u64(rank), rank_o)
            np.testing.assert_array_equal(host_u64(root), root_o)


def test_host_variant(kb, oracle_mod):
    n = 300_000
    succ_h = oracle_mod.gen_list(n, 9, 1)
    w_h = oracle_mod.gen_weights(n, 10, 16)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    root, rank = kb.rank_list_host(succ_h, w_h)
    np.testing.assert_array_equal(root, root_o)
    np.testing.assert_array_equal(rank, rank_o)


def test_host_calls_odd_sizes_offset_outputs_and_an_unsynced_async_call(kb, oracle_mod):
    """Host-buffer calls on one context: odd sizes from 1 to 9 Mi elements
    (the context's arena grows between them), output buffers that start 8 B
    past an aligned address (pageable numpy memory), and an async call that is
    followed by another call on the same context without kascade_ctx_sync
    (the async call's outputs are complete all the same)."""
    import ctypes

    ctx = kb.Context()
    for n in (1, 7, 4097, (9 << 20) + 3):
        succ_h = oracle_mod.gen_list(n, 0x51 + n, 0)
        w_h = oracle_mod.gen_weights(n, 0x52, 16)
        root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
        root, rank = kb.rank_list_host(succ_h, w_h, ctx=ctx)
        np.testing.assert_array_equal(root, root_o)
        np.testing.assert_array_equal(rank, rank_o)
        # outputs 8 B past a 32 B boundary (pageable numpy memory)
        big_r = np.zeros(n + 1, np.uint64)
        big_k = np.zeros(n + 1, np.uint64)
        o = kb.GpuTuning().to_opts()
        st = kb.lib.kascade_rank_list_host(ctx.handle, succ_h.ctypes.data, w_h.ctypes.data, n,
                                           big_r[1:].ctypes.data, big_k[1:].ctypes.data, ctypes.byref(o),
                                           torch.cuda.current_stream().cuda_stream)
        kb._lib.check(st, "kascade_rank_list_host", ctx.handle)
        np.testing.assert_array_equal(big_r[1:], root_o)
        np.testing.assert_array_equal(big_k[1:], rank_o)
        assert big_r[0] == 0 and big_k[0] == 0
    # an async call, then a forest call on the same context before any sync
    n = 300_001
    succ_h = oracle_mod.gen_list(n, 0x53, 1)
    root_o, rank_o = oracle_mod.rank_list(succ_h)
    par_h = oracle_mod.gen_forest(n, 0x54, 0, 5)
    froot_o, depth_o = oracle_mod.root_forest(par_h)
    r1 = np.zeros(n, np.uint64)
    k1 = np.zeros(n, np.uint64)
    o = kb.GpuTuning(async_=True).to_opts()
    s = torch.cuda.current_stream().cuda_stream
    kb._lib.check(kb.lib.kascade_rank_list_host(ctx.handle, succ_h.ctypes.data, None, n, r1.ctypes.data,
                                                k1.ctypes.data, ctypes.byref(o), s), "async call", ctx.handle)
    froot, depth = kb.root_forest_host(par_h, ctx=ctx)
    np.testing.assert_array_equal(r1, root_o)
    np.testing.assert_array_equal(k1, rank_o)
    np.testing.assert_array_equal(froot, froot_o)
    np.testing.assert_array_equal(depth, depth_o)
    ctx.close()


def test_seed_independence(kb, oracle_mod):
    """Ruler choice cannot change the result."""
    n = 250_000
    succ_h = oracle_mod.gen_list(n, 3, 0)
    w_h = oracle_mod.gen_weights(n, 4, 16)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    for seed in (1, 2, 3, 0xDEADBEEF):
        root, rank = kb.rank_list(dev64(succ_h), dev32(w_h), tuning=kb.GpuTuning(seed=seed, ruler_spacing=7))
        np.testing.assert_array_equal(host_u64(rank), rank_o)
        np.testing.assert_array_equal(host_u64(root), root_o)


def test_profile_and_levels(kb):
    ctx = kb.Context()
    succ = kb.gen_list(1 << 20, 1, 0)
    kb.rank_list(succ, tuning=kb.GpuTuning(profile=True), ctx=ctx)
    times = ctx.kernel_times()
    assert "chase" in times and "propagate" in times and "prepare" in times
    lv = ctx.levels()
    assert lv[0] == 1 << 20 and len(lv) >= 2 and lv[1] < lv[0] // 8
    ctx.close()


def test_host_async_pipelined_on_two_contexts(kb, oracle_mod):
    """Host-buffer calls with async set, alternating over two contexts and two
    streams from pinned buffers (a call's copy-out overlaps the next call's
    copy-in): every call's outputs equal the oracle's once its context has
    been synced, lists and forests alike."""
    import ctypes

    n = 1 << 18
    succ_h = oracle_mod.gen_list(n, 21, 0)
    w_h = oracle_mod.gen_weights(n, 22, 16)
    par_h = oracle_mod.gen_forest(n, 23, 0, 4)
    want_list = oracle_mod.rank_list(succ_h, w_h)
    want_forest = oracle_mod.root_forest(par_h)
    pin = lambda a, dt: torch.from_numpy(a.view(dt)).pin_memory()
    in_succ, in_w, in_par = pin(succ_h, np.int64), pin(w_h, np.int32), pin(par_h, np.int64)
    ctxs = [kb.Context(), kb.Context()]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [(torch.empty(n, dtype=torch.int64).pin_memory(), torch.empty(n, dtype=torch.int64).pin_memory())
            for _ in range(2)]
    o = kb.GpuTuning(async_=True).to_opts()
    pending = [None, None]

    def finish(i):
        kb._lib.check(kb.lib.kascade_ctx_sync(ctxs[i].handle, streams[i].cuda_stream), "kascade_ctx_sync",
                      ctxs[i].handle)
        root_o, rank_o = want_list if pending[i] == "list" else want_forest
        np.testing.assert_array_equal(outs[i][0].numpy().view(np.uint64), root_o, err_msg=pending[i])
        np.testing.assert_array_equal(outs[i][1].numpy().view(np.uint64), rank_o, err_msg=pending[i])
        outs[i][0].fill_(-1)
        outs[i][1].fill_(-1)

    for step in range(6):
        i = step % 2
        if pending[i]:
            finish(i)
        kind = "list" if step % 3 != 2 else "forest"
        if kind == "list":
            st = kb.lib.kascade_rank_list_host(ctxs[i].handle, in_succ.data_ptr(), in_w.data_ptr(), n,
                                               outs[i][0].data_ptr(), outs[i][1].data_ptr(), ctypes.byref(o),
                                               streams[i].cuda_stream)
        else:
            st = kb.lib.kascade_root_forest_host(ctxs[i].handle, in_par.data_ptr(), n, outs[i][0].data_ptr(),
                                                 outs[i][1].data_ptr(), ctypes.byref(o), streams[i].cuda_stream)
        kb._lib.check(st, "host-buffer call", ctxs[i].handle)
        pending[i] = kind
    for i in range(2):
        finish(i)


@pytest.mark.parametrize("shape", ["all_roots", "short_lists"])
def test_host_call_rerun_when_a_level_outgrows_the_device_recursion(kb, oracle_mod, shape):
    """Host-buffer calls rank with the device-driven recursion; an input whose
    level outgrows it (every element a root, or 2^18 lists of four elements)
    is ranked again on the host-driven path -- at once for a synchronous
    call, inside kascade_ctx_sync for an async one -- with the same results."""
    import ctypes

    n = 1 << 20
    if shape == "all_roots":
        succ_h = np.arange(n, dtype=np.uint64)
    else:
        succ_h = np.arange(1, n + 1, dtype=np.uint64)
        succ_h[3::4] = np.arange(3, n, 4, dtype=np.uint64)  # every fourth element ends a list
    w_h = oracle_mod.gen_weights(n, 5, 16)
    root_o, rank_o = oracle_mod.rank_list(succ_h, w_h)
    root, rank = kb.rank_list_host(succ_h, w_h)
    np.testing.assert_array_equal(root, root_o)
    np.testing.assert_array_equal(rank, rank_o)
    ctx = kb.Context()
    stream = torch.cuda.Stream()
    in_s = torch.from_numpy(succ_h.view(np.int64)).pin_memory()
    in_w = torch.from_numpy(w_h.view(np.int32)).pin_memory()
    out_r = torch.full((n,), -1, dtype=torch.int64).pin_memory()
    out_k = torch.full((n,), -1, dtype=torch.int64).pin_memory()
    o = kb.GpuTuning(async_=True).to_opts()
    for _ in range(2):
        kb._lib.check(kb.lib.kascade_rank_list_host(ctx.handle, in_s.data_ptr(), in_w.data_ptr(), n, out_r.data_ptr(),
                                                    out_k.data_ptr(), ctypes.byref(o), stream.cuda_stream),
                      "kascade_rank_list_host", ctx.handle)
        kb._lib.check(kb.lib.kascade_ctx_sync(ctx.handle, stream.cuda_stream), "kascade_ctx_sync", ctx.handle)
        np.testing.assert_array_equal(out_r.numpy().view(np.uint64), root_o)
        np.testing.assert_array_equal(out_k.numpy().view(np.uint64), rank_o)
        out_r.fill_(-1)
        out_k.fill_(-1)
    ctx.close()
