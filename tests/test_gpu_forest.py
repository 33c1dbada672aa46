"""Tree rooting (Euler tour + ranking) on the GPU against the oracle and the
reference's own outputs."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gpu_util import DEEP, SPARSE, dev64, host_i64, host_u64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kb():
    import kascade_b200

    return kascade_b200


def _forests(oracle_mod):
    rng = np.random.default_rng(5)
    out = {
        "rrt_64": oracle_mod.gen_forest(1 << 16, 1, 0, 64),
        "rrt_1": oracle_mod.gen_forest(100_000, 2, 0, 1),
        "cat": oracle_mod.gen_forest(1 << 17, 3, 1, 4, 1 << 14),
        "path": np.maximum(np.arange(-1, 40_000), 0).astype(np.uint64),
        "heap": np.maximum((np.arange(70_000) - 1) // 2, 0).astype(np.uint64),
        "star": np.zeros(30_000, np.uint64),
        "all_roots": np.arange(20_000, dtype=np.uint64),
        "single": np.array([0], np.uint64),
    }
    par = np.array([i if (i == 0 or rng.random() < 0.05) else rng.integers(0, i) for i in range(50_000)], np.uint64)
    perm = rng.permutation(50_000).astype(np.uint64)
    relab = np.empty_like(par)
    relab[perm] = perm[par]
    out["random_many_roots"] = relab
    return out


def test_golden_forests(kb, golden_cases):
    for tuning in ({}, DEEP, SPARSE, dict(DEEP, level0_mode=2)):
        t = kb.GpuTuning(**tuning)
        for name, c in golden_cases.items():
            if "w" in c:
                continue  # weighted cases are lists with weights
            if c["kind"][0] != "forest" and not name.startswith(("list_", "single", "pair", "all_roots")):
                continue
            # a list is a forest of paths too
            root, depth = kb.root_forest(dev64(c["succ"]), tuning=t)
            np.testing.assert_array_equal(host_u64(root), c["root"], err_msg=name)
            np.testing.assert_array_equal(host_i64(depth), c["rank"], err_msg=name)


@pytest.mark.parametrize("tuning", [{}, DEEP, SPARSE, dict(DEEP, level0_mode=2), dict(SPARSE, level0_mode=2),
                                    dict(DEEP, level0_mode=2, max_chain=2)])
def test_forests_vs_oracle(kb, oracle_mod, tuning):
    for name, par in _forests(oracle_mod).items():
        root_o, depth_o = oracle_mod.root_forest(par)
        root, depth = kb.root_forest(dev64(par), tuning=kb.GpuTuning(**tuning))
        np.testing.assert_array_equal(host_u64(root), root_o, err_msg=name)
        np.testing.assert_array_equal(host_u64(depth), depth_o, err_msg=name)


@pytest.mark.parametrize("n,kind,blocks,spine", [(1 << 20, 0, 64, 0), (1 << 20, 1, 8, 1 << 16)])
def test_generated_forests(kb, oracle_mod, n, kind, blocks, spine):
    par_h = oracle_mod.gen_forest(n, 0xC2, kind, blocks, spine)
    par = kb.gen_forest(n, 0xC2, kind, blocks, spine)
    np.testing.assert_array_equal(host_u64(par), par_h)
    root_o, depth_o = oracle_mod.root_forest(par_h)
    root, depth = kb.root_forest(par)
    np.testing.assert_array_equal(host_u64(root), root_o)
    np.testing.assert_array_equal(host_u64(depth), depth_o)


@pytest.mark.parametrize("level0_mode", [0, 2])
@pytest.mark.parametrize("kind,blocks,spine", [(0, 40, 0), (1, 4, 1 << 18)])
def test_forest_several_placement_windows(kb, oracle_mod, level0_mode, kind, blocks, spine):
    """Forests whose up records span several 2^20-slot windows of the tour
    placement (the last one partial), random recursive trees and deep
    caterpillars, on both level-0 paths of the tour ranking, against the
    oracle."""
    n = 3 * (1 << 20) + 777
    par_h = oracle_mod.gen_forest(n, 0xC9, kind, blocks, spine)
    root_o, depth_o = oracle_mod.root_forest(par_h)
    root, depth = kb.root_forest(dev64(par_h), tuning=kb.GpuTuning(level0_mode=level0_mode))
    np.testing.assert_array_equal(host_u64(root), root_o)
    np.testing.assert_array_equal(host_u64(depth), depth_o)


def test_compute_euler_tour_kat(kb, kat):
    e = kat["euler_tour_small"]
    tour = kb.compute_euler_tour(dev64(np.array(e["parent"], np.uint64)))
    assert host_u64(tour).tolist() == e["tour_succ"]


def test_compute_euler_tour_vs_oracle(kb, oracle_mod):
    for name, par in _forests(oracle_mod).items():
        if par.size > 70_000:
            continue
        ts, tw, es, ed, up = oracle_mod.euler_tour(par)
        tour = kb.compute_euler_tour(dev64(par))
        np.testing.assert_array_equal(host_u64(tour), ts, err_msg=name)


def test_rank_via_euler_tour_in_place(kb, oracle_mod):
    """Roots keep their input values; non-roots get root and depth."""
    par = oracle_mod.gen_forest(50_000, 8, 0, 16)
    s_o = par.copy()
    r_o = np.where(par == np.arange(par.size, dtype=np.uint64), 7, 1).astype(np.int64)
    r_in = r_o.copy()
    oracle_mod.rank_via_euler_tour(s_o, r_o)
    s = dev64(par)
    r = dev64(r_in)
    kb.rank_via_euler_tour(kb.EulerTourConfig(), s, r)
    np.testing.assert_array_equal(host_u64(s), s_o)
    np.testing.assert_array_equal(host_i64(r), r_o)


def test_root_forest_host(kb, oracle_mod):
    par = oracle_mod.gen_forest(200_000, 11, 1, 5, 10_000)
    root_o, depth_o = oracle_mod.root_forest(par)
    root, depth = kb.root_forest_host(par)
    np.testing.assert_array_equal(root, root_o)
    np.testing.assert_array_equal(depth, depth_o)


@pytest.mark.parametrize("level0_mode", [0, 2])
def test_forest_with_rootless_cycle_reports_error(kb, oracle_mod, level0_mode):
    """Parents that close a cycle without a root (not a forest): the call
    reports an error status instead of a result, for a short cycle (likely
    without a ruler) and a long one, and the context stays usable."""
    rng = np.random.default_rng(0xCA)
    ctx = kb.Context()
    for k in (3, 40_000):
        par = oracle_mod.gen_forest(200_000, 0xCB, 0, 8).copy()
        cyc = rng.permutation(200_000)[:k].astype(np.uint64)
        par[cyc] = np.roll(cyc, -1)
        with pytest.raises(kb.KascadeError) as e:
            kb.root_forest(dev64(par), tuning=kb.GpuTuning(level0_mode=level0_mode), ctx=ctx)
        assert e.value.name in ("CYCLE", "NOT_A_LIST")
    good = oracle_mod.gen_forest(100_000, 0xCC, 0, 8)
    root_o, depth_o = oracle_mod.root_forest(good)
    root, depth = kb.root_forest(dev64(good), ctx=ctx)
    np.testing.assert_array_equal(host_u64(root), root_o)
    np.testing.assert_array_equal(host_u64(depth), depth_o)
    ctx.close()


def test_compute_euler_tour_vs_reference_transcription(kb, oracle_mod):
    """kascade_compute_euler_tour against the statement-by-statement
    transcription of the reference's tour construction (reverse_rooted_tree,
    make_graph, compute_euler_tour_impl) on forests with several roots,
    isolated roots, a star and vertices of high degree."""
    rng = np.random.default_rng(0xE8)
    forests = [np.array([0], np.uint64), np.array([0, 1, 2], np.uint64), np.array([0] * 6, np.uint64),
               np.array([1, 2, 3, 4, 4], np.uint64),
               np.array([3, 3, 3, 3, 2, 2, 6, 6, 9, 9, 0, 6, 11, 13], np.uint64)]
    for n in (24, 41, 64, 500):
        par = np.arange(n, dtype=np.uint64)
        for v in range(1, n):
            if rng.random() < 0.85:
                par[v] = rng.integers(0, v)
        perm = rng.permutation(n)
        lab = np.empty(n, np.uint64)
        lab[perm] = np.arange(n, dtype=np.uint64)
        p2 = np.empty(n, np.uint64)
        p2[lab] = lab[par]
        forests.append(p2)
    for par in forests:
        exp, _, _ = oracle_mod.euler_tour_transcribed(par)
        tour = kb.compute_euler_tour(dev64(par))
        np.testing.assert_array_equal(host_u64(tour), exp, err_msg=str(par[:16]))


def test_high_degree_handling_flag_gives_the_same_results(kb, oracle_mod):
    """use_high_degree_handling=True: the same tour from compute_euler_tour
    and the same roots and depths from rank_via_euler_tour (on one rank the
    reference's proxy construction creates no proxy)."""
    for par in (np.zeros(3000, np.uint64), oracle_mod.gen_forest(20000, 31, 0, 3),
                oracle_mod.gen_forest(20000, 32, 1, 2, 2000)):
        t0 = kb.compute_euler_tour(dev64(par))
        t1 = kb.compute_euler_tour(dev64(par), use_high_degree_handling=True)
        assert torch.equal(t0, t1)
        s_o = par.copy()
        r_o = np.where(par == np.arange(par.size, dtype=np.uint64), 0, 1).astype(np.int64)
        oracle_mod.rank_via_euler_tour(s_o, r_o)
        s = dev64(par)
        r = dev64(np.where(par == np.arange(par.size, dtype=np.uint64), 0, 1).astype(np.int64))
        kb.rank_via_euler_tour(kb.EulerTourConfig(use_high_degree_handling=True), s, r)
        np.testing.assert_array_equal(host_u64(s), s_o)
        np.testing.assert_array_equal(host_i64(r), r_o)


@pytest.mark.parametrize("shape", ["all_roots", "pairs"])
def test_forest_host_call_rerun_when_a_level_outgrows_the_device_recursion(kb, oracle_mod, shape):
    """Forests whose tour gives ~n rulers (every vertex a root, or 2^19
    two-vertex trees) outgrow the device-driven recursion: the host-buffer
    call roots them again on the host-driven path -- at once when
    synchronous, inside kascade_ctx_sync when async -- and the device-pointer
    call likewise; the results equal the oracle's."""
    import ctypes

    n = 1 << 20
    par = np.arange(n, dtype=np.uint64)
    if shape == "pairs":
        par[1::2] = np.arange(0, n, 2, dtype=np.uint64)
    root_o, depth_o = oracle_mod.root_forest(par)
    root, depth = kb.root_forest_host(par)
    np.testing.assert_array_equal(root, root_o)
    np.testing.assert_array_equal(depth, depth_o)
    root_d, depth_d = kb.root_forest(dev64(par))
    np.testing.assert_array_equal(host_u64(root_d), root_o)
    np.testing.assert_array_equal(host_u64(depth_d), depth_o)
    ctx = kb.Context()
    stream = torch.cuda.Stream()
    in_p = torch.from_numpy(par.view(np.int64)).pin_memory()
    out_r = torch.full((n,), -1, dtype=torch.int64).pin_memory()
    out_d = torch.full((n,), -1, dtype=torch.int64).pin_memory()
    o = kb.GpuTuning(async_=True).to_opts()
    for _ in range(2):
        kb._lib.check(kb.lib.kascade_root_forest_host(ctx.handle, in_p.data_ptr(), n, out_r.data_ptr(),
                                                      out_d.data_ptr(), ctypes.byref(o), stream.cuda_stream),
                      "kascade_root_forest_host", ctx.handle)
        kb._lib.check(kb.lib.kascade_ctx_sync(ctx.handle, stream.cuda_stream), "kascade_ctx_sync", ctx.handle)
        np.testing.assert_array_equal(out_r.numpy().view(np.uint64), root_o)
        np.testing.assert_array_equal(out_d.numpy().view(np.uint64), depth_o)
        out_r.fill_(-1)
        out_d.fill_(-1)
    ctx.close()


def test_forest_levels_report_the_tour_length(kb, oracle_mod):
    """The device-driven tour ranking sizes its records for 2n but reports
    the tour's length (n + vertices with a down edge) as level 0."""
    n = 1 << 21
    par = oracle_mod.gen_forest(n, 77, 0, 4)
    ctx = kb.Context()
    kb.root_forest(dev64(par), ctx=ctx)
    torch.cuda.synchronize()
    lv = ctx.levels()
    internal = np.zeros(n, bool)
    nonroot = par != np.arange(n, dtype=np.uint64)
    internal[par[nonroot].astype(np.int64)] = True
    downs = int((internal & nonroot).sum())
    assert lv[0] == n + downs, (lv[:2], n, downs)
    ctx.close()
