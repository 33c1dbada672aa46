"""The multi-core CPU rankers (the CPU baseline beside the reference's
sequential GatherChase) are exact: the ruling set and pointer doubling
restatements against the reference's own GatherChase (oracle/_ref) where it
was built, else against the oracle's restatement of it."""
from __future__ import annotations

import numpy as np
import pytest


def _gather_chase(oracle_mod, succ, rank):
    s, r = succ.copy(), rank.copy()
    if oracle_mod.has_ref():
        oracle_mod.ref_local_pointer_chasing(s, r)
    else:
        oracle_mod.local_pointer_chasing(s, r)
    return s, r


def _many_lists(n, k, seed):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    cuts = np.sort(rng.choice(np.arange(1, n), k, replace=False))
    succ = np.empty(n, np.uint64)
    for seg in np.split(perm, cuts):
        succ[seg[:-1]] = seg[1:]
        succ[seg[-1]] = seg[-1]
    return succ


def _lists(oracle_mod):
    n = 1 << 18
    yield "random", oracle_mod.gen_list(n, 0xC1, 0)
    yield "runs", oracle_mod.gen_list(n, 0xC1, 1)
    yield "path", oracle_mod.gen_list(n + 7, 3, 2)
    yield "many", _many_lists(300_000, 4000, 5)


@pytest.mark.parametrize("threads", [0, 3])
def test_cpu_ruling_set_equals_gather_chase(oracle_mod, threads):
    for name, succ in _lists(oracle_mod):
        n = succ.size
        rng = np.random.default_rng(n)
        for kind in ("unit", "weighted", "signed"):
            if kind == "unit":
                rank = np.ones(n, np.int64)
            elif kind == "weighted":
                rank = rng.integers(0, 1 << 16, n).astype(np.int64)
            else:
                rank = rng.integers(-1000, 1000, n).astype(np.int64)
            rank[succ == np.arange(n, dtype=np.uint64)] = 0
            s_o, r_o = _gather_chase(oracle_mod, succ, rank)
            for spacing in (4, 32):
                s, r = succ.copy(), rank.copy()
                oracle_mod.cpu_sparse_ruling_set(s, r, spacing=spacing, threads=threads)
                np.testing.assert_array_equal(s, s_o, err_msg=f"{name} {kind} {spacing}")
                np.testing.assert_array_equal(r, r_o, err_msg=f"{name} {kind} {spacing}")


def test_cpu_pointer_doubling_equals_gather_chase(oracle_mod):
    cases = list(_lists(oracle_mod))
    cases.append(("forest", oracle_mod.gen_forest(200_000, 9, 0, 16)))
    cases.append(("caterpillar", oracle_mod.gen_forest(120_000, 4, 1, 3, 20_000)))
    for name, succ in cases:
        n = succ.size
        rank = np.random.default_rng(1).integers(0, 1 << 16, n).astype(np.int64)
        rank[succ == np.arange(n, dtype=np.uint64)] = 0
        s_o, r_o = _gather_chase(oracle_mod, succ, rank)
        s, r = succ.copy(), rank.copy()
        rounds = oracle_mod.cpu_pointer_doubling(s, r, threads=4)
        assert rounds >= 1
        np.testing.assert_array_equal(s, s_o, err_msg=name)
        np.testing.assert_array_equal(r, r_o, err_msg=name)


def test_cpu_rankers_report_cycles_and_bad_indices(oracle_mod):
    n = 100_000
    succ = np.roll(np.arange(n, dtype=np.uint64), 1)  # one rootless cycle
    with pytest.raises(ValueError):
        oracle_mod.cpu_pointer_doubling(succ.copy(), np.ones(n, np.int64))
    bad = oracle_mod.gen_list(n, 2, 0)
    bad[17] = n + 5
    with pytest.raises(ValueError):
        oracle_mod.cpu_sparse_ruling_set(bad.copy(), np.ones(n, np.int64))
    with pytest.raises(ValueError):
        oracle_mod.cpu_pointer_doubling(bad.copy(), np.ones(n, np.int64))


def test_cpu_generators_equal_sequential(oracle_mod):
    np.testing.assert_array_equal(oracle_mod.cpu_gen_list(100_003, 7, 0), oracle_mod.gen_list(100_003, 7, 0))
    np.testing.assert_array_equal(oracle_mod.cpu_gen_list(100_003, 7, 1), oracle_mod.gen_list(100_003, 7, 1))
    np.testing.assert_array_equal(oracle_mod.cpu_gen_weights(100_003, 8, 16), oracle_mod.gen_weights(100_003, 8, 16))
    np.testing.assert_array_equal(oracle_mod.cpu_gen_forest(100_003, 9, 1, 64, 500),
                                  oracle_mod.gen_forest(100_003, 9, 1, 64, 500))
    assert oracle_mod.cpu_threads() >= 1
