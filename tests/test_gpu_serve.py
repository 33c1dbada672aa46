"""The serving loop: every result equals the oracle and the same request
ranked alone; admission under a tight budget; device-side submission;
release; statistics."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kb():
    import kascade_b200

    return kascade_b200


def _requests(oracle_mod, count, seed, lo=8, hi=17):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(2 ** rng.uniform(lo, hi))
        if rng.random() < 0.7:
            succ = oracle_mod.gen_list(n, seed * 1000 + i, int(rng.integers(0, 2)))
            w = oracle_mod.gen_weights(n, seed * 1000 + i, 16) if rng.random() < 0.5 else None
            out.append((0, succ, w))
        else:
            out.append((1, oracle_mod.gen_forest(n, seed * 1000 + i, 0, max(1, n >> 12)), None))
    return out


def _expected(oracle_mod, kind, inp, w):
    return oracle_mod.rank_list(inp, w) if kind == 0 else oracle_mod.root_forest(inp)


def test_results_same_alone_and_in_the_mix(kb, oracle_mod):
    reqs = _requests(oracle_mod, 80, seed=1)
    srv = kb.Server(small_max=1 << 12, small_batch_elements=1 << 15)
    ids = [None] * len(reqs)

    def submitter(part):
        for i in part:
            kind, inp, w = reqs[i]
            ids[i] = srv.submit(kind, inp, w)

    threads = [threading.Thread(target=submitter, args=(range(k, len(reqs), 4),)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i, (kind, inp, w) in enumerate(reqs):
        srv.wait(ids[i], 120.0)
        root, rank = srv.fetch(ids[i])
        r_o, k_o = _expected(oracle_mod, kind, inp, w)
        np.testing.assert_array_equal(root, r_o, err_msg=f"request {i}")
        np.testing.assert_array_equal(rank, k_o, err_msg=f"request {i}")
        # the same request ranked alone through the plain calls
        if kind == 0:
            r_a, k_a = kb.rank_list_host(inp, w)
        else:
            r_a, k_a = kb.root_forest_host(inp)
        np.testing.assert_array_equal(root, r_a)
        np.testing.assert_array_equal(rank, k_a)
        srv.release(ids[i])
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["bytes_in_use"] == 0
    assert st["batches"] >= 2 and st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_admission_under_a_tight_budget(kb, oracle_mod):
    reqs = _requests(oracle_mod, 24, seed=2, lo=14, hi=18)
    # room for only a few requests at a time: the rest wait and are admitted
    # as earlier ones are released
    srv = kb.Server(hbm_budget=256 << 20, small_max=1 << 15)
    pending = []
    for kind, inp, w in reqs:
        pending.append((srv.submit(kind, inp, w), kind, inp, w))
    for rid, kind, inp, w in pending:
        srv.wait(rid, 120.0)
        root, rank = srv.fetch(rid)
        r_o, k_o = _expected(oracle_mod, kind, inp, w)
        np.testing.assert_array_equal(root, r_o)
        np.testing.assert_array_equal(rank, k_o)
        srv.release(rid)
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()


def test_device_submission_and_results(kb, oracle_mod):
    srv = kb.Server()
    n = 300_000
    succ_h = oracle_mod.gen_list(n, 5, 0)
    w_h = oracle_mod.gen_weights(n, 6, 16)
    succ = torch.from_numpy(succ_h.view(np.int64)).cuda()
    w = torch.from_numpy(w_h.view(np.int32)).cuda()
    par_h = oracle_mod.gen_forest(200_000, 7, 1, 3, 20_000)
    par = torch.from_numpy(par_h.view(np.int64)).cuda()
    a = srv.submit(kb.SEG_LIST, succ, w)
    b = srv.submit(kb.SEG_FOREST, par)
    srv.wait(a, 120.0)
    srv.wait(b, 120.0)
    root, rank = srv.result_device(a)
    r_o, k_o = oracle_mod.rank_list(succ_h, w_h)
    np.testing.assert_array_equal(root.cpu().numpy(), r_o)
    np.testing.assert_array_equal(rank.cpu().numpy(), k_o)
    root, depth = srv.result_device(b)
    r_o, d_o = oracle_mod.root_forest(par_h)
    np.testing.assert_array_equal(root.cpu().numpy(), r_o)
    np.testing.assert_array_equal(depth.cpu().numpy(), d_o)
    srv.release(a)
    srv.release(b)
    srv.close()


def test_continuous_batching_overlaps_and_results_exact(kb, oracle_mod):
    """Requests up to 2^22 elements, large ones submitted first and small ones
    streamed while the large batches run: both lanes run batches, some
    requests are admitted and some batches start while another batch is in
    flight (the server's own counters), and every result equals the oracle
    and the same request ranked alone."""
    rng = np.random.default_rng(0x5E)
    large = _requests(oracle_mod, 16, seed=21, lo=18, hi=22)
    small = _requests(oracle_mod, 120, seed=22, lo=8, hi=16)
    srv = kb.Server(small_max=1 << 16, small_batch_elements=1 << 19)
    ids_l = [srv.submit(kind, inp, w) for kind, inp, w in large]
    ids_s = []
    for kind, inp, w in small:
        ids_s.append(srv.submit(kind, inp, w))
        time.sleep(float(rng.exponential(2e-4)))
    for rid, (kind, inp, w) in zip(ids_l + ids_s, large + small):
        srv.wait(rid, 300.0)
        root, rank = srv.fetch(rid)
        r_o, k_o = _expected(oracle_mod, kind, inp, w)
        np.testing.assert_array_equal(root, r_o)
        np.testing.assert_array_equal(rank, k_o)
        if kind == 0:
            r_a, k_a = kb.rank_list_host(inp, w)
        else:
            r_a, k_a = kb.root_forest_host(inp)
        np.testing.assert_array_equal(root, r_a)
        np.testing.assert_array_equal(rank, k_a)
        srv.release(rid)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(large) + len(small)
    assert st["lane_batches"][0] > 0 and st["lane_batches"][1] > 0, st
    assert st["admitted_while_running"] > 0, st
    assert st["batches_started_overlapping"] > 0, st
