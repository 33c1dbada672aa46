"""kascade_rank_list_noalloc: the entry point for callers that may not
allocate device memory (it keeps its scratch in a fixed device array of the
library).  Checked through the C ABI against kascade_rank_list on the same
inputs, on two calls in a row; the results are integers and must match
exactly.  This file is collected last so that a failure here comes after
every other test has run."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _reference_rank(lib, ctx, succ, w):
    n = succ.numel()
    root = torch.empty(n, dtype=torch.int64, device="cuda")
    rank = torch.empty(n, dtype=torch.int64, device="cuda")
    st = lib.kascade_rank_list(ctx, succ.data_ptr(), w.data_ptr() if w is not None else None, n, root.data_ptr(),
                               rank.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert st == 0
    return root, rank


def _noalloc_rank(lib, succ, w):
    n = succ.numel()
    root = torch.full((n,), -7, dtype=torch.int64, device="cuda")
    rank = torch.full((n,), -7, dtype=torch.int64, device="cuda")
    st = lib.kascade_rank_list_noalloc(succ.data_ptr(), w.data_ptr() if w is not None else None, n, root.data_ptr(),
                                       rank.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return st, root, rank


def test_noalloc_matches_rank_list_on_two_calls():
    import kascade_b200 as kb
    import oracle

    lib = kb.lib
    ctx = ctypes.c_void_p()
    assert lib.kascade_ctx_create(0, ctypes.byref(ctx)) == 0
    try:
        # call 1: a weighted random list at the maximum size
        n1 = 65536
        s1 = torch.from_numpy(oracle.gen_list(n1, 0xA1, 0).view(np.int64)).cuda()
        w1 = torch.from_numpy(oracle.gen_weights(n1, 0xA2, 16).view(np.int32)).cuda()
        # call 2: a smaller forest of trees with unit weights (the array keeps
        # call 1's contents; the result must not depend on them)
        s2 = torch.from_numpy(oracle.gen_forest(5000, 0xA3, 0, 7).view(np.int64)).cuda()
        r1_ref, k1_ref = _reference_rank(lib, ctx, s1, w1)
        r2_ref, k2_ref = _reference_rank(lib, ctx, s2, None)
        torch.cuda.synchronize()
        st1, r1, k1 = _noalloc_rank(lib, s1, w1)
        st2, r2, k2 = _noalloc_rank(lib, s2, None)
        assert st1 == 0 and st2 == 0
        assert torch.equal(r1, r1_ref) and torch.equal(k1, k1_ref)
        assert torch.equal(r2, r2_ref) and torch.equal(k2, k2_ref)
        # and once more on the first input after the second call
        st3, r3, k3 = _noalloc_rank(lib, s1, w1)
        assert st3 == 0 and torch.equal(r3, r1_ref) and torch.equal(k3, k1_ref)
    finally:
        lib.kascade_ctx_destroy(ctx)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import kascade_b200 as kb

    n = 65537
    s = torch.arange(n, dtype=torch.int64, device="cuda")
    st, _, _ = _noalloc_rank(kb.lib, s, None)
    assert kb._lib.STATUS_NAMES[st] == "TOO_LARGE"


def test_noalloc_allocates_no_device_memory():
    import kascade_b200 as kb
    import oracle

    n = 30000
    s = torch.from_numpy(oracle.gen_list(n, 0xA4, 1).view(np.int64)).cuda()
    root = torch.empty(n, dtype=torch.int64, device="cuda")
    rank = torch.empty(n, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # first call: may load the library's device code on this GPU
    assert kb.lib.kascade_rank_list_noalloc(s.data_ptr(), None, n, root.data_ptr(), rank.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert kb.lib.kascade_rank_list_noalloc(s.data_ptr(), None, n, root.data_ptr(), rank.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    exp_root, exp_rank = oracle.rank_list(oracle.gen_list(n, 0xA4, 1))
    assert np.array_equal(rank.cpu().numpy().view(np.uint64), exp_rank)
    assert np.array_equal(root.cpu().numpy().view(np.uint64), exp_root)


def test_noalloc_error_statuses_then_a_valid_call():
    """An out-of-range successor and rootless cycles (two elements, and one
    long cycle) return their statuses; the next valid call still equals
    kascade_rank_list."""
    import kascade_b200 as kb
    import oracle

    names = kb._lib.STATUS_NAMES
    n = 5000
    bad = oracle.gen_list(n, 0xA5, 0)
    bad[123] = n + 9
    st, _, _ = _noalloc_rank(kb.lib, torch.from_numpy(bad.view(np.int64)).cuda(), None)
    assert names[st] == "OUT_OF_RANGE"
    two = np.arange(n, dtype=np.uint64)
    two[10], two[11] = 11, 10  # a rootless 2-cycle beside n - 2 roots
    st, _, _ = _noalloc_rank(kb.lib, torch.from_numpy(two.view(np.int64)).cuda(), None)
    assert names[st] == "CYCLE"
    ring = np.roll(np.arange(40000, dtype=np.uint64), 1)  # one rootless cycle
    st, _, _ = _noalloc_rank(kb.lib, torch.from_numpy(ring.view(np.int64)).cuda(), None)
    assert names[st] == "CYCLE"
    ctx = ctypes.c_void_p()
    assert kb.lib.kascade_ctx_create(0, ctypes.byref(ctx)) == 0
    try:
        s = torch.from_numpy(oracle.gen_list(20000, 0xA6, 1).view(np.int64)).cuda()
        r_ref, k_ref = _reference_rank(kb.lib, ctx, s, None)
        st, r, k = _noalloc_rank(kb.lib, s, None)
        assert st == 0 and torch.equal(r, r_ref) and torch.equal(k, k_ref)
    finally:
        kb.lib.kascade_ctx_destroy(ctx)
