"""The C-ABI library loads and exports what include/kascade_b200.h declares
(no compute calls: this runs without a GPU)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_library_loads_and_exports_every_declared_symbol():
    import kascade_b200 as kb

    declared = kb.declared_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(kb.lib, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_declarations_parsed_from_every_header():
    text = "".join(p.read_text() for p in (ROOT / "include").glob("*.h"))
    n = len(re.findall(r"\bkascade_\w+\s*\(", text))
    import kascade_b200 as kb

    assert len(set(kb.declared_symbols())) <= n


def test_status_strings_and_opts():
    import kascade_b200 as kb
    from kascade_b200._lib import Opts

    assert kb.lib.kascade_version().startswith(b"kascade_b200")
    for code in range(10):
        assert kb.lib.kascade_status_string(code)
    o = Opts()
    kb.lib.kascade_opts_init(ctypes.byref(o))
    assert o.struct_size == ctypes.sizeof(Opts) == 56
    assert o.algorithm == 4
    assert kb.lib.kascade_scratch_bytes_rank_list(1 << 20) < kb.lib.kascade_scratch_bytes_rank_list(1 << 28)


def test_library_is_the_in_tree_build():
    import kascade_b200 as kb

    assert Path(kb.LIB_PATH).resolve().parent == (ROOT / "kascade_b200").resolve()


def test_ctx_create_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import kascade_b200 as kb

    h = ctypes.c_void_p()
    st = kb.lib.kascade_ctx_create(0, ctypes.byref(h))
    assert st != 0 and not h.value


def test_config_mapping():
    from kascade_b200 import RulerSelectionStrategy, SparseRulingSetConfig

    c = SparseRulingSetConfig(ruler_selection=RulerSelectionStrategy.heuristic, heuristic_factor=0.05)
    assert c.tuning().ruler_spacing == 20
    c = SparseRulingSetConfig(ruler_selection=RulerSelectionStrategy.limit_rounds, round_limit=64,
                              sparse_ruling_set_rounds=3)
    t = c.tuning()
    assert t.ruler_spacing == 64 and t.max_levels == 3
    assert SparseRulingSetConfig().tuning().ruler_spacing == 0


def test_noalloc_source_names_no_allocating_call():
    """The no-allocation entry point's source calls no device or host
    allocator: no cudaMalloc* (pool and async forms included), cudaFree*,
    cudaHostAlloc / cudaMallocHost, and no allocation through the library's
    context arena."""
    src = (Path(__file__).resolve().parents[1] / "kascade_b200" / "csrc" / "noalloc.cu").read_text()
    code = "\n".join(line.split("//")[0] for line in src.splitlines())
    banned = re.findall(r"\b(cudaMalloc\w*|cudaFree\w*|cudaHostAlloc|cudaMallocHost|cuMem\w*|alloc<|malloc|"
                        r"new\s+\w+\[|kascade_ctx_create)\b", code)
    assert banned == [], banned
