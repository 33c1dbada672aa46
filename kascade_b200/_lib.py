"""ctypes binding of libkascade_b200.so (the C ABI in include/kascade_b200.h).

The shared library is built in-tree (``python -m kascade_b200.build`` or
``__graft_entry__.build()``).  There is no fallback: if the library is absent
or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("KASCADE_B200_LIB", _PKG / "libkascade_b200.so"))

if not LIB_PATH.exists():
    raise ImportError(
        f"kascade_b200: native library {LIB_PATH} is missing; build it with "
        "`python -m kascade_b200.build` (nvcc for sm_100a is required)"
    )

lib = ctypes.CDLL(str(LIB_PATH))

c_void_p = ctypes.c_void_p
c_u64 = ctypes.c_uint64
c_u32 = ctypes.c_uint32
c_int = ctypes.c_int
P = ctypes.POINTER


class Segment(ctypes.Structure):
    """Mirror of ``kascade_segment``."""

    _fields_ = [("offset", ctypes.c_uint64), ("size", ctypes.c_uint64), ("kind", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class ShardDesc(ctypes.Structure):
    """Mirror of ``kascade_shard_desc``."""

    _fields_ = [("lo", c_u64), ("n_local", c_u64), ("n_global", c_u64), ("num_shards", c_u32), ("self", c_u32),
                ("offsets", c_void_p), ("ruler_base", c_u64), ("num_sampled", c_u64), ("fixup_base", c_u64)]


class ServerConfig(ctypes.Structure):
    """Mirror of ``kascade_server_config``."""

    _fields_ = [("struct_size", c_u32), ("device", c_int), ("hbm_budget_bytes", c_u64),
                ("max_batch_requests", c_u32), ("reserved", c_u32), ("max_batch_elements", c_u64),
                ("small_max", c_u64), ("small_batch_elements", c_u64), ("latency_sms", c_u32),
                ("small_reserve_pct", c_u32), ("result_heap_bytes", c_u64)]


class ServerStats(ctypes.Structure):
    """Mirror of ``kascade_server_stats``."""

    _fields_ = [("completed", c_u64), ("completed_small", c_u64), ("batches", c_u64), ("elements", c_u64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("p50_small_ms", ctypes.c_double),
                ("p99_small_ms", ctypes.c_double), ("elements_per_s", ctypes.c_double),
                ("requests_per_s", ctypes.c_double), ("bytes_in_use", c_u64), ("lane_batches", c_u64 * 2),
                ("lane_elements", c_u64 * 2), ("lane_busy_ms", ctypes.c_double * 2),
                ("lane_max_batch_ms", ctypes.c_double * 2), ("partition_sms", c_u64),
                ("partition_batches", c_u64), ("admitted_while_running", c_u64),
                ("batches_started_overlapping", c_u64)]


class Stats(ctypes.Structure):
    """Mirror of ``kascade_stats``."""

    _fields_ = [("num_trees", c_u64), ("max_rank", ctypes.c_int64), ("avg_rank", ctypes.c_double),
                ("ext_num_trees", c_u64), ("num_nontrivial_trees", c_u64), ("nontrivial_size_sum", c_u64),
                ("nontrivial_rank_sum", ctypes.c_int64), ("max_size", c_u64), ("avg_size", ctypes.c_double),
                ("nontrivial_avg_size", ctypes.c_double), ("nontrivial_avg_rank", ctypes.c_double)]


class Opts(ctypes.Structure):
    """Mirror of ``kascade_opts``."""

    _fields_ = [
        ("struct_size", c_u32),
        ("algorithm", c_u32),
        ("ruler_spacing", c_u32),
        ("ruler_spacing_deep", c_u32),
        ("max_levels", c_u32),
        ("base_case_size", c_u32),
        ("chains_per_thread", c_u32),
        ("block_size", c_u32),
        ("validate", c_u32),
        ("async_", c_u32),
        ("profile", c_u32),
        ("seed", c_u32),
        ("level0_mode", c_u32),
        ("max_chain", c_u32),
    ]


_ctx_p = c_void_p
_status = c_int

_SIGS = {
    "kascade_version": (ctypes.c_char_p, []),
    "kascade_status_string": (ctypes.c_char_p, [c_int]),
    "kascade_opts_init": (None, [P(Opts)]),
    "kascade_ctx_create": (_status, [c_int, P(c_void_p)]),
    "kascade_ctx_destroy": (_status, [_ctx_p]),
    "kascade_ctx_reserve": (_status, [_ctx_p, c_u64]),
    "kascade_scratch_bytes_rank_list": (c_u64, [c_u64]),
    "kascade_scratch_bytes_root_forest": (c_u64, [c_u64]),
    "kascade_ctx_sync": (_status, [_ctx_p, c_void_p]),
    "kascade_ctx_error_info": (c_u64, [_ctx_p]),
    "kascade_ctx_kernel_times": (
        c_int,
        [_ctx_p, P(ctypes.c_char_p), P(ctypes.c_double), P(c_u64), c_int],
    ),
    "kascade_ctx_reset_kernel_times": (None, [_ctx_p]),
    "kascade_ctx_last_levels": (c_int, [_ctx_p, P(c_u64), c_int]),
    "kascade_rank_list": (
        _status,
        [_ctx_p, c_void_p, c_void_p, c_u64, c_void_p, c_void_p, P(Opts), c_void_p],
    ),
    "kascade_rank_list_host": (
        _status,
        [_ctx_p, c_void_p, c_void_p, c_u64, c_void_p, c_void_p, P(Opts), c_void_p],
    ),
    "kascade_sparse_ruling_set": (_status, [_ctx_p, P(Opts), c_void_p, c_void_p, c_u64, c_void_p]),
    "kascade_pointer_doubling": (_status, [_ctx_p, P(Opts), c_void_p, c_void_p, c_u64, c_void_p]),
    "kascade_rank_on_root": (_status, [_ctx_p, c_void_p, c_void_p, c_u64, c_void_p]),
    "kascade_set_initial_ranking_state": (
        _status,
        [_ctx_p, c_void_p, c_void_p, c_void_p, c_u64, c_void_p],
    ),
    "kascade_is_list": (_status, [_ctx_p, c_void_p, c_u64, P(c_int), c_void_p]),
    "kascade_root_forest": (
        _status,
        [_ctx_p, c_void_p, c_u64, c_void_p, c_void_p, P(Opts), c_void_p],
    ),
    "kascade_root_forest_host": (
        _status,
        [_ctx_p, c_void_p, c_u64, c_void_p, c_void_p, P(Opts), c_void_p],
    ),
    "kascade_rank_via_euler_tour": (_status, [_ctx_p, P(Opts), c_void_p, c_void_p, c_u64, c_void_p]),
    "kascade_compute_euler_tour": (_status, [_ctx_p, c_void_p, c_u64, c_void_p, P(c_u64), c_void_p]),
    "kascade_pack": (
        _status,
        [_ctx_p, c_void_p, c_void_p, c_u64, c_void_p, c_u64, c_void_p, c_void_p, c_void_p],
    ),
    "kascade_unpack": (
        _status,
        [_ctx_p, c_void_p, c_void_p, c_void_p, c_u64, c_void_p, c_void_p, c_u64, c_void_p],
    ),
    "kascade_gen_list": (_status, [c_u64, c_u64, c_u32, c_void_p, c_void_p]),
    "kascade_gen_weights": (_status, [c_u64, c_u64, c_u32, c_void_p, c_void_p]),
    "kascade_gen_forest": (_status, [c_u64, c_u64, c_u32, c_u64, c_u64, c_void_p, c_void_p]),
    "kascade_calibrate_random_access": (_status, [_ctx_p, c_u64, c_u32, c_u32, P(ctypes.c_double)]),
    "kascade_rank_list_noalloc": (_status, [c_void_p, c_void_p, c_u64, c_void_p, c_void_p, c_void_p]),
    "kascade_rank_batch": (
        _status,
        [_ctx_p, P(Segment), c_u32, c_void_p, c_void_p, c_u64, c_void_p, c_void_p, P(Opts), c_void_p],
    ),
    "kascade_ctx_set_size_classes": (_status, [_ctx_p, P(c_u64), P(c_u32), c_u32]),
    "kascade_ctx_get_size_classes": (c_int, [_ctx_p, P(c_u64), P(c_u32), c_int]),
    "kascade_ctx_set_class_launch": (_status, [_ctx_p, P(c_u32), P(c_u32), P(c_u32), c_u32]),
    "kascade_batch_plan_create": (_status, [c_int, c_void_p, c_u32, c_void_p, c_void_p, c_u64, c_void_p, c_void_p,
                                            c_void_p, P(c_void_p)]),
    "kascade_batch_plan_launch": (_status, [c_void_p, c_void_p]),
    "kascade_batch_plan_destroy": (_status, [c_void_p]),
    "kascade_compute_stats": (_status, [_ctx_p, c_void_p, c_void_p, c_u64, c_int, P(Stats), c_void_p, c_u64,
                                        P(c_u64), c_void_p]),
    "kascade_ctx_get_class_launch": (c_int, [_ctx_p, P(c_u32), P(c_u32), P(c_u32), c_int]),
    "kascade_ctx_set_sm_budget": (_status, [_ctx_p, c_int]),
    "kascade_shard_prepare": (_status, [_ctx_p, P(ShardDesc), c_void_p, c_void_p, c_u64, c_u32, c_u32, c_void_p,
                                        c_void_p, P(c_u64), c_void_p]),
    "kascade_shard_chase": (_status, [_ctx_p, P(ShardDesc), c_void_p, c_void_p, c_u64, c_void_p, c_u64, c_void_p,
                                      c_u64, c_void_p, P(c_u64), c_void_p, P(c_u64), c_u64, c_void_p]),
    "kascade_shard_unreached": (_status, [_ctx_p, P(ShardDesc), c_void_p, c_void_p, c_u64, P(c_u64), c_void_p]),
    "kascade_shard_ruler_globals": (_status, [_ctx_p, c_void_p, c_u64, c_u64, c_u64, c_void_p, c_void_p]),
    "kascade_shard_sublist": (_status, [_ctx_p, c_void_p, c_u64, c_u64, c_void_p, c_void_p, c_void_p]),
    "kascade_shard_propagate": (_status, [_ctx_p, P(ShardDesc), c_void_p, c_void_p, c_void_p, c_void_p, c_u64,
                                          c_void_p, c_void_p, c_void_p]),
    "kascade_server_config_init": (None, [P(ServerConfig)]),
    "kascade_server_create": (_status, [P(ServerConfig), P(c_void_p)]),
    "kascade_server_destroy": (_status, [c_void_p]),
    "kascade_server_submit": (_status, [c_void_p, c_u32, c_void_p, c_void_p, c_u64, P(c_u64)]),
    "kascade_server_submit_device": (_status, [c_void_p, c_u32, c_void_p, c_void_p, c_u64, P(c_u64)]),
    "kascade_server_wait": (_status, [c_void_p, c_u64, ctypes.c_double]),
    "kascade_server_result_device": (_status, [c_void_p, c_u64, P(c_void_p), P(c_void_p)]),
    "kascade_server_fetch": (_status, [c_void_p, c_u64, c_void_p, c_void_p]),
    "kascade_server_release": (_status, [c_void_p, c_u64]),
    "kascade_server_get_stats": (_status, [c_void_p, P(ServerStats)]),
    "kascade_server_reset_stats": (_status, [c_void_p]),
}

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


STATUS_NAMES = {
    0: "OK",
    1: "INVALID_ARG",
    2: "OUT_OF_RANGE",
    3: "CYCLE",
    4: "NOT_A_LIST",
    5: "TIMEOUT",
    6: "OOM",
    7: "CUDA",
    8: "TOO_LARGE",
    9: "UNSUPPORTED",
}


class KascadeError(RuntimeError):
    """A non-OK ``kascade_status``; ``.status`` holds the code."""

    def __init__(self, status: int, where: str, info: int | None = None):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        msg = lib.kascade_status_string(status).decode()
        detail = f" (info {info})" if info else ""
        super().__init__(f"{where}: KASCADE_ERR_{self.name}: {msg}{detail}")


def check(status: int, where: str, ctx=None) -> None:
    if status != 0:
        info = lib.kascade_ctx_error_info(ctx) if ctx else None
        raise KascadeError(status, where, info)


def declared_symbols(header: Path | None = None) -> list[str]:
    """Function names declared with KASCADE_API in the public C headers."""
    import re

    inc = _PKG.parent / "include"
    names: list[str] = []
    for h in [header] if header else sorted(inc.glob("*.h")):
        text = Path(h).read_text()
        names += re.findall(r"KASCADE_API[^;{(]*?\b(kascade_\w+)\s*\(", text, flags=re.S)
    return names
