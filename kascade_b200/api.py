"""Python mirror of kascade's list-ranking API on one B200.

Function names, argument meaning and in-place behaviour follow the reference
library ``lib/kascade`` (niklas-uhl/kascade); every call goes through the C ABI
of libkascade_b200.so.  Device arrays are CUDA ``torch`` tensors used as plain
memory (uint64 data travels in int64/uint64 tensors, uint32 weights in
int32/uint32 tensors); host arrays are numpy arrays.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Optional

import numpy as np
import torch

from ._lib import Stats, KascadeError, Opts, Segment, ServerConfig, ServerStats, check, lib


class Algorithm(IntEnum):
    """kascade::Algorithm (lib/kascade/configuration.hpp:9-18)."""

    GatherChase = 0
    PointerDoubling = 1
    AsyncPointerDoubling = 2
    RMAPointerDoubling = 3
    SparseRulingSet = 4
    EulerTour = 5


class RulerSelectionStrategy(IntEnum):
    """configuration.hpp:49-57; on one GPU only the mean spacing matters."""

    dehne = 0
    heuristic = 1
    sanders = 2
    ultimate = 3
    ultimate_sanders = 4
    limit_rounds = 5


@dataclass
class GpuTuning:
    """B200 tunables (kascade_opts); 0 = autotuned default."""

    ruler_spacing: int = 0
    ruler_spacing_deep: int = 0
    max_levels: int = 0
    base_case_size: int = 0
    chains_per_thread: int = 0
    block_size: int = 0
    validate: bool = False
    profile: bool = False
    seed: int = 0
    async_: bool = False
    level0_mode: int = 0
    max_chain: int = 0

    def to_opts(self, algorithm: Algorithm = Algorithm.SparseRulingSet) -> Opts:
        o = Opts()
        lib.kascade_opts_init(ctypes.byref(o))
        o.algorithm = int(algorithm)
        o.ruler_spacing = self.ruler_spacing
        o.ruler_spacing_deep = self.ruler_spacing_deep
        o.max_levels = self.max_levels
        o.base_case_size = self.base_case_size
        o.chains_per_thread = self.chains_per_thread
        o.block_size = self.block_size
        o.validate = int(self.validate)
        o.profile = int(self.profile)
        o.seed = self.seed
        o.async_ = int(self.async_)
        o.level0_mode = self.level0_mode
        o.max_chain = self.max_chain
        return o


@dataclass
class PointerDoublingConfig:
    """configuration.hpp:39-47.  The message-layer options (grid
    communication, aggregation, owner caching, request schemes, allgather
    fallback) have no counterpart on one GPU and are accepted unchanged."""

    use_local_preprocessing: bool = True
    use_grid_communication: bool = False
    use_local_first_request_scheme: bool = True
    cache_succ_owners: bool = True
    fallback_allgather_size_ratio: float = 0.0
    gpu: GpuTuning = field(default_factory=GpuTuning)


@dataclass
class SparseRulingSetConfig:
    """configuration.hpp:65-95.  ``heuristic_factor`` (heuristic strategy) and
    ``round_limit`` (limit_rounds strategy) map to the GPU's mean ruler
    spacing; the p-dependent strategies (dehne, sanders, ultimate,
    ultimate_sanders) use the autotuned spacing; ``sparse_ruling_set_rounds``
    bounds the recursion depth when set above its default of 1; the messaging
    switches (sync, spawn, post_invert, grid communication, ...) describe MPI
    exchanges that do not exist on one GPU."""

    ruler_selection: RulerSelectionStrategy = RulerSelectionStrategy.sanders
    base_algorithm: Algorithm = Algorithm.PointerDoubling
    sparse_ruling_set_rounds: int = 1
    heuristic_factor: float = 0.01
    round_limit: int = 100
    sync: bool = True
    spawn: bool = False
    post_invert: bool = False
    use_local_contraction: bool = False
    gpu: GpuTuning = field(default_factory=GpuTuning)

    def tuning(self) -> GpuTuning:
        t = GpuTuning(**vars(self.gpu))
        if t.ruler_spacing == 0:
            if self.ruler_selection == RulerSelectionStrategy.heuristic and self.heuristic_factor > 0:
                t.ruler_spacing = max(2, int(round(1.0 / self.heuristic_factor)))
            elif self.ruler_selection == RulerSelectionStrategy.limit_rounds and self.round_limit > 0:
                t.ruler_spacing = max(2, int(self.round_limit))
        if t.max_levels == 0 and self.sparse_ruling_set_rounds > 1:
            t.max_levels = int(self.sparse_ruling_set_rounds)
        return t


@dataclass
class EulerTourConfig:
    """configuration.hpp:97-103."""

    algorithm: Algorithm = Algorithm.SparseRulingSet
    use_high_degree_handling: bool = False
    algo_config: object = None
    gpu: GpuTuning = field(default_factory=GpuTuning)


# ---------------------------------------------------------------------------
# Context
# ---------------------------------------------------------------------------
class Context:
    """A kascade_ctx: owns the device scratch arena and status word."""

    def __init__(self, device: int | None = None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = int(device)
        h = ctypes.c_void_p()
        check(lib.kascade_ctx_create(self.device, ctypes.byref(h)), "kascade_ctx_create")
        self.handle = h

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.kascade_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, nbytes: int) -> None:
        check(lib.kascade_ctx_reserve(self.handle, nbytes), "kascade_ctx_reserve", self.handle)

    def kernel_times(self) -> dict[str, tuple[float, int]]:
        cap = 64
        names = (ctypes.c_char_p * cap)()
        ms = (ctypes.c_double * cap)()
        cnt = (ctypes.c_uint64 * cap)()
        k = lib.kascade_ctx_kernel_times(self.handle, names, ms, cnt, cap)
        return {names[i].decode(): (ms[i], int(cnt[i])) for i in range(min(k, cap))}

    def reset_kernel_times(self) -> None:
        lib.kascade_ctx_reset_kernel_times(self.handle)

    def levels(self) -> list[int]:
        buf = (ctypes.c_uint64 * 32)()
        k = lib.kascade_ctx_last_levels(self.handle, buf, 32)
        return [int(buf[i]) for i in range(min(k, 32))]

    def sync(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        s = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        check(lib.kascade_ctx_sync(self.handle, s), "kascade_ctx_sync", self.handle)


_contexts: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    if device is None:
        device = torch.cuda.current_device()
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = _contexts[device] = Context(device)
    return ctx


def _ctx_for(t: torch.Tensor, ctx: Optional[Context]) -> Context:
    return ctx if ctx is not None else default_context(t.device.index)


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _dev64(t: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype not in (torch.int64, torch.uint64):
        raise TypeError(f"{name} must hold 64-bit integers, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


def _dev32(t: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype not in (torch.int32, torch.uint32):
        raise TypeError(f"{name} must hold 32-bit integers, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


# ---------------------------------------------------------------------------
# Plain forms
# ---------------------------------------------------------------------------
def rank_list(succ: torch.Tensor, weights: Optional[torch.Tensor] = None, *, tuning: Optional[GpuTuning] = None,
              algorithm: Algorithm = Algorithm.SparseRulingSet, root_out: Optional[torch.Tensor] = None,
              rank_out: Optional[torch.Tensor] = None, ctx: Optional[Context] = None):
    """Rank a forest of lists: returns (root, rank) as int64 tensors.
    rank[i] = sum of weights from i to its root, excluding the root."""
    _dev64(succ, "succ")
    n = succ.numel()
    if weights is not None:
        _dev32(weights, "weights")
        if weights.numel() != n:
            raise ValueError("weights must have one entry per element")
    root_out = root_out if root_out is not None else torch.empty(n, dtype=torch.int64, device=succ.device)
    rank_out = rank_out if rank_out is not None else torch.empty(n, dtype=torch.int64, device=succ.device)
    c = _ctx_for(succ, ctx)
    o = (tuning or GpuTuning()).to_opts(algorithm)
    st = lib.kascade_rank_list(c.handle, succ.data_ptr(), weights.data_ptr() if weights is not None else None, n,
                               root_out.data_ptr(), rank_out.data_ptr(), ctypes.byref(o), _stream(succ))
    check(st, "kascade_rank_list", c.handle)
    return root_out, rank_out


def rank_list_host(succ: np.ndarray, weights: Optional[np.ndarray] = None, *, tuning: Optional[GpuTuning] = None,
                   ctx: Optional[Context] = None):
    """Host-array form: numpy in, numpy out (copies inside the call)."""
    succ = np.ascontiguousarray(succ, dtype=np.uint64)
    n = succ.size
    if weights is not None:
        weights = np.ascontiguousarray(weights, dtype=np.uint32)
    root = np.empty(n, np.uint64)
    rank = np.empty(n, np.uint64)
    c = ctx or default_context()
    o = (tuning or GpuTuning()).to_opts()
    o.async_ = 0  # the arrays are returned: the call completes first
    st = lib.kascade_rank_list_host(c.handle, succ.ctypes.data, weights.ctypes.data if weights is not None else None,
                                    n, root.ctypes.data, rank.ctypes.data, ctypes.byref(o),
                                    torch.cuda.current_stream(c.device).cuda_stream)
    check(st, "kascade_rank_list_host", c.handle)
    return root, rank


def root_forest(parent: torch.Tensor, *, tuning: Optional[GpuTuning] = None, ctx: Optional[Context] = None,
                root_out: Optional[torch.Tensor] = None, depth_out: Optional[torch.Tensor] = None):
    """Root every vertex of a forest given as a parent array: (root, depth)."""
    _dev64(parent, "parent")
    n = parent.numel()
    root_out = root_out if root_out is not None else torch.empty(n, dtype=torch.int64, device=parent.device)
    depth_out = depth_out if depth_out is not None else torch.empty(n, dtype=torch.int64, device=parent.device)
    c = _ctx_for(parent, ctx)
    o = (tuning or GpuTuning()).to_opts()
    st = lib.kascade_root_forest(c.handle, parent.data_ptr(), n, root_out.data_ptr(), depth_out.data_ptr(),
                                 ctypes.byref(o), _stream(parent))
    check(st, "kascade_root_forest", c.handle)
    return root_out, depth_out


def root_forest_host(parent: np.ndarray, *, tuning: Optional[GpuTuning] = None, ctx: Optional[Context] = None):
    parent = np.ascontiguousarray(parent, dtype=np.uint64)
    n = parent.size
    root = np.empty(n, np.uint64)
    depth = np.empty(n, np.uint64)
    c = ctx or default_context()
    o = (tuning or GpuTuning()).to_opts()
    o.async_ = 0  # the arrays are returned: the call completes first
    st = lib.kascade_root_forest_host(c.handle, parent.ctypes.data, n, root.ctypes.data, depth.ctypes.data,
                                      ctypes.byref(o), torch.cuda.current_stream(c.device).cuda_stream)
    check(st, "kascade_root_forest_host", c.handle)
    return root, depth


# ---------------------------------------------------------------------------
# Reference-shaped in-place calls
# ---------------------------------------------------------------------------
def set_initial_ranking_state(succ_array: torch.Tensor, root_array: Optional[torch.Tensor] = None,
                              rank_array: Optional[torch.Tensor] = None, ctx: Optional[Context] = None):
    """list_ranking.hpp:47-50: root := succ, rank := 1 (0 at roots)."""
    _dev64(succ_array, "succ_array")
    n = succ_array.numel()
    root_array = root_array if root_array is not None else torch.empty(n, dtype=torch.int64, device=succ_array.device)
    rank_array = rank_array if rank_array is not None else torch.empty(n, dtype=torch.int64, device=succ_array.device)
    c = _ctx_for(succ_array, ctx)
    check(lib.kascade_set_initial_ranking_state(c.handle, succ_array.data_ptr(), root_array.data_ptr(),
                                                 rank_array.data_ptr(), n, _stream(succ_array)),
          "kascade_set_initial_ranking_state", c.handle)
    return root_array, rank_array


def _inplace(fn, where: str, opts: Optional[Opts], succ_array: torch.Tensor, rank_array: torch.Tensor,
             ctx: Optional[Context]):
    _dev64(succ_array, "succ_array")
    _dev64(rank_array, "rank_array")
    if succ_array.numel() != rank_array.numel():
        raise ValueError("succ_array and rank_array differ in length")
    c = _ctx_for(succ_array, ctx)
    args = [c.handle]
    if opts is not None:
        args.append(ctypes.byref(opts))
    args += [succ_array.data_ptr(), rank_array.data_ptr(), succ_array.numel(), _stream(succ_array)]
    check(fn(*args), where, c.handle)


def sparse_ruling_set(config: SparseRulingSetConfig, succ_array: torch.Tensor, rank_array: torch.Tensor,
                      ctx: Optional[Context] = None) -> None:
    """kascade::sparse_ruling_set (sparse_ruling_set.hpp:13-18), in place."""
    o = config.tuning().to_opts(Algorithm.SparseRulingSet)
    _inplace(lib.kascade_sparse_ruling_set, "kascade_sparse_ruling_set", o, succ_array, rank_array, ctx)


def pointer_doubling(config: PointerDoublingConfig, succ_array: torch.Tensor, rank_array: torch.Tensor,
                     ctx: Optional[Context] = None) -> None:
    """kascade::pointer_doubling (pointer_doubling.hpp:18-23), in place."""
    o = config.gpu.to_opts(Algorithm.PointerDoubling)
    _inplace(lib.kascade_pointer_doubling, "kascade_pointer_doubling", o, succ_array, rank_array, ctx)


def async_pointer_doubling(config, succ_array: torch.Tensor, rank_array: torch.Tensor,
                           ctx: Optional[Context] = None) -> None:
    """kascade::async_pointer_doubling (pointer_doubling.hpp:29-33): on one GPU
    the asynchronous message queue disappears; the jump kernel runs."""
    o = GpuTuning().to_opts(Algorithm.AsyncPointerDoubling)
    _inplace(lib.kascade_pointer_doubling, "kascade_pointer_doubling", o, succ_array, rank_array, ctx)


def rma_pointer_doubling(config, succ_array: torch.Tensor, rank_array: torch.Tensor,
                         ctx: Optional[Context] = None) -> None:
    """kascade::rma_pointer_doubling (pointer_doubling.hpp:38-43); one-sided
    windows disappear into HBM; the jump kernel runs (and, unlike the
    reference's RMA variant, zero weights are handled)."""
    o = GpuTuning().to_opts(Algorithm.RMAPointerDoubling)
    _inplace(lib.kascade_pointer_doubling, "kascade_pointer_doubling", o, succ_array, rank_array, ctx)


def rank_on_root(succ_array: torch.Tensor, rank_array: torch.Tensor, ctx: Optional[Context] = None) -> None:
    """kascade::rank_on_root (list_ranking.hpp:19-22): GatherChase contract."""
    _inplace(lib.kascade_rank_on_root, "kascade_rank_on_root", None, succ_array, rank_array, ctx)


def local_pointer_chasing(succ_array: torch.Tensor, rank_array: torch.Tensor, ctx: Optional[Context] = None) -> None:
    """kascade::local_pointer_chasing (list_ranking.hpp:24): same contract."""
    rank_on_root(succ_array, rank_array, ctx)


def is_list(succ_array: torch.Tensor, ctx: Optional[Context] = None) -> bool:
    """kascade::is_list (successor_utils.hpp:19-24)."""
    _dev64(succ_array, "succ_array")
    c = _ctx_for(succ_array, ctx)
    out = ctypes.c_int(0)
    check(lib.kascade_is_list(c.handle, succ_array.data_ptr(), succ_array.numel(), ctypes.byref(out),
                              _stream(succ_array)), "kascade_is_list", c.handle)
    return bool(out.value)


STATS_NONE, STATS_BASIC, STATS_REDUCED_EXTENSIVE, STATS_EXTENSIVE = 1, 2, 3, 4


def compute_stats(root_array: torch.Tensor, rank_array: torch.Tensor, level: int = STATS_EXTENSIVE,
                  ctx: Optional[Context] = None):
    """The bench's compute_stats (bench/detail/stats.hpp:46-49) on the device:
    (figures dict, non-trivial trees as an (k, 4) int64 array of root, size,
    max rank, rank sum ordered by root; empty below STATS_EXTENSIVE)."""
    _dev64(root_array, "root_array")
    _dev64(rank_array, "rank_array")
    n = root_array.numel()
    c = _ctx_for(root_array, ctx)
    st = Stats()
    cnt = ctypes.c_uint64(0)
    per_tree = None
    if level >= STATS_EXTENSIVE and n:
        per_tree = torch.empty((n // 2 + 1, 4), dtype=torch.int64, device=root_array.device)
    check(lib.kascade_compute_stats(c.handle, root_array.data_ptr(), rank_array.data_ptr(), n, level,
                                    ctypes.byref(st), per_tree.data_ptr() if per_tree is not None else None,
                                    per_tree.shape[0] if per_tree is not None else 0, ctypes.byref(cnt),
                                    _stream(root_array)), "kascade_compute_stats", c.handle)
    figs = {f: getattr(st, f) for f, _ in Stats._fields_}
    trees = per_tree[:cnt.value].cpu().numpy() if per_tree is not None else np.zeros((0, 4), np.int64)
    return figs, trees


def rank_via_euler_tour(config: EulerTourConfig, succ_array: torch.Tensor, rank_array: torch.Tensor,
                        ctx: Optional[Context] = None) -> None:
    """kascade::rank_via_euler_tour (eulertour.hpp:22-27), in place: parents in,
    roots and depths out for non-roots.  use_high_degree_handling selects the
    reference's proxy construction (successor_utils.cpp:302-418), which on
    one rank creates no proxy (proxies stand in for remote parents only) and
    builds the same tree, so it changes nothing here."""
    o = config.gpu.to_opts(Algorithm.SparseRulingSet)
    _inplace(lib.kascade_rank_via_euler_tour, "kascade_rank_via_euler_tour", o, succ_array, rank_array, ctx)


def compute_euler_tour(parent_array: torch.Tensor, use_high_degree_handling: bool = False,
                       ctx: Optional[Context] = None) -> torch.Tensor:
    """kascade::compute_euler_tour (eulertour.hpp:32-34): the tour's successor
    array in the reference's element numbering (one rank).  With
    use_high_degree_handling the reference builds the same tour on one rank
    (no remote parent, so no proxy vertex; successor_utils.cpp:322-339)."""
    _dev64(parent_array, "parent_array")
    n = parent_array.numel()
    out = torch.empty(max(2 * n, 1), dtype=torch.int64, device=parent_array.device)
    m = ctypes.c_uint64(0)
    c = _ctx_for(parent_array, ctx)
    check(lib.kascade_compute_euler_tour(c.handle, parent_array.data_ptr(), n, out.data_ptr(), ctypes.byref(m),
                                         _stream(parent_array)), "kascade_compute_euler_tour", c.handle)
    return out[: m.value]


def pack(succ_array: torch.Tensor, rank_array: torch.Tensor, active_indices: torch.Tensor,
         ctx: Optional[Context] = None):
    """kascade::pack (pack.hpp:23-80) on one rank: returns the packed arrays."""
    for t, nm in ((succ_array, "succ_array"), (rank_array, "rank_array"), (active_indices, "active_indices")):
        _dev64(t, nm)
    k = active_indices.numel()
    sp = torch.empty(max(k, 1), dtype=torch.int64, device=succ_array.device)
    rp = torch.empty(max(k, 1), dtype=torch.int64, device=succ_array.device)
    c = _ctx_for(succ_array, ctx)
    check(lib.kascade_pack(c.handle, succ_array.data_ptr(), rank_array.data_ptr(), succ_array.numel(),
                           active_indices.data_ptr(), k, sp.data_ptr(), rp.data_ptr(), _stream(succ_array)),
          "kascade_pack", c.handle)
    return sp[:k], rp[:k]


def unpack(succ_packed: torch.Tensor, rank_packed: torch.Tensor, succ_array: torch.Tensor, rank_array: torch.Tensor,
           active_indices: torch.Tensor, ctx: Optional[Context] = None) -> None:
    """The unpack closure of kascade::pack (pack.hpp:81-175), in place."""
    for t, nm in ((succ_packed, "succ_packed"), (rank_packed, "rank_packed"), (succ_array, "succ_array"),
                  (rank_array, "rank_array"), (active_indices, "active_indices")):
        _dev64(t, nm)
    c = _ctx_for(succ_array, ctx)
    check(lib.kascade_unpack(c.handle, succ_packed.data_ptr(), rank_packed.data_ptr(), active_indices.data_ptr(),
                             active_indices.numel(), succ_array.data_ptr(), rank_array.data_ptr(),
                             succ_array.numel(), _stream(succ_array)), "kascade_unpack", c.handle)


# ---------------------------------------------------------------------------
# Batched ranking
# ---------------------------------------------------------------------------
SEG_LIST, SEG_FOREST = 0, 1


def make_segments(sizes, kinds) -> "ctypes.Array":
    """Segment table for instances of the given sizes and kinds (SEG_LIST /
    SEG_FOREST), concatenated in order."""
    arr = (Segment * len(sizes))()
    off = 0
    for i, (sz, kd) in enumerate(zip(sizes, kinds)):
        arr[i].offset, arr[i].size, arr[i].kind, arr[i].reserved = off, int(sz), int(kd), 0
        off += int(sz)
    return arr


def rank_batch(inputs: torch.Tensor, segments, weights: Optional[torch.Tensor] = None, *,
               tuning: Optional[GpuTuning] = None, root_out: Optional[torch.Tensor] = None,
               rank_out: Optional[torch.Tensor] = None, ctx: Optional[Context] = None):
    """Rank many independent lists and forests at once (kascade_rank_batch).
    `inputs` holds every instance's successor (list) or parent (forest) array,
    concatenated, with instance-local indices; `segments` comes from
    make_segments.  Returns (root, rank_or_depth), roots instance-local."""
    _dev64(inputs, "inputs")
    n = inputs.numel()
    if weights is not None:
        _dev32(weights, "weights")
    root_out = root_out if root_out is not None else torch.empty(n, dtype=torch.int64, device=inputs.device)
    rank_out = rank_out if rank_out is not None else torch.empty(n, dtype=torch.int64, device=inputs.device)
    c = _ctx_for(inputs, ctx)
    o = (tuning or GpuTuning()).to_opts()
    check(lib.kascade_rank_batch(c.handle, segments, len(segments), inputs.data_ptr(),
                                 weights.data_ptr() if weights is not None else None, n, root_out.data_ptr(),
                                 rank_out.data_ptr(), ctypes.byref(o), _stream(inputs)), "kascade_rank_batch",
          c.handle)
    return root_out, rank_out


class BatchPlan:
    """A batch captured once as a CUDA graph and replayed
    (kascade_batch_plan_*).  The segment table and the tensors are fixed at
    creation; their contents may change between launches."""

    def __init__(self, inputs: torch.Tensor, segments, weights: Optional[torch.Tensor] = None, *,
                 root_out: Optional[torch.Tensor] = None, rank_out: Optional[torch.Tensor] = None,
                 tuning: Optional[GpuTuning] = None):
        _dev64(inputs, "inputs")
        if weights is not None:
            _dev32(weights, "weights")
        n = inputs.numel()
        self.inputs, self.weights, self.segments = inputs, weights, segments
        self.root = root_out if root_out is not None else torch.empty(n, dtype=torch.int64, device=inputs.device)
        self.rank = rank_out if rank_out is not None else torch.empty(n, dtype=torch.int64, device=inputs.device)
        o = (tuning or GpuTuning()).to_opts()
        h = ctypes.c_void_p()
        torch.cuda.synchronize(inputs.device)
        check(lib.kascade_batch_plan_create(inputs.device.index or 0, segments, len(segments), inputs.data_ptr(),
                                            weights.data_ptr() if weights is not None else None, n,
                                            self.root.data_ptr(), self.rank.data_ptr(), ctypes.byref(o),
                                            ctypes.byref(h)), "kascade_batch_plan_create")
        self.handle = h

    def launch(self):
        """Replay on the current stream; returns (root, rank)."""
        check(lib.kascade_batch_plan_launch(self.handle, _stream(self.inputs)), "kascade_batch_plan_launch")
        return self.root, self.rank

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.kascade_batch_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def set_size_classes(ctx: Context, max_sizes, spacings) -> None:
    """Install a size-class table (max instance size -> mean ruler spacing)."""
    k = len(max_sizes)
    ms = (ctypes.c_uint64 * k)(*[int(x) for x in max_sizes])
    sp = (ctypes.c_uint32 * k)(*[int(x) for x in spacings])
    check(lib.kascade_ctx_set_size_classes(ctx.handle, ms, sp, k), "kascade_ctx_set_size_classes", ctx.handle)


def get_size_classes(ctx: Context):
    ms = (ctypes.c_uint64 * 64)()
    sp = (ctypes.c_uint32 * 64)()
    k = lib.kascade_ctx_get_size_classes(ctx.handle, ms, sp, 64)
    return [int(ms[i]) for i in range(k)], [int(sp[i]) for i in range(k)]


def set_class_launch(ctx: Context, chains, blocks, single_spacing=None) -> None:
    """Per size class: chains per chase thread (1, 2, 4), chase block size
    (128, 256, 512) and, optionally, the ruler spacing of calls that rank one
    instance on their own; one entry per class of the current table."""
    k = len(chains)
    ch = (ctypes.c_uint32 * k)(*[int(x) for x in chains])
    bl = (ctypes.c_uint32 * k)(*[int(x) for x in blocks])
    ss = None if single_spacing is None else (ctypes.c_uint32 * k)(*[int(x) for x in single_spacing])
    check(lib.kascade_ctx_set_class_launch(ctx.handle, ch, bl, ss, k), "kascade_ctx_set_class_launch", ctx.handle)


def get_class_launch(ctx: Context):
    """(chains, blocks, single-call spacings) per size class."""
    ch = (ctypes.c_uint32 * 64)()
    bl = (ctypes.c_uint32 * 64)()
    ss = (ctypes.c_uint32 * 64)()
    k = lib.kascade_ctx_get_class_launch(ctx.handle, ch, bl, ss, 64)
    return [int(ch[i]) for i in range(k)], [int(bl[i]) for i in range(k)], [int(ss[i]) for i in range(k)]


def load_tuning(ctx: Context, table: dict) -> None:
    """Install an autotuner table (the dict autotune.tune returns)."""
    cls = table["classes"]
    set_size_classes(ctx, [c["max"] for c in cls], [c["spacing"] for c in cls])
    set_class_launch(ctx, [c["chains"] for c in cls], [c["block"] for c in cls],
                     [c.get("spacing_single", c["spacing"]) for c in cls])


def batch_sizes(count: int, seed: int, lo_log2: int = 6, hi_log2: int = 22, total: Optional[int] = None,
                list_share: float = 0.7):
    """Instance sizes log-uniform in [2^lo, 2^hi] (rescaled to sum to `total`
    when given, never below 2^lo) and kinds (list with probability
    list_share, else forest), from a seeded generator."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(2.0 ** rng.uniform(lo_log2, hi_log2, count)).astype(np.int64)
    if total:
        sizes = np.maximum((sizes * (total / sizes.sum())).astype(np.int64), 1 << lo_log2)
    kinds = np.where(rng.random(count) < list_share, SEG_LIST, SEG_FOREST)
    return sizes, kinds


def gen_batch(sizes, kinds, seed: int, device=None, wbits: int = 16):
    """Concatenated seeded instances: lists in random order, forests of
    random recursive trees (one tree per 2^16 vertices, at least one); plus
    uint32 weights for the whole array."""
    total = int(np.sum(sizes))
    dev = device or "cuda"
    out = torch.empty(total, dtype=torch.int64, device=dev)
    off = 0
    for i, (sz, kd) in enumerate(zip(sizes, kinds)):
        sz = int(sz)
        part = out[off:off + sz]
        if kd == SEG_LIST:
            gen_list(sz, seed + 7919 * i, LAYOUT_RANDOM, out=part)
        else:
            gen_forest(sz, seed + 7919 * i, FOREST_RRT, max(1, sz >> 16), 0, out=part)
        off += sz
    w = gen_weights(total, seed ^ 0x5A5A, wbits, device=dev)
    return out, w


# ---------------------------------------------------------------------------
# Serving
# ---------------------------------------------------------------------------
class _DevView:
    """A device array described by __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<u8", "data": (ptr, False), "version": 3}


class Server:
    """The library's request loop (kascade_server_*): admission by HBM
    footprint, device-resident inputs and results, two lanes of continuous
    batching.  kind: SEG_LIST (successors, optional uint32 weights) or
    SEG_FOREST (parents)."""

    def __init__(self, device: int = 0, hbm_budget: int = 40 << 30, small_max: int = 1 << 20,
                 small_batch_elements: int = 1 << 23, max_batch_elements: int = 1 << 27,
                 max_batch_requests: int = 4096, latency_sms: int = 32, small_reserve_pct: int = 10):
        cfg = ServerConfig()
        lib.kascade_server_config_init(ctypes.byref(cfg))
        cfg.device = device
        cfg.hbm_budget_bytes = hbm_budget
        cfg.small_max = small_max
        cfg.small_batch_elements = small_batch_elements
        cfg.max_batch_elements = max_batch_elements
        cfg.max_batch_requests = max_batch_requests
        cfg.latency_sms = latency_sms
        cfg.small_reserve_pct = small_reserve_pct
        h = ctypes.c_void_p()
        check(lib.kascade_server_create(ctypes.byref(cfg), ctypes.byref(h)), "kascade_server_create")
        self.handle = h
        self.device = device
        self._n: dict[int, int] = {}
        self._viewed: set[int] = set()

    def submit(self, kind: int, inp, weights=None) -> int:
        rid = ctypes.c_uint64(0)
        if isinstance(inp, torch.Tensor):
            _dev64(inp, "input")
            w = weights
            if w is not None:
                _dev32(w, "weights")
            st = lib.kascade_server_submit_device(self.handle, kind, inp.data_ptr(),
                                                  w.data_ptr() if w is not None else None, inp.numel(),
                                                  ctypes.byref(rid))
            n = inp.numel()
        else:
            a = np.ascontiguousarray(inp, dtype=np.uint64)
            w = None if weights is None else np.ascontiguousarray(weights, dtype=np.uint32)
            st = lib.kascade_server_submit(self.handle, kind, a.ctypes.data, w.ctypes.data if w is not None else None,
                                           a.size, ctypes.byref(rid))
            n = a.size
        check(st, "kascade_server_submit")
        self._n[rid.value] = n
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> None:
        check(lib.kascade_server_wait(self.handle, rid, timeout), "kascade_server_wait")

    def fetch(self, rid: int):
        n = self._n[rid]
        root = np.empty(n, np.uint64)
        rank = np.empty(n, np.uint64)
        check(lib.kascade_server_fetch(self.handle, rid, root.ctypes.data, rank.ctypes.data), "kascade_server_fetch")
        return root, rank

    def result_device(self, rid: int):
        """(root, rank) as CUDA tensors viewing the server's result buffers
        (valid until release)."""
        r, k = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib.kascade_server_result_device(self.handle, rid, ctypes.byref(r), ctypes.byref(k)),
              "kascade_server_result_device")
        n = self._n[rid]
        dev = f"cuda:{self.device}"
        self._viewed.add(rid)
        return (torch.as_tensor(_DevView(r.value or 0, n), device=dev),
                torch.as_tensor(_DevView(k.value or 0, n), device=dev))

    def release(self, rid: int) -> None:
        """Drop a completed request.  Its result memory is reused by later
        batches at once, so work queued on the views from result_device must
        finish first: the current stream is synchronised for such requests."""
        if rid in self._viewed:
            torch.cuda.current_stream(self.device).synchronize()
            self._viewed.discard(rid)
        check(lib.kascade_server_release(self.handle, rid), "kascade_server_release")
        self._n.pop(rid, None)

    def stats(self) -> dict:
        st = ServerStats()
        check(lib.kascade_server_get_stats(self.handle, ctypes.byref(st)), "kascade_server_get_stats")
        out = {}
        for f, _ in ServerStats._fields_:
            v = getattr(st, f)
            out[f] = list(v) if isinstance(v, ctypes.Array) else v
        return out

    def reset_stats(self) -> None:
        check(lib.kascade_server_reset_stats(self.handle), "kascade_server_reset_stats")

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.kascade_server_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Seeded inputs
# ---------------------------------------------------------------------------
LAYOUT_RANDOM, LAYOUT_RUNS, LAYOUT_IDENTITY = 0, 1, 2
FOREST_RRT, FOREST_CATERPILLAR = 0, 1


def gen_list(n: int, seed: int, layout: int = LAYOUT_RANDOM, device=None, out=None) -> torch.Tensor:
    out = out if out is not None else torch.empty(n, dtype=torch.int64, device=device or "cuda")
    check(lib.kascade_gen_list(n, seed, layout, out.data_ptr(), _stream(out)), "kascade_gen_list")
    return out


def gen_weights(n: int, seed: int, wbits: int = 16, device=None, out=None) -> torch.Tensor:
    out = out if out is not None else torch.empty(n, dtype=torch.int32, device=device or "cuda")
    check(lib.kascade_gen_weights(n, seed, wbits, out.data_ptr(), _stream(out)), "kascade_gen_weights")
    return out


def gen_forest(n: int, seed: int, kind: int = FOREST_RRT, blocks: int = 64, spine: int = 0, device=None,
               out=None) -> torch.Tensor:
    out = out if out is not None else torch.empty(n, dtype=torch.int64, device=device or "cuda")
    check(lib.kascade_gen_forest(n, seed, kind, blocks, spine, out.data_ptr(), _stream(out)), "kascade_gen_forest")
    return out


# ---------------------------------------------------------------------------
# Plug-in shaped like the reference bench's AbstractAlgorithm
# (bench/detail/algorithm.hpp:7-20): ingest / run / get_rank_array /
# get_root_array.
# ---------------------------------------------------------------------------
class B200Ranking:
    """Ranks on the GPU; arrays are numpy on the host like the reference's
    std::vector members.  algorithm: any Algorithm; EulerTour treats the
    ingested array as a parent array."""

    def __init__(self, algorithm: Algorithm = Algorithm.SparseRulingSet, tuning: Optional[GpuTuning] = None,
                 device: int | None = None):
        self.algorithm = Algorithm(algorithm)
        self.tuning = tuning or GpuTuning()
        self.device = torch.cuda.current_device() if device is None else device
        self._succ: Optional[torch.Tensor] = None
        self._rank = np.empty(0, np.int64)
        self._root = np.empty(0, np.uint64)

    def ingest(self, succ_array) -> None:
        a = np.ascontiguousarray(succ_array, dtype=np.uint64)
        self._succ = torch.from_numpy(a.view(np.int64)).to(f"cuda:{self.device}")

    def run(self) -> None:
        assert self._succ is not None, "ingest() first"
        root, rank = set_initial_ranking_state(self._succ)
        if self.algorithm == Algorithm.EulerTour:
            rank_via_euler_tour(EulerTourConfig(gpu=self.tuning), root, rank)
        elif self.algorithm == Algorithm.SparseRulingSet:
            sparse_ruling_set(SparseRulingSetConfig(gpu=self.tuning), root, rank)
        else:
            o = self.tuning.to_opts(self.algorithm)
            _inplace(lib.kascade_pointer_doubling, "kascade_pointer_doubling", o, root, rank, None)
        self._root = root.cpu().numpy().view(np.uint64)
        self._rank = rank.cpu().numpy()

    def get_rank_array(self) -> np.ndarray:
        return self._rank

    def get_root_array(self) -> np.ndarray:
        return self._root
