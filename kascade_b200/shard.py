"""Sharded list ranking: one list spread over several GPUs by index ranges.

The reference ranks a list distributed over MPI ranks by contiguous index
ranges (``Distribution``, lib/kascade/distribution.hpp:16-113) with the
sparse ruling set's synchronous ruler chase: rounds of one all-to-all
exchange of ruler messages (sparse_ruling_set_detail/ruler_chasing_engine.hpp:
57-101).  Here every process owns one GPU and one shard; the shard's work runs
in the library's kernels (``kascade_shard_*``) and the rounds, exchanges and
gathers go over ``torch.distributed`` (NCCL over NVLink):

  1. every shard builds its records and samples rulers (roots included);
     global ruler ids follow from every shard's count (an all-gather)
  2. chase rounds: chains walk while their element is local, and leave the
     shard as 16 B messages (target, ruler, distance); one all-to-all per
     round, until no shard sends (an all-reduce)
  3. unreached elements (list heads ahead of their first ruler) become
     rulers, as the reference's fixup_unreached does, and are chased
  4. every shard gathers all chain ends (one per ruler) and the rulers'
     elements, and ranks the ruler sub-list on its own GPU
  5. every shard writes its elements' roots (global indices) and ranks

Every rank takes the same collective steps in the same order; an error on any
shard (an index out of range, a second predecessor, a rootless cycle) is
shared by an all-reduce before anyone raises, so no rank is left waiting.

``rank_list_sharded`` is the call for one process per GPU.
``rank_list_sharded_local`` runs several shards in one process (one device,
shard after shard, the exchanges done in memory): the same protocol and
kernels, without a second GPU.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Generator, Optional, Sequence

import torch

from . import _lib
from ._lib import KascadeError, ShardDesc, check, lib

STATUS_CYCLE = 3
DEFAULT_SPACING = 16


class Distribution:
    """Index ranges of the shards, as the reference's Distribution
    (lib/kascade/distribution.hpp:16-113): shard s owns global indices
    [offsets[s], offsets[s + 1]), built from every shard's local size."""

    def __init__(self, local_sizes: Sequence[int]):
        self.offsets = [0]
        for k in local_sizes:
            self.offsets.append(self.offsets[-1] + int(k))

    def get_owner(self, idx: int) -> int:
        import bisect

        if not 0 <= idx < self.get_global_size():
            raise IndexError(idx)
        return bisect.bisect_right(self.offsets, idx) - 1

    def counts(self) -> list[int]:
        return [b - a for a, b in zip(self.offsets, self.offsets[1:])]

    def index_range_begin(self, rank: int) -> int:
        return self.offsets[rank]

    def index_range_end(self, rank: int) -> int:
        return self.offsets[rank + 1]

    def is_local(self, idx: int, rank: int) -> bool:
        return self.offsets[rank] <= idx < self.offsets[rank + 1]

    def get_local_idx(self, idx: int, rank: int) -> int:
        return idx - self.offsets[rank]

    def get_global_idx(self, idx: int, rank: int) -> int:
        return idx + self.offsets[rank]

    def get_global_size(self) -> int:
        return self.offsets[-1]

    def get_local_size(self, rank: int) -> int:
        return self.offsets[rank + 1] - self.offsets[rank]


class CudaShardOps:
    """One shard's device work, through the library's kascade_shard_* calls.
    Buffers are CUDA tensors on `device`; every call returns once complete."""

    def __init__(self, device, ctx=None):
        from .api import Context

        self.device = torch.device(device)
        self.ctx = ctx or Context(self.device.index or 0)
        self.stream = torch.cuda.current_stream(self.device)
        self.desc = ShardDesc()
        self._regions = self._send = None
        self.num_ends = ctypes.c_uint64(0)

    def _s(self):
        return self.stream.cuda_stream

    def _empty(self, *shape, dtype=torch.int64):
        return torch.empty(*shape, dtype=dtype, device=self.device)

    def setup(self, me: int, offsets: list[int], succ: torch.Tensor, weights: Optional[torch.Tensor]) -> None:
        self.me = me
        self.succ, self.weights = succ, weights
        self.n_local = succ.numel()
        self.offsets_t = torch.tensor(offsets, dtype=torch.int64, device=self.device)
        d = self.desc
        d.lo, d.n_local, d.n_global = offsets[me], self.n_local, offsets[-1]
        d.num_shards, d.self = len(offsets) - 1, me
        d.offsets = self.offsets_t.data_ptr()
        self.rec = self._empty(max(self.n_local, 1), 2)
        self.ruler_elem = self._empty(max(self.n_local, 1), dtype=torch.int32)
        self.ends = self._empty(2 * self.n_local + 2, 2)

    def prepare(self, spacing: int, seed: int) -> tuple[int, int]:
        r = ctypes.c_uint64(0)
        w = self.weights.data_ptr() if self.weights is not None else None
        st = lib.kascade_shard_prepare(self.ctx.handle, ctypes.byref(self.desc), self.succ.data_ptr(), w,
                                       self.desc.n_global, spacing, seed, self.rec.data_ptr(),
                                       self.ruler_elem.data_ptr(), ctypes.byref(r), self._s())
        return int(r.value), st

    def set_ruler_ids(self, ruler_base: int, num_sampled: int, fixup_base: int) -> None:
        self.desc.ruler_base, self.desc.num_sampled, self.desc.fixup_base = ruler_base, num_sampled, fixup_base

    def chase(self, first: int, count: int, incoming: Optional[torch.Tensor]) -> tuple[torch.Tensor, list[int], int]:
        n_in = 0 if incoming is None else incoming.shape[0]
        work = count + n_in
        P = self.desc.num_shards
        cap = max(work, 1)
        if self._regions is None or self._regions.shape[0] < P * cap:
            self._regions = self._empty(P * cap, 2)
            self._send = self._empty(cap, 2)
        if self._send.shape[0] < cap:
            self._send = self._empty(cap, 2)
        counts = (ctypes.c_uint64 * P)()
        starts = self.ruler_elem.data_ptr() + 4 * first if count else None
        inc = incoming.contiguous() if n_in else None
        st = lib.kascade_shard_chase(self.ctx.handle, ctypes.byref(self.desc), self.rec.data_ptr(), starts, count,
                                     inc.data_ptr() if n_in else None, n_in, self._regions.data_ptr(), cap,
                                     self._send.data_ptr(), counts, self.ends.data_ptr(), ctypes.byref(self.num_ends),
                                     self.ends.shape[0], self._s())
        cnt = [int(counts[d]) for d in range(P)]
        return self._send[:sum(cnt)], cnt, st

    def unreached(self, first_lid: int) -> tuple[int, int]:
        u = ctypes.c_uint64(0)
        st = lib.kascade_shard_unreached(self.ctx.handle, ctypes.byref(self.desc), self.rec.data_ptr(),
                                         self.ruler_elem.data_ptr(), first_lid, ctypes.byref(u), self._s())
        return int(u.value), st

    def ruler_globals(self, first: int, count: int) -> torch.Tensor:
        out = self._empty(max(count, 1), 1)
        check(lib.kascade_shard_ruler_globals(self.ctx.handle, self.ruler_elem.data_ptr(), self.desc.lo, first,
                                              count, out.data_ptr(), self._s()), "kascade_shard_ruler_globals",
              self.ctx.handle)
        return out[:count]

    def chain_ends(self) -> torch.Tensor:
        return self.ends[:int(self.num_ends.value)]

    def rank_sublist(self, ends: torch.Tensor, num_rulers: int) -> tuple[torch.Tensor, torch.Tensor, int]:
        succ2 = self._empty(max(num_rulers, 1))
        w2 = self._empty(max(num_rulers, 1))
        e = ends.contiguous()
        st = lib.kascade_shard_sublist(self.ctx.handle, e.data_ptr() if e.numel() else None, e.shape[0], num_rulers,
                                       succ2.data_ptr(), w2.data_ptr(), self._s())
        if st == 0 and num_rulers:
            st = lib.kascade_sparse_ruling_set(self.ctx.handle, None, succ2.data_ptr(), w2.data_ptr(), num_rulers,
                                               self._s())
        return succ2, w2, st

    def propagate(self, sub_root, sub_rank, elem_of, num_rulers) -> tuple[torch.Tensor, torch.Tensor, int]:
        root = self._empty(self.n_local)
        rank = self._empty(self.n_local)
        st = lib.kascade_shard_propagate(self.ctx.handle, ctypes.byref(self.desc), self.rec.data_ptr(),
                                         sub_root.data_ptr(), sub_rank.data_ptr(), elem_of.data_ptr(), num_rulers,
                                         root.data_ptr(), rank.data_ptr(), self._s())
        return root, rank, st


# ---------------------------------------------------------------------------
# The protocol of one shard, as a generator of collective requests:
#   ("allgather", int)          -> list of every shard's int
#   ("max", [ints])             -> element-wise maximum over shards
#   ("alltoallv", rows, counts) -> the rows every shard sent here, by shard
#   ("allgather_rows", rows)    -> every shard's rows, concatenated by shard
# `rows` are int64 tensors of shape (k, w).
# ---------------------------------------------------------------------------
def _shard_protocol(ops, me: int, succ: torch.Tensor, weights: Optional[torch.Tensor], spacing: int,
                    seed: int) -> Generator:
    def agree(err: int):
        # every shard learns of an error before anyone raises
        e = (yield ("max", [err]))[0]
        if e:
            raise KascadeError(e, f"sharded ranking (shard {me})")

    counts = yield ("allgather", succ.numel())
    dist = Distribution(counts)
    if dist.get_global_size() > 0xFFFFFFFE:
        yield from agree(8)  # KASCADE_ERR_TOO_LARGE
    ops.setup(me, dist.offsets, succ, weights)
    r, err = ops.prepare(spacing, seed)
    yield from agree(err)
    rs = yield ("allgather", r)
    R0 = sum(rs)
    ops.set_ruler_ids(sum(rs[:me]), r, 0)

    def chase_rounds(first: int, count: int):
        send, cnt, err = ops.chase(first, count, None)
        rounds = 0
        while True:
            pending, e = yield ("max", [int(sum(cnt) > 0), err])
            if e:
                raise KascadeError(e, f"sharded ranking (shard {me}), chase round {rounds}")
            if not pending:
                return rounds
            if rounds > dist.get_global_size() + 2:  # the same decision on every shard
                raise KascadeError(STATUS_CYCLE, f"sharded ranking (shard {me}): rounds exhausted")
            recv = yield ("alltoallv", send, cnt)
            send, cnt, err = ops.chase(0, 0, recv)
            rounds += 1

    rounds = yield from chase_rounds(0, r)
    u, err = ops.unreached(r)
    yield from agree(err)
    us = yield ("allgather", u)
    F = sum(us)
    ops.set_ruler_ids(sum(rs[:me]), r, R0 + sum(us[:me]))
    if F:
        rounds += yield from chase_rounds(r, u)
    R = R0 + F
    ends = yield ("allgather_rows", ops.chain_ends())
    sampled = yield ("allgather_rows", ops.ruler_globals(0, r))
    fixup = yield ("allgather_rows", ops.ruler_globals(r, u))
    elem_of = torch.cat([sampled.reshape(-1), fixup.reshape(-1)])
    sub_root, sub_rank, err = ops.rank_sublist(ends, R)
    yield from agree(err)
    root, rank, err = ops.propagate(sub_root, sub_rank, elem_of, R)
    yield from agree(err)
    return root, rank, {"rounds": rounds, "rulers": R, "fixup_rulers": F, "offsets": dist.offsets}


def _run_lockstep(gens: list) -> list:
    """Drive several shards' protocols in one process: each collective is
    fulfilled once every shard has asked for it."""
    P = len(gens)
    replies = [None] * P
    done = [None] * P
    while True:
        reqs = []
        for s in range(P):
            try:
                reqs.append(gens[s].send(replies[s]))
            except StopIteration as stop:
                done[s] = stop.value
                reqs.append(None)
        if all(d is not None for d in done):
            return done
        if any(q is None for q in reqs):
            raise RuntimeError("shards left the protocol at different steps")
        kind = reqs[0][0]
        if any(q[0] != kind for q in reqs):
            raise RuntimeError("shards asked for different collectives")
        if kind == "allgather":
            vals = [int(q[1]) for q in reqs]
            replies = [list(vals) for _ in range(P)]
        elif kind == "max":
            m = [max(int(q[1][i]) for q in reqs) for i in range(len(reqs[0][1]))]
            replies = [list(m) for _ in range(P)]
        elif kind == "alltoallv":
            parts = []
            for q in reqs:
                rows, cnt = q[1], q[2]
                offs = [0]
                for c in cnt:
                    offs.append(offs[-1] + c)
                parts.append([rows[offs[d]:offs[d + 1]] for d in range(P)])
            replies = [torch.cat([parts[s][d] for s in range(P)]) for d in range(P)]
        elif kind == "allgather_rows":
            allr = torch.cat([q[1] for q in reqs])
            replies = [allr for _ in range(P)]
        else:
            raise RuntimeError(f"unknown collective {kind}")


def _run_distributed(gen, group=None):
    """Drive this process's shard over torch.distributed (NCCL for CUDA
    tensors, gloo for CPU tensors); every rank takes the same steps."""
    import torch.distributed as dist

    P = dist.get_world_size(group)
    reply = None
    dev = None
    while True:
        try:
            req = gen.send(reply)
        except StopIteration as stop:
            return stop.value
        kind = req[0]
        if dev is None:
            dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else \
                torch.device("cpu")
        if kind == "allgather":
            t = torch.tensor([int(req[1])], dtype=torch.int64, device=dev)
            out = [torch.empty_like(t) for _ in range(P)]
            dist.all_gather(out, t, group=group)
            reply = [int(x.item()) for x in out]
        elif kind == "max":
            t = torch.tensor([int(v) for v in req[1]], dtype=torch.int64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
            reply = [int(v) for v in t.tolist()]
        elif kind == "alltoallv":
            rows, cnt = req[1], req[2]
            width = rows.shape[1] if rows.dim() == 2 else 2
            send_counts = torch.tensor(cnt, dtype=torch.int64, device=dev)
            recv_counts = torch.empty_like(send_counts)
            dist.all_to_all_single(recv_counts, send_counts, group=group)
            rc = [int(x) for x in recv_counts.tolist()]
            recv = torch.empty((sum(rc), width), dtype=torch.int64, device=rows.device)
            dist.all_to_all_single(recv, rows.reshape(-1, width).contiguous(), output_split_sizes=rc,
                                   input_split_sizes=list(cnt), group=group)
            reply = recv
        elif kind == "allgather_rows":
            rows = req[1]
            width = rows.shape[1]
            k = torch.tensor([rows.shape[0]], dtype=torch.int64, device=dev)
            ks = [torch.empty_like(k) for _ in range(P)]
            dist.all_gather(ks, k, group=group)
            ks = [int(x.item()) for x in ks]
            m = max(ks + [1])
            pad = torch.zeros((m, width), dtype=torch.int64, device=rows.device)
            pad[:rows.shape[0]] = rows
            out = [torch.empty_like(pad) for _ in range(P)]
            dist.all_gather(out, pad, group=group)
            reply = torch.cat([o[:c] for o, c in zip(out, ks)])
        else:
            raise RuntimeError(f"unknown collective {kind}")


def rank_list_sharded(succ: torch.Tensor, weights: Optional[torch.Tensor] = None, *, group=None, ctx=None,
                      spacing: int = DEFAULT_SPACING, seed: int = 0x5EED, ops=None):
    """Rank one list whose elements are spread over the processes of `group`
    (one GPU each, torch.distributed with NCCL): this process holds the
    shard's successors (global indices, int64 CUDA tensor) and optional
    uint32 weights; shards are ordered by rank.  Returns this shard's (root,
    rank) -- roots as global indices, ranks with 0 at roots -- and a dict
    with the rounds and ruler counts.  Collective: every rank must call it."""
    import torch.distributed as dist

    me = dist.get_rank(group)
    ops = ops or CudaShardOps(succ.device, ctx)
    root, rank, info = _run_distributed(_shard_protocol(ops, me, succ, weights, spacing, seed), group)
    return root, rank, info


def rank_list_sharded_local(shards: Sequence[tuple], *, ctx=None, spacing: int = DEFAULT_SPACING,
                            seed: int = 0x5EED, ops_factory: Optional[Callable] = None):
    """The sharded protocol with every shard in this process: `shards` is a
    list of (succ, weights) per shard, in index-range order.  Returns
    [(root, rank, info)] per shard."""
    if ops_factory is None:
        def ops_factory(i, succ):
            return CudaShardOps(succ.device, ctx)
    gens = [_shard_protocol(ops_factory(i, s), i, s, w, spacing, seed) for i, (s, w) in enumerate(shards)]
    return _run_lockstep(gens)


__all__ = ["Distribution", "CudaShardOps", "rank_list_sharded", "rank_list_sharded_local"]
_ = _lib  # the binding module (keeps the import for the ctypes declarations)
