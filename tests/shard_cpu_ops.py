"""A CPU stand-in for one shard's device work in the sharded ranking protocol
(kascade_b200/shard.py): the same operations as CudaShardOps, written in
numpy on CPU tensors, so that the protocol -- routing, rounds, termination,
fix-up rulers, the gathered sub-list -- runs on gloo ranks without a GPU.
Test infrastructure only: the sub-list is ranked by the oracle."""
from __future__ import annotations

import numpy as np
import torch

import oracle

UNREACHED = -1
NOT_A_LIST, OUT_OF_RANGE, CYCLE = 4, 2, 3


def _sampled(g: np.ndarray, spacing: int, seed: int) -> np.ndarray:
    h = (g.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)) >> np.uint64(40)
    return (h % np.uint64(max(spacing, 2))) == 0


class CpuShardOps:
    def setup(self, me, offsets, succ, weights):
        self.me, self.offsets = me, list(offsets)
        self.lo, self.hi = offsets[me], offsets[me + 1]
        self.n = self.hi - self.lo
        self.P = len(offsets) - 1
        self.succ = succ.numpy().view(np.uint64).astype(np.int64)
        self.w = (weights.numpy().view(np.uint32).astype(np.int64) if weights is not None
                  else np.ones(self.n, np.int64))
        self.tag = np.full(self.n, UNREACHED, np.int64)   # ruler local id, or -1
        self.stamp = np.full(self.n, UNREACHED, np.int64)  # ruler global id of a reached element
        self.dist = np.zeros(self.n, np.int64)
        self.ruler_elem = []
        self.ends = []

    def prepare(self, spacing, seed):
        g = np.arange(self.lo, self.hi, dtype=np.int64)
        if np.any((self.succ < 0) | (self.succ >= self.offsets[-1])):
            return 0, OUT_OF_RANGE
        root = self.succ == g
        self.w[root] = 0
        rul = np.flatnonzero(root | _sampled(g, spacing, seed))
        self.tag[rul] = np.arange(rul.size)
        self.ruler_elem = list(rul)
        return int(rul.size), 0

    def set_ruler_ids(self, ruler_base, num_sampled, fixup_base):
        self.rb, self.ns, self.fb = ruler_base, num_sampled, fixup_base

    def gid(self, lid):
        return self.rb + lid if lid < self.ns else self.fb + (lid - self.ns)

    def owner(self, g):
        return int(np.searchsorted(self.offsets, g, side="right") - 1)

    def chase(self, first, count, incoming):
        work = []
        for lid in range(first, first + count):
            x = self.ruler_elem[lid]
            if self.succ[x] == self.lo + x:
                self.ends.append((self.gid(lid), self.gid(lid), 0))
                continue
            work.append((int(self.succ[x]), self.gid(lid), int(self.w[x])))
        if incoming is not None:
            raw = incoming.numpy().reshape(-1, 2)
            for row in raw:
                t = int(row[0] & 0xFFFFFFFF)
                r = int((row[0] >> 32) & 0xFFFFFFFF)
                work.append((t, r, int(row[1])))
        out = [[] for _ in range(self.P)]
        err = 0
        for cur, ruler, d in work:
            hops = 0
            while True:
                if not self.lo <= cur < self.hi:
                    out[self.owner(cur)].append((cur, ruler, d))
                    break
                x = cur - self.lo
                if self.tag[x] >= 0:
                    self.ends.append((ruler, self.gid(int(self.tag[x])), d))
                    break
                if self.stamp[x] >= 0 or hops > self.n:
                    err = NOT_A_LIST
                    break
                self.stamp[x], self.dist[x] = ruler, d
                d += int(self.w[x])
                cur = int(self.succ[x])
                hops += 1
        counts = [len(o) for o in out]
        rows = [((t | (r << 32)), d) for o in out for (t, r, d) in o]
        send = torch.tensor(rows, dtype=torch.int64).reshape(-1, 2)
        return send, counts, err

    def unreached(self, first_lid):
        u = np.flatnonzero((self.tag < 0) & (self.stamp < 0))
        self.tag[u] = first_lid + np.arange(u.size)
        self.ruler_elem += list(u)
        return int(u.size), 0

    def ruler_globals(self, first, count):
        return torch.tensor([self.lo + int(x) for x in self.ruler_elem[first:first + count]],
                            dtype=torch.int64).reshape(-1, 1)

    def chain_ends(self):
        rows = [((r | (nx << 32)), d) for (r, nx, d) in self.ends]
        return torch.tensor(rows, dtype=torch.int64).reshape(-1, 2)

    def rank_sublist(self, ends, num_rulers):
        e = ends.numpy().reshape(-1, 2)
        if e.shape[0] != num_rulers:
            return None, None, CYCLE if e.shape[0] < num_rulers else NOT_A_LIST
        succ2 = np.full(num_rulers, -1, np.int64)
        w2 = np.zeros(num_rulers, np.int64)
        r = (e[:, 0] & 0xFFFFFFFF).astype(np.int64)
        nx = ((e[:, 0] >> 32) & 0xFFFFFFFF).astype(np.int64)
        succ2[r] = nx
        w2[r] = e[:, 1]
        if np.any(succ2 < 0):
            return None, None, CYCLE
        s, k = succ2.astype(np.uint64), w2.copy()
        try:
            oracle.local_pointer_chasing(s, k)
        except ValueError:
            return None, None, CYCLE
        si = s.astype(np.int64)
        if np.any(si[si] != si):  # a rootless cycle no leaf leads into
            return None, None, CYCLE
        return si, k, 0

    def propagate(self, sub_root, sub_rank, elem_of, num_rulers):
        elem = elem_of.numpy().astype(np.int64)
        root = np.empty(self.n, np.int64)
        rank = np.empty(self.n, np.int64)
        for x in range(self.n):
            if self.tag[x] >= 0:
                g, d = self.gid(int(self.tag[x])), 0
            elif self.stamp[x] >= 0:
                g, d = int(self.stamp[x]), int(self.dist[x])
            else:
                return None, None, CYCLE
            root[x] = elem[sub_root[g]]
            rank[x] = sub_rank[g] - d
        return torch.from_numpy(root), torch.from_numpy(rank), 0
