"""ctypes wrappers around the oracle shared libraries (test infrastructure)."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libkascade_oracle.so"
REF_SO = HERE / "_ref" / "libkascade_ref.so"

__all__ = [
    "compute_stats", "compute_stats_transcribed", "euler_tour_transcribed",
    "build", "has_ref", "rank_list", "root_forest", "local_pointer_chasing", "pointer_doubling",
    "euler_tour", "rank_via_euler_tour", "is_list", "pack", "unpack", "gen_list", "gen_weights",
    "gen_forest", "ref_gather_rank", "ref_local_pointer_chasing",
    "cpu_threads", "cpu_sparse_ruling_set", "cpu_pointer_doubling", "cpu_gen_list", "cpu_gen_weights",
    "cpu_gen_forest",
]


def build() -> None:
    """Build the oracle (and oracle/_ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


_lib = None
_ref = None


def _o():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        _lib = ctypes.CDLL(str(ORACLE_SO))
    return _lib


def has_ref() -> bool:
    return REF_SO.exists()


def _r():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (reference source tree absent)")
        _ref = ctypes.CDLL(str(REF_SO))
    return _ref


def _p(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


U64 = ctypes.c_uint64
U32 = ctypes.c_uint32


def rank_list(succ: np.ndarray, weights: np.ndarray | None = None):
    succ = np.ascontiguousarray(succ, np.uint64)
    w = None if weights is None else np.ascontiguousarray(weights, np.uint32)
    root = np.empty_like(succ)
    rank = np.empty(succ.size, np.uint64)
    rc = _o().oracle_rank_list(_p(succ), _p(w), U64(succ.size), _p(root), _p(rank))
    if rc != 0:
        raise ValueError("oracle: cycle without a root")
    return root, rank


def root_forest(parent: np.ndarray):
    parent = np.ascontiguousarray(parent, np.uint64)
    root = np.empty_like(parent)
    depth = np.empty(parent.size, np.uint64)
    rc = _o().oracle_root_forest(_p(parent), U64(parent.size), _p(root), _p(depth))
    if rc != 0:
        raise ValueError("oracle: cycle without a root")
    return root, depth


def local_pointer_chasing(succ: np.ndarray, rank: np.ndarray) -> None:
    assert succ.dtype == np.uint64 and rank.dtype == np.int64
    if _o().oracle_local_pointer_chasing(_p(succ), _p(rank), U64(succ.size)) != 0:
        raise ValueError("oracle: cycle without a root")


def pointer_doubling(succ: np.ndarray, rank: np.ndarray) -> int:
    assert succ.dtype == np.uint64 and rank.dtype == np.int64
    return _o().oracle_pointer_doubling(_p(succ), _p(rank), U64(succ.size))


def euler_tour(parent: np.ndarray):
    """The reference-numbered tour: (succ, weight, src, dst, is_up)."""
    parent = np.ascontiguousarray(parent, np.uint64)
    n = parent.size
    lib = _o()
    lib.oracle_euler_tour_size.restype = ctypes.c_uint64
    m = int(lib.oracle_euler_tour_size(_p(parent), U64(n)))
    ts = np.empty(max(m, 1), np.uint64)
    tw = np.empty(max(m, 1), np.int64)
    es = np.empty(max(m, 1), np.uint64)
    ed = np.empty(max(m, 1), np.uint64)
    up = np.empty(max(m, 1), np.uint8)
    lib.oracle_euler_tour(_p(parent), U64(n), _p(ts), _p(tw), _p(es), _p(ed), _p(up))
    return ts[:m], tw[:m], es[:m], ed[:m], up[:m].astype(bool)


def rank_via_euler_tour(succ: np.ndarray, rank: np.ndarray) -> None:
    assert succ.dtype == np.uint64 and rank.dtype == np.int64
    if _o().oracle_rank_via_euler_tour(_p(succ), _p(rank), U64(succ.size)) != 0:
        raise ValueError("oracle: cycle without a root")


def is_list(succ: np.ndarray) -> bool:
    succ = np.ascontiguousarray(succ, np.uint64)
    return bool(_o().oracle_is_list(_p(succ), U64(succ.size)))


def pack(succ: np.ndarray, rank: np.ndarray, active: np.ndarray):
    succ = np.ascontiguousarray(succ, np.uint64)
    rank = np.ascontiguousarray(rank, np.int64)
    active = np.ascontiguousarray(active, np.uint64)
    sp = np.empty(active.size, np.uint64)
    rp = np.empty(active.size, np.int64)
    rc = _o().oracle_pack(_p(succ), _p(rank), U64(succ.size), _p(active), U64(active.size), _p(sp), _p(rp))
    if rc != 0:
        raise ValueError("oracle: an active element's successor is not active")
    return sp, rp


def unpack(sp: np.ndarray, rp: np.ndarray, active: np.ndarray, succ: np.ndarray, rank: np.ndarray) -> None:
    assert succ.dtype == np.uint64 and rank.dtype == np.int64
    sp = np.ascontiguousarray(sp, np.uint64)  # keep the converted arrays alive
    rp = np.ascontiguousarray(rp, np.int64)
    active = np.ascontiguousarray(active, np.uint64)
    _o().oracle_unpack(_p(sp), _p(rp), _p(active), U64(active.size), _p(succ), _p(rank))


def cpu_threads() -> int:
    """Host threads the multi-core rankers use (all online cores, or
    KASCADE_CPU_THREADS)."""
    return int(_o().cpu_threads())


def cpu_sparse_ruling_set(succ: np.ndarray, rank: np.ndarray, spacing: int = 32, seed: int = 42,
                          threads: int = 0) -> None:
    """In place, the multi-core restatement of the reference's sparse ruling
    set (oracle/cpu_parallel.c): succ -> root, rank -> distance to the root."""
    assert succ.dtype == np.uint64 and rank.dtype == np.int64 and succ.flags.c_contiguous and rank.flags.c_contiguous
    rc = _o().cpu_sparse_ruling_set(_p(succ), _p(rank), U64(succ.size), U32(spacing), U64(seed),
                                    ctypes.c_int(threads))
    if rc != 0:
        raise ValueError("cpu_sparse_ruling_set: index out of range or a cycle without a root")


def cpu_pointer_doubling(succ: np.ndarray, rank: np.ndarray, threads: int = 0) -> int:
    """In place, multi-core synchronous pointer doubling; returns the rounds."""
    assert succ.dtype == np.uint64 and rank.dtype == np.int64 and succ.flags.c_contiguous and rank.flags.c_contiguous
    rounds = _o().cpu_pointer_doubling(_p(succ), _p(rank), U64(succ.size), ctypes.c_int(threads))
    if rounds < 0:
        raise ValueError("cpu_pointer_doubling: index out of range or a cycle without a root")
    return rounds


def cpu_gen_list(n: int, seed: int, layout: int = 0) -> np.ndarray:
    out = np.empty(n, np.uint64)
    _o().cpu_gen_list(U64(n), U64(seed), U32(layout), _p(out))
    return out


def cpu_gen_weights(n: int, seed: int, wbits: int = 16) -> np.ndarray:
    out = np.empty(n, np.uint32)
    _o().cpu_gen_weights(U64(n), U64(seed), U32(wbits), _p(out))
    return out


def cpu_gen_forest(n: int, seed: int, kind: int = 0, blocks: int = 64, spine: int = 0) -> np.ndarray:
    out = np.empty(n, np.uint64)
    _o().cpu_gen_forest(U64(n), U64(seed), U32(kind), U64(blocks), U64(spine), _p(out))
    return out


def gen_list(n: int, seed: int, layout: int = 0) -> np.ndarray:
    out = np.empty(n, np.uint64)
    _o().oracle_gen_list(U64(n), U64(seed), U32(layout), _p(out))
    return out


def gen_weights(n: int, seed: int, wbits: int = 16) -> np.ndarray:
    out = np.empty(n, np.uint32)
    _o().oracle_gen_weights(U64(n), U64(seed), U32(wbits), _p(out))
    return out


def gen_forest(n: int, seed: int, kind: int = 0, blocks: int = 64, spine: int = 0) -> np.ndarray:
    out = np.empty(n, np.uint64)
    _o().oracle_gen_forest(U64(n), U64(seed), U32(kind), U64(blocks), U64(spine), _p(out))
    return out


def ref_gather_rank(succ: np.ndarray):
    """The reference's own GatherRank path (set_initial_ranking_state +
    local_pointer_chasing from lib/kascade, compiled from source)."""
    succ = np.ascontiguousarray(succ, np.uint64)
    root = np.empty_like(succ)
    rank = np.empty(succ.size, np.int64)
    _r().ref_gather_rank(_p(succ), U64(succ.size), _p(root), _p(rank))
    return root, rank


def ref_local_pointer_chasing(succ: np.ndarray, rank: np.ndarray) -> None:
    """In place, the reference's lib/kascade/local_pointer_chasing.cpp."""
    assert succ.dtype == np.uint64 and rank.dtype == np.int64
    _r().ref_local_pointer_chasing(_p(succ), _p(rank), U64(succ.size))


def compute_stats(root: np.ndarray, rank: np.ndarray, level: int) -> tuple[dict, list]:
    """The bench's compute_stats (bench/detail/stats.cpp:110-143 basic, 24-108
    per tree) on one rank: level 2 basic, 3 reduced extensive, 4 extensive
    (also the non-trivial trees, here ordered by root).  numpy restatement."""
    root = np.asarray(root, dtype=np.uint64)
    rank = np.asarray(rank).view(np.int64) if np.asarray(rank).dtype == np.uint64 else np.asarray(rank, np.int64)
    n = root.size
    out = {"num_trees": 0, "max_rank": 0, "avg_rank": 0.0}
    if level < 2 or n == 0:
        return out, []
    idx = np.arange(n, dtype=np.uint64)
    out["num_trees"] = int(np.count_nonzero(root == idx))  # stats.cpp:117-119 (is_root)
    out["max_rank"] = int(rank.max())                        # stats.cpp:121-123
    # stats.cpp:124-126 fold into a std::size_t: the sum as an unsigned value
    total = int(np.sum(rank.view(np.uint64), dtype=np.uint64))
    out["avg_rank"] = float(total) / float(n)                # stats.cpp:136-137
    if level < 3:
        return out, []
    keys, inv = np.unique(root, return_inverse=True)         # one entry per tree (stats.cpp:32-39)
    size = np.bincount(inv, minlength=keys.size).astype(np.int64)
    rsum = np.zeros(keys.size, np.int64)
    np.add.at(rsum, inv, rank)
    rmax = np.zeros(keys.size, np.int64)                     # TreeStats::max_rank = 0 (stats.hpp:23-27)
    np.maximum.at(rmax, inv, rank)
    nt = size > 1                                            # stats.cpp:58-68
    out["ext_num_trees"] = int(keys.size)
    out["num_nontrivial_trees"] = int(nt.sum())
    out["nontrivial_size_sum"] = int(size[nt].sum())
    out["nontrivial_rank_sum"] = int(np.sum(rsum[nt], dtype=np.int64))
    out["max_size"] = int(size.max())
    trivial = out["ext_num_trees"] - out["num_nontrivial_trees"]
    div = lambda a, b: 0.0 if b == 0 else float(a) / float(b)  # noqa: E731  (stats.cpp:19-22)
    out["avg_size"] = div(out["nontrivial_size_sum"] + trivial, out["ext_num_trees"])
    out["nontrivial_avg_size"] = div(out["nontrivial_size_sum"], out["num_nontrivial_trees"])
    out["nontrivial_avg_rank"] = div(out["nontrivial_rank_sum"], out["nontrivial_size_sum"])
    trees = []
    if level >= 4:
        trees = [(int(k), int(a), int(b), int(c)) for k, a, b, c in zip(keys[nt], size[nt], rmax[nt], rsum[nt])]
    return out, trees



def compute_stats_transcribed(root, rank, level: int) -> tuple[dict, list]:
    """compute_stats of bench/detail/stats.cpp transcribed statement by
    statement for one rank (one Distribution slice = the whole array), in
    plain Python loops for small inputs.  An independent check of the numpy
    restatement above: a dict stands in for the absl hash map, C integer
    widths are applied where the reference converts (std::size_t sums,
    int64 per-tree sums), and the non-trivial trees come back ordered by root
    (the reference's order is the hash map's iteration order, unspecified).
    """
    M64 = (1 << 64) - 1

    def s64(x):  # two's complement int64 of a Python int
        x &= M64
        return x - (1 << 64) if x >> 63 else x

    root = [int(x) for x in np.asarray(root, dtype=np.uint64)]
    rank = [s64(int(x)) for x in np.asarray(rank).view(np.uint64)]
    n = len(root)
    if level < 2 or n == 0:  # StatsLevel::none (stats.cpp:150-152)
        return {"num_trees": 0, "max_rank": 0, "avg_rank": 0.0}, []
    # compute_basic_stats (stats.cpp:110-143)
    local_num_roots = sum(1 for i in range(n) if root[i] == i)      # is_root, successor_utils.cpp:65-70
    local_max_rank = max(rank) & M64                                # std::size_t (stats.cpp:121-123)
    local_rank_sum = 0
    for v in rank:                                                  # fold_left over int64 (stats.cpp:124-126)
        local_rank_sum = s64(local_rank_sum + v)
    global_rank_sum = local_rank_sum & M64                          # std::size_t (stats.cpp:132-134)
    basic = {"num_trees": local_num_roots,
             "avg_rank": float(global_rank_sum) / float(n),         # stats.cpp:136-137
             "max_rank": s64(local_max_rank)}                       # stats.cpp:139-141
    if level == 2:
        return basic, []
    # compute_per_tree_stats (stats.cpp:24-108)
    local_stats: dict = {}
    for i in range(n):
        t = local_stats.setdefault(root[i], {"size": 0, "max_rank": 0, "rank_sum": 0})
        t["size"] += 1
        t["rank_sum"] = s64(t["rank_sum"] + rank[i])
        t["max_rank"] = max(t["max_rank"], rank[i])
    ext = {"ext_num_trees": 0, "num_nontrivial_trees": 0, "nontrivial_size_sum": 0, "nontrivial_rank_sum": 0,
           "max_size": 0}
    per_tree = []
    for r in sorted(local_stats):
        t = local_stats[r]
        ext["ext_num_trees"] += 1
        ext["max_size"] = max(ext["max_size"], t["size"])
        if t["size"] > 1:
            ext["num_nontrivial_trees"] += 1
            ext["nontrivial_size_sum"] += t["size"]
            ext["nontrivial_rank_sum"] = s64(ext["nontrivial_rank_sum"] + t["rank_sum"])
            per_tree.append((r, t["size"], t["max_rank"], t["rank_sum"]))

    def safe_division(a, b):  # stats.cpp:19-22
        return 0.0 if b == 0 else float(a) / float(b)

    trivial = ext["ext_num_trees"] - ext["num_nontrivial_trees"]
    ext["avg_size"] = safe_division(ext["nontrivial_size_sum"] + trivial, ext["ext_num_trees"])
    ext["nontrivial_avg_size"] = safe_division(ext["nontrivial_size_sum"], ext["num_nontrivial_trees"])
    ext["nontrivial_avg_rank"] = safe_division(ext["nontrivial_rank_sum"], s64(ext["nontrivial_size_sum"]))
    out = dict(basic)
    out.update(ext)
    return out, (per_tree if level >= 4 else [])


def euler_tour_transcribed(parent, high_degree: bool = False) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """compute_euler_tour for one rank, transcribed statement by statement in
    plain Python (small inputs): the forest as reverse_rooted_tree(...,
    add_back_edge=true) sends it (lib/kascade/successor_utils.cpp:265-300;
    high_degree: the resolve_high_degree_tag variant, successor_utils.cpp:
    302-418, which on one rank finds no remote parent, creates no proxy and
    sends, for each non-root i, the edge from the parent first and then the
    back edge),
    the CSR graph as make_graph fills it -- each vertex's adjacency from its
    end backwards, in arrival order (successor_utils.cpp:236-260) -- and the
    tour as compute_euler_tour_impl builds it (lib/kascade/eulertour.cpp:
    33-127): edge ids in CSR order, succ[(u_prev, v)] = (v, u) with u_prev
    the neighbour before u in v's rotation, the first edge into each root
    (with neighbours) pointing at that root's dummy element, elements without
    a message left as self loops.  Returns (succ, weight, is_upward).  An
    independent check of the C restatement, which derives the same numbering
    by formulas."""
    parent = [int(x) for x in np.asarray(parent, dtype=np.uint64)]
    n = len(parent)
    # reverse_rooted_tree, one rank: the back edge first, then the edge to
    # the parent's owner (the same rank), for each non-root i in order
    recv_edges = []
    for i in range(n):
        if parent[i] == i:  # is_root (successor_utils.cpp:65-70)
            continue
        if high_degree:
            # every parent is owned by this rank: no entry in remote_info, no
            # proxy (successor_utils.cpp:322-339); edge to the parent's new
            # name, then the back edge (:381-389)
            recv_edges.append((parent[i], i))
            recv_edges.append((i, parent[i]))
        else:
            recv_edges.append((i, parent[i]))
            recv_edges.append((parent[i], i))
    # make_graph
    xadj = [0] * (n + 1)
    adjncy = [0] * len(recv_edges)
    for src, _ in recv_edges:
        xadj[src] += 1
    for k in range(1, n + 1):  # std::inclusive_scan
        xadj[k] += xadj[k - 1]
    for src, dst in recv_edges:
        xadj[src] -= 1
        adjncy[xadj[src]] = dst
    # compute_euler_tour_impl
    is_root = {v for v in range(n) if parent[v] == v}
    num_list_elems = len(adjncy) + len(is_root)
    weight = [0] * num_list_elems
    upward = [False] * num_list_elems
    edge_to_index = {}
    messages = []
    next_id = 0
    root_index = len(adjncy)
    for v in range(n):
        neighbors = adjncy[xadj[v]:xadj[v + 1]]
        degree = len(neighbors)
        for i in range(degree):
            u_prev = neighbors[(i + degree - 1) % degree]
            u = neighbors[i]
            edge_to_index[(v, u)] = next_id
            up = parent[v] == u
            weight[next_id] = 1 if up else -1
            upward[next_id] = up
            if v in is_root and i == 0:
                messages.append((u_prev, v, root_index))
                weight[root_index] = 0
                upward[root_index] = False
                edge_to_index[(v, v)] = root_index
                root_index += 1
            else:
                messages.append((u_prev, v, next_id))
            next_id += 1
    succ = list(range(num_list_elems))
    for u, v, nxt in messages:
        succ[edge_to_index[(u, v)]] = nxt
    return np.array(succ, np.uint64), np.array(weight, np.int64), np.array(upward, bool)
