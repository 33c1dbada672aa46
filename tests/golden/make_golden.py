"""Generate the golden fixtures under tests/golden/.

  chase_cases.npz  Inputs from the seeded generators and the outputs of the
                   reference's own GatherChase (lib/kascade/
                   local_pointer_chasing.cpp, compiled from the reference
                   source tree into oracle/_ref by oracle/Makefile).  GatherRank
                   on a parent array gives (root, depth), on a successor array
                   (root, rank); weighted cases put the weights in the rank
                   array (roots 0), as the reference's in-place contract does.
  kat.json         Known answers: the arrays of the reference's
                   tests/pack_test.cpp (PackTest.works on 4 ranks, concatenated
                   into one index space, and PackTest.sanity_check), and an
                   Euler tour worked by hand from eulertour.cpp:33-127 and
                   successor_utils.cpp:236-300.

Run from the repository root with the reference tree present:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def ref_rank(succ: np.ndarray, weights: np.ndarray | None):
    s = succ.astype(np.uint64).copy()
    if weights is None:
        return oracle.ref_gather_rank(s)
    r = weights.astype(np.int64)
    r[s == np.arange(s.size, dtype=np.uint64)] = 0
    oracle.ref_local_pointer_chasing(s, r)
    return s, r


def many_lists(n: int, parts: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    order = rng.permutation(n).astype(np.uint64)
    cuts = np.sort(rng.choice(np.arange(1, n), size=parts - 1, replace=False))
    succ = np.empty(n, np.uint64)
    for seg in np.split(order, cuts):
        succ[seg[:-1]] = seg[1:]
        succ[seg[-1]] = seg[-1]
    return succ


def random_forest(n: int, root_prob: float, seed: int) -> np.ndarray:
    """parent[i] uniform in [0, i) (or a root), then relabelled."""
    rng = np.random.default_rng(seed)
    par = np.empty(n, np.uint64)
    for i in range(n):
        par[i] = i if (i == 0 or rng.random() < root_prob) else rng.integers(0, i)
    perm = rng.permutation(n).astype(np.uint64)
    out = np.empty(n, np.uint64)
    out[perm] = perm[par]
    return out


def main() -> None:
    if not oracle.has_ref():
        oracle.build()
    assert oracle.has_ref(), "oracle/_ref must be built from the reference tree"
    cases: dict[str, np.ndarray] = {}

    def add(name: str, succ: np.ndarray, weights: np.ndarray | None = None, kind: str = "list") -> None:
        root, rank = ref_rank(succ, weights)
        cases[f"{name}__succ"] = succ.astype(np.uint64)
        if weights is not None:
            cases[f"{name}__w"] = weights.astype(np.uint32)
        cases[f"{name}__root"] = root.astype(np.uint64)
        cases[f"{name}__rank"] = rank.astype(np.int64)
        cases[f"{name}__kind"] = np.array([kind])

    add("list_random_1000", oracle.gen_list(1000, 0xC0, 0))
    add("list_runs_4096", oracle.gen_list(4096, 5, 1))
    add("list_path_9000", oracle.gen_list(9000, 0, 2))
    add("list_weighted_3000", oracle.gen_list(3000, 11, 0), oracle.gen_weights(3000, 12, 16))
    w0 = oracle.gen_weights(2500, 13, 2)  # many zeros
    add("list_zero_weights_2500", oracle.gen_list(2500, 14, 0), w0)
    add("lists_many_5000", many_lists(5000, 97, 31))
    add("lists_many_weighted_4000", many_lists(4000, 13, 32), oracle.gen_weights(4000, 33, 16))
    add("single_1", np.array([0], np.uint64))
    add("pair_2", np.array([1, 1], np.uint64))
    add("all_roots_100", np.arange(100, dtype=np.uint64))
    add("forest_rrt_5000", oracle.gen_forest(5000, 21, 0, 7), kind="forest")
    add("forest_cat_6000", oracle.gen_forest(6000, 22, 1, 3, 1500), kind="forest")
    add("forest_random_3000", random_forest(3000, 0.01, 41), kind="forest")
    star = np.zeros(2000, np.uint64)
    add("forest_star_2000", star, kind="forest")
    np.savez_compressed(OUT / "chase_cases.npz", **cases)

    kat = {
        "source": "reference tests/pack_test.cpp (PackTest.works, PackTest.sanity_check); "
        "Euler tour worked by hand from lib/kascade/eulertour.cpp:33-127",
        "pack_works": {
            # ranks 0..3 of the 4-rank test, concatenated: global indices
            # 0-7 | 8-13 | 14-15 | 16-19 (distribution.hpp block offsets)
            "succ": [0, 6, 0, 0, 0, 0, 8, 0, 10, 0, 14, 0, 0, 0, 15, 18, 0, 0, 18, 0],
            "rank": [42, 1, 42, 42, 42, 42, 1, 42, 1, 42, 1, 42, 42, 42, 1, 1, 42, 42, 0, 42],
            "active": [1, 6, 8, 10, 14, 15, 18],
            "packed_succ": [1, 2, 3, 4, 5, 6, 6],
            "packed_rank": [1, 1, 1, 1, 1, 1, 0],
            # the test then sets every packed successor to 6 and rank 6 - i
            "ranked_packed_succ": [6, 6, 6, 6, 6, 6, 6],
            "ranked_packed_rank": [6, 5, 4, 3, 2, 1, 0],
            "unpacked_succ": [0, 18, 0, 0, 0, 0, 18, 0, 18, 0, 18, 0, 0, 0, 18, 18, 0, 0, 18, 0],
            "unpacked_rank": [42, 6, 42, 42, 42, 42, 5, 42, 4, 42, 3, 42, 42, 42, 2, 1, 42, 42, 0, 42],
        },
        "pack_sanity": {
            "succ": list(range(1, 12)) + [11],
            "rank": [1] * 11 + [0],
        },
        "euler_tour_small": {
            # root 0 with children 1 and 3; 2 below 1
            "parent": [0, 0, 1, 0],
            # CSR: nbrs(0)=[3,1], nbrs(1)=[2,0], nbrs(2)=[1], nbrs(3)=[0];
            # ids (0,3)=0 (0,1)=1 (1,2)=2 (1,0)=3 (2,1)=4 (3,0)=5, dummy 6
            "tour_succ": [5, 2, 4, 6, 3, 1, 6],
            "depth": [0, 1, 2, 1],
            "root": [0, 0, 0, 0],
        },
    }
    (OUT / "kat.json").write_text(json.dumps(kat, indent=1) + "\n")
    print(f"wrote {len(cases)} arrays to chase_cases.npz and kat.json")


if __name__ == "__main__":
    main()
