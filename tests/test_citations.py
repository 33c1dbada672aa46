"""Every `file:line` citation of the reference in the library, its headers,
the oracle and the design/integration notes resolves to lines that exist in
the reference source tree, and the key entry points land on the function
they name.  Skipped when the reference tree is not beside this repository
(set KASCADE_REFERENCE_TREE to point elsewhere)."""
from __future__ import annotations

import os
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("KASCADE_REFERENCE_TREE", ROOT.parent / "reference"))
SCANNED = ["include", "kascade_b200", "oracle", "DESIGN.md", "INTEGRATION.md", "bench.py", "__graft_entry__.py",
           "tests"]
SUFFIXES = {".h", ".hpp", ".cu", ".cuh", ".py", ".c", ".cpp", ".md", ".json"}
CITE = re.compile(r"([A-Za-z0-9_./-]+\.(?:hpp|cpp|h|yaml|cmake|toml))"
                  r":(\d+(?:-\d+)?(?:, ?\d+(?:-\d+)?)*)")
# (file, first cited line) -> text that line must contain: the reference
# functions the boundary replaces
ANCHORS = {
    ("lib/kascade/list_ranking.hpp", 47): "set_initial_ranking_state",
    ("lib/kascade/list_ranking.hpp", 19): "rank_on_root",
    ("lib/kascade/list_ranking.cpp", 60): "set_initial_ranking_state",
    ("lib/kascade/list_ranking.cpp", 29): "rank_on_root",
    ("lib/kascade/local_pointer_chasing.cpp", 18): "local_pointer_chasing",
    ("lib/kascade/eulertour.cpp", 33): "compute_euler_tour_impl",
    ("lib/kascade/eulertour.cpp", 235): "map_euler_tour_back",
    ("lib/kascade/eulertour.cpp", 337): "rank_via_euler_tour",
    ("lib/kascade/eulertour.cpp", 379): "compute_euler_tour",
    ("lib/kascade/successor_utils.cpp", 302): "reverse_rooted_tree",
    ("lib/kascade/eulertour.hpp", 22): "rank_via_euler_tour",
    ("lib/kascade/sparse_ruling_set.hpp", 13): "sparse_ruling_set",
    ("lib/kascade/pointer_doubling.hpp", 18): "pointer_doubling",
    ("lib/kascade/successor_utils.cpp", 236): "make_graph",
    ("lib/kascade/successor_utils.cpp", 265): "reverse_rooted_tree",
    ("bench/detail/algorithm_impl.hpp", 81): "class GatherRank",
    ("bench/detail/algorithm_impl.hpp", 183): "class EulerTour",
    ("bench/detail/algorithm.hpp", 7): "class AbstractAlgorithm",
    ("bench/detail/stats.cpp", 24): "compute_per_tree_stats",
    ("bench/detail/stats.cpp", 110): "compute_basic_stats",
    ("bench/detail/stats.hpp", 23): "struct TreeStats",
}

pytestmark = pytest.mark.skipif(not (REF / "lib" / "kascade").is_dir(), reason="reference source tree not present")


def _scanned_files():
    for name in SCANNED:
        p = ROOT / name
        if p.is_file():
            yield p
            continue
        for q in sorted(p.rglob("*")):
            if q.is_file() and q.suffix in SUFFIXES and not {"_build", "_ref", "__pycache__"} & set(q.parts):
                yield q


def _citations():
    out = []
    for f in _scanned_files():
        if f.name == "test_citations.py":
            continue
        for ln, line in enumerate(f.read_text(errors="replace").splitlines(), 1):
            for m in CITE.finditer(line):
                out.append((f"{f.relative_to(ROOT)}:{ln}", m.group(1), m.group(2)))
    return out


def _resolve(name: str, index: dict) -> list[Path]:
    """Reference files a cited name can mean: an exact relative path, or every
    file whose path ends with the cited (possibly shortened) name."""
    exact = REF / name
    if exact.is_file():
        return [exact]
    return [p for p in index.get(Path(name).name, []) if str(p).endswith("/" + name) or p.name == name]


def test_every_citation_is_inside_its_file():
    index: dict = {}
    for p in REF.rglob("*"):
        if p.is_file() and ".git" not in p.parts:
            index.setdefault(p.name, []).append(p)
    cites = _citations()
    assert len(cites) > 100
    lengths: dict = {}
    bad = []
    for where, name, ranges in cites:
        cands = _resolve(name, index)
        if not cands:
            bad.append(f"{where}: {name} is not a file of the reference")
            continue
        spans = []
        for part in ranges.split(","):
            a, _, b = part.strip().partition("-")
            spans.append((int(a), int(b or a)))
        # a shortened name may match several files: one that holds every span
        ok = False
        for c in cands:
            n = lengths.setdefault(c, len(c.read_text(errors="replace").splitlines()))
            if all(1 <= a <= b <= n for a, b in spans):
                ok = True
                break
        if not ok:
            bad.append(f"{where}: {name}:{ranges} runs past the end of the file")
    assert not bad, "\n".join(bad)


def test_no_citation_without_a_file_name():
    """A shorthand like `eulertour.hpp:22-27, .cpp:337-377` cannot be checked:
    every citation names its file."""
    bare = re.compile(r"(?<![A-Za-z0-9_/-])\.(?:cpp|hpp|h):\d")
    bad = []
    for f in _scanned_files():
        if f.name == "test_citations.py":
            continue
        for ln, line in enumerate(f.read_text(errors="replace").splitlines(), 1):
            if bare.search(line):
                bad.append(f"{f.relative_to(ROOT)}:{ln}: {line.strip()}")
    assert not bad, "\n".join(bad)


def test_key_citations_land_on_their_functions():
    cited = {(name, int(r.split(",")[0].split("-")[0])) for _, name, r in _citations()}
    checked = 0
    for (path, line), needle in ANCHORS.items():
        text = (REF / path).read_text().splitlines()
        assert needle in text[line - 1], f"{path}:{line} is `{text[line - 1].strip()}`, not {needle}"
        short = {path, path.split("/", 2)[-1] if path.startswith("lib/") else path, Path(path).name}
        checked += any((s, line) in cited for s in short)
    assert checked >= len(ANCHORS) // 2
