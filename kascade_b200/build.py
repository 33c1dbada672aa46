"""Build recipe for libkascade_b200.so (sm_100a) -- in-tree, no JIT cache.

Every ``csrc/*.cu`` is compiled by nvcc for ``sm_100a`` into ``_build/`` and
linked, with the CUDA runtime linked statically, into
``kascade_b200/libkascade_b200.so``.  Objects are rebuilt only when a source
or header is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libkascade_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I",
    str(INCLUDE),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build kascade_b200")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    deps = _headers()
    srcs = sorted(CSRC.glob("*.cu"))
    flags = NVCC_FLAGS + list(extra_flags or [])
    jobs = []
    for src in srcs:
        obj = BUILD / (src.stem + ".o")
        if _stale(obj, src, deps):
            jobs.append([cc, *flags, "-c", str(src), "-o", str(obj)])

    def run(cmd: list[str]) -> None:
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        if verbose and res.stderr.strip():
            print(res.stderr, file=sys.stderr)

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            list(ex.map(run, jobs))
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    if jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        link = [cc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        run(link)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
