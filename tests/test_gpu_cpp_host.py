"""The C++ host interface (include/kascade_b200.hpp) compiled against the
in-tree library and run."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_cpp_plugin(tmp_path):
    cxx = shutil.which("g++") or "g++"
    exe = tmp_path / "plugin_check"
    cmd = [cxx, "-std=c++20", "-O2", f"-I{ROOT / 'include'}", f"-I{ROOT / 'kascade_b200' / 'csrc'}",
           str(ROOT / "tests" / "cpp" / "plugin_check.cpp"), "-o", str(exe), f"-L{ROOT / 'kascade_b200'}",
           "-lkascade_b200", f"-Wl,-rpath,{ROOT / 'kascade_b200'}"]
    subprocess.run(cmd, check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.count(": ok") == 4
