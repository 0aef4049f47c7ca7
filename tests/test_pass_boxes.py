"""The CPML pass boxes of the tile step (host code, csrc/pass_boxes.h):
compiled with the host compiler and checked on random grids and face
layouts by tests/pass_boxes_check.cpp (exactly-once cover of the cells each
pass must handle, per-box face masks, block ranges)."""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_pass_boxes_cover_each_cell_once_with_its_faces(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "pass_boxes_check"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", str(ROOT / "magnelio_b200" / "csrc"),
                    str(ROOT / "tests" / "pass_boxes_check.cpp"), "-o", str(exe)], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:]
    assert res.stdout.startswith("ok 1200 layouts"), res.stdout
