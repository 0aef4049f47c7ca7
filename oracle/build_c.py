"""Compile the C port of the step (``oracle/fitstep.c``) for the host CPU --
TEST INFRASTRUCTURE AND CPU BASELINE ONLY.

The library goes to ``oracle/_build/libfitc.so`` (git-ignored).  It is
compiled with ``-march=native`` on the machine that runs it, the way the
reference's Numba kernels are JIT-compiled for the host they run on.
"""

from __future__ import annotations

import os
import platform
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "fitstep.c"
OUT_DIR = HERE / "_build"


def lib_path() -> Path:
    tag = platform.node().replace("/", "_") or "host"
    return OUT_DIR / f"libfitc_{tag}.so"


def build(force: bool = False) -> Path:
    out = lib_path()
    if out.exists() and not force and out.stat().st_mtime >= SRC.stat().st_mtime:
        return out
    OUT_DIR.mkdir(exist_ok=True)
    objs = []
    for real, sfx in (("float", "f32"), ("double", "f64")):
        obj = OUT_DIR / f"fitstep_{sfx}.o"
        cmd = ["gcc", "-O3", "-march=native", "-fopenmp", "-fPIC", "-std=c11", f"-DREAL={real}", f"-DSFX={sfx}",
               "-c", str(SRC), "-o", str(obj)]
        subprocess.run(cmd, check=True, capture_output=True, text=True)
        objs.append(str(obj))
    tmp = out.with_suffix(".tmp")
    subprocess.run(["gcc", "-shared", "-fopenmp", "-o", str(tmp), *objs], check=True, capture_output=True, text=True)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force=True))
