"""Build oracle/libcbimp.so, the FP32 OpenMP C restatement (test and CPU
baseline infrastructure; the product never loads it).

    python oracle/build_cbimp.py [--force]

x86-64 hosts get -mavx2 -mfma (every AVX2-era server CPU); others build
with the compiler's baseline ISA.
"""
from __future__ import annotations

import os
import platform
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "cbimp.c"
LIB = HERE / "libcbimp.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    flags = ["-O3", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-D_GNU_SOURCE"]
    if platform.machine() in ("x86_64", "AMD64"):
        flags += ["-mavx2", "-mfma"]
    # $CC first; a compiler without an OpenMP runtime falls through to the
    # system gcc
    candidates = [c for c in (os.environ.get("CC"), shutil.which("gcc"), "/usr/bin/gcc") if c]
    last = None
    for cc in dict.fromkeys(candidates):
        cmd = [cc, *flags, str(SRC), "-o", str(LIB), "-lm"]
        print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            return LIB
        last = r.stderr.strip().splitlines()[-1:] or [f"exit {r.returncode}"]
        print(f"  failed: {last[0]}", flush=True)
    raise RuntimeError(f"could not build {LIB.name}: {last}")


if __name__ == "__main__":
    build(force="--force" in sys.argv)
