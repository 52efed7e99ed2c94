"""Build oracle/_ref/libbimpref.so: the reference's own BIMP device kernels
(daniel-koudouna/cuda-bimp, bimp/include/detection/cuda_bimp.cuh, compiled
unmodified from where the reference lies) with the harness
oracle/ref_harness/harness.cu that drives them in DoFullGPUFiltering's order
with cuFFT.  Test infrastructure: only the tests and the golden-fixture script
load it; the product never does.

    python oracle/build_ref.py [--force] [--reference DIR]

The reference tree is needed only to build (it is not read at run time); the
built library travels with the repository's other built files.  The
OpenCV types that the reference header names come from the small stand-ins
under oracle/ref_harness/stubs.  Needs nvcc (sm_100a) and cuFFT.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
HARNESS = HERE / "ref_harness" / "harness.cu"
STUBS = HERE / "ref_harness" / "stubs"
OUT = HERE / "_ref" / "libbimpref.so"
DEFAULT_REFERENCE = Path("/root/reference")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def reference_include(reference: Path) -> Path:
    return reference / "bimp" / "include" / "detection"


def available(reference: Path = DEFAULT_REFERENCE) -> bool:
    return (reference_include(reference) / "cuda_bimp.cuh").exists()


def build(force: bool = False, reference: Path = DEFAULT_REFERENCE) -> Path | None:
    """Builds the library when the reference tree is present; returns its
    path (or None when neither the tree nor a built library exists)."""
    inc = reference_include(reference)
    if not available(reference):
        return OUT if OUT.exists() else None
    deps = [HARNESS, *STUBS.rglob("*.hpp"), *inc.glob("*")]
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= Path(d).stat().st_mtime for d in deps):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    # nvcc's defaults for the device code (as the reference's CMake build,
    # which sets no device flags), sm_100a only
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-Xcompiler", "-fPIC",
           "-shared", f"-I{STUBS}", f"-I{inc}", str(HARNESS), "-o", str(OUT), "-lcufft"]
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    ref = DEFAULT_REFERENCE
    if "--reference" in sys.argv:
        ref = Path(sys.argv[sys.argv.index("--reference") + 1])
    out = build(force="--force" in sys.argv, reference=ref)
    print(out if out else "reference tree not found; nothing built")
