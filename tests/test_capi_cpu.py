"""CPU checks of the C ABI: the library loads, exports every function the
public headers declare, and its host-only helpers agree with the oracle."""
import re
from pathlib import Path

import numpy as np

from bimp_b200 import _lib as L
from bimp_b200 import api
from oracle import bimp_oracle as O

ROOT = Path(__file__).resolve().parent.parent


def _declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(?:int|void|const char\*)\s+(bimp_\w+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    declared = _declared_functions()
    assert len(declared) >= 20
    h = L.lib()
    missing = [n for n in sorted(declared) if not hasattr(h, n)]
    assert not missing, missing
    # the Python binding covers the same surface
    assert declared <= set(L.EXPORTED), sorted(declared - set(L.EXPORTED))


def test_version_and_defaults():
    assert b"sm_100a" in L.lib().bimp_version()
    p = api.default_params()
    assert (p.gamma, p.sigma_ratio, p.size_ratio, p.offset_ratio) == (0.5, 0.56, 7.0, 0.6)
    assert (p.level_max, p.radial_gain, p.w_tan, p.w_rad, p.thresh_ratio) == (7.5, 16.0, 1.0, 1.0, 0.104)


def test_make_lambdas_match_oracle():
    for args in [(4, 45.26, 2), (4, 64, 2), (4, 32, 1), (3.5, 100, 3)]:
        assert api.makeLambdasLog(*args) == O.make_lambdas_log(*args)
    assert api.makeLambdasLin(4, 8, 5) == O.make_lambdas_lin(4, 8, 5)


def test_snap_transform_size_matches_oracle():
    for n in list(range(1, 2200, 7)) + [2160, 3840, 4096, 5000]:
        assert api.snapTransformSize(n) == O.snap_transform_size(n)


def test_null_arguments_rejected_without_gpu():
    import ctypes as C
    assert L.lib().bimp_ctx_create(None, 64, 64, None, 0, None) == L.BIMP_ERR_INVALID
    h = C.c_void_p()
    assert L.lib().bimp_ctx_create(C.byref(h), 64, 64, None, 0, None) == L.BIMP_ERR_INVALID
    assert L.lib().bimp_ctx_destroy(None) == L.BIMP_OK
    n = C.c_int()
    assert L.lib().bimp_detect_host(None, None, 0, 0, 0, None, 0, C.byref(n), None) == L.BIMP_ERR_INVALID
    assert L.lib().bimp_make_lambdas_log(4.0, 8.0, 0, None, 0, C.byref(n)) == L.BIMP_ERR_INVALID
    assert L.lib().bimp_batch_create(None, None, None, 0, None, 0, None, 0) == L.BIMP_ERR_INVALID
    assert b"null" in L.lib().bimp_last_error() or L.lib().bimp_last_error() != b""


def test_keypoint_struct_layout_is_cv_keypoint():
    import ctypes as C
    assert C.sizeof(L.KeyPointC) == 28
    assert [f for f, _ in L.KeyPointC._fields_] == ["x", "y", "size", "angle", "response", "octave", "class_id"]
    assert C.sizeof(L.Params) == 9 * 8


def _build_shim_demo():
    import subprocess
    out = ROOT / "cuda-bimp_b200" / "_build" / "shim_demo"
    out.parent.mkdir(parents=True, exist_ok=True)
    lib = ROOT / "cuda-bimp_b200" / "lib"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "cpp" / "shim_demo.cpp"), f"-L{lib}", "-lbimp_b200",
                    f"-Wl,-rpath,{lib}", "-o", str(out)], check=True)
    return out


def test_cpp_shim_compiles_and_links():
    assert _build_shim_demo().exists()
