"""The reference's own BIMP device kernels, run per scale (test infrastructure).

ctypes wrapper of oracle/_ref/libbimpref.so, built by oracle/build_ref.py
from daniel-koudouna/cuda-bimp's bimp/include/detection/cuda_bimp.cuh
(compiled unmodified) and the harness oracle/ref_harness/harness.cu.  The
harness drives FilterSimpleCells_kernel, complexResponse_kernel,
endStoppedResponse_kernel, inhibitionResponse_kernel, inhibitKeypoints_kernel
and identifyKeypoints_kernel in DoFullGPUFiltering's order
(bimp/src/cuda_bimp.cu:462-559, :714-743) with cuFFT R2C/C2R.

This module is a CHECKER, like the rest of oracle/: only tests/ and the
golden-fixture script use it.  It needs a CUDA device.  Inputs it cannot get
from the reference because they live in OpenCV-CUDA or in host code that
needs OpenCV come from the FP64 oracle (oracle/bimp_oracle.py):

* the uint8 pyramid levels (cv::cuda::pyrDown -> bimp_oracle.pyr_down_u8,
  pinned to cv2.pyrDown away from .5 ties);
* the per-scale geometry, the float32 Gabor taps and the stencil offsets
  (host arithmetic of the CudaStuff constructor, bimp/src/cuda_bimp.cu:222-349,
  and of DoFullGPUFiltering, :533-550).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from oracle import bimp_oracle as O

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libbimpref.so"
_LIB = None

RECORD_DTYPE = np.dtype([("x", "f4"), ("y", "f4"), ("size", "f4"), ("angle", "f4"), ("response", "f4"),
                         ("octave", "i4"), ("class_id", "i4")])


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is not built (python oracle/build_ref.py, needs the reference tree)")
        L = C.CDLL(str(LIB_PATH))
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        L.bref_scale.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, fp, fp,
                                 ip, ip, C.c_float, C.c_float, fp, fp, fp, fp, C.c_int, ip]
        L.bref_scale.restype = C.c_int
        L.bref_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def level_u8(img_u8: np.ndarray, sc: O.Scale) -> np.ndarray:
    """The scale's uint8 level, cropped to dataH x dataW (cuda_bimp.cu:473-486)."""
    cur = img_u8
    for _ in range(sc.levels):
        cur = O.pyr_down_u8(cur)
    return np.ascontiguousarray(cur[:sc.dataH, :sc.dataW])


def run_scale(img_u8: np.ndarray, sc: O.Scale, keep_c: bool = False, cap: int = 1 << 18,
              p: O.Params = O.Params()) -> dict:
    """One scale through the reference kernels.  Returns D, S (float32,
    dataH x dataW), C (8 x fftH x fftW, when keep_c) and the keypoint
    records sorted by (y, x), with their total count."""
    lvl = level_u8(img_u8, sc)
    even = np.empty((8, sc.kW, sc.kW), np.float32)
    odd = np.empty((8, sc.kW, sc.kW), np.float32)
    for o in range(8):
        even[o], odd[o] = O.gabor_taps(sc, o, p)
    es = np.ascontiguousarray(np.array(sc.es_off, dtype=np.int32).reshape(16))
    inh = np.ascontiguousarray(np.array(sc.in_off, dtype=np.int32).reshape(16))
    D = np.empty((sc.dataH, sc.dataW), np.float32)
    S = np.empty_like(D)
    Cm = np.empty((8, sc.fftH, sc.fftW), np.float32) if keep_c else None
    kp = np.zeros((7, cap), np.float32)
    n = C.c_int(0)
    rc = lib().bref_scale(lvl.ctypes.data, lvl.strides[0], sc.dataW, sc.dataH, sc.fftW, sc.fftH, sc.kW, sc.kX,
                          _fptr(even), _fptr(odd), _iptr(es), _iptr(inh), sc.lam, sc.pyrstep, _fptr(D), _fptr(S),
                          _fptr(Cm) if keep_c else None, _fptr(kp), cap, C.byref(n))
    if rc != 0:
        raise RuntimeError("reference harness: " + lib().bref_last_error().decode())
    total = n.value
    m = min(total, cap)
    rec = np.zeros(m, dtype=RECORD_DTYPE)
    rec["x"] = kp[0, :m]
    rec["y"] = kp[1, :m]
    rec["class_id"] = kp[2, :m].view(np.int32)
    rec["octave"] = kp[3, :m].view(np.int32)
    rec["size"] = kp[4, :m]
    rec["angle"] = kp[5, :m]
    rec["response"] = kp[6, :m]
    # the reference's slots are atomic-order: sort by level position
    order = np.lexsort((rec["x"], rec["y"]))
    return {"scale": sc, "D": D, "S": S, "C": Cm, "kp": rec[order], "count": total}


def run(img_u8: np.ndarray, lambdas, keep_c: bool = False, p: O.Params = O.Params()) -> list:
    """Every scale of one image (the scales sorted as the CudaStuff
    constructor sorts them, bimp/src/cuda_bimp.cu:224)."""
    H, W = img_u8.shape
    return [run_scale(img_u8, sc, keep_c=keep_c, p=p) for sc in O.scale_geometry(W, H, lambdas, p)]


def records(result: list) -> np.ndarray:
    """All scales' records in one array, in scale order."""
    return np.concatenate([r["kp"] for r in result]) if result else np.zeros(0, RECORD_DTYPE)
