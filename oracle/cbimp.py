"""ctypes wrapper of oracle/libcbimp.so, the FP32 OpenMP C restatement of the
reference pipeline (test infrastructure and timed CPU baseline only).

    with CBimp(w, h, lambdas) as cb:
        records, total = cb.detect(img_u8)     # structured cv::KeyPoint rows
        D = cb.dense_map(scale)                # summed keypoint map
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_LIB = None
KEYPOINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("size", "<f4"), ("angle", "<f4"),
                           ("response", "<f4"), ("octave", "<i4"), ("class_id", "<i4")])


def lib(build_if_missing: bool = True):
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(__file__).resolve().parent / "libcbimp.so"
    if not path.exists() and build_if_missing:
        from oracle import build_cbimp
        build_cbimp.build()
    L = C.CDLL(str(path))
    L.cbimp_create.restype = C.c_void_p
    L.cbimp_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_double)]
    L.cbimp_destroy.argtypes = [C.c_void_p]
    L.cbimp_num_scales.argtypes = [C.c_void_p]
    L.cbimp_scale_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.cbimp_detect.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.cbimp_dense_map.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.cbimp_set_threads.argtypes = [C.c_int]
    L.cbimp_snap_transform_size.argtypes = [C.c_int]
    _LIB = L
    return L


class CBimp:
    """One wavelength bank for width x height u8 images."""

    def __init__(self, width: int, height: int, lambdas, params=None, threads: int | None = None):
        L = lib()
        if threads:
            L.cbimp_set_threads(int(threads))
        lam = (C.c_float * len(lambdas))(*[float(x) for x in lambdas])
        p = None
        if params is not None:
            vals = [params.gamma, params.sigma_ratio, params.size_ratio, params.offset_ratio, params.level_max,
                    params.radial_gain, params.w_tan, params.w_rad, params.thresh_ratio]
            p = (C.c_double * 9)(*vals)
        self._h = L.cbimp_create(int(width), int(height), lam, len(lambdas), p)
        if not self._h:
            raise ValueError("cbimp_create failed (invalid size or wavelengths)")
        self.width, self.height = int(width), int(height)
        self.scales = []
        for s in range(L.cbimp_num_scales(self._h)):
            info = (C.c_int * 7)()
            L.cbimp_scale_info(self._h, s, info)
            self.scales.append(dict(zip(("data_w", "data_h", "fft_w", "fft_h", "kw", "off", "level"), info)))

    def detect(self, img: np.ndarray, capacity: int = 1 << 20):
        img = np.ascontiguousarray(img, dtype=np.uint8)
        assert img.shape == (self.height, self.width)
        out = np.zeros(capacity, dtype=KEYPOINT_DTYPE)
        total = C.c_int()
        n = lib().cbimp_detect(self._h, img.ctypes.data, img.strides[0], out.ctypes.data, capacity, C.byref(total))
        if n < 0:
            raise RuntimeError("cbimp_detect failed")
        return out[:n], total.value

    def dense_map(self, scale: int, which: int = 0) -> np.ndarray:
        s = self.scales[scale]
        out = np.empty((s["data_h"], s["data_w"]), dtype=np.float32)
        if lib().cbimp_dense_map(self._h, scale, which, out.ctypes.data) != 0:
            raise IndexError(scale)
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().cbimp_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def max_threads() -> int:
    return int(lib().cbimp_max_threads())
