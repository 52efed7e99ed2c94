"""ctypes binding of libbimp_b200.so (the C ABI in include/bimp_b200.h).

Loading fails loudly when the shared library has not been built: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent.parent / "lib" / "libbimp_b200.so"

BIMP_OK = 0
BIMP_ERR_INVALID = -1
BIMP_ERR_CUDA = -2
BIMP_ERR_NOMEM = -3
BIMP_ERR_CAPACITY = -4
BIMP_ERR_NO_DEVICE = -5
BIMP_ERR_UNSUPPORTED = -6

STATUS_NAMES = {
    BIMP_OK: "BIMP_OK",
    BIMP_ERR_INVALID: "BIMP_ERR_INVALID",
    BIMP_ERR_CUDA: "BIMP_ERR_CUDA",
    BIMP_ERR_NOMEM: "BIMP_ERR_NOMEM",
    BIMP_ERR_CAPACITY: "BIMP_ERR_CAPACITY",
    BIMP_ERR_NO_DEVICE: "BIMP_ERR_NO_DEVICE",
    BIMP_ERR_UNSUPPORTED: "BIMP_ERR_UNSUPPORTED",
}

KP_VECTOR_LENGTH = 7
KP_MAX_POINTS = 8000
NUM_ORI = 8


class TilePlan(C.Structure):
    """bimp_tile_plan (include/bimp_b200_batch.h)."""
    _fields_ = [("policy", C.c_int), ("order", C.c_int), ("kernel", C.c_int), ("grid", C.c_int),
                ("tiles", C.c_int), ("ms", C.c_float)]

    def as_dict(self) -> dict:
        return {"policy": self.policy, "order": self.order, "kernel": self.kernel, "grid": self.grid,
                "tiles": self.tiles, "ms": round(float(self.ms), 4)}


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "gamma", "sigma_ratio", "size_ratio", "offset_ratio", "level_max",
        "radial_gain", "w_tan", "w_rad", "thresh_ratio")]


class KeyPointC(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("size", C.c_float), ("angle", C.c_float),
                ("response", C.c_float), ("octave", C.c_int32), ("class_id", C.c_int32)]


class ScaleInfo(C.Structure):
    _fields_ = [("lambda_full", C.c_float), ("lambda_level", C.c_float), ("pyrstep", C.c_float),
                ("kernel_w", C.c_int), ("kernel_x", C.c_int), ("data_w", C.c_int),
                ("data_h", C.c_int), ("fft_w", C.c_int), ("fft_h", C.c_int), ("margin", C.c_int)]


# (name, restype, argtypes)
_PROTOS = [
    ("bimp_version", C.c_char_p, []),
    ("bimp_last_error", C.c_char_p, []),
    ("bimp_default_params", None, [C.POINTER(Params)]),
    ("bimp_make_lambdas_log", C.c_int, [C.c_float, C.c_float, C.c_int, C.POINTER(C.c_float), C.c_int,
                                        C.POINTER(C.c_int)]),
    ("bimp_make_lambdas_lin", C.c_int, [C.c_float, C.c_float, C.c_int, C.POINTER(C.c_float), C.c_int,
                                        C.POINTER(C.c_int)]),
    ("bimp_snap_transform_size", C.c_int, [C.c_int]),
    ("bimp_ctx_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int,
                                  C.POINTER(Params)]),
    ("bimp_ctx_destroy", C.c_int, [C.c_void_p]),
    ("bimp_ctx_create_for_input", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.POINTER(C.c_float), C.c_int, C.POINTER(Params)]),
    ("bimp_device_alloc", C.c_int, [C.POINTER(C.c_void_p), C.c_size_t]),
    ("bimp_device_free", C.c_int, [C.c_void_p]),
    ("bimp_copy_2d", C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t,
                               C.c_void_p]),
    ("bimp_ctx_num_scales", C.c_int, [C.c_void_p]),
    ("bimp_ctx_scale_info", C.c_int, [C.c_void_p, C.c_int, C.POINTER(ScaleInfo)]),
    ("bimp_detect_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p,
                                     C.c_size_t, C.c_int, C.POINTER(C.c_int), C.c_void_p]),
    ("bimp_detect_device_async", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int,
                                           C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_void_p]),
    ("bimp_detect_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int,
                                   C.POINTER(KeyPointC), C.c_int, C.POINTER(C.c_int), C.c_void_p]),
    ("bimp_pipeline_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int,
                                       C.POINTER(Params), C.c_int, C.c_int]),
    ("bimp_pipeline_destroy", C.c_int, [C.c_void_p]),
    ("bimp_pipeline_push", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int]),
    ("bimp_pipeline_pop", C.c_int, [C.c_void_p, C.POINTER(KeyPointC), C.c_int, C.POINTER(C.c_int)]),
    ("bimp_pipeline_in_flight", C.c_int, [C.c_void_p]),
    ("bimp_dense_map", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_complex_map", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_detect_lines_edges", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_min_size_dims", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_double)]),
    ("bimp_gpu_image", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                 C.c_size_t, C.c_void_p]),
    ("bimp_color_features", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t, C.c_int, C.c_int,
                                      C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_extract_keypoints_noalloc", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_float, C.c_float,
                                                 C.c_double, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p,
                                                 C.c_void_p]),
    ("bimp_ctx_kernel_launches", C.c_int, [C.c_void_p]),
    ("bimp_ctx_run_stage", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("bimp_download_keypoints", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(KeyPointC),
                                          C.c_void_p]),
    ("bimp_upload_keypoints", C.c_int, [C.POINTER(KeyPointC), C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_adjoint_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float),
                                      C.c_int, C.POINTER(Params)]),
    ("bimp_adjoint_destroy", C.c_int, [C.c_void_p]),
    ("bimp_adjoint_num_scales", C.c_int, [C.c_void_p]),
    ("bimp_adjoint_mask_layout", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("bimp_adjoint_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("bimp_adjoint_backward", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    ("bimp_adjoint_dense_map", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_adjoint_complex_map", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t,
                                           C.c_void_p]),
    ("bimp_adjoint_device_bytes", C.c_size_t, [C.c_void_p]),
    ("bimp_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int,
                                    C.POINTER(C.c_float), C.c_int, C.POINTER(Params), C.c_int]),
    ("bimp_batch_destroy", C.c_int, [C.c_void_p]),
    ("bimp_batch_num_images", C.c_int, [C.c_void_p]),
    ("bimp_batch_image", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    ("bimp_batch_run", C.c_int, [C.c_void_p, C.c_void_p]),
    ("bimp_batch_set_tile_plan", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("bimp_batch_autotune", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(TilePlan), C.POINTER(TilePlan),
                                      C.c_int, C.POINTER(C.c_int)]),
    ("bimp_batch_counts", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("bimp_batch_keypoints_device", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_size_t)]),
    ("bimp_batch_scale_info", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(ScaleInfo)]),
    ("bimp_batch_dense_map", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bimp_batch_detect_host", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                                         C.POINTER(C.POINTER(KeyPointC)), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.c_void_p]),
]

EXPORTED = [p[0] for p in _PROTOS]

_lib = None


def lib() -> C.CDLL:
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} not built: run `python cuda-bimp_b200/build.py`")
        h = C.CDLL(str(LIB_PATH))
        for name, res, args in _PROTOS:
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


class BimpError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().bimp_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(code: int, where: str) -> int:
    if code != BIMP_OK:
        raise BimpError(code, where)
    return code
