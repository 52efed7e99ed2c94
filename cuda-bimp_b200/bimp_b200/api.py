"""Python mirror of the daniel-koudouna/cuda-bimp keypoint API over the C ABI.

Names follow the reference (bimp/include/detection/cuda_bimp.hpp,
bimp/include/detection/bimp.hpp, bimp/include/detection/utils.hpp):

* ``CudaStuff(width, height, lambdas)``        -> bimp_ctx_create
* ``getKeypoints(gpu_image, cs)``               -> bimp_detect_device, returns the
  7 x n device matrix (SURF_CUDA row layout), like the GpuMat colRange view
* ``downloadKeypoints(kp)`` / ``uploadKeypoints`` (utils.cpp:109-150)
* ``makeLambdasLog`` / ``makeLambdasLin`` / ``snapTransformSize``
* ``Context(image)`` with ``getKeypoints()``, ``getKeypointsAndDownload()``,
  ``loadImage()``, ``getResponses()`` (bimp.cpp:7-129)

Device memory and streams come from torch; every computation runs in
libbimp_b200.so.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import sys
import warnings
from dataclasses import dataclass

import numpy as np

from . import _lib as L

KP_MAX_POINTS = L.KP_MAX_POINTS
KP_VECTOR_LENGTH = L.KP_VECTOR_LENGTH
NUM_ORI = L.NUM_ORI
X_ROW, Y_ROW, LAPLACIAN_ROW, OCTAVE_ROW, SIZE_ROW, ANGLE_ROW, HESSIAN_ROW = range(7)


def _torch():
    import torch  # plumbing only: device memory and streams
    return torch


def _stream_ptr(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


@dataclass
class KeyPoint:
    """Field-for-field stand-in of cv::KeyPoint."""
    pt: tuple
    size: float
    angle: float
    response: float
    octave: int
    class_id: int


def default_params() -> L.Params:
    p = L.Params()
    L.lib().bimp_default_params(C.byref(p))
    return p


def makeLambdasLog(start: float, end: float, scales_per_octave: int) -> list:
    n = C.c_int(0)
    L.check(L.lib().bimp_make_lambdas_log(start, end, scales_per_octave, None, 0, C.byref(n)),
            "makeLambdasLog")
    buf = (C.c_float * max(n.value, 1))()
    L.check(L.lib().bimp_make_lambdas_log(start, end, scales_per_octave, buf, n.value, C.byref(n)),
            "makeLambdasLog")
    return [float(buf[i]) for i in range(n.value)]


def makeLambdasLin(start: float, end: float, num_scales: int) -> list:
    n = C.c_int(0)
    buf = (C.c_float * max(num_scales, 1))()
    L.check(L.lib().bimp_make_lambdas_lin(start, end, num_scales, buf, num_scales, C.byref(n)),
            "makeLambdasLin")
    return [float(buf[i]) for i in range(n.value)]


def snapTransformSize(n: int) -> int:
    return int(L.lib().bimp_snap_transform_size(int(n)))


def _params(params) -> L.Params | None:
    if params is None:
        return None
    p = default_params()
    items = params.items() if isinstance(params, dict) else vars(params).items()
    for k, v in items:
        if not hasattr(p, k):
            raise ValueError(f"unknown parameter {k!r}")
        setattr(p, k, float(v))
    return p


class CudaStuff:
    """bimp::cuda::CudaStuff: filter bank + buffers for one image size."""

    def __init__(self, width: int, height: int, lambdas, params=None, input_size=None):
        """input_size (default (width, height)): the size of the images a
        detection takes; a larger input is filtered on the top-left window of
        each pyramid level (bimp_ctx_create_for_input), as the reference's
        Context does for upscaled small images."""
        lam = (C.c_float * len(lambdas))(*[float(x) for x in lambdas])
        h = C.c_void_p()
        p = _params(params)
        iw, ih = (int(width), int(height)) if input_size is None else (int(input_size[0]), int(input_size[1]))
        L.check(L.lib().bimp_ctx_create_for_input(C.byref(h), int(width), int(height), iw, ih, lam, len(lambdas),
                                                  C.byref(p) if p is not None else None), "CudaStuff")
        self._h = h
        self.width, self.height = int(width), int(height)
        self.input_width, self.input_height = iw, ih
        self.ks = [self.scale_info(i) for i in range(L.lib().bimp_ctx_num_scales(h))]

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("CudaStuff already released")
        return self._h

    def scale_info(self, i: int) -> dict:
        si = L.ScaleInfo()
        L.check(L.lib().bimp_ctx_scale_info(self._h, i, C.byref(si)), "scale_info")
        return {f: getattr(si, f) for f, _ in L.ScaleInfo._fields_}

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.lib().bimp_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- dense maps of the last detection ---------------------------------
    def dense_map(self, scale: int, which: int = 0):
        torch = _torch()
        k = self.ks[scale]
        out = torch.empty((k["data_h"], k["data_w"]), dtype=torch.float32, device="cuda")
        L.check(L.lib().bimp_dense_map(self.handle, scale, which, C.c_void_p(out.data_ptr()),
                                       out.stride(0), _stream_ptr()), "dense_map")
        return out

    def complex_map(self, scale: int, orientation: int):
        torch = _torch()
        k = self.ks[scale]
        out = torch.empty((k["data_h"] + 1, k["data_w"] + 1), dtype=torch.float32, device="cuda")
        L.check(L.lib().bimp_complex_map(self.handle, scale, orientation, C.c_void_p(out.data_ptr()),
                                         out.stride(0), _stream_ptr()), "complex_map")
        return out

    def lines_edges(self, scale: int, ch=None):
        """Line/edge detection on one scale of the last detection
        (bimp_detect_lines_edges): (strength, orientation, type) maps.
        ch: optional summed complex response (data_h x data_w float32 CUDA
        tensor); default the sum of the scale's complex cells."""
        torch = _torch()
        k = self.ks[scale]
        h, w = k["data_h"], k["data_w"]
        res = torch.empty((h, w), dtype=torch.float32, device="cuda")
        ori = torch.empty((h, w), dtype=torch.float32, device="cuda")
        typ = torch.empty((h, w), dtype=torch.int8, device="cuda")
        chp, chld = (None, 0) if ch is None else (C.c_void_p(ch.data_ptr()), ch.stride(0))
        L.check(L.lib().bimp_detect_lines_edges(self.handle, scale, chp, chld, C.c_void_p(res.data_ptr()),
                                                C.c_void_p(ori.data_ptr()), C.c_void_p(typ.data_ptr()), w,
                                                _stream_ptr()), "detect_lines_edges")
        return res, ori, typ


def _as_gpu_u8(image):
    torch = _torch()
    if isinstance(image, np.ndarray):
        image = torch.from_numpy(np.ascontiguousarray(image)).cuda()
    if image.dtype != torch.uint8 or image.dim() != 2 or not image.is_cuda:
        raise ValueError("expected a 2-D uint8 CUDA tensor")
    if image.stride(1) != 1:
        image = image.contiguous()
    return image


def getKeypoints(input, cs: CudaStuff, capacity: int = KP_MAX_POINTS, return_count: bool = False):
    """bimp::cuda::getKeypoints(GpuMat&, CudaStuff&) (cuda_bimp.cu:129-140).

    Returns the 7 x n float32 device matrix; like the reference, more than
    ``capacity`` keypoints produce a warning and the first ``capacity`` are
    kept ((scale, y, x) order).
    """
    torch = _torch()
    img = _as_gpu_u8(input)
    kp = torch.zeros((KP_VECTOR_LENGTH, max(capacity, 1)), dtype=torch.float32, device="cuda")
    n = C.c_int(0)
    rc = L.lib().bimp_detect_device(cs.handle, C.c_void_p(img.data_ptr()), img.stride(0),
                                    img.shape[1], img.shape[0], C.c_void_p(kp.data_ptr()),
                                    kp.stride(0), capacity, C.byref(n), _stream_ptr())
    if rc == L.BIMP_ERR_CAPACITY:
        warnings.warn(f"Keypoints ({n.value}) exceed current keypoint maximum ({capacity}).")
    elif rc != L.BIMP_OK:
        L.check(rc, "getKeypoints")
    rows = min(n.value, capacity)
    view = kp[:, :rows]
    return (view, n.value) if return_count else view


def downloadKeypoints(kp) -> list:
    """bimp::utils::downloadKeypoints (utils.cpp:130-150)."""
    n = kp.shape[1]
    out = (L.KeyPointC * max(n, 1))()
    L.check(L.lib().bimp_download_keypoints(C.c_void_p(kp.data_ptr()), kp.stride(0), n, out,
                                            _stream_ptr()), "downloadKeypoints")
    return [KeyPoint((k.x, k.y), k.size, k.angle, k.response, k.octave, k.class_id) for k in out[:n]]


def uploadKeypoints(points) -> "object":
    """bimp::utils::uploadKeypoints (utils.cpp:109-128)."""
    torch = _torch()
    n = len(points)
    arr = (L.KeyPointC * max(n, 1))()
    for i, p in enumerate(points):
        arr[i] = L.KeyPointC(p.pt[0], p.pt[1], p.size, p.angle, p.response, p.octave, p.class_id)
    kp = torch.empty((KP_VECTOR_LENGTH, max(n, 1)), dtype=torch.float32, device="cuda")
    L.check(L.lib().bimp_upload_keypoints(arr, n, C.c_void_p(kp.data_ptr()), kp.stride(0),
                                          _stream_ptr()), "uploadKeypoints")
    return kp[:, :n]


# cv::KeyPoint field order of the host records (bimp_keypoint)
_HOST_RECORD = np.dtype([("x", "<f4"), ("y", "<f4"), ("size", "<f4"), ("angle", "<f4"), ("response", "<f4"),
                         ("octave", "<i4"), ("class_id", "<i4")])


def detect_host(cs: CudaStuff, image: np.ndarray, capacity: int = KP_MAX_POINTS):
    """Host image in, host records out through bimp_detect_host.

    Returns (structured array of cv::KeyPoint fields, total count, status)."""
    img = np.ascontiguousarray(image, dtype=np.uint8)
    out = (L.KeyPointC * max(capacity, 1))()
    n = C.c_int(0)
    rc = L.lib().bimp_detect_host(cs.handle, C.c_void_p(img.ctypes.data), img.strides[0], img.shape[1],
                                  img.shape[0], out, capacity, C.byref(n), _stream_ptr())
    if rc not in (L.BIMP_OK, L.BIMP_ERR_CAPACITY):
        L.check(rc, "detect_host")
    m = min(n.value, capacity)
    rec = np.frombuffer(out, dtype=_HOST_RECORD, count=m).copy()
    return rec, n.value, rc


def min_size_dims(width: int, height: int) -> tuple:
    """getGPUImage's size rule (bimp_min_size_dims): (out_w, out_h)."""
    ow, oh = C.c_int(), C.c_int()
    L.check(L.lib().bimp_min_size_dims(int(width), int(height), C.byref(ow), C.byref(oh), None), "min_size_dims")
    return ow.value, oh.value


def gpu_image_device(image: np.ndarray, grayscale: bool = True):
    """getGPUImage (cuda_bimp.cu:156-180) keeping the result on the device:
    uint8 CUDA tensor (h, w) for grey output, (h, w * 3) for BGR."""
    torch = _torch()
    img = np.ascontiguousarray(image, dtype=np.uint8)
    h, w = img.shape[:2]
    cn = 1 if img.ndim == 2 else img.shape[2]
    ow, oh = min_size_dims(w, h)
    ocn = 1 if (grayscale or cn == 1) else cn
    src = torch.from_numpy(img.reshape(h, w * cn)).cuda()
    dst = torch.empty((oh, ow * ocn), dtype=torch.uint8, device="cuda")
    L.check(L.lib().bimp_gpu_image(C.c_void_p(src.data_ptr()), src.stride(0), w, h, cn, int(bool(grayscale)),
                                   C.c_void_p(dst.data_ptr()), dst.stride(0), _stream_ptr()), "gpu_image")
    return dst


def gpu_image(image: np.ndarray, grayscale: bool = True) -> np.ndarray:
    """getGPUImage (cuda_bimp.cu:156-180): upscale below 350 px and BGR -> grey
    on the device; returns the host copy of the result."""
    torch = _torch()
    img = np.ascontiguousarray(image, dtype=np.uint8)
    h, w = img.shape[:2]
    cn = 1 if img.ndim == 2 else img.shape[2]
    ow, oh = C.c_int(), C.c_int()
    L.check(L.lib().bimp_min_size_dims(w, h, C.byref(ow), C.byref(oh), None), "min_size_dims")
    ocn = 1 if (grayscale or cn == 1) else cn
    src = torch.from_numpy(img.reshape(h, w * cn)).cuda()
    dst = torch.empty((oh.value, ow.value * ocn), dtype=torch.uint8, device="cuda")
    L.check(L.lib().bimp_gpu_image(C.c_void_p(src.data_ptr()), src.stride(0), w, h, cn, int(bool(grayscale)),
                                   C.c_void_p(dst.data_ptr()), dst.stride(0), _stream_ptr()), "gpu_image")
    out = dst.cpu().numpy()
    return out if ocn == 1 else out.reshape(oh.value, ow.value, ocn)


def color_features(kp, bgr: np.ndarray) -> np.ndarray:
    """addColorFeatures (cuda_bimp.cu:950-958): 24-bin colour histograms of
    the keypoints in the 7 x n device matrix over a BGR image."""
    torch = _torch()
    img = np.ascontiguousarray(bgr, dtype=np.uint8)
    h, w = img.shape[:2]
    n = kp.shape[1]
    src = torch.from_numpy(img.reshape(h, w * 3)).cuda()
    desc = torch.empty((max(n, 1), 24), dtype=torch.float32, device="cuda")
    L.check(L.lib().bimp_color_features(C.c_void_p(kp.data_ptr()), kp.stride(0), n, C.c_void_p(src.data_ptr()),
                                        src.stride(0), w, h, C.c_void_p(desc.data_ptr()), desc.stride(0),
                                        _stream_ptr()), "color_features")
    return desc[:n].cpu().numpy()


def keypoint_matrix_to_records(kp) -> np.ndarray:
    """7 x n device matrix -> structured numpy array (host)."""
    h = kp.detach().cpu().numpy()
    rec = np.zeros(h.shape[1], dtype=[("x", "f4"), ("y", "f4"), ("size", "f4"), ("angle", "f4"),
                                      ("response", "f4"), ("octave", "i4"), ("class_id", "i4")])
    rec["x"] = h[X_ROW]
    rec["y"] = h[Y_ROW]
    rec["size"] = h[SIZE_ROW]
    rec["angle"] = h[ANGLE_ROW]
    rec["response"] = h[HESSIAN_ROW]
    rec["octave"] = h[OCTAVE_ROW].view(np.int32)
    rec["class_id"] = h[LAPLACIAN_ROW].view(np.int32)
    return rec


class Context:
    """bimp::Context (bimp.hpp:19-51, bimp.cpp:7-129) for grey or BGR uint8
    images.

    As in the reference: the bank is makeLambdasLog(4, 64, 2) (bimp.cpp:8);
    the image goes through getGPUImage (grey; upscaled when a side is below
    350 pixels; the colour image is kept for the colour histogram);
    CudaStuff is built from the image's own size (bimp.cpp:7-8), so an
    upscaled image is filtered on the top-left window of each pyramid level;
    width()/height() are the uploaded image's.
    """

    def __init__(self, image, lambdas=None, params=None):
        img = np.asarray(image)
        if img.dtype != np.uint8 or img.ndim not in (2, 3) or (img.ndim == 3 and img.shape[2] != 3):
            raise ValueError("Context expects a grey or BGR uint8 image")
        self.lambdas = list(lambdas) if lambdas is not None else makeLambdasLog(4, 64, 2)
        h, w = img.shape[:2]
        self.cuda_data = CudaStuff(w, h, self.lambdas, params, input_size=min_size_dims(w, h))
        self.current_keypoints = None
        self.capacity = KP_MAX_POINTS   # keypoint limit, as KP_MAX_POINTS (bimp::Context::capacity)
        self.loadImage(img)

    def width(self) -> int:
        return int(self.current_image.shape[1])

    def height(self) -> int:
        return int(self.current_image.shape[0])

    def loadImage(self, new_image):
        """A host image (numpy, through getGPUImage) or a grey uint8 CUDA
        tensor of the uploaded size (loadImage(GpuMat))."""
        torch = _torch()
        if isinstance(new_image, torch.Tensor):
            grey, colour = _as_gpu_u8(new_image), None
        else:
            img = np.asarray(new_image)
            grey = gpu_image_device(img, grayscale=True)
            colour = gpu_image_device(img, grayscale=False) if img.ndim == 3 else None
        if tuple(grey.shape) != (self.cuda_data.input_height, self.cuda_data.input_width):
            raise ValueError("loadImage: size differs from the context's")
        self.current_image = grey
        self.current_image_color = colour
        self.has_changed_keypoints = True

    def getKeypoints(self):
        if self.has_changed_keypoints:
            self.current_keypoints = getKeypoints(self.current_image, self.cuda_data, capacity=self.capacity)
            self.has_changed_keypoints = False
        return self.current_keypoints

    def getKeypointsAndDownload(self) -> list:
        return downloadKeypoints(self.getKeypoints())

    def getResponses(self) -> list:
        """Per-scale geometry with the summed keypoint map D and the
        single-stopped map S."""
        self.getKeypoints()
        out = []
        for i, k in enumerate(self.cuda_data.ks):
            out.append(dict(k, D=self.cuda_data.dense_map(i, 0), S=self.cuda_data.dense_map(i, 1)))
        return out

    def getColorFeatures(self) -> np.ndarray:
        """24-bin colour histograms of the current keypoints (n x 24)."""
        if self.current_image_color is None:
            raise ValueError("the image has no colour")
        h, w3 = self.current_image_color.shape
        img = self.current_image_color.cpu().numpy().reshape(h, w3 // 3, 3)
        return color_features(self.getKeypoints(), img)


class Pipeline:
    """Host frames in flight (bimp_pipeline_*): push() enqueues a uint8 host
    frame and returns at once, pop() returns the oldest frame's records as a
    structured array (the layout of detect_host).  Up to `depth` frames are
    in flight, so one frame's copies overlap another's kernels.  A pushed
    frame's memory must stay unchanged until it is popped (this class keeps a
    reference to it)."""

    def __init__(self, width: int, height: int, lambdas, depth: int = 3, capacity: int = KP_MAX_POINTS,
                 params=None):
        lam = (C.c_float * len(lambdas))(*[float(x) for x in lambdas])
        p = _params(params)
        h = C.c_void_p()
        L.check(L.lib().bimp_pipeline_create(C.byref(h), int(width), int(height), lam, len(lambdas),
                                             C.byref(p) if p is not None else None, int(depth), int(capacity)),
                "Pipeline")
        self._h = h
        self.width, self.height, self.depth, self.capacity = int(width), int(height), int(depth), int(capacity)
        self._frames = []
        self._out = (L.KeyPointC * self.capacity)()

    def in_flight(self) -> int:
        return int(L.lib().bimp_pipeline_in_flight(self._h))

    def push(self, image: np.ndarray):
        img = np.asarray(image)
        if img.dtype != np.uint8 or img.shape != (self.height, self.width) or img.strides[1] != 1:
            raise ValueError("expected a uint8 host image of the pipeline's size (rows contiguous)")
        L.check(L.lib().bimp_pipeline_push(self._h, C.c_void_p(img.ctypes.data), img.strides[0], self.width,
                                           self.height), "pipeline_push")
        self._frames.append(img)

    def pop(self, capacity: int | None = None):
        """(records, total, status) of the oldest frame in flight."""
        cap = self.capacity if capacity is None else int(capacity)
        n = C.c_int(0)
        rc = L.lib().bimp_pipeline_pop(self._h, self._out, cap, C.byref(n))
        if rc not in (L.BIMP_OK, L.BIMP_ERR_CAPACITY):
            L.check(rc, "pipeline_pop")
        self._frames.pop(0)
        m = min(n.value, cap, self.capacity)
        rec = np.frombuffer(self._out, dtype=_HOST_RECORD, count=m).copy()
        return rec, n.value, rc

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.lib().bimp_pipeline_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many images of mixed sizes, one CUDA-graph replay per detection."""

    def __init__(self, sizes, lambdas, params=None, kp_capacity: int = 65536):
        n = len(sizes)
        ws = (C.c_int * n)(*[int(w) for w, h in sizes])
        hs = (C.c_int * n)(*[int(h) for w, h in sizes])
        lam = (C.c_float * len(lambdas))(*[float(x) for x in lambdas])
        p = _params(params)
        h = C.c_void_p()
        L.check(L.lib().bimp_batch_create(C.byref(h), ws, hs, n, lam, len(lambdas),
                                          C.byref(p) if p is not None else None, kp_capacity),
                "Batch")
        self._h = h
        self.sizes = [(int(w), int(hh)) for w, hh in sizes]
        self.kp_capacity = kp_capacity
        self._inputs = []
        torch = _torch()
        for i in range(n):
            ptr = C.c_void_p()
            pitch = C.c_size_t()
            L.check(L.lib().bimp_batch_image(h, i, C.byref(ptr), C.byref(pitch)), "batch_image")
            self._inputs.append((ptr.value, pitch.value))
        self._counts = torch.zeros(n, dtype=torch.int32, device="cuda")

    def input_view(self, i: int):
        """(pointer, pitch) of image i's device input buffer."""
        return self._inputs[i]

    def input_tensor(self, i: int):
        """uint8 CUDA tensor (h x w, row stride = pitch) aliasing image i's input."""
        ptr, pitch = self._inputs[i]
        w, h = self.sizes[i]
        return _wrap_device(ptr, (h, w), (pitch, 1), "|u1")

    def load(self, images, stream=None):
        """Copy uint8 images (numpy or CUDA tensors) into the batch inputs."""
        torch = _torch()
        with torch.cuda.stream(stream) if stream is not None else _nullcontext():
            for i, img in enumerate(images):
                img = _as_gpu_u8(img)
                if tuple(img.shape) != (self.sizes[i][1], self.sizes[i][0]):
                    raise ValueError(f"image {i} has shape {tuple(img.shape)}, batch expects {self.sizes[i]}")
                self.input_tensor(i).copy_(img, non_blocking=True)

    def run(self, stream=None):
        L.check(L.lib().bimp_batch_run(self._h, _stream_ptr(stream)), "batch_run")

    def set_tile_plan(self, policy: int, order: int, grid: int = 0, kernel: int = 1):
        """Use a tile plan (bimp_batch_set_tile_plan); grid <= 0: one CTA per
        tile; kernel 1: warp-specialised tile kernel where it fits, 0: phased."""
        L.check(L.lib().bimp_batch_set_tile_plan(self._h, int(policy), int(order), int(grid), int(kernel)),
                "batch_tile_plan")

    def autotune(self, reps: int = 5, stream=None) -> dict:
        """Time every tile plan on the loaded images, keep the fastest
        (bimp_batch_autotune); returns the chosen plan and all timings."""
        chosen = L.TilePlan()
        tried = (L.TilePlan * 32)()
        n = C.c_int()
        L.check(L.lib().bimp_batch_autotune(self._h, _stream_ptr(stream), int(reps), C.byref(chosen), tried, 32,
                                            C.byref(n)), "batch_autotune")
        return {"chosen": chosen.as_dict(), "tried": [tried[i].as_dict() for i in range(n.value)]}

    def counts(self, stream=None):
        L.check(L.lib().bimp_batch_counts(self._h, C.c_void_p(self._counts.data_ptr()),
                                          _stream_ptr(stream)), "batch_counts")
        return self._counts

    def scale_info(self, i: int, scale: int) -> dict:
        """Geometry of image i at one scale (bimp_batch_scale_info)."""
        si = L.ScaleInfo()
        L.check(L.lib().bimp_batch_scale_info(self._h, int(i), int(scale), C.byref(si)), "batch_scale_info")
        return {f: getattr(si, f) for f, _ in L.ScaleInfo._fields_}

    def dense_map(self, i: int, scale: int):
        """Summed keypoint map D of image i, scale `scale` from the last run
        (bimp_batch_dense_map)."""
        torch = _torch()
        k = self.scale_info(i, scale)
        out = torch.empty((k["data_h"], k["data_w"]), dtype=torch.float32, device="cuda")
        L.check(L.lib().bimp_batch_dense_map(self._h, int(i), int(scale), C.c_void_p(out.data_ptr()),
                                             out.stride(0), _stream_ptr()), "batch_dense_map")
        return out

    def keypoints(self, i: int):
        torch = _torch()
        ptr = C.c_void_p()
        ld = C.c_size_t()
        L.check(L.lib().bimp_batch_keypoints_device(self._h, i, C.byref(ptr), C.byref(ld)),
                "batch_keypoints")
        n = int(self.counts()[i].item())
        n = min(n, self.kp_capacity)
        # wrap the internal matrix without copying
        buf = _wrap_device(ptr.value, (KP_VECTOR_LENGTH, ld.value), (4 * ld.value, 4), "<f4")
        return buf[:, :n]

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.lib().bimp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """Gradient of L = sum M * D (summed keypoint maps) for n float images.

    forward(images, masks) -> loss; backward() -> (dL/dimages, dL/d(alpha,
    rho, w_tan, w_rad)).  images: float32 CUDA tensor (n, H, W); masks: float32
    CUDA tensor of n * mask_stride elements laid out by mask_views().
    """

    def __init__(self, width: int, height: int, n_images: int, lambdas, params=None):
        lam = (C.c_float * len(lambdas))(*[float(x) for x in lambdas])
        p = _params(params)
        h = C.c_void_p()
        L.check(L.lib().bimp_adjoint_create(C.byref(h), int(width), int(height), int(n_images), lam, len(lambdas),
                                            C.byref(p) if p is not None else None), "Adjoint")
        self._h = h
        self.params = p if p is not None else default_params()
        self.width, self.height, self.n = int(width), int(height), int(n_images)
        self.layout = []
        for s in range(L.lib().bimp_adjoint_num_scales(h)):
            w, hh, off, stride = C.c_int(), C.c_int(), C.c_size_t(), C.c_size_t()
            L.check(L.lib().bimp_adjoint_mask_layout(h, s, C.byref(w), C.byref(hh), C.byref(off), C.byref(stride)),
                    "mask_layout")
            self.layout.append((off.value, w.value, hh.value))
            self.mask_stride = stride.value
        torch = _torch()
        self._loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        self._gp = torch.zeros(4, dtype=torch.float64, device="cuda")

    def mask_views(self, masks):
        """[(image, scale) -> (h, w) view] of a flat mask tensor."""
        return [[masks[i * self.mask_stride + off:i * self.mask_stride + off + w * h].view(h, w)
                 for (off, w, h) in self.layout] for i in range(self.n)]

    def forward(self, images, masks, stream=None):
        assert images.dtype == _torch().float32 and images.is_contiguous() and masks.is_contiguous()
        L.check(L.lib().bimp_adjoint_forward(self._h, C.c_void_p(images.data_ptr()), images.shape[-1],
                                             C.c_void_p(masks.data_ptr()), C.c_void_p(self._loss.data_ptr()),
                                             _stream_ptr(stream)), "adjoint_forward")
        return self._loss

    def backward(self, grad=None, stream=None):
        torch = _torch()
        if grad is None:
            grad = torch.empty((self.n, self.height, self.width), dtype=torch.float32, device="cuda")
        L.check(L.lib().bimp_adjoint_backward(self._h, C.c_void_p(grad.data_ptr()), grad.shape[-1],
                                              C.c_void_p(self._gp.data_ptr()), _stream_ptr(stream)),
                "adjoint_backward")
        return grad, self._gp

    def dense_map(self, image: int, scale: int):
        torch = _torch()
        off, w, h = self.layout[scale]
        out = torch.empty((h, w), dtype=torch.float32, device="cuda")
        L.check(L.lib().bimp_adjoint_dense_map(self._h, image, scale, C.c_void_p(out.data_ptr()), out.stride(0),
                                               _stream_ptr()), "adjoint_dense_map")
        return out

    def complex_map(self, image: int, scale: int, orientation: int):
        """|e + i o| of the last forward over the stencil window, (h+1, w+1)."""
        torch = _torch()
        off, w, h = self.layout[scale]
        out = torch.empty((h + 1, w + 1), dtype=torch.float32, device="cuda")
        L.check(L.lib().bimp_adjoint_complex_map(self._h, image, scale, orientation, C.c_void_p(out.data_ptr()),
                                                 out.stride(0), _stream_ptr()), "adjoint_complex_map")
        return out

    def device_bytes(self) -> int:
        return int(L.lib().bimp_adjoint_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.lib().bimp_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _wrap_device(ptr: int, shape, strides_bytes, typestr: str):
    """A CUDA tensor aliasing library-owned device memory (no copy)."""
    torch = _torch()

    class _Arr:
        __cuda_array_interface__ = {"shape": tuple(shape), "strides": tuple(strides_bytes),
                                    "typestr": typestr, "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Arr(), device="cuda")


class _nullcontext:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


__all__ = ["KeyPoint", "CudaStuff", "Context", "Batch", "getKeypoints", "downloadKeypoints",
           "uploadKeypoints", "makeLambdasLog", "makeLambdasLin", "snapTransformSize", "detect_host",
           "keypoint_matrix_to_records", "default_params", "KP_MAX_POINTS", "gpu_image", "color_features", "Adjoint"]

if sys.version_info < (3, 8):  # pragma: no cover
    raise RuntimeError("python >= 3.8 required")
