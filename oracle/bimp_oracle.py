"""FP64 CPU oracle for BIMP keypoint extraction (test infrastructure only).

This module is the CHECKER for the CUDA path.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it; the product path never does.

It restates, in float64 numpy, the per-scale pipeline of
daniel-koudouna/cuda-bimp (files cited relative to the reference project):

* wavelength list ............ bimp/src/cuda_bimp.cu:927-937 (makeLambdasLog)
* per-scale geometry ......... bimp/src/cuda_bimp.cu:222-256, :200-219
* Gabor taps ................. bimp/src/cuda_bimp.cu:241-250, :304-331
* pyramid + conversion ....... bimp/src/cuda_bimp.cu:472-486 (cv::cuda::pyrDown,
                               convertTo 255/65536, collectCVMemory
                               bimp/include/detection/cuda_bimp.cuh:151-163)
* torus padding .............. bimp/include/detection/convolutionFFT2D.cuh:31-49
                               (kernel, centre at (0,0) with wrap) and :56-85
                               (data: copy / clamp-to-last / clamp-to-first)
* spectral filtering ......... bimp/include/detection/cuda_bimp.cuh:226-248 and
                               the R2C/C2R calls at bimp/src/cuda_bimp.cu:498-515
* complex cells .............. bimp/include/detection/cuda_bimp.cuh:165-180
* end-stopped cells .......... bimp/include/detection/cuda_bimp.cuh:436-467,
                               offsets bimp/src/cuda_bimp.cu:533-539
* inhibition ................. bimp/include/detection/cuda_bimp.cuh:469-502,
                               offsets bimp/src/cuda_bimp.cu:541-550
* summed keypoint map ........ bimp/include/detection/cuda_bimp.cuh:504-517
* threshold + NMS ............ bimp/src/cuda_bimp.cu:714-743, :960-966, :73-85
* keypoint records ........... bimp/include/detection/cuda_bimp.cuh:86-148,
                               bimp/src/utils.cpp:130-150 (downloadKeypoints)

Parity status: UNPINNED against the reference's own outputs.  The reference
has no tests, golden vectors or fixtures, and it cannot be built in this
environment (C++ OpenCV 3.x with CUDA/contrib modules, CUDA-samples helper
headers and CUDA<=11 texture references are all required).  The pyramid stage
alone is pinned against ``cv2.pyrDown`` (the reference's ``resize_cpu``
branch, bimp/src/cuda_bimp.cu:657-667) away from exact rounding ties, and the
restatement is cross-checked against the independent FP32 C restatement in
``oracle/cbimp.c``.

Deliberate, documented choices where the reference is undefined:

* The stencils address the complex-cell buffer as ``y*fftW + x`` with an
  inclusive upper bound, so they can read one row past the data.  When
  ``fftH == dataH`` that row lies outside the level's FFT grid (the reference
  reads stale or out-of-allocation memory).  Here the flat index wraps modulo
  ``fftH*fftW``.
* When a Gabor kernel is larger than the FFT grid the reference's padKernel
  writes out of bounds; here taps wrap onto the torus and add.
* The uint8 pyramid rounds exact .5 ties half-to-even (CUDA ``cvt.rni``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

NUM_ORI = 8
KP_MAX_POINTS = 8000

f32 = np.float32


# ---------------------------------------------------------------------------
# parameters (the reference hard-codes these; names follow the reference)
# ---------------------------------------------------------------------------
@dataclass
class Params:
    """Model constants of bimp/src/cuda_bimp.cu (defaults = reference values)."""

    gamma: float = 0.5          # :241 aspect, multiplies the squared term
    sigma_ratio: float = 0.56   # :243 sigma = 0.56 * lambda
    size_ratio: float = 7.0     # :245 filtersize = 7 * lambda
    offset_ratio: float = 0.6   # :535 offsets = round(0.6 * lambda * trig)
    level_max: float = 7.5      # :236 pyramid step while lambda/pyrstep >= 7.5
    radial_gain: float = 16.0   # cuda_bimp.cuh:497 radial inhibition gain
    w_tan: float = 1.0          # cuda_bimp.cuh:514 weight of tangential inhibition
    w_rad: float = 1.0          # cuda_bimp.cuh:514 weight of radial inhibition
    thresh_ratio: float = 0.104  # cuda_bimp.cu:721


# ---------------------------------------------------------------------------
# wavelength lists and per-scale geometry
# ---------------------------------------------------------------------------
def make_lambdas_log(start: float, end: float, scales_per_octave: int) -> list[float]:
    """float32 restatement of makeLambdasLog (bimp/src/cuda_bimp.cu:927-937)."""
    mult = f32(2.0 ** (1.0 / scales_per_octave))
    lam = f32(start)
    out = []
    while float(lam) <= float(f32(end)) * 1.05:
        out.append(float(lam))
        lam = f32(lam * mult)
    return out


def make_lambdas_lin(start: float, end: float, num: int) -> list[float]:
    """float32 restatement of makeLambdasLin (bimp/src/cuda_bimp.cu:905-921)."""
    step = f32(1.0)
    if num > 1:
        step = f32((f32(end) - f32(start)) / f32(num - 1))
    return [float(f32(f32(start) + f32(s - 1) * step)) for s in range(1, num + 1)]


def snap_transform_size(n: int) -> int:
    """snapTransformSize (bimp/src/cuda_bimp.cu:200-219)."""
    n = (n + 15) // 16 * 16
    hi = n.bit_length() - 1
    if (1 << hi) == n:
        return n
    if (1 << (hi + 1)) <= 1024:
        return 1 << (hi + 1)
    return (n + 511) // 512 * 512


@dataclass
class Scale:
    lambda2: float        # requested wavelength (full resolution)
    pyrstep: float        # power-of-two pyramid step
    lam: float            # wavelength at the pyramid level
    filtersize: float     # float filter size (used by the DC correction)
    kW: int
    kX: int
    dataW: int
    dataH: int
    fftW: int
    fftH: int
    levels: int           # number of pyrDown applications
    es_off: list = field(default_factory=list)   # end-stop (o1 row, o2 col)
    in_off: list = field(default_factory=list)   # inhibition (o1 row, o2 col)
    off: int = 0          # keypoint margin (int)lambda


def _round_half_away(v: float) -> int:
    return int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)


def scale_geometry(width: int, height: int, lambdas, p: Params = Params()) -> list[Scale]:
    """CudaStuff constructor geometry (bimp/src/cuda_bimp.cu:222-256)."""
    out = []
    for l2 in sorted(float(f32(x)) for x in lambdas):
        l2f = f32(l2)
        pyr = f32(1.0)
        while float(f32(l2f / pyr)) >= p.level_max:
            pyr = f32(pyr * 2)
        lam = f32(l2f / pyr)
        fs = f32(f32(p.size_ratio) * lam)
        if int(fs) % 2 == 0:
            fs = f32(fs + 1)
        kX = int(math.floor(float(f32(fs / f32(2)))))
        kW = int(fs)
        dataH = int(f32(height) / pyr)
        dataW = int(f32(width) / pyr)
        sc = Scale(lambda2=float(l2f), pyrstep=float(pyr), lam=float(lam), filtersize=float(fs),
                   kW=kW, kX=kX, dataW=dataW, dataH=dataH,
                   fftW=snap_transform_size(dataW), fftH=snap_transform_size(dataH),
                   levels=int(round(math.log2(float(pyr)))))
        for o in range(NUM_ORI):
            th = f32(o * math.pi / NUM_ORI)
            c = float(np.cos(th, dtype=np.float32))
            s = float(np.sin(th, dtype=np.float32))
            # cuda_bimp.cu:535-536 and :546-547 (double products, C round())
            sc.es_off.append((_round_half_away(p.offset_ratio * float(lam) * c),
                              _round_half_away(p.offset_ratio * float(lam) * s)))
            sc.in_off.append((_round_half_away(p.offset_ratio * float(lam) * s),
                              _round_half_away(p.offset_ratio * float(lam) * c)))
        sc.off = int(lam)  # cuda_bimp.cu:737 int off = k.lambda
        out.append(sc)
    return out


# ---------------------------------------------------------------------------
# Gabor bank (float32 arithmetic as on the reference host)
# ---------------------------------------------------------------------------
def gabor_taps(sc: Scale, o: int, p: Params = Params()):
    """Even/odd Gabor taps of one orientation (bimp/src/cuda_bimp.cu:304-331).

    Returns float32 arrays (kW, kW); the even kernel has its DC removed with
    the reference's float ``filtersize`` divisor.
    """
    lam = f32(sc.lam)
    sigma = f32(float(lam) * p.sigma_ratio)
    sigsq = f32(sigma * sigma)
    gamma = f32(p.gamma)
    phi = f32(-math.pi / 2)
    th = f32(o * math.pi / NUM_ORI)
    s = np.sin(th, dtype=np.float32)
    c = np.cos(th, dtype=np.float32)
    n = sc.kW
    idx = np.arange(n, dtype=np.int64)
    x = (idx[None, :] - sc.kX).astype(np.float32)
    y = (idx[:, None] - sc.kX).astype(np.float32)
    a = (x * c + y * s).astype(np.float32)
    b = (y * c - x * s).astype(np.float32)
    coef = f32(f32(-1.0) / f32(f32(2.0) * sigsq))
    quad = (a * a + (gamma * b) * b).astype(np.float32)
    env = np.exp((coef * quad).astype(np.float32)).astype(np.float32)
    freq = (2.0 * math.pi * a.astype(np.float64) / float(lam)).astype(np.float32)
    even = (env * np.cos(freq).astype(np.float32)).astype(np.float32)
    odd = (env * np.cos((freq + phi).astype(np.float32)).astype(np.float32)).astype(np.float32)
    evensum = f32(0.0)
    for v in even.ravel():          # row-major float accumulation (:326)
        evensum = f32(evensum + v)
    fs = f32(sc.filtersize)
    even = (even - f32(evensum / f32(fs * fs))).astype(np.float32)
    return even, odd


# ---------------------------------------------------------------------------
# pyramid (uint8, 5-tap Gaussian, reflect-101, round half to even)
# ---------------------------------------------------------------------------
def _reflect101(i: np.ndarray, n: int) -> np.ndarray:
    if n == 1:
        return np.zeros_like(i)
    period = 2 * n - 2
    i = np.abs(i) % period
    return np.where(i >= n, period - i, i)


def pyr_down_u8(img: np.ndarray) -> np.ndarray:
    """cv::cuda::pyrDown on CV_8UC1 (called at bimp/src/cuda_bimp.cu:476).

    out(y,x) = rint(sum_ij w_i w_j src(r101(2y+i), r101(2x+j)) / 256) with
    w = [1,4,6,4,1]; the sum is an exact integer so the only rounding is the
    final half-to-even conversion.  Output size ceil(w/2) x ceil(h/2).
    """
    h, w = img.shape
    oh, ow = (h + 1) // 2, (w + 1) // 2
    wts = (1, 4, 6, 4, 1)
    src = img.astype(np.int64)
    rows = _reflect101(2 * np.arange(oh)[:, None] + np.arange(-2, 3)[None, :], h)
    tmp = sum(wts[k] * src[rows[:, k], :] for k in range(5))
    cols = _reflect101(2 * np.arange(ow)[:, None] + np.arange(-2, 3)[None, :], w)
    acc = sum(wts[k] * tmp[:, cols[:, k]] for k in range(5))
    q, r = np.divmod(acc, 256)
    up = (r > 128) | ((r == 128) & (q % 2 == 1))
    return np.clip(q + up, 0, 255).astype(np.uint8)


def pyr_down_f(img: np.ndarray) -> np.ndarray:
    """Float pyramid step (no uint8 rounding), used by the adjoint workload."""
    h, w = img.shape
    oh, ow = (h + 1) // 2, (w + 1) // 2
    wts = np.array([1, 4, 6, 4, 1], dtype=np.float64) / 16.0
    rows = _reflect101(2 * np.arange(oh)[:, None] + np.arange(-2, 3)[None, :], h)
    tmp = sum(wts[k] * img[rows[:, k], :] for k in range(5))
    cols = _reflect101(2 * np.arange(ow)[:, None] + np.arange(-2, 3)[None, :], w)
    return sum(wts[k] * tmp[:, cols[:, k]] for k in range(5))


def level_image(img_u8: np.ndarray, sc: Scale) -> np.ndarray:
    """dataH x dataW float64 level image = 255*u8/65536 of the repeated pyrDown.

    bimp/src/cuda_bimp.cu:473-486: the top-left dataW x dataH window is kept
    when pyrDown's ceil() size exceeds the floor() data size.
    """
    cur = img_u8
    for _ in range(sc.levels):
        cur = pyr_down_u8(cur)
    return cur[:sc.dataH, :sc.dataW].astype(np.float64) * (255.0 / 65536.0)


# ---------------------------------------------------------------------------
# torus filtering
# ---------------------------------------------------------------------------
def pad_map(n_fft: int, n_data: int, k_half: int) -> np.ndarray:
    """Source index of each padded row/col (convolutionFFT2D.cuh:56-85)."""
    t = np.arange(n_fft)
    return np.where(t < n_data, t, np.where(t < n_data + k_half, n_data - 1, 0))


def padded_image(data: np.ndarray, sc: Scale) -> np.ndarray:
    ry = pad_map(sc.fftH, sc.dataH, sc.kX)
    rx = pad_map(sc.fftW, sc.dataW, sc.kX)
    return data[ry[:, None], rx[None, :]]


def padded_kernel(taps: np.ndarray, sc: Scale) -> np.ndarray:
    """Kernel centre at (0,0) with wrap (convolutionFFT2D.cuh:31-49); taps add."""
    out = np.zeros((sc.fftH, sc.fftW), dtype=np.float64)
    k = np.arange(sc.kW)
    ry = (k - sc.kX) % sc.fftH
    rx = (k - sc.kX) % sc.fftW
    np.add.at(out, (ry[:, None], rx[None, :]), taps.astype(np.float64))
    return out


def complex_cells(data: np.ndarray, sc: Scale, p: Params = Params()):
    """C_o = |circconv(Ip, Pe_o) + i circconv(Ip, Po_o)| on the fftH x fftW torus.

    Returns (C[8, fftH, fftW], E[8], O[8]) in float64.
    """
    Ip = padded_image(data, sc)
    X = np.fft.rfft2(Ip)
    C = np.empty((NUM_ORI, sc.fftH, sc.fftW))
    E = np.empty_like(C)
    O = np.empty_like(C)
    for o in range(NUM_ORI):
        ke, ko = gabor_taps(sc, o, p)
        E[o] = np.fft.irfft2(X * np.fft.rfft2(padded_kernel(ke, sc)), s=Ip.shape)
        O[o] = np.fft.irfft2(X * np.fft.rfft2(padded_kernel(ko, sc)), s=Ip.shape)
        C[o] = np.sqrt(E[o] ** 2 + O[o] ** 2)
    return C, E, O


def stencil_window(Ct: np.ndarray, sc: Scale) -> np.ndarray:
    """(dataH+1) x (dataW+1) window read by the stencils with flat addressing.

    Element (r, c) is C_flat[(r*fftW + c) mod (fftH*fftW)] (cuda_bimp.cuh:442).
    """
    F = sc.fftH * sc.fftW
    r = np.arange(sc.dataH + 1)[:, None]
    c = np.arange(sc.dataW + 1)[None, :]
    flat = (r * sc.fftW + c) % F
    return Ct.reshape(Ct.shape[:-2] + (F,))[..., flat]


def stencil_masks(sc: Scale, o1: int, o2: int) -> np.ndarray:
    """Pixels where the reference's bounds test passes (cuda_bimp.cuh:445-449)."""
    y = np.arange(sc.dataH)[:, None]
    x = np.arange(sc.dataW)[None, :]
    ok = np.ones((sc.dataH, sc.dataW), dtype=bool)
    for m in (1, 2):
        for sgn in (-1, 1):
            xx = x + sgn * m * o2
            yy = y + sgn * m * o1
            ok &= (xx >= 0) & (xx <= sc.dataW) & (yy >= 0) & (yy <= sc.dataH)
    return ok


def _shift(Cw: np.ndarray, dy: int, dx: int, dataH: int, dataW: int) -> np.ndarray:
    """Cw[y+dy, x+dx] for the data grid, clipped (masked entries are unused)."""
    y = np.clip(np.arange(dataH) + dy, 0, dataH)
    x = np.clip(np.arange(dataW) + dx, 0, dataW)
    return Cw[y[:, None], x[None, :]]


def keypoint_maps(Cw: np.ndarray, sc: Scale, p: Params = Params()):
    """End-stopping, inhibition and the summed keypoint map in float64.

    Cw: (8, dataH+1, dataW+1) stencil windows.  Returns dict with S, D (after
    inhibition), T, R and the pre-inhibition D0/S0 (cuda_bimp.cuh:436-517).
    """
    H, W = sc.dataH, sc.dataW
    S = np.zeros((H, W))
    D = np.zeros((H, W))
    T = np.zeros((H, W))
    R = np.zeros((H, W))
    for o in range(NUM_ORI):
        o1, o2 = sc.es_off[o]
        m = stencil_masks(sc, o1, o2)
        C = Cw[o]
        s = np.maximum(_shift(C, -o1, o2, H, W) - _shift(C, o1, -o2, H, W), 0.0)
        d = np.maximum(_shift(C, 0, 0, H, W) - 0.5 * _shift(C, -2 * o1, 2 * o2, H, W)
                       - 0.5 * _shift(C, 2 * o1, -2 * o2, H, W), 0.0)
        S += np.where(m, s, 0.0)
        D += np.where(m, d, 0.0)
    for o in range(NUM_ORI):
        op = (o + NUM_ORI // 2) % NUM_ORI
        o1, o2 = sc.in_off[o]
        m = stencil_masks(sc, o1, o2)
        C = Cw[o]
        Cp = Cw[op]
        centre = _shift(C, 0, 0, H, W)
        t = np.maximum(_shift(C, -o1, -o2, H, W) - centre, 0.0)
        h1 = _round_half_away(0.5 * o1)
        h2 = _round_half_away(0.5 * o2)
        r = np.maximum(centre - p.radial_gain * _shift(Cp, h1, h2, H, W), 0.0)
        r = np.maximum(r + centre - p.radial_gain * _shift(Cp, -h1, -h2, H, W), 0.0)
        T += np.where(m, t, 0.0)
        R += np.where(m, r, 0.0)
    inhib = p.w_tan * T + p.w_rad * R
    return {"S0": S, "D0": D, "T": T, "R": R, "D": D - inhib, "S": S - inhib}


# ---------------------------------------------------------------------------
# keypoint extraction
# ---------------------------------------------------------------------------
def dilate8(D: np.ndarray) -> np.ndarray:
    """3x3 max with the centre masked out, reflect-101 border (cuda_bimp.cu:73-85)."""
    H, W = D.shape
    ry = _reflect101(np.arange(-1, H + 1), H)
    rx = _reflect101(np.arange(-1, W + 1), W)
    P = D[ry[:, None], rx[None, :]]
    out = np.full_like(D, -np.inf)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dy == 0 and dx == 0:
                continue
            out = np.maximum(out, P[1 + dy:1 + dy + H, 1 + dx:1 + dx + W])
    return out


@dataclass
class ScaleKeypoints:
    scale: int
    ix: np.ndarray        # integer level position
    iy: np.ndarray
    x: np.ndarray         # full-resolution subpixel position
    y: np.ndarray
    size: float
    octave: int
    response: np.ndarray
    thresh: float
    dmax: float
    # decision margins (for the tie rule): min over all tests of |margin|
    cand_margin: np.ndarray   # per candidate-region pixel
    region: tuple             # (y0, y1, x0, x1) of the candidate region


def extract_keypoints(D: np.ndarray, sc: Scale, scale_index: int, p: Params = Params()):
    """cuda_gpu_keypoints + identifyKeypoints_kernel (cuda_bimp.cu:714-743,
    cuda_bimp.cuh:86-148) in float64, deterministic (scale, y, x) order."""
    H, W = D.shape
    dmax = float(D.max())
    thresh = p.thresh_ratio * dmax
    dil = dilate8(D)
    off = sc.off
    # off < i < W-off (cuda_bimp.cuh:102); the 3x3 support must stay inside
    # the map, which only binds when off == 0
    y0, y1, x0, x1 = off + 1, min(H - off, H - 1), off + 1, min(W - off, W - 1)
    if y1 <= y0 or x1 <= x0:
        z = np.zeros(0)
        return ScaleKeypoints(scale_index, z.astype(int), z.astype(int), z, z,
                              float(f32(f32(sc.lam) * f32(sc.pyrstep))),
                              int(f32(f32(sc.lam) * f32(sc.pyrstep))), z, thresh, dmax,
                              np.zeros((0, 0)), (y0, y1, x0, x1))
    Dr = D[y0:y1, x0:x1]
    loc = Dr - dil[y0:y1, x0:x1]
    keep = (loc > 0) & (Dr > thresh)
    # distance of the decision (loc > 0 and D > thresh) from flipping: a
    # keypoint flips when either margin reaches 0, a non-keypoint only when
    # every failing test is near 0
    dth = Dr - thresh
    margin = np.where(keep, np.minimum(loc, dth),
                      np.maximum(np.where(loc <= 0, -loc, 0.0), np.where(dth <= 0, -dth, 0.0)))
    iy, ix = np.nonzero(keep)
    iy = iy + y0
    ix = ix + x0
    v2 = D[iy, ix]
    xv1, xv3 = D[iy, ix - 1], D[iy, ix + 1]
    yv1, yv3 = D[iy - 1, ix], D[iy + 1, ix]
    dxn = xv1 + xv3 - 2 * v2
    dyn = yv1 + yv3 - 2 * v2
    with np.errstate(divide="ignore", invalid="ignore"):
        xs = ix + np.where(dxn != 0, 0.5 * (xv1 - xv3) / np.where(dxn != 0, dxn, 1), 0.0)
        ys = iy + np.where(dyn != 0, 0.5 * (yv1 - yv3) / np.where(dyn != 0, dyn, 1), 0.0)
    lp = float(f32(f32(sc.lam) * f32(sc.pyrstep)))
    return ScaleKeypoints(scale_index, ix, iy, xs * sc.pyrstep, ys * sc.pyrstep, lp,
                          int(f32(f32(sc.lam) * f32(sc.pyrstep))), v2, thresh, dmax,
                          margin, (y0, y1, x0, x1))


# ---------------------------------------------------------------------------
# whole pipeline
# ---------------------------------------------------------------------------
def run(img_u8: np.ndarray, lambdas, p: Params = Params(), keep_maps: bool = True, geometry_size=None):
    """Full BIMP on one uint8 grayscale image: per-scale maps and keypoints.

    geometry_size (W, H), default the image's own: the size the CudaStuff is
    built for.  The reference's Context builds it from the size of the image
    before getGPUImage upscales it (bimp/src/bimp.cpp:7-8,
    bimp/src/cuda_bimp.cu:156-168); each scale then takes the top-left
    dataW x dataH window of its level of the larger image (convertTo and
    collectCVMemory, bimp/src/cuda_bimp.cu:481-486), which level_image does.
    """
    H, W = img_u8.shape if geometry_size is None else (geometry_size[1], geometry_size[0])
    scales = scale_geometry(W, H, lambdas, p)
    out = []
    for i, sc in enumerate(scales):
        data = level_image(img_u8, sc)
        Ct, _, _ = complex_cells(data, sc, p)
        Cw = stencil_window(Ct, sc)
        maps = keypoint_maps(Cw, sc, p)
        kp = extract_keypoints(maps["D"], sc, i, p)
        rec = {"scale": sc, "kp": kp, "D": maps["D"], "S": maps["S"]}
        if keep_maps:
            rec.update({"Cw": Cw, "T": maps["T"], "R": maps["R"], "data": data})
        out.append(rec)
    return out


def keypoint_table(result) -> np.ndarray:
    """Structured array (scale, iy, ix, x, y, size, octave, response) in order."""
    rows = []
    for r in result:
        kp = r["kp"]
        for j in range(len(kp.ix)):
            rows.append((kp.scale, int(kp.iy[j]), int(kp.ix[j]), float(kp.x[j]), float(kp.y[j]),
                         kp.size, kp.octave, float(kp.response[j])))
    dt = [("scale", "i4"), ("iy", "i4"), ("ix", "i4"), ("x", "f8"), ("y", "f8"),
          ("size", "f8"), ("octave", "i4"), ("response", "f8")]
    return np.array(rows, dtype=dt)


# ---------------------------------------------------------------------------
# input preprocessing (getGPUImage) and the colour histogram
# ---------------------------------------------------------------------------
MIN_SIZE = 350   # bimp/src/cuda_bimp.cu:158


def min_size_dims(width: int, height: int):
    """Upscale rule of getGPUImage (bimp/src/cuda_bimp.cu:160-168): float factor,
    output size rounded to nearest (cv::resize with fx = fy = sf)."""
    sf = 1.0
    if height < MIN_SIZE and width >= MIN_SIZE:
        sf = float(f32(MIN_SIZE / (1.0 * height)))
    elif width < MIN_SIZE:
        sf = float(f32(MIN_SIZE / (1.0 * width)))
    if sf == 1.0:
        return width, height, 1.0
    return int(np.rint(width * sf)), int(np.rint(height * sf)), sf


def _lin_coefs(n_out: int, scale: float, n_in: int):
    f = ((np.arange(n_out) + 0.5) * scale - 0.5).astype(np.float32)
    s = np.floor(f).astype(np.int64)
    f = (f - s).astype(np.float32)
    lo = s < 0
    f = np.where(lo, f32(0), f)
    s = np.where(lo, 0, s)
    hi = s >= n_in - 1
    f = np.where(hi, f32(0), f)
    s = np.where(hi, n_in - 1, s)
    a0 = np.rint((f32(1) - f).astype(np.float32) * f32(2048)).astype(np.int64)
    a1 = np.rint(f * f32(2048)).astype(np.int64)
    return s, np.minimum(s + 1, n_in - 1), a0, a1


def resize_linear_u8(img: np.ndarray, sf: float, out_w: int, out_h: int) -> np.ndarray:
    """cv::resize INTER_LINEAR on uint8 (per channel): 11-bit weights,
    horizontal taps in int, vertical blend with 16-bit multiply-high rounding.
    Unpinned at about 0.1% of pixels (+-1) against cv2 4.13, whose rounding
    depends on the code path; the reference's OpenCV 3.3.1 is not available."""
    src = img.astype(np.int64)
    if src.ndim == 2:
        src = src[..., None]
    H, W = src.shape[:2]
    xs0, xs1, a0, a1 = _lin_coefs(out_w, 1.0 / sf, W)
    ys0, ys1, b0, b1 = _lin_coefs(out_h, 1.0 / sf, H)
    hz = src[:, xs0, :] * a0[None, :, None] + src[:, xs1, :] * a1[None, :, None]
    h0 = hz[ys0] >> 4
    h1 = hz[ys1] >> 4
    y = ((b0[:, None, None] * h0) >> 16) + ((b1[:, None, None] * h1) >> 16)
    out = np.clip((y + 2) >> 2, 0, 255).astype(np.uint8)
    return out[..., 0] if img.ndim == 2 else out


def bgr_to_gray(img: np.ndarray) -> np.ndarray:
    """cv::cuda::cvtColor COLOR_BGR2GRAY: 14-bit fixed-point weights
    round(0.114, 0.587, 0.299 * 2^14) = 1868, 9617, 4899."""
    b, g, r = (img[..., i].astype(np.int64) for i in range(3))
    return ((b * 1868 + g * 9617 + r * 4899 + 8192) >> 14).astype(np.uint8)


def gpu_image(img: np.ndarray, grayscale: bool = True) -> np.ndarray:
    """getGPUImage (bimp/src/cuda_bimp.cu:156-180): upscale, then BGR->grey."""
    h, w = img.shape[:2]
    ow, oh, sf = min_size_dims(w, h)
    out = img if sf == 1.0 else resize_linear_u8(img, sf, ow, oh)
    if img.ndim == 3 and grayscale:
        out = bgr_to_gray(out)
    return out


def color_features(kp_x, kp_y, kp_size, bgr: np.ndarray) -> np.ndarray:
    """addColorFeatures_kernel (bimp/include/detection/cuda_bimp.cuh:8-71).

    8 bins per channel over the open intervals (31.875k, 31.875(k+1)); the
    channel bytes are compared as signed char (values >= 128 count nowhere);
    window [im - p, im + p) with p = (int)(log2(size)/2); each visited pixel
    adds 3 to the normaliser; desc = 0.5 * count / visited (double, stored
    as float).  The reference's test admits one row/column past the image
    (iy == rows, ix == cols); those pixels are counted as visited, not read.
    """
    h, w = bgr.shape[:2]
    thresh = f32(255.0 / 8.0)
    edges = [float(f32(thresh * f32(k))) for k in range(9)]
    out = np.zeros((len(kp_x), 24), dtype=np.float32)
    for i, (x, y, size) in enumerate(zip(kp_x, kp_y, kp_size)):
        cnt = np.zeros(24)
        ix0, iy0 = int(np.float32(x)), int(np.float32(y))
        p = int(np.log2(float(np.float32(size))) / 2.0)
        found = 0
        for iy in range(iy0 - p, iy0 + p):
            if iy < 0 or iy > h:
                continue
            for ix in range(ix0 - p, ix0 + p):
                if ix < 0 or ix > w:
                    continue
                found += 3
                if iy >= h or ix >= w:
                    continue
                for c in range(3):
                    v = int(bgr[iy, ix, c])
                    v = v - 256 if v >= 128 else v
                    for k in range(8):
                        if edges[k] < v < edges[k + 1]:
                            cnt[c * 8 + k] += 1
        with np.errstate(invalid="ignore", divide="ignore"):
            out[i] = (0.5 * cnt) / (found * 1.0)
    return out


# ---------------------------------------------------------------------------
# line and edge detection (detectLE_kernel)
# ---------------------------------------------------------------------------
LE_THRESH = 0.1   # bimp/include/detection/cuda_bimp.cuh:392


def detect_lines_edges(E: np.ndarray, Od: np.ndarray, Ct: np.ndarray, sc: Scale, ch=None):
    """detectLE_kernel (bimp/include/detection/cuda_bimp.cuh:362-432) on the
    data pixels of one scale, from the torus maps E, O, C (8, fftH, fftW).

    ch: summed complex response (dataH, dataW); default sum_o C_o.  Returns
    (result, ori, type, margin): result = C at detected pixels else 0, ori =
    float32(o * 0.392699) there else 0, type 1..4 (positive/negative line,
    positive/negative edge; edges override lines) else 0, and per pixel the
    smallest gap of any comparison the decision made (threshold, dominant
    orientation, extrema, zero crossings, complex-cell maximum).  A pixel
    whose one-pixel step leaves the data is not detected (the reference
    reads past the data there).
    """
    H, W = sc.dataH, sc.dataW
    C = Ct[:, :H, :W]
    if ch is None:
        ch = C.sum(axis=0)
    res = np.zeros((H, W))
    ori = np.zeros((H, W), dtype=np.float32)
    typ = np.zeros((H, W), dtype=np.int8)
    margin = np.full((H, W), np.inf)
    for y in range(H):
        for x in range(W):
            chv = ch[y, x]
            m = abs(chv - LE_THRESH)
            if chv < LE_THRESH:
                margin[y, x] = m
                continue
            c = C[:, y, x]
            maxori, maxresp = -1, 0.0
            for o in range(NUM_ORI):
                if c[o] > maxresp:
                    maxresp, maxori = c[o], o
            srt = np.sort(c)
            m = min(m, srt[-1] - srt[-2], abs(srt[-1]))
            if maxori < 0:
                margin[y, x] = m
                continue
            th = f32(maxori * 0.392699)
            ox = _round_half_away(float(np.cos(th, dtype=np.float32)))
            oy = _round_half_away(float(np.sin(th, dtype=np.float32)))
            xp, yp, xm, ym = x + ox, y + oy, x - ox, y - oy
            if not (0 <= xp < W and 0 <= yp < H and 0 <= xm < W and 0 <= ym < H):
                margin[y, x] = m
                continue
            o0, op, om = Od[maxori, y, x], Od[maxori, yp, xp], Od[maxori, ym, xm]
            e0, ep, em = E[maxori, y, x], E[maxori, yp, xp], E[maxori, ym, xm]
            c0, cp, cm = C[maxori, y, x], C[maxori, yp, xp], C[maxori, ym, xm]
            romax, romin, rozc = o0 > op and o0 > om, o0 < op and o0 < om, op * om < 0
            remax, remin, rezc = e0 > ep and e0 > em, e0 < ep and e0 < em, ep * em < 0
            m = min(m, abs(o0 - op), abs(o0 - om), abs(e0 - ep), abs(e0 - em), abs(op), abs(om), abs(ep),
                    abs(em), abs(c0 - cp), abs(c0 - cm))
            margin[y, x] = m
            if (romax or romin or remax or remin) and (rezc or rozc) and not (c0 <= cp or c0 <= cm):
                t = 4 if (rezc and romin) else 3 if (rezc and romax) else 2 if (rozc and remin) else \
                    1 if (rozc and remax) else 0
                typ[y, x] = t
                ori[y, x] = th
                res[y, x] = c0
    return res, ori, typ, margin
