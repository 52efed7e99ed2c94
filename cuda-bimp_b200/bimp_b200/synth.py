"""Seeded synthetic images for the BIMP workloads.

Content model: a 1/f^2 power-spectrum noise field (mean 128, std 30) with
random filled polygons (3-6 vertices, uniform intensity in [0, 255]) drawn on
top, clipped to [0, 255] and stored as uint8.  No public dataset is used.

Workloads (sizes and banks follow the detector's published configurations):

* ``vga``      one 640x480 image, 20 polygons, wavelengths 4, 8, 16, 32
* ``hd``       one 1920x1080 image, 150 polygons, 8 scales (4*2^(k/2))
* ``mixed``    64 images, W in [320,1920], H in [240,1080] (multiples of 16),
               about 7 polygons per 100k pixels, 8 scales
* ``adjoint``  16 float 512x512 images (the uint8 content / 255), 6 scales
* ``uhd``      32 correlated 3840x2160 frames (subpixel shifts <= 2 px plus
               N(0,2) noise), 12 scales
"""
from __future__ import annotations

import numpy as np


def _noise_field(rng: np.random.Generator, h: int, w: int) -> np.ndarray:
    white = rng.standard_normal((h, w))
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    amp = np.zeros_like(f)
    amp[f > 0] = 1.0 / f[f > 0]          # power ~ 1/f^2  <=>  amplitude ~ 1/f
    field = np.fft.irfft2(np.fft.rfft2(white) * amp, s=(h, w))
    field -= field.mean()
    sd = field.std()
    if sd > 0:
        field /= sd
    return 128.0 + 30.0 * field


def _fill_polygon(img: np.ndarray, xs: np.ndarray, ys: np.ndarray, value: float) -> None:
    """Even-odd fill of pixel centres inside the polygon (xs, ys)."""
    h, w = img.shape
    x0 = max(int(np.floor(xs.min())), 0)
    x1 = min(int(np.ceil(xs.max())) + 1, w)
    y0 = max(int(np.floor(ys.min())), 0)
    y1 = min(int(np.ceil(ys.max())) + 1, h)
    if x1 <= x0 or y1 <= y0:
        return
    px = np.arange(x0, x1)[None, :] + 0.0
    py = np.arange(y0, y1)[:, None] + 0.0
    inside = np.zeros((y1 - y0, x1 - x0), dtype=bool)
    n = len(xs)
    for i in range(n):
        xa, ya = xs[i], ys[i]
        xb, yb = xs[(i + 1) % n], ys[(i + 1) % n]
        if ya == yb:
            continue
        crosses = (ya > py) != (yb > py)
        xint = xa + (py - ya) * (xb - xa) / (yb - ya)
        inside ^= crosses & (px < xint)
    img[y0:y1, x0:x1][inside] = value


def synth_image(width: int, height: int, n_polygons: int, seed: int) -> np.ndarray:
    """One uint8 grayscale image (height x width)."""
    rng = np.random.default_rng(seed)
    img = _noise_field(rng, height, width)
    scale = min(width, height)
    for _ in range(n_polygons):
        nv = int(rng.integers(3, 7))
        cx = rng.uniform(0, width)
        cy = rng.uniform(0, height)
        rad = rng.uniform(0.02, 0.15) * scale
        ang = np.sort(rng.uniform(0, 2 * np.pi, nv))
        rr = rad * rng.uniform(0.5, 1.0, nv)
        _fill_polygon(img, cx + rr * np.cos(ang), cy + rr * np.sin(ang), rng.uniform(0, 255))
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def lambdas_log(start: float, end: float, spo: int) -> list[float]:
    """float32-accumulated wavelength list (same rule as the detector's makeLambdasLog)."""
    mult = np.float32(2.0 ** (1.0 / spo))
    lam = np.float32(start)
    out = []
    while float(lam) <= float(np.float32(end)) * 1.05:
        out.append(float(lam))
        lam = np.float32(lam * mult)
    return out


def bank(n_scales: int) -> list[float]:
    """lambda = 4*2^(k/2), k = 0..n-1, accumulated in float32."""
    return lambdas_log(4.0, 4.0 * 2.0 ** ((n_scales - 1) / 2.0) + 0.01, 2)[:n_scales]


VGA_LAMBDAS = [4.0, 8.0, 16.0, 32.0]


def dequantised(img_u8: np.ndarray, seed: int) -> np.ndarray:
    """float32 (u8 + U(-0.5, 0.5)) / 255: the same picture without exactly
    flat regions."""
    rng = np.random.default_rng(seed)
    return ((img_u8.astype(np.float64) + rng.uniform(-0.5, 0.5, img_u8.shape)) / 255.0).astype(np.float32)


def workload(name: str, seed_base: int = 1000):
    """Return (images, lambdas) for a named workload."""
    if name == "vga":
        return [synth_image(640, 480, 20, seed_base + 0)], list(VGA_LAMBDAS)
    if name == "hd":
        return [synth_image(1920, 1080, 150, seed_base + 1)], bank(8)
    if name == "mixed":
        rng = np.random.default_rng(seed_base + 2)
        imgs = []
        for i in range(64):
            w = int(rng.integers(20, 121)) * 16
            h = int(rng.integers(15, 68)) * 16
            npoly = max(1, int(round(7 * w * h / 1e5)))
            imgs.append(synth_image(w, h, npoly, seed_base + 100 + i))
        return imgs, bank(8)
    if name == "adjoint":
        imgs = [synth_image(512, 512, 20, seed_base + 300 + i).astype(np.float32) / np.float32(255.0)
                for i in range(16)]
        return imgs, bank(6)
    if name == "uhd":
        return uhd_frames(32, seed_base + 4), bank(12)
    raise ValueError(f"unknown workload {name!r}")


def uhd_frames(n: int, seed: int, width: int = 3840, height: int = 2160) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    base = synth_image(width, height, int(round(20 * width * height / (640 * 480))), seed).astype(np.float64)
    frames = [base.astype(np.uint8)]
    cur = base
    fy = np.fft.fftfreq(height)[:, None]
    fx = np.fft.rfftfreq(width)[None, :]
    for _ in range(1, n):
        dx, dy = rng.uniform(-2, 2, 2)
        ph = np.exp(-2j * np.pi * (fx * dx + fy * dy))
        cur = np.fft.irfft2(np.fft.rfft2(cur) * ph, s=cur.shape)
        noisy = cur + rng.normal(0.0, 2.0, cur.shape)
        frames.append(np.clip(np.rint(noisy), 0, 255).astype(np.uint8))
    return frames
