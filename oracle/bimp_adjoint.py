"""FP64 CPU reference for the adjoint of the summed keypoint map (test
infrastructure only: used by tests/ and the CPU legs of bench.py).

Loss  L = sum_s sum_{y,x} M_s[y,x] * D_s[y,x]  for seeded masks M_s, where
D_s is the summed keypoint map of scale s (double-stopped cells minus
w_tan * tangential minus w_rad * radial inhibition,
bimp/include/detection/cuda_bimp.cuh:436-517).  Gradients with respect to

* the float input image X (a float pyramid without uint8 rounding feeds the
  levels; level value = (255*255/65536) * X, the uint8 path's scale for
  X = u8/255),
* alpha: every level wavelength is alpha * lambda (geometry -- kernel size,
  offsets, pyramid step, margins -- frozen at the nominal lambda; the DC
  correction divisor filtersize scales as size_ratio * alpha * lambda),
* rho: sigma = rho * lambda (nominal 0.56),
* w_tan, w_rad: the inhibition weights (nominal 1).

The forward restates bimp_oracle's per-scale pipeline in float64 with taps
computed from the Gabor formula (bimp/src/cuda_bimp.cu:304-331) as
differentiable functions of (alpha, rho); the backward is written out by hand
and checked against central finite differences.  ReLU derivatives are 0 at
0, and |e + i o| <= MAG_FLOOR passes no gradient.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import bimp_oracle as O

KAPPA = 255.0 * 255.0 / 65536.0
# |e + i o| at or below this passes no gradient (the minimal-norm subgradient
# of |z| at 0): exactly flat image regions give z = 0 up to rounding, where
# z/|z| is the direction of rounding noise.  Same value as the CUDA backward.
MAG_FLOOR = 3.0e-5


@dataclass
class Theta:
    alpha: float = 1.0
    rho: float = 0.56
    w_tan: float = 1.0
    w_rad: float = 1.0


def _grid(sc: O.Scale):
    n = sc.kW
    idx = np.arange(n, dtype=np.float64) - sc.kX
    x = idx[None, :]
    y = idx[:, None]
    return x, y


def taps_f64(sc: O.Scale, o: int, th: Theta, p: O.Params = O.Params()):
    """Even/odd taps and their derivatives with respect to alpha and rho.

    Returns dict with e, o, de_da, do_da, de_dr, do_dr (kW x kW float64).
    """
    lam0 = float(sc.lam)
    fs_extra = sc.filtersize - p.size_ratio * lam0          # 0 or 1 (frozen)
    lam = th.alpha * lam0
    sig = th.rho * lam
    fs = p.size_ratio * lam + fs_extra
    t = float(np.float32(o * math.pi / O.NUM_ORI))
    c, s = math.cos(t), math.sin(t)
    x, y = _grid(sc)
    a = x * c + y * s
    b = y * c - x * s
    Q = a * a + p.gamma * b * b
    env = np.exp(-Q / (2 * sig * sig))
    f = 2 * math.pi * a / lam
    cf, sf = np.cos(f), np.sin(f)
    e_raw = env * cf
    od = env * sf
    # partial derivatives at fixed sigma (lambda) and fixed lambda (sigma)
    e_l = env * sf * (f / lam)
    o_l = -env * cf * (f / lam)
    env_s = env * Q / sig ** 3
    e_s = env_s * cf
    o_s = env_s * sf
    S = e_raw.sum()
    e = e_raw - S / fs ** 2
    # alpha: d lambda = lam0, d sigma = rho * lam0, d fs = size_ratio * lam0
    e_raw_a = lam0 * e_l + th.rho * lam0 * e_s
    de_da = e_raw_a - e_raw_a.sum() / fs ** 2 + 2 * S * p.size_ratio * lam0 / fs ** 3
    do_da = lam0 * o_l + th.rho * lam0 * o_s
    # rho: d sigma = lam
    e_raw_r = lam * e_s
    de_dr = e_raw_r - e_raw_r.sum() / fs ** 2
    do_dr = lam * o_s
    return {"e": e, "o": od, "de_da": de_da, "do_da": do_da, "de_dr": de_dr, "do_dr": do_dr}


def float_pyramid(X: np.ndarray, levels: int):
    P = [np.asarray(X, dtype=np.float64)]
    for _ in range(levels):
        P.append(O.pyr_down_f(P[-1]))
    return P


def pyr_down_f_adjoint(g: np.ndarray, shape_in) -> np.ndarray:
    """Transpose of bimp_oracle.pyr_down_f (reflect-101 taps add)."""
    h, w = shape_in
    oh, ow = g.shape
    wts = np.array([1, 4, 6, 4, 1], dtype=np.float64) / 16.0
    rows = O._reflect101(2 * np.arange(oh)[:, None] + np.arange(-2, 3)[None, :], h)
    cols = O._reflect101(2 * np.arange(ow)[:, None] + np.arange(-2, 3)[None, :], w)
    tmp = np.zeros((oh, w))
    for k in range(5):
        np.add.at(tmp, (slice(None), cols[:, k]), wts[k] * g)
    out = np.zeros((h, w))
    for k in range(5):
        np.add.at(out, rows[:, k], wts[k] * tmp)
    return out


def _flat_index(sc: O.Scale):
    F = sc.fftH * sc.fftW
    r = np.arange(sc.dataH + 1)[:, None]
    c = np.arange(sc.dataW + 1)[None, :]
    return (r * sc.fftW + c) % F


def _shift_idx(sc, dy, dx):
    y = np.clip(np.arange(sc.dataH) + dy, 0, sc.dataH)
    x = np.clip(np.arange(sc.dataW) + dx, 0, sc.dataW)
    return y[:, None], x[None, :]


def forward_scale(data: np.ndarray, sc: O.Scale, th: Theta, p: O.Params = O.Params(), need_grad=False):
    """One scale: returns dict with D and the intermediates the adjoint needs."""
    Ip = O.padded_image(data, sc)
    Xh = np.fft.rfft2(Ip)
    flat = _flat_index(sc)
    E = np.empty((O.NUM_ORI, sc.fftH, sc.fftW))
    Od = np.empty_like(E)
    taps = []
    for o in range(O.NUM_ORI):
        tp = taps_f64(sc, o, th, p)
        taps.append(tp)
        E[o] = np.fft.irfft2(Xh * np.fft.rfft2(O.padded_kernel(tp["e"], sc)), s=Ip.shape)
        Od[o] = np.fft.irfft2(Xh * np.fft.rfft2(O.padded_kernel(tp["o"], sc)), s=Ip.shape)
    Ct = np.sqrt(E * E + Od * Od)
    Cw = Ct.reshape(O.NUM_ORI, -1)[:, flat]
    pp = O.Params(**{**p.__dict__, "w_tan": th.w_tan, "w_rad": th.w_rad})
    maps = O.keypoint_maps(Cw, sc, pp)
    out = {"D": maps["D"], "T": maps["T"], "R": maps["R"]}
    if need_grad:
        out.update({"Ip": Ip, "Xh": Xh, "E": E, "O": Od, "Ct": Ct, "Cw": Cw, "flat": flat, "taps": taps})
    return out


def loss(X, lambdas, masks, th: Theta = Theta(), p: O.Params = O.Params()) -> float:
    H, W = X.shape
    scales = O.scale_geometry(W, H, lambdas, p)
    P = float_pyramid(X, max(s.levels for s in scales))
    total = 0.0
    for s, sc in enumerate(scales):
        data = KAPPA * P[sc.levels][:sc.dataH, :sc.dataW]
        total += float((masks[s] * forward_scale(data, sc, th, p)["D"]).sum())
    return total


def _relu_states(Cw: np.ndarray, sc: O.Scale, p: O.Params, fp32: bool):
    """Per orientation, the ReLU states of the stencils at every pixel:
    d > 0 (double-stopped), t > 0 (tangential), r > 0 and r1 > 0 (radial),
    each gated by its bounds test.  fp32=True evaluates the arguments from
    float32 cells with the CUDA kernels' float operation order (fused
    multiply-adds round once), so the states are the ones the device took."""
    f = (lambda v: v.astype(np.float32).astype(np.float64)) if fp32 else (lambda v: v)
    yc, xc = _shift_idx(sc, 0, 0)
    out = []
    for o in range(O.NUM_ORI):
        C = Cw[o]
        Cp = Cw[(o + O.NUM_ORI // 2) % O.NUM_ORI]
        o1, o2 = sc.es_off[o]
        ya, xa = _shift_idx(sc, -2 * o1, 2 * o2)
        yb, xb = _shift_idx(sc, 2 * o1, -2 * o2)
        c0 = C[yc, xc]
        if fp32:
            d = f(f(c0 - 0.5 * C[ya, xa]) - 0.5 * C[yb, xb])
        else:
            d = c0 - 0.5 * C[ya, xa] - 0.5 * C[yb, xb]
        i1, i2 = sc.in_off[o]
        m_in = O.stencil_masks(sc, i1, i2)
        yt, xt = _shift_idx(sc, -i1, -i2)
        t = f(C[yt, xt] - c0)
        h1 = O._round_half_away(0.5 * i1)
        h2 = O._round_half_away(0.5 * i2)
        yp, xp = _shift_idx(sc, h1, h2)
        ym, xm = _shift_idx(sc, -h1, -h2)
        r1 = f(c0 - p.radial_gain * Cp[yp, xp])
        r = f(np.maximum(r1, 0.0) + f(c0 - p.radial_gain * Cp[ym, xm]))
        out.append({"d": O.stencil_masks(sc, o1, o2) & (d > 0), "t": m_in & (t > 0), "r": m_in & (r > 0),
                    "r1": r1 > 0})
    return out


def stencil_backward(Cw: np.ndarray, M: np.ndarray, sc: O.Scale, th: Theta, p: O.Params = O.Params(),
                     decide: np.ndarray | None = None):
    """Gradient of sum(M * D) with respect to the stencil window Cw
    (8, dataH+1, dataW+1).  The ReLU states come from Cw in float64, or, when
    `decide` (float32 cells of the same window) is given, from those with the
    device's float arithmetic."""
    st = _relu_states(Cw if decide is None else decide.astype(np.float64), sc, p, fp32=decide is not None)
    g = np.zeros_like(Cw)
    gT = -th.w_tan * M
    gR = -th.w_rad * M
    yc, xc = _shift_idx(sc, 0, 0)
    for o in range(O.NUM_ORI):
        o1, o2 = sc.es_off[o]
        ya, xa = _shift_idx(sc, -2 * o1, 2 * o2)
        yb, xb = _shift_idx(sc, 2 * o1, -2 * o2)
        gd = np.where(st[o]["d"], M, 0.0)
        np.add.at(g[o], (np.broadcast_to(yc, gd.shape), np.broadcast_to(xc, gd.shape)), gd)
        np.add.at(g[o], (np.broadcast_to(ya, gd.shape), np.broadcast_to(xa, gd.shape)), -0.5 * gd)
        np.add.at(g[o], (np.broadcast_to(yb, gd.shape), np.broadcast_to(xb, gd.shape)), -0.5 * gd)
    for o in range(O.NUM_ORI):
        op = (o + O.NUM_ORI // 2) % O.NUM_ORI
        i1, i2 = sc.in_off[o]
        yt, xt = _shift_idx(sc, -i1, -i2)
        gt = np.where(st[o]["t"], gT, 0.0)
        np.add.at(g[o], (np.broadcast_to(yt, gt.shape), np.broadcast_to(xt, gt.shape)), gt)
        np.add.at(g[o], (np.broadcast_to(yc, gt.shape), np.broadcast_to(xc, gt.shape)), -gt)
        h1 = O._round_half_away(0.5 * i1)
        h2 = O._round_half_away(0.5 * i2)
        yp, xp = _shift_idx(sc, h1, h2)
        ym, xm = _shift_idx(sc, -h1, -h2)
        gr = np.where(st[o]["r"], gR, 0.0)
        gr1 = np.where(st[o]["r1"], gr, 0.0)
        np.add.at(g[o], (np.broadcast_to(yc, gr.shape), np.broadcast_to(xc, gr.shape)), gr + gr1)
        np.add.at(g[op], (np.broadcast_to(ym, gr.shape), np.broadcast_to(xm, gr.shape)), -p.radial_gain * gr)
        np.add.at(g[op], (np.broadcast_to(yp, gr.shape), np.broadcast_to(xp, gr.shape)), -p.radial_gain * gr1)
    return g


def gradient(X, lambdas, masks, th: Theta = Theta(), p: O.Params = O.Params(), decide=None):
    """Loss and its gradient: (L, dL/dX, {alpha, rho, w_tan, w_rad}).

    decide: optional list (per scale) of float32 complex-cell windows
    (8, dataH+1, dataW+1), e.g. the device's; the piecewise choices (ReLU
    states and the magnitude floor) are then taken from them, so that the
    gradient is that of the same linear piece the device evaluated.  A float32
    forward sits within its rounding of ReLU kinks wherever an argument is
    within ~1e-7 of the map peak of zero, and each such kink moves the
    gradient by one pixel's share."""
    H, W = X.shape
    scales = O.scale_geometry(W, H, lambdas, p)
    maxl = max(s.levels for s in scales)
    P = float_pyramid(X, maxl)
    gP = [np.zeros_like(q) for q in P]
    gth = {"alpha": 0.0, "rho": 0.0, "w_tan": 0.0, "w_rad": 0.0}
    total = 0.0
    for s, sc in enumerate(scales):
        data = KAPPA * P[sc.levels][:sc.dataH, :sc.dataW]
        f = forward_scale(data, sc, th, p, need_grad=True)
        M = masks[s]
        total += float((M * f["D"]).sum())
        gth["w_tan"] += float(-(M * f["T"]).sum())
        gth["w_rad"] += float(-(M * f["R"]).sum())
        dec = None if decide is None else decide[s]
        gCw = stencil_backward(f["Cw"], M, sc, th, p, decide=dec)
        gCt = np.zeros((O.NUM_ORI, sc.fftH * sc.fftW))
        for o in range(O.NUM_ORI):
            np.add.at(gCt[o], f["flat"].ravel(), gCw[o].ravel())
        gCt = gCt.reshape(O.NUM_ORI, sc.fftH, sc.fftW)
        Ct = f["Ct"]
        if dec is None:
            Cdec = Ct
        else:
            Cdec = np.zeros((O.NUM_ORI, sc.fftH * sc.fftW))
            Cdec[:, f["flat"].ravel()] = dec.reshape(O.NUM_ORI, -1)
            Cdec = Cdec.reshape(Ct.shape)
        with np.errstate(divide="ignore", invalid="ignore"):
            gE = np.where(Cdec > MAG_FLOOR, gCt * f["E"] / Ct, 0.0)
            gO = np.where(Cdec > MAG_FLOOR, gCt * f["O"] / Ct, 0.0)
        gIp = np.zeros((sc.fftH, sc.fftW))
        for o in range(O.NUM_ORI):
            tp = f["taps"][o]
            Ke = np.fft.rfft2(O.padded_kernel(tp["e"], sc))
            Ko = np.fft.rfft2(O.padded_kernel(tp["o"], sc))
            GE = np.fft.rfft2(gE[o])
            GO = np.fft.rfft2(gO[o])
            # adjoint of circular convolution = circular correlation
            gIp += np.fft.irfft2(GE * np.conj(Ke) + GO * np.conj(Ko), s=gIp.shape)
            for name, ke, ko in (("alpha", tp["de_da"], tp["do_da"]), ("rho", tp["de_dr"], tp["do_dr"])):
                dE = np.fft.irfft2(f["Xh"] * np.fft.rfft2(O.padded_kernel(ke, sc)), s=gIp.shape)
                dO = np.fft.irfft2(f["Xh"] * np.fft.rfft2(O.padded_kernel(ko, sc)), s=gIp.shape)
                gth[name] += float((gE[o] * dE + gO[o] * dO).sum())
        ry = O.pad_map(sc.fftH, sc.dataH, sc.kX)
        rx = O.pad_map(sc.fftW, sc.dataW, sc.kX)
        gdata = np.zeros((sc.dataH, sc.dataW))
        np.add.at(gdata, (ry[:, None], rx[None, :]), gIp)
        gP[sc.levels][:sc.dataH, :sc.dataW] += KAPPA * gdata
    for l in range(maxl, 0, -1):
        gP[l - 1] += pyr_down_f_adjoint(gP[l], P[l - 1].shape)
    return total, gP[0], gth


def masks_for(X_shape, lambdas, seed: int, p: O.Params = O.Params()):
    H, W = X_shape
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((sc.dataH, sc.dataW)) for sc in O.scale_geometry(W, H, lambdas, p)]
