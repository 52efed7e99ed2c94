"""Comparison helpers for GPU-vs-oracle parity tests.

Tolerances (written here, used by the tests):

* response maps (complex cells C, summed keypoint map D, single map S):
  peak-relative error max|gpu - ref| / max|ref| <= MAP_TOL (1e-4) per scale,
  plus the element-wise relative error |gpu - ref| / max(|ref|, ELEM_FLOOR *
  max|ref|) <= MAP_TOL for the complex cells: every magnitude above 5% of the
  map peak is within 1e-4 of the oracle element-wise.  The floor is needed
  because an FP32 FFT's error is absolute, about 1e-7..1e-6 of the peak at
  every pixel, so near-zero magnitudes have no meaningful relative error;
* keypoints: identical (scale, integer x, integer y) sets except where the
  oracle's decision is within TIE_EPS * max|D| of a tie (with a neighbour, or
  with the threshold), and subpixel positions within SUBPIX_TOL pixels
  of the scale's pyramid level (the parabola is fitted on the level grid;
  records carry level position x pyrstep).
"""
from __future__ import annotations

import numpy as np

MAP_TOL = 1e-4
ELEM_FLOOR = 5e-2
TIE_EPS = 1e-5
SUBPIX_TOL = 2e-3


def peak_rel_error(gpu, ref) -> float:
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    assert g.shape == r.shape, (g.shape, r.shape)
    m = np.abs(r).max()
    if m == 0:
        return float(np.abs(g).max())
    return float(np.abs(g - r).max() / m)


def elem_rel_error(gpu, ref, floor_frac: float = 1e-3) -> float:
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    floor = floor_frac * np.abs(r).max()
    return float((np.abs(g - r) / np.maximum(np.abs(r), max(floor, 1e-300))).max())


def records_by_scale(rec: np.ndarray, oracle_result) -> dict:
    """Split GPU records into {scale: {(ix, iy): (x, y, response)}}.

    The scale of a record is identified by its size (lambda * pyrstep), the
    integer level position by rounding x/pyrstep (the parabolic offset is
    strictly inside (-0.5, 0.5) at a strict maximum).
    """
    out = {}
    sizes = {}
    for r in oracle_result:
        kp = r["kp"]
        sizes.setdefault(np.float32(kp.size), []).append(kp.scale)
    for r in oracle_result:
        out[r["kp"].scale] = {}
    for k in rec:
        cand = sizes.get(np.float32(k["size"]))
        assert cand is not None, f"record with unknown size {k['size']}"
        s = cand[0]
        pyr = oracle_result[s]["scale"].pyrstep
        ix = int(np.rint(k["x"] / pyr))
        iy = int(np.rint(k["y"] / pyr))
        assert (ix, iy) not in out[s], f"duplicate keypoint {(s, ix, iy)}"
        out[s][(ix, iy)] = (float(k["x"]), float(k["y"]), float(k["response"]))
    return out


def compare_keypoints(rec: np.ndarray, oracle_result, tie_eps: float = TIE_EPS) -> dict:
    """Compare GPU records with the oracle; returns a report dict."""
    got = records_by_scale(rec, oracle_result)
    report = {"missing": [], "extra": [], "ties_excluded": 0, "matched": 0, "max_subpix": 0.0,
              "max_resp_rel": 0.0}
    for r in oracle_result:
        kp = r["kp"]
        s = kp.scale
        D = r["D"]
        scale = np.abs(D).max()
        y0, y1, x0, x1 = kp.region
        tie = np.zeros(D.shape, dtype=bool)
        if kp.cand_margin.size:
            tie[y0:y1, x0:x1] = kp.cand_margin < tie_eps * scale
        report["ties_excluded"] += int(tie.sum())
        ref = {(int(x), int(y)): (float(a), float(b), float(v))
               for x, y, a, b, v in zip(kp.ix, kp.iy, kp.x, kp.y, kp.response)}
        g = got.get(s, {})
        for key, val in ref.items():
            if tie[key[1], key[0]]:
                continue
            if key not in g:
                report["missing"].append((s, key))
                continue
            report["matched"] += 1
            gx, gy, gv = g[key]
            pyr = r["scale"].pyrstep
            report["max_subpix"] = max(report["max_subpix"], abs(gx - val[0]) / pyr, abs(gy - val[1]) / pyr)
            report["max_resp_rel"] = max(report["max_resp_rel"], abs(gv - val[2]) / scale)
        for key in g:
            if key in ref:
                continue
            x, y = key
            inside = y0 <= y < y1 and x0 <= x < x1
            if inside and tie[y, x]:
                continue
            report["extra"].append((s, key))
    return report
