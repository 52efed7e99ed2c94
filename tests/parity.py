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


def decision_margin(D, thresh_ratio: float = 0.104) -> np.ndarray:
    """Per-pixel distance of the keypoint decision (strict 8-neighbour
    maximum, and above thresh_ratio * max) from flipping, from a summed
    keypoint map."""
    H, W = D.shape
    P = np.pad(D, 1, mode="reflect")
    dil = np.full(D.shape, -np.inf)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dy or dx:
                dil = np.maximum(dil, P[1 + dy:1 + dy + H, 1 + dx:1 + dx + W])
    loc = D - dil
    dth = D - np.float32(np.float64(D.max()) * thresh_ratio)
    return np.minimum(np.abs(loc), np.abs(dth))


def check_against_c_restatement(cb, ref: np.ndarray, lambdas, rec: np.ndarray, dense_maps,
                                tie_frac: float = 1e-4) -> dict:
    """Records `rec` and per-scale summed keypoint maps of one image against
    the FP32 C restatement `cb` (oracle.cbimp.CBimp) and its records `ref`
    from cb.detect on the same image: maps within MAP_TOL of the peak;
    keypoint (scale, x, y) sets equal except where the restatement's decision
    is within tie_frac of the map peak of a tie (at most max(2, n/1000) such
    pixels per scale).  A record keys to the pixel nearest its subpixel
    position; where a neighbour ties the maximum the parabolic offset is
    +-0.5 and the two sides can round to adjacent pixels, so a record that
    the other side has within SUBPIX_TOL level pixels counts as present.
    Returns the worst map error and the symmetric difference per scale."""
    out = {"map_err": 0.0, "symdiff": [], "keypoints": 0, "split_rounding": 0}
    lam = sorted(float(np.float32(x)) for x in lambdas)
    for s, info in enumerate(cb.scales):
        D = cb.dense_map(s)
        out["map_err"] = max(out["map_err"], peak_rel_error(dense_maps[s], D))
        pyr = 2 ** info["level"]
        size = np.float32(np.float32(np.float32(lam[s]) / np.float32(pyr)) * np.float32(pyr))

        def keyed(r):
            d = {}
            for k in r[r["size"] == size]:
                x, y = float(k["x"]) / pyr, float(k["y"]) / pyr
                d[(int(np.rint(x)), int(np.rint(y)))] = (x, y)
            return d

        a, b = keyed(ref), keyed(rec)
        marg = decision_margin(D)
        peak = np.abs(D).max()
        diff = 0
        for key in set(a) ^ set(b):
            own, other = (a, b) if key in a else (b, a)
            x, y = own[key]
            if any(abs(ox - x) <= SUBPIX_TOL and abs(oy - y) <= SUBPIX_TOL
                   for dk in ((-1, 0), (1, 0), (0, -1), (0, 1))
                   for ox, oy in [other.get((key[0] + dk[0], key[1] + dk[1]), (np.inf, np.inf))]):
                out["split_rounding"] += 1
                continue
            # the pixel the record came from: the nearest one, or either
            # neighbour when the parabolic offset is +-0.5 (a neighbour tie)
            xs = {int(np.floor(x + 0.5 - 1e-3)), int(np.floor(x + 0.5 + 1e-3))}
            ys = {int(np.floor(y + 0.5 - 1e-3)), int(np.floor(y + 0.5 + 1e-3))}
            m = min(marg[yy, xx] for xx in xs for yy in ys if 0 <= yy < D.shape[0] and 0 <= xx < D.shape[1])
            assert m < tie_frac * peak, (s, key, (x, y), m / peak)
            diff += 1
        assert diff <= max(2, len(a) // 1000), (s, diff, len(a))
        out["symdiff"].append(diff)
        out["keypoints"] += len(a)
    assert out["map_err"] <= MAP_TOL, out["map_err"]
    return out
