"""Parity pinned to the reference's own device kernels.

oracle/_ref/libbimpref.so runs daniel-koudouna/cuda-bimp's BIMP kernels
(bimp/include/detection/cuda_bimp.cuh, compiled unmodified) with cuFFT in
DoFullGPUFiltering's order (bimp/src/cuda_bimp.cu:462-559, :714-743).  On the
same images it must agree with the FP64 oracle (so the oracle restates the
reference) and with this library's CUDA path (so the product matches the
reference), within the tolerances of tests/parity.py:

* summed keypoint maps D (and S, complex cells C on small tori): peak-relative
  error <= 1e-4 per scale;
* keypoints: identical (scale, integer x, integer y) sets except where the
  oracle's decision is within 1e-5 of the map peak of a tie; subpixel
  positions within 2e-3 level pixels; responses within 1e-4 of the peak.
"""
import numpy as np
import pytest

from bimp_b200 import api, synth
from oracle import bimp_oracle as O
from oracle import refrun
from parity import MAP_TOL, SUBPIX_TOL, TIE_EPS, compare_keypoints, peak_rel_error, records_by_scale

pytestmark = pytest.mark.gpu


def _product(img, lam):
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    kp = api.getKeypoints(img, cs, capacity=1 << 20)
    return cs, api.keypoint_matrix_to_records(kp)


def _tie_pixels(res):
    """Per scale, the candidate-region pixels whose oracle decision is within
    TIE_EPS of the map peak of flipping."""
    out = {}
    for r in res:
        kp = r["kp"]
        y0, y1, x0, x1 = kp.region
        t = set()
        if kp.cand_margin.size:
            ys, xs = np.nonzero(kp.cand_margin < TIE_EPS * np.abs(r["D"]).max())
            t = {(int(x) + x0, int(y) + y0) for x, y in zip(xs, ys)}
        out[kp.scale] = t
    return out


def _pin(img, lam, keep_c):
    assert refrun.available(), "oracle/_ref/libbimpref.so is missing: build it with python oracle/build_ref.py"
    ref = refrun.run(img, lam, keep_c=keep_c)
    res = O.run(img, lam)
    cs, rec = _product(img, lam)
    worst = {"D_ref_vs_oracle": 0.0, "S_ref_vs_oracle": 0.0, "D_product_vs_ref": 0.0, "C_ref_vs_oracle": 0.0}
    for s, (a, r) in enumerate(zip(ref, res)):
        worst["D_ref_vs_oracle"] = max(worst["D_ref_vs_oracle"], peak_rel_error(a["D"], r["D"]))
        worst["S_ref_vs_oracle"] = max(worst["S_ref_vs_oracle"], peak_rel_error(a["S"], r["S"]))
        worst["D_product_vs_ref"] = max(worst["D_product_vs_ref"],
                                        peak_rel_error(cs.dense_map(s, 0).cpu().numpy(), a["D"]))
        if keep_c:
            cw = O.stencil_window(a["C"], r["scale"])
            for o in range(8):
                worst["C_ref_vs_oracle"] = max(worst["C_ref_vs_oracle"], peak_rel_error(cw[o], r["Cw"][o]))
    # the reference's keypoints against the oracle (tie rule on the oracle's margins)
    rref = refrun.records(ref)
    rep = compare_keypoints(rref, res)
    # the product's keypoints against the reference's, directly
    ties = _tie_pixels(res)
    a = records_by_scale(rref, res)
    b = records_by_scale(rec, res)
    sym = []
    for s in a:
        for key in set(a[s]) ^ set(b.get(s, {})):
            if key not in ties[s]:
                sym.append((s, key))
    subpix = 0.0
    for s in a:
        pyr = res[s]["scale"].pyrstep
        for key in set(a[s]) & set(b.get(s, {})):
            (xa, ya, _), (xb, yb, _) = a[s][key], b[s][key]
            subpix = max(subpix, abs(xa - xb) / pyr, abs(ya - yb) / pyr)
    n_ref = sum(len(v) for v in a.values())
    print({**worst, "ref_keypoints": n_ref, "matched_ref_vs_oracle": rep["matched"],
           "ties_excluded": rep["ties_excluded"], "product_vs_ref_symdiff": len(sym), "subpix_product_vs_ref": subpix})
    for k, v in worst.items():
        assert v <= MAP_TOL, (k, v)
    assert not rep["missing"] and not rep["extra"], (rep["missing"][:5], rep["extra"][:5])
    assert rep["max_subpix"] <= SUBPIX_TOL and rep["max_resp_rel"] <= MAP_TOL
    assert not sym, sym[:10]
    assert subpix <= SUBPIX_TOL
    cs.close()
    return worst, n_ref


def test_reference_pins_vga_config():
    """640x480, wavelengths 4, 8, 16, 32 (four pyramid levels)."""
    imgs, lam = synth.workload("vga")
    _, n = _pin(imgs[0], lam, keep_c=True)
    assert n > 1000


@pytest.mark.parametrize("w,h,lam", [
    (512, 512, [4.0, 5.656854, 8.0]),          # fftW == dataW and fftH == dataH: flat reads past the torus
    (333, 277, [4.0, 6.0, 11.0]),              # odd sizes, three pyramid levels
    (1024, 200, [4.0, 7.9999995, 16.0]),       # fftW == dataW at every level
    (130, 1100, [4.0, 5.656854]),               # fft height above 1024 (multiple of 512)
])
def test_reference_pins_torus_edge_cases(w, h, lam):
    img = synth.synth_image(w, h, max(2, w * h // 15000), seed=7 + w + h)
    _pin(img, lam, keep_c=True)


def test_reference_pins_hd_config():
    """1920x1080, the 8-scale bank (float-accumulated 4 * 2^(k/2))."""
    imgs, lam = synth.workload("hd")
    _, n = _pin(imgs[0], lam, keep_c=False)
    assert n > 10000
