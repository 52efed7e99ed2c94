"""The FP32 C restatement (oracle/cbimp.c) against the FP64 oracle.

The C restatement is the timed CPU baseline; these tests pin it to the
oracle with the same tolerances the GPU parity tests use (response maps within
1e-4 of the peak, identical keypoint sets outside decision ties).
"""
import ctypes as C

import numpy as np
import pytest

from bimp_b200 import synth
from oracle import bimp_oracle as O
from oracle import cbimp
from parity import MAP_TOL, SUBPIX_TOL, compare_keypoints, peak_rel_error


@pytest.fixture(scope="module")
def L():
    lib = cbimp.lib()
    lib.cbimp_fft2.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    return lib


@pytest.mark.parametrize("h,w", [(8, 8), (16, 24), (40, 8), (56, 64), (1536, 8), (8, 2560), (8, 3584)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_fft2_matches_numpy(L, h, w, inverse):
    rng = np.random.default_rng(h * 7 + w)
    x = rng.standard_normal((h, w)) + 1j * rng.standard_normal((h, w))
    re = np.ascontiguousarray(x.real, dtype=np.float32)
    im = np.ascontiguousarray(x.imag, dtype=np.float32)
    assert L.cbimp_fft2(re.ctypes.data, im.ctypes.data, h, w, inverse) == 0
    ref = np.fft.ifft2(x) * (h * w) if inverse else np.fft.fft2(x)
    assert np.abs(re + 1j * im - ref).max() / np.abs(ref).max() < 1e-6


def test_fft2_rejects_unsupported_sizes(L):
    a = np.zeros((8, 8 * 67), dtype=np.float32)
    assert L.cbimp_fft2(a.ctypes.data, a.ctypes.data, 8, 8 * 67, 0) == -1   # prime factor 67 > 64
    assert L.cbimp_fft2(a.ctypes.data, a.ctypes.data, 8, 12, 0) == -1       # not a multiple of 8


def test_snap_transform_size(L):
    for n in list(range(1, 2200, 5)) + [2160, 3840, 4096, 5000]:
        assert L.cbimp_snap_transform_size(n) == O.snap_transform_size(n)


def _check(img, lam):
    res = O.run(img, lam)
    with cbimp.CBimp(img.shape[1], img.shape[0], lam) as cb:
        rec, total = cb.detect(img)
        assert total == len(rec)
        for i, r in enumerate(res):
            assert peak_rel_error(cb.dense_map(i), r["D"]) <= MAP_TOL
            assert peak_rel_error(cb.dense_map(i, 1), r["S"]) <= MAP_TOL
    rep = compare_keypoints(rec, res)
    assert not rep["missing"] and not rep["extra"], (rep["missing"][:5], rep["extra"][:5])
    assert rep["max_subpix"] <= SUBPIX_TOL
    assert rep["max_resp_rel"] <= MAP_TOL
    return rec, rep


def test_vga_matches_oracle():
    imgs, lam = synth.workload("vga")
    rec, rep = _check(imgs[0], lam)
    assert rep["matched"] > 1000
    # (scale, y, x) order: sizes non-decreasing
    assert np.all(np.diff(rec["size"]) >= 0)
    assert np.all(rec["angle"] == -1) and np.all(rec["class_id"] == 1)


@pytest.mark.parametrize("w,h,lam", [
    (512, 512, [4.0, 5.656854, 8.0]),
    (333, 277, [4.0, 6.0, 11.0]),
    (48, 40, [4.0, 5.5]),
    (1024, 200, [4.0, 7.9999995, 16.0]),
    (130, 1100, [4.0, 5.656854]),
])
def test_torus_edge_cases_match_oracle(w, h, lam):
    img = synth.synth_image(w, h, max(2, w * h // 15000), seed=7 + w + h)
    _check(img, lam)


def test_golden_fixture_keypoints():
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "oracle_small.npz")
    img = g["image"]
    lam = [float(x) for x in g["lambdas"]]
    with cbimp.CBimp(img.shape[1], img.shape[0], lam) as cb:
        rec, _ = cb.detect(img)
        for i in range(len(lam)):
            d = g[f"D{i}"]
            assert np.abs(cb.dense_map(i) - d).max() <= MAP_TOL * np.abs(d).max()
    assert len(rec) == len(g["kp_ix"])
    assert np.allclose(rec["x"], g["kp_x"], atol=SUBPIX_TOL * 8)
    assert np.allclose(rec["y"], g["kp_y"], atol=SUBPIX_TOL * 8)


def test_capacity_truncates_and_counts():
    imgs, lam = synth.workload("vga")
    with cbimp.CBimp(640, 480, lam) as cb:
        full, total = cb.detect(imgs[0])
        part, total2 = cb.detect(imgs[0], capacity=100)
    assert total == total2 == len(full)
    assert len(part) == 100
    assert np.array_equal(part, full[:100])


def test_invalid_arguments():
    with pytest.raises(ValueError):
        cbimp.CBimp(1, 480, [4.0])
    with pytest.raises(ValueError):
        cbimp.CBimp(640, 480, [-1.0])
