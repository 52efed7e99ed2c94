"""CPU tests of the FP64 oracle: pins against cv2.pyrDown, hand-built known
answers for each stage, and the committed golden fixtures."""
import math

import numpy as np
import pytest

from bimp_b200 import synth
from oracle import bimp_oracle as O


def test_snap_transform_size_cases():
    # snapTransformSize (cuda_bimp.cu:200-219)
    cases = {1: 16, 16: 16, 17: 32, 480: 512, 640: 1024, 1024: 1024, 1025: 1536, 1080: 1536,
             1920: 2048, 2160: 2560, 3840: 4096, 67: 128, 33: 64, 135: 256, 512: 512, 1536: 1536}
    for n, want in cases.items():
        assert O.snap_transform_size(n) == want, n


def test_make_lambdas_log_float_accumulation():
    lam = O.make_lambdas_log(4, 45.26, 2)
    assert len(lam) == 8
    assert lam[2] == float(np.float32(7.9999995))      # not exactly 8
    assert O.make_lambdas_log(4, 32, 1) == [4.0, 8.0, 16.0, 32.0]
    assert len(O.make_lambdas_log(4, 64, 2)) == 9       # Context's bank (bimp.cpp:8)
    assert synth.lambdas_log(4, 45.26, 2) == lam


def test_scale_geometry_hd():
    sc = O.scale_geometry(1920, 1080, O.make_lambdas_log(4, 45.26, 2))
    assert [s.kW for s in sc] == [29, 39, 27, 39, 27, 39, 27, 39]
    assert [s.pyrstep for s in sc] == [1, 1, 2, 2, 4, 4, 8, 8]
    assert [(s.fftW, s.fftH) for s in sc[:4:2]] == [(2048, 1536), (1024, 1024)]
    assert [s.off for s in sc] == [4, 5, 3, 5, 3, 5, 3, 5]
    assert sc[0].es_off == [(2, 0), (2, 1), (2, 2), (1, 2), (0, 2), (-1, 2), (-2, 2), (-2, 1)]
    assert sc[0].in_off == [(0, 2), (1, 2), (2, 2), (2, 1), (2, 0), (2, -1), (2, -2), (1, -2)]


def test_pyramid_matches_cv2_away_from_ties():
    cv2 = pytest.importorskip("cv2")
    img = synth.synth_image(321, 247, 15, seed=3)
    a = O.pyr_down_u8(img).astype(int)
    b = cv2.pyrDown(img).astype(int)
    assert a.shape == b.shape == (124, 161)
    # exact integer sums: cv2 rounds .5 up, the CUDA pyrDown rounds half to even
    diff = a != b
    assert np.all(np.abs(a - b)[diff] == 1)
    assert np.all(a[diff] % 2 == 0) and np.all(b[diff] % 2 == 1)


def test_pyramid_tie_rounding():
    img = np.zeros((5, 5), np.uint8)
    img[2, 2] = 128          # centre weight 36/256 -> 18.0 exactly
    assert O.pyr_down_u8(img)[1, 1] == 18
    img[2, 2] = 64 + 32      # 96*36 = 3456 = 13.5*256 -> tie, rounds to even 14
    assert O.pyr_down_u8(img)[1, 1] == 14


def test_gabor_taps_symmetry_and_dc():
    sc = O.scale_geometry(640, 480, [5.656854])[0]
    for o in range(8):
        e, od = O.gabor_taps(sc, o)
        assert e.shape == (39, 39)
        assert np.array_equal(e, e[::-1, ::-1])                 # point-symmetric
        assert np.max(np.abs(od + od[::-1, ::-1])) < 1e-6       # antisymmetric up to float
        # DC removed with the float filtersize divisor (39.598^2, not 39^2)
        resid = float(e.astype(np.float64).sum())
        assert abs(resid) < 0.5


def test_delta_image_gives_flipped_taps():
    # A delta inside the data gives the torus convolution = the (flipped) taps.
    sc = O.scale_geometry(96, 96, [4.0])[0]
    data = np.zeros((sc.dataH, sc.dataW))
    data[40, 50] = 1.0
    Ip = O.padded_image(data, sc)
    X = np.fft.rfft2(Ip)
    e, od = O.gabor_taps(sc, 3)
    E = np.fft.irfft2(X * np.fft.rfft2(O.padded_kernel(e, sc)), s=Ip.shape)
    k = sc.kX
    patch = E[40 - k:40 + k + 1, 50 - k:50 + k + 1]
    assert np.allclose(patch, e[::-1, ::-1], atol=1e-12)


def test_padding_semantics():
    # rows < dataH copy, then kY clamp-to-last rows, then clamp-to-first
    m = O.pad_map(64, 40, 14)
    assert list(m[:40]) == list(range(40))
    assert set(m[40:54]) == {39} and set(m[54:]) == {0}
    m2 = O.pad_map(48, 40, 14)            # torus shorter than data + half kernel
    assert list(m2[40:]) == [39] * 8


def test_stencil_window_flat_addressing():
    sc = O.scale_geometry(32, 32, [4.0])[0]     # fft == data: flat wrap cases
    assert (sc.fftW, sc.fftH) == (32, 32)
    Ct = np.arange(32 * 32, dtype=float).reshape(32, 32)
    Cw = O.stencil_window(Ct, sc)
    assert Cw.shape == (33, 33)
    assert Cw[3, 32] == Ct[4, 0]          # column dataW -> next row, column 0
    assert Cw[32, 5] == Ct[0, 5]          # row dataH wraps modulo fftH*fftW
    assert Cw[32, 32] == Ct[1, 0]


def test_end_stop_on_hand_map():
    # A single bright complex-cell spot: the double-stopped response at the
    # spot is C - 0.5*0 - 0.5*0 for every orientation whose bounds hold.
    sc = O.scale_geometry(40, 40, [4.0])[0]
    Cw = np.zeros((8, sc.dataH + 1, sc.dataW + 1))
    Cw[:, 20, 20] = 1.0
    maps = O.keypoint_maps(Cw, sc)
    assert maps["D0"][20, 20] == pytest.approx(8.0)
    # tangential inhibition at a neighbour that sees the spot at -offset
    o1, o2 = sc.in_off[0]
    assert maps["T"][20 + o1, 20 + o2] >= 1.0 - 1e-12


def test_nms_and_subpixel_on_hand_map():
    sc = O.scale_geometry(20, 20, [4.0])[0]
    D = np.zeros((20, 20))
    D[10, 10] = 1.0
    D[10, 11] = 0.5
    D[9, 10] = 0.25
    D[11, 10] = 0.25
    D[15, 15] = 0.05        # below 0.104*max
    kp = O.extract_keypoints(D, sc, 0)
    assert list(zip(kp.ix, kp.iy)) == [(10, 10)]
    # parabola through (0, 1, 0.5): x + 0.5*(0-0.5)/(0+0.5-2) = 10 + 1/6
    assert kp.x[0] == pytest.approx(10 + 1 / 6)
    assert kp.y[0] == pytest.approx(10.0)
    assert kp.octave == 4 and kp.size == 4.0


def test_float_pyramid_is_linear():
    rng = np.random.default_rng(0)
    a, b = rng.random((37, 29)), rng.random((37, 29))
    assert np.allclose(O.pyr_down_f(a + 2 * b), O.pyr_down_f(a) + 2 * O.pyr_down_f(b))


def test_golden_fixture():
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "oracle_small.npz")
    img = g["image"]
    lam = list(g["lambdas"])
    res = O.run(img, lam)
    for i, r in enumerate(res):
        assert np.allclose(r["D"], g[f"D{i}"], rtol=0, atol=1e-9 * np.abs(g[f"D{i}"]).max())
    tab = O.keypoint_table(res)
    assert np.array_equal(tab["ix"], g["kp_ix"]) and np.array_equal(tab["iy"], g["kp_iy"])
    assert np.array_equal(tab["scale"], g["kp_scale"])


def test_min_size_rule():
    # cuda_bimp.cu:160-168: rows < 350 (cols >= 350) -> 350/rows; else cols < 350 -> 350/cols
    assert O.min_size_dims(640, 480) == (640, 480, 1.0)
    w, h, sf = O.min_size_dims(500, 250)
    assert (w, h) == (700, 350) and sf == float(np.float32(350 / 250))
    w, h, sf = O.min_size_dims(300, 900)
    assert (w, h) == (350, 1050)
    w, h, sf = O.min_size_dims(123, 77)     # cols < 350 branch wins for small images
    assert w == 350 and sf == float(np.float32(350 / 123))


def test_resize_and_gray_against_cv2():
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(2)
    img = rng.integers(0, 256, (120, 300, 3), dtype=np.uint8)
    w, h, sf = O.min_size_dims(300, 120)
    ref = cv2.resize(img, None, fx=sf, fy=sf)
    mine = O.resize_linear_u8(img, sf, w, h)
    assert mine.shape == ref.shape
    d = np.abs(mine.astype(int) - ref)
    assert d.max() <= 1 and (d > 0).mean() < 0.005      # rounding path differs at ~0.1%
    # grey: 14-bit weights (CUDA colour conversion) vs cv2's 15-bit CPU weights
    g = O.bgr_to_gray(img).astype(int)
    gc = cv2.cvtColor(img, cv2.COLOR_BGR2GRAY).astype(int)
    assert np.abs(g - gc).max() <= 1 and (g != gc).mean() < 0.01


def test_color_features_quirks():
    bgr = np.zeros((20, 20, 3), np.uint8)
    bgr[..., 0] = 10      # bin 0 of B
    bgr[..., 1] = 100     # bin 3 of G
    bgr[..., 2] = 200     # signed char -56: counted nowhere
    f = O.color_features([10.0], [10.0], [16.0], bgr)[0]   # p = 2: 4x4 window, 48 samples
    assert f[0] == pytest.approx(0.5 * 16 / 48) and f[8 + 3] == pytest.approx(0.5 * 16 / 48)
    assert f[16:].sum() == 0 and f[1:8].sum() == 0
    bgr[..., 0] = 0       # open interval: 0 is not in (0, 31.875)
    assert O.color_features([10.0], [10.0], [16.0], bgr)[0][:8].sum() == 0


def test_lines_edges_known_answers():
    """detectLE restatement: a bright 1-pixel line is a positive line, a dark
    one a negative line; opposite step edges get opposite edge types; all at
    the dominant orientation 0 (vertical structures)."""
    sc = O.scale_geometry(128, 96, [4.0])[0]

    def run(img):
        C, E, Od = O.complex_cells(O.level_image(img, sc), sc)
        return O.detect_lines_edges(E, Od, C, sc)

    line = np.full((96, 128), 60, np.uint8)
    line[:, 64] = 200
    r, o, ty, _ = run(line)
    assert (ty[20:76, 64] == 1).all() and (o[20:76, 64] == 0).all() and (r[20:76, 64] > 0).all()
    assert (ty[20:76, 40:60] == 0).all()
    r, o, ty, _ = run(255 - line)
    assert (ty[20:76, 64] == 2).all()
    step = np.full((96, 128), 60, np.uint8)
    step[:, 64:] = 200
    t_up = run(step)[2][20:76, 64]
    t_down = run(255 - step)[2][20:76, 64]
    assert set(np.unique(t_up)) | set(np.unique(t_down)) == {3, 4}
    assert (t_up != t_down).all()


def test_oracle_matches_reference_kernels_golden():
    """The FP64 oracle against outputs of the reference's own BIMP device
    kernels (bimp/include/detection/cuda_bimp.cuh compiled unmodified, driven
    in DoFullGPUFiltering's order with cuFFT; fixture made by
    tests/golden/make_ref_golden.py): summed keypoint maps D and single-stopped
    maps S within 1e-4 of the map peak, identical keypoint sets outside
    decision ties, subpixel positions within 2e-3 level pixels.  Case b has
    fftW == dataW and fftH == dataH, so the stencils' flat reads pass the
    torus."""
    from pathlib import Path

    from parity import MAP_TOL, SUBPIX_TOL, compare_keypoints, peak_rel_error
    g = np.load(Path(__file__).parent / "golden" / "ref_small.npz")
    for name in ("a", "b"):
        img = g[f"{name}_image"]
        lam = [float(x) for x in g[f"{name}_lambdas"]]
        res = O.run(img, lam)
        for i, r in enumerate(res):
            assert peak_rel_error(g[f"{name}_D{i}"], r["D"]) <= MAP_TOL, (name, i)
            assert peak_rel_error(g[f"{name}_S{i}"], r["S"]) <= MAP_TOL, (name, i)
        rec = np.zeros(len(g[f"{name}_kp_x"]), dtype=[("x", "f4"), ("y", "f4"), ("size", "f4"), ("response", "f4")])
        for f in ("x", "y", "size", "response"):
            rec[f] = g[f"{name}_kp_{f}"]
        assert len(rec) > 100
        rep = compare_keypoints(rec, res)
        assert not rep["missing"] and not rep["extra"], (name, rep["missing"][:5], rep["extra"][:5])
        assert rep["max_subpix"] <= SUBPIX_TOL and rep["max_resp_rel"] <= MAP_TOL
        assert (g[f"{name}_kp_class_id"] == 1).all() and (g[f"{name}_kp_angle"] == -1).all()
