"""GPU parity: the CUDA path through the C ABI against the FP64 oracle."""
import numpy as np
import pytest

from bimp_b200 import api, synth
from oracle import bimp_oracle as O
from parity import ELEM_FLOOR, MAP_TOL, SUBPIX_TOL, compare_keypoints, elem_rel_error, peak_rel_error

pytestmark = pytest.mark.gpu


def _run_gpu(img, lambdas, capacity=200000):
    cs = api.CudaStuff(img.shape[1], img.shape[0], lambdas)
    kp, n = api.getKeypoints(img, cs, capacity=capacity, return_count=True)
    rec = api.keypoint_matrix_to_records(kp)
    return cs, rec, n


def _map_errors(cs, res):
    worst = {"C": 0.0, "Cel": 0.0, "D": 0.0, "S": 0.0}
    for i, r in enumerate(res):
        for o in range(8):
            g = cs.complex_map(i, o).cpu().numpy()
            worst["C"] = max(worst["C"], peak_rel_error(g, r["Cw"][o]))
            worst["Cel"] = max(worst["Cel"], elem_rel_error(g, r["Cw"][o], ELEM_FLOOR))
        worst["D"] = max(worst["D"], peak_rel_error(cs.dense_map(i, 0).cpu().numpy(), r["D"]))
        worst["S"] = max(worst["S"], peak_rel_error(cs.dense_map(i, 1).cpu().numpy(), r["S"]))
    print("map errors", worst)
    return worst


def _check_scale_maps(cs, res):
    worst = _map_errors(cs, res)
    assert worst["C"] <= MAP_TOL and worst["Cel"] <= MAP_TOL
    assert worst["D"] <= MAP_TOL and worst["S"] <= MAP_TOL
    return worst


def _check_keypoints(rec, res):
    rep = compare_keypoints(rec, res)
    print({k: (v if not isinstance(v, list) else len(v)) for k, v in rep.items()})
    assert not rep["missing"], rep["missing"][:10]
    assert not rep["extra"], rep["extra"][:10]
    assert rep["max_subpix"] <= SUBPIX_TOL
    assert rep["max_resp_rel"] <= MAP_TOL
    return rep


def test_vga_maps_and_keypoints():
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    res = O.run(img, lam)
    cs, rec, n = _run_gpu(img, lam)
    assert n == len(rec)
    _map_errors(cs, res)
    _check_keypoints(rec, res)
    _check_scale_maps(cs, res)
    # deterministic (scale, y, x) order
    order = [(r["size"], r["y"], r["x"]) for r in rec]
    assert len(order) == n


@pytest.mark.parametrize("w,h,lam", [
    (512, 512, [4.0, 5.656854, 8.0]),          # fftW == dataW and fftH == dataH (pure torus)
    (333, 277, [4.0, 6.0, 11.0]),              # odd sizes, three pyramid levels
    (48, 40, [4.0, 5.5]),                       # torus smaller than a tile: multiple wraps
    (1024, 200, [4.0, 7.9999995, 16.0]),       # wrapW at every level
    (130, 1100, [4.0, 5.656854]),               # fft height > 1024 (align 512)
])
def test_torus_edge_cases(w, h, lam):
    img = synth.synth_image(w, h, max(2, w * h // 15000), seed=7 + w + h)
    res = O.run(img, lam)
    cs, rec, n = _run_gpu(img, lam)
    _check_scale_maps(cs, res)
    _check_keypoints(rec, res)


def test_hd_keypoints_and_maps():
    imgs, lam = synth.workload("hd")
    img = imgs[0]
    res = O.run(img, lam)
    cs, rec, n = _run_gpu(img, lam)
    _check_scale_maps(cs, res)
    rep = _check_keypoints(rec, res)
    assert rep["matched"] > 1000


def test_uhd_coarse_scales_match_oracle():
    """3840x2160, the coarse half of the 12-scale bank (pyramid levels 3-5;
    level 5 keeps 67 of pyrDown's 68 rows)."""
    img = synth.uhd_frames(1, seed=1004)[0]
    lam = synth.bank(12)[6:]
    res = O.run(img, lam)
    assert res[-1]["scale"].dataH == 67
    cs, rec, n = _run_gpu(img, lam)
    _check_scale_maps(cs, res)
    _check_keypoints(rec, res)


def _decision_margin(D, off, thresh_ratio=0.104):
    """Per-pixel distance of the keypoint decision from flipping (strict
    8-neighbour max and threshold), from a summed keypoint map."""
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


def test_uhd_full_bank_against_c_restatement():
    """All 12 scales of a 3840x2160 frame against the FP32 C restatement of
    the reference pipeline (itself pinned to the oracle on CPU): maps within
    1e-4 of the peak; keypoints identical except where the restatement's
    decision is within 1e-4 of the peak of a tie."""
    from oracle.cbimp import CBimp
    img = synth.uhd_frames(2, seed=1004)[1]
    lam = synth.bank(12)
    cs, rec, n = _run_gpu(img, lam)
    with CBimp(img.shape[1], img.shape[0], lam) as cb:
        ref, total = cb.detect(img, capacity=1 << 21)
        assert total == len(ref)
        sizes = sorted({float(s) for s in ref["size"]} | {float(s) for s in rec["size"]})
        assert len(sizes) <= len(lam)
        for s in range(len(lam)):
            D = cb.dense_map(s)
            assert peak_rel_error(cs.dense_map(s, 0).cpu().numpy(), D) <= MAP_TOL
            info = cb.scales[s]
            pyr = 2 ** info["level"]
            size = np.float32(np.float32(lam[s] / pyr) * np.float32(pyr))
            a = {(int(np.rint(k["x"] / pyr)), int(np.rint(k["y"] / pyr))) for k in ref if k["size"] == size}
            b = {(int(np.rint(k["x"] / pyr)), int(np.rint(k["y"] / pyr))) for k in rec if k["size"] == size}
            marg = _decision_margin(D, info["off"])
            peak = np.abs(D).max()
            for (x, y) in a ^ b:
                assert marg[y, x] < 1e-4 * peak, (s, x, y, marg[y, x] / peak)
            assert len(a ^ b) <= max(2, len(a) // 1000), (s, len(a ^ b), len(a))


def test_detect_host_matches_device():
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    kp, n = api.getKeypoints(img, cs, capacity=100000, return_count=True)
    dev = api.keypoint_matrix_to_records(kp)
    host, n2, rc = api.detect_host(cs, img, capacity=100000)
    assert rc == 0 and n2 == n
    assert np.array_equal(dev, host)


def test_detect_host_sequence_of_counts():
    """One context, host path, images whose keypoint counts rise and fall
    (including none): every call equals the device path."""
    imgs, lam = synth.workload("vga")
    base = imgs[0]
    half = base.copy()
    half[:, : base.shape[1] // 2] = 128   # about half the keypoints
    seq = [base, np.full_like(base, 128), base[:, ::-1].copy(), base[::-1].copy(), half, base, np.full_like(base, 7),
           base]
    cs = api.CudaStuff(base.shape[1], base.shape[0], lam)
    for img in seq:
        kp, n = api.getKeypoints(img, cs, capacity=100000, return_count=True)
        dev = api.keypoint_matrix_to_records(kp)
        host, n2, rc = api.detect_host(cs, img, capacity=100000)
        assert rc == 0 and n2 == n
        assert np.array_equal(dev, host)


def test_repeatable_bitwise():
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    a = api.keypoint_matrix_to_records(api.getKeypoints(img, cs, capacity=100000))
    d1 = cs.dense_map(0).cpu().numpy()
    b = api.keypoint_matrix_to_records(api.getKeypoints(img, cs, capacity=100000))
    d2 = cs.dense_map(0).cpu().numpy()
    assert np.array_equal(a, b) and np.array_equal(d1, d2)


def test_capacity_overflow_truncates_in_order():
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    full = api.keypoint_matrix_to_records(api.getKeypoints(img, cs, capacity=100000))
    with pytest.warns(UserWarning):
        kp, n = api.getKeypoints(img, cs, capacity=1000, return_count=True)
    part = api.keypoint_matrix_to_records(kp)
    assert n == len(full) and len(part) == 1000
    assert np.array_equal(part, full[:1000])
    host, n2, rc = api.detect_host(cs, img, capacity=1000)
    assert rc == -4 and n2 == n and np.array_equal(host, full[:1000])


def test_errors_are_status_codes():
    import ctypes as C
    from bimp_b200 import _lib as L
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    n = C.c_int()
    # wrong size
    rc = L.lib().bimp_detect_device(cs.handle, C.c_void_p(1), 640, 320, 240, None, 0, 0, C.byref(n), None)
    assert rc == L.BIMP_ERR_INVALID
    # null image
    rc = L.lib().bimp_detect_device(cs.handle, None, 640, 640, 480, None, 0, 0, C.byref(n), None)
    assert rc == L.BIMP_ERR_INVALID
    # capacity without a matrix
    rc = L.lib().bimp_detect_device(cs.handle, C.c_void_p(1), 640, 640, 480, None, 0, 10, C.byref(n), None)
    assert rc == L.BIMP_ERR_INVALID
    # empty wavelength list / unsupported wavelength geometry
    h = C.c_void_p()
    assert L.lib().bimp_ctx_create(C.byref(h), 64, 64, None, 0, None) == L.BIMP_ERR_INVALID
    p = api.default_params()
    p.level_max = 40.0   # kernels wider than the tile supports
    lam1 = (C.c_float * 1)(30.0)
    assert L.lib().bimp_ctx_create(C.byref(h), 640, 480, lam1, 1, C.byref(p)) == L.BIMP_ERR_INVALID
    # the context still works afterwards
    kp, n2 = api.getKeypoints(img, cs, capacity=100000, return_count=True)
    assert n2 > 0


def test_context_mirror():
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    ctx = api.Context(img, lambdas=lam)
    pts = ctx.getKeypointsAndDownload()
    assert len(pts) > 0 and all(p.class_id == 1 and p.angle == -1 for p in pts)
    resp = ctx.getResponses()
    assert len(resp) == len(lam) and resp[0]["D"].shape == (480, 640)
    ctx.loadImage(np.ascontiguousarray(img[:, ::-1]))
    pts2 = ctx.getKeypointsAndDownload()
    assert len(pts2) > 0


def test_upload_download_roundtrip():
    pts = [api.KeyPoint((1.5, 2.25), 4.0, -1.0, 0.5, 4, 1), api.KeyPoint((10.0, 20.0), 8.0, -1.0, 2.0, 7, 1)]
    kp = api.uploadKeypoints(pts)
    back = api.downloadKeypoints(kp)
    assert back == pts


def test_batch_matches_single():
    rng = np.random.default_rng(5)
    sizes = [(int(rng.integers(20, 60)) * 16, int(rng.integers(15, 40)) * 16) for _ in range(5)]
    imgs = [synth.synth_image(w, h, 10, seed=50 + i) for i, (w, h) in enumerate(sizes)]
    lam = synth.bank(8)
    b = api.Batch(sizes, lam, kp_capacity=100000)
    b.load(imgs)
    b.run()
    for i, img in enumerate(imgs):
        cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
        ref = api.keypoint_matrix_to_records(api.getKeypoints(img, cs, capacity=100000))
        got = api.keypoint_matrix_to_records(b.keypoints(i))
        assert np.array_equal(ref, got), i
    # replay again: same answer
    b.run()
    got0 = api.keypoint_matrix_to_records(b.keypoints(0))
    cs = api.CudaStuff(imgs[0].shape[1], imgs[0].shape[0], lam)
    assert np.array_equal(got0, api.keypoint_matrix_to_records(api.getKeypoints(imgs[0], cs, capacity=100000)))


def test_batch_tile_plans_and_autotune():
    """Every tile plan keeps parity with the oracle; plans of one policy and
    kernel variant are bitwise identical (tile order, grid); the autotuner
    times all 24 (2 kernels x 2 policies x 2 orders x 3 grids) and keeps the
    fastest."""
    rng = np.random.default_rng(9)
    sizes = [(int(rng.integers(20, 50)) * 16, int(rng.integers(15, 35)) * 16) for _ in range(3)]
    imgs = [synth.synth_image(w, h, 8, seed=90 + i) for i, (w, h) in enumerate(sizes)]
    lam = synth.bank(8)
    refs = [O.run(img, lam) for img in imgs]
    b = api.Batch(sizes, lam, kp_capacity=100000)
    b.load(imgs)
    outs = {}
    for policy in (0, 1):
        for order, grid, kernel in ((0, 0, 1), (1, 148, 1), (0, 0, 0), (1, 296, 0)):
            b.set_tile_plan(policy, order, grid, kernel)
            b.run()
            outs[(policy, order, kernel)] = [api.keypoint_matrix_to_records(b.keypoints(i)) for i in range(len(imgs))]
        for i in range(len(imgs)):
            # tile order and grid leave every record bitwise unchanged
            for kernel in (0, 1):
                assert np.array_equal(outs[(policy, 0, kernel)][i], outs[(policy, 1, kernel)][i]), kernel
                _check_keypoints(outs[(policy, 0, kernel)][i], refs[i])
    rep = b.autotune(reps=2)
    assert len(rep["tried"]) == 24 and rep["chosen"]["ms"] > 0
    assert {t["kernel"] for t in rep["tried"]} == {0, 1}
    assert rep["chosen"]["ms"] == min(t["ms"] for t in rep["tried"])
    b.run()
    ch = rep["chosen"]
    for i in range(len(imgs)):
        got = api.keypoint_matrix_to_records(b.keypoints(i))
        assert np.array_equal(got, outs[(ch["policy"], 0, ch["kernel"])][i])
    b.close()


@pytest.mark.parametrize("grid", ["7", "0", "1000"])
def test_tile_plans_bitwise_equal(monkeypatch, grid):
    """The default plan (the tiles' orientations split over one persistent
    CTA per SM) against: 7 CTAs, each walking many tiles and orientation runs
    (the G ring's phases carry across items); one CTA per tile (0); and more
    CTAs than the plan can use (1000: runs of one orientation).  Every
    (tile, orientation) is computed the same way in all of them, so maps and
    records are bitwise equal."""
    imgs, lam = synth.workload("vga")
    img = imgs[0]
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    ref = api.keypoint_matrix_to_records(api.getKeypoints(img, cs, capacity=100000))
    d_ref = [cs.dense_map(i).cpu().numpy() for i in range(len(lam))]
    monkeypatch.setenv("BIMP_TILE_GRID", grid)
    cs2 = api.CudaStuff(img.shape[1], img.shape[0], lam)
    got = api.keypoint_matrix_to_records(api.getKeypoints(img, cs2, capacity=100000))
    assert np.array_equal(ref, got)
    for i in range(len(lam)):
        assert np.array_equal(d_ref[i], cs2.dense_map(i).cpu().numpy())


def _shim_image(w, h, cn, seed):
    grey = synth.synth_image(w, h, max(3, w * h // 15000), seed=seed)
    if cn == 1:
        return grey
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(np.stack([grey, np.roll(grey, 7, 1), rng.integers(0, 256, grey.shape, dtype=np.uint8)],
                                         -1))


@pytest.mark.parametrize("w,h,cn", [(640, 480, 1), (640, 480, 3), (300, 200, 3), (200, 500, 1)])
def test_cpp_context_shim_matches_python_api(tmp_path, w, h, cn):
    """bimp::Context (include/bimp/bimp.hpp) from a C++ program, on grey and
    BGR images, including images below 350 pixels (getGPUImage upscales them
    and the context's geometry stays that of the original size, as in the
    reference): the device keypoint matrix, the responses and the colour
    histograms equal the Python mirror's, whose keypoints and maps match the
    FP64 oracle run on the same upscaled image with the original geometry."""
    import subprocess
    from test_capi_cpu import _build_shim_demo
    exe = _build_shim_demo()
    img = _shim_image(w, h, cn, seed=w + 3 * h + cn)
    lam = [4.0, 5.656854, 8.0, 16.0]
    raw = tmp_path / "img.raw"
    raw.write_bytes(img.tobytes())
    res = subprocess.run([str(exe), str(w), str(h), str(cn), str(raw)] + [repr(x) for x in lam],
                         check=True, capture_output=True, text=True)
    lines = [ln.split() for ln in res.stdout.splitlines()]
    kps = [ln[1:] for ln in lines if ln[0] == "kp"]
    ctx_line = next(ln for ln in lines if ln[0] == "ctx")
    low = next(ln for ln in lines if ln[0] == "lowlevel")
    assert int(low[1]) == int(ctx_line[3]) and low[2] == "1"
    resp = [ln for ln in lines if ln[0] == "resp"]
    ctx = api.Context(img, lambdas=lam)
    ctx.capacity = 1 << 20   # as the C++ program sets it
    uw, uh = api.min_size_dims(w, h)
    assert (int(ctx_line[1]), int(ctx_line[2])) == (ctx.width(), ctx.height()) == (uw, uh)
    ref = api.keypoint_matrix_to_records(ctx.getKeypoints())
    assert int(ctx_line[3]) == len(ref) == len(kps) > 0
    got = np.array([[float(r[0]), float(r[1]), float(r[2]), float(r[3])] for r in kps], dtype=np.float32)
    assert np.array_equal(got[:, 0], ref["x"]) and np.array_equal(got[:, 1], ref["y"])
    assert np.array_equal(got[:, 2], ref["size"]) and np.array_equal(got[:, 3], ref["response"])
    assert all(int(r[5]) == 1 and float(r[6]) == -1.0 for r in kps)
    py_resp = ctx.getResponses()
    assert len(resp) == len(py_resp) == len(lam)
    for ln, r in zip(resp, py_resp):
        D = r["D"].cpu().numpy().astype(np.float64)
        S = r["S"].cpu().numpy().astype(np.float64)
        assert (int(ln[2]), int(ln[3])) == (r["data_w"], r["data_h"])
        assert float(ln[4]) == np.float32(D.max())
        assert abs(float(ln[5]) - D.sum()) <= 1e-6 * np.abs(D).sum()
        assert abs(float(ln[6]) - S.sum()) <= 1e-6 * np.abs(S).sum()
    if cn == 3:
        col = next(ln for ln in lines if ln[0] == "color")
        feats = ctx.getColorFeatures()
        assert int(col[1]) == len(ref) == feats.shape[0]
        s_py = float(np.sum(feats, dtype=np.float64))
        assert (np.isnan(s_py) and col[2] == "nan") or abs(float(col[2]) - s_py) <= 1e-6 * abs(s_py)
    # the Python mirror against the FP64 oracle on the same upscaled image
    grey = O.gpu_image(img, grayscale=True)
    res_o = O.run(grey, lam, geometry_size=(w, h))
    for i, r in enumerate(res_o):
        assert peak_rel_error(ctx.cuda_data.dense_map(i, 0).cpu().numpy(), r["D"]) <= MAP_TOL
    _check_keypoints(ref, res_o)


@pytest.mark.parametrize("w,h,cn", [(300, 120, 3), (640, 480, 3), (200, 500, 1), (123, 77, 3)])
def test_gpu_image_matches_oracle(w, h, cn):
    import torch
    rng = np.random.default_rng(w * h)
    img = rng.integers(0, 256, (h, w, cn) if cn == 3 else (h, w), dtype=np.uint8)
    for gray in (1, 0):
        if cn == 1 and gray == 0:
            continue
        ref = O.gpu_image(img, grayscale=bool(gray))
        got = api.gpu_image(img, grayscale=bool(gray))
        assert got.shape == ref.shape and np.array_equal(got, ref), (w, h, cn, gray)


def test_color_features_match_oracle():
    import torch
    imgs, lam = synth.workload("vga")
    gray = imgs[0]
    rng = np.random.default_rng(9)
    bgr = np.stack([gray, np.roll(gray, 5, 0), rng.integers(0, 256, gray.shape, dtype=np.uint8)], -1)
    cs = api.CudaStuff(640, 480, lam)
    kp = api.getKeypoints(gray, cs, capacity=100000)
    rec = api.keypoint_matrix_to_records(kp)
    got = api.color_features(kp, bgr)
    ref = O.color_features(rec["x"], rec["y"], rec["size"], bgr)
    assert got.shape == (len(rec), 24)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    assert np.array_equal(np.nan_to_num(got), np.nan_to_num(ref))


@pytest.mark.parametrize("w,h,lam", [(320, 240, [4.0, 5.656854, 8.0]), (512, 512, [4.0, 11.313707])])
def test_lines_edges_match_oracle(w, h, lam):
    """bimp_detect_lines_edges against the FP64 restatement of detectLE:
    identical types and orientations except where a decision of the oracle is
    within 1e-4 of the map peak of a tie; strengths within 1e-4 of the peak."""
    img = synth.synth_image(w, h, 12, seed=41 + w)
    res = O.run(img, lam)
    cs, rec, n = _run_gpu(img, lam)
    for i, r in enumerate(res):
        sc = r["scale"]
        Ct, E, Od = O.complex_cells(r["data"], sc)
        ref, ori, typ, margin = O.detect_lines_edges(E, Od, Ct, sc)
        g_res, g_ori, g_typ = (t.cpu().numpy() for t in cs.lines_edges(i))
        peak = Ct.max()
        near = margin < 1e-4 * peak
        diff = (g_typ != typ) & ~near
        assert not diff.any(), (i, int(diff.sum()), np.argwhere(diff)[:5])
        both = (g_typ == typ) & (typ > 0)
        assert both.sum() > 0.9 * (typ > 0).sum()
        assert np.array_equal(g_ori[both], ori[both])
        assert np.abs(g_res[both] - ref[both]).max() <= 1e-4 * peak
        # the caller's summed map gives the same as the default
        import torch
        ch = torch.from_numpy(np.ascontiguousarray(Ct[:, :sc.dataH, :sc.dataW].sum(0), dtype=np.float32)).cuda()
        g2 = cs.lines_edges(i, ch=ch)[2].cpu().numpy()
        assert ((g2 != g_typ) & ~near).sum() == 0


def test_async_detection_captured_in_a_caller_graph():
    """bimp_detect_device_async recorded into the caller's own CUDA graph and
    replayed writes the same keypoints as a direct call, also when direct
    calls into another keypoint matrix run before and after the replay (the
    context's keypoint destination is rewritten in stream order)."""
    import ctypes as C

    import torch
    from bimp_b200 import _lib as L
    imgs, lam = synth.workload("vga")
    cs = api.CudaStuff(640, 480, lam)
    ref, n_ref = api.getKeypoints(imgs[0], cs, return_count=True)
    ref = ref.clone()
    img = torch.from_numpy(imgs[0]).cuda().contiguous()
    cap = 8192
    lib = L.lib()

    def call(out, count, stream):
        L.check(lib.bimp_detect_device_async(cs.handle, C.c_void_p(img.data_ptr()), img.stride(0), 640, 480,
                                             C.c_void_p(out.data_ptr()), out.stride(0), cap,
                                             C.c_void_p(count.data_ptr()), C.c_void_p(stream.cuda_stream)),
                "bimp_detect_device_async")

    kp = torch.zeros((7, cap), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    other = torch.zeros_like(kp)
    cnt2 = torch.zeros_like(cnt)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        call(kp, cnt, s)
    call(other, cnt2, torch.cuda.current_stream())
    torch.cuda.synchronize()
    assert int(cnt2.item()) == n_ref <= cap
    assert torch.equal(other[:, :n_ref], ref[:, :n_ref])
    g.replay()
    torch.cuda.synchronize()
    assert int(cnt.item()) == n_ref
    assert torch.equal(kp[:, :n_ref], ref[:, :n_ref])
    other.zero_()
    call(other, cnt2, torch.cuda.current_stream())
    torch.cuda.synchronize()
    assert torch.equal(other[:, :n_ref], ref[:, :n_ref])
    del g


@pytest.mark.parametrize("depth", [1, 3])
def test_pipeline_matches_detect_host(depth):
    """bimp_pipeline_*: frames pushed ahead of their pops give the same
    records as bimp_detect_host one by one, including frames with no
    keypoints, a count far above the previous frame's (the records beyond the
    speculative copy) and a capacity overflow on pop."""
    imgs, lam = synth.workload("vga")
    base = imgs[0]
    seq = [base, np.full_like(base, 128), base[:, ::-1].copy(), np.full_like(base, 9), base[::-1].copy(), base,
           base[:, ::-1].copy()]
    cs = api.CudaStuff(640, 480, lam)
    refs = [api.detect_host(cs, im, capacity=100000) for im in seq]
    pl = api.Pipeline(640, 480, lam, depth=depth, capacity=100000)
    got = []
    for im in seq:
        if pl.in_flight() == depth:
            got.append(pl.pop())
        pl.push(im)
    while pl.in_flight():
        got.append(pl.pop())
    assert len(got) == len(seq)
    for (r, n, rc), (g, m, rc2) in zip(refs, got):
        assert rc == rc2 == 0 and n == m and np.array_equal(r, g)
    # a full pipeline refuses another frame
    for im in seq[:depth]:
        pl.push(im)
    import ctypes as C
    from bimp_b200 import _lib as L
    assert L.lib().bimp_pipeline_push(pl._h, C.c_void_p(base.ctypes.data), 640, 640, 480) == L.BIMP_ERR_INVALID
    # capacity overflow on pop: the first records and the true total
    rec, n, rc = pl.pop(capacity=100)
    assert rc == L.BIMP_ERR_CAPACITY and n == refs[0][1] and np.array_equal(rec, refs[0][0][:100])
    while pl.in_flight():
        pl.pop()
    pl.close()
    cs.close()


def test_device_allocation_failure_is_a_status():
    """A batch whose arena exceeds the device memory (four 32767 x 32767
    images, about 400 GB) fails with BIMP_ERR_NOMEM and a message, allocates
    nothing, and the library keeps working afterwards."""
    import ctypes as C
    from bimp_b200 import _lib as L
    n = 4
    ws = (C.c_int * n)(*[32767] * n)
    hs = (C.c_int * n)(*[32767] * n)
    lam = synth.bank(8)
    la = (C.c_float * len(lam))(*lam)
    h = C.c_void_p()
    rc = L.lib().bimp_batch_create(C.byref(h), ws, hs, n, la, len(lam), None, 1024)
    assert rc == L.BIMP_ERR_NOMEM and not h.value
    assert b"cudaMalloc" in L.lib().bimp_last_error()
    imgs, lam2 = synth.workload("vga")
    cs = api.CudaStuff(640, 480, lam2)
    kp, n_found = api.getKeypoints(imgs[0], cs, capacity=100000, return_count=True)
    assert n_found > 0
    cs.close()
