"""The allocation-free keypoint extraction entry point.

bimp_extract_keypoints_noalloc serves callers that cannot allocate device
memory while they run (real-time loops that must never enter the allocator,
whose calls can block on a device synchronisation, or hosts whose device
memory all belongs to an external pool): its scratch lives in a fixed
file-scope device array.  Its records must equal the
extraction step of the existing bimp_detect_device entry point on the same
summed keypoint map, on consecutive calls that reuse the shared scratch.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_extraction_matches_detect_on_two_calls():
    import torch

    from bimp_b200 import _lib as L
    from bimp_b200 import api, synth

    imgs, lam = synth.workload("vga")
    img = imgs[0]
    cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
    full = api.keypoint_matrix_to_records(api.getKeypoints(img, cs, capacity=100000))
    p = api.default_params()
    stream = C.c_void_p(int(torch.cuda.current_stream().cuda_stream))
    cap = 50000
    # two calls in a row; the larger map first so that stale scratch from the
    # first call would show up in the second
    for scale in (0, 1):
        info = cs.ks[scale]
        dmap = cs.dense_map(scale)
        kp = torch.full((7, cap), -7.0, dtype=torch.float32, device="cuda")
        cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        rc = L.lib().bimp_extract_keypoints_noalloc(
            C.c_void_p(dmap.data_ptr()), dmap.stride(0), info["data_w"], info["data_h"], info["lambda_level"],
            info["pyrstep"], p.thresh_ratio, C.c_void_p(kp.data_ptr()), kp.stride(0), cap,
            C.c_void_p(cnt.data_ptr()), stream)
        assert rc == 0, L.lib().bimp_last_error()
        n = int(cnt.item())
        got = api.keypoint_matrix_to_records(kp[:, :n])
        size = np.float32(np.float32(info["lambda_level"]) * np.float32(info["pyrstep"]))
        ref = full[full["size"] == size]
        assert n == len(ref) > 0
        # same kernels on the same map: records are bit-identical
        assert np.array_equal(got, ref)


def test_noalloc_rejects_oversized_maps():
    import torch

    from bimp_b200 import _lib as L

    d = torch.zeros((1, 4), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    # 20000 rows exceed the fixed scratch (16384 candidate rows); rejected
    # before any GPU work
    rc = L.lib().bimp_extract_keypoints_noalloc(C.c_void_p(d.data_ptr()), 4, 4, 20000, 4.0, 1.0, 0.104, None, 0, 0,
                                                C.c_void_p(cnt.data_ptr()), None)
    assert rc == L.BIMP_ERR_UNSUPPORTED
    assert b"16384" in L.lib().bimp_last_error()
