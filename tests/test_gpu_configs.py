"""Parity at each workload configuration's own size.

* 64 mixed-size images (W in [320, 1920], H in [240, 1080]) in one batch:
  every image's keypoints equal the single-image path bit for bit under the
  default tile plan, and four images (the largest among them) match the FP32
  C restatement of the reference pipeline (oracle/cbimp.c) under the default
  and under the autotuned tile plan.
* 32 correlated 3840x2160 frames with the 12-scale bank in one batch: frames
  0 and 31 against the C restatement, frame 0 also bit for bit against the
  single-image path.

Tolerances (tests/parity.py): summed keypoint maps within 1e-4 of the map
peak; keypoint (scale, x, y) sets equal except where the restatement's
decision is within 1e-4 of the map peak of a tie, at most max(2, n/1000) such
pixels per scale.
"""
import numpy as np
import pytest

from bimp_b200 import api, synth
from parity import check_against_c_restatement

pytestmark = pytest.mark.gpu


def _records(kp):
    return api.keypoint_matrix_to_records(kp)


def _batch_maps(b, i, n_scales):
    return [b.dense_map(i, s).cpu().numpy() for s in range(n_scales)]


def _c_check(img, lam, rec, maps):
    from oracle.cbimp import CBimp
    with CBimp(img.shape[1], img.shape[0], lam) as cb:
        ref, total = cb.detect(img, capacity=1 << 21)
        assert total == len(ref)
        return check_against_c_restatement(cb, ref, lam, rec, maps)


def test_mixed_batch_of_64_images():
    imgs, lam = synth.workload("mixed")
    sizes = [(im.shape[1], im.shape[0]) for im in imgs]
    assert len(imgs) == 64
    b = api.Batch(sizes, lam, kp_capacity=1 << 17)
    b.load(imgs)
    b.run()
    n_kp = 0
    for i, img in enumerate(imgs):
        cs = api.CudaStuff(img.shape[1], img.shape[0], lam)
        ref = _records(api.getKeypoints(img, cs, capacity=1 << 17))
        got = _records(b.keypoints(i))
        assert np.array_equal(ref, got), i
        for s in range(len(lam)):
            assert np.array_equal(cs.dense_map(s).cpu().numpy(), b.dense_map(i, s).cpu().numpy()), (i, s)
        n_kp += len(got)
        cs.close()
    largest = int(np.argmax([w * h for w, h in sizes]))
    picks = [largest] + [i for i in (0, 21, 42, 63) if i != largest][:3]
    worst = {"map_err": 0.0, "symdiff": 0}
    for i in picks:
        rep = _c_check(imgs[i], lam, _records(b.keypoints(i)), _batch_maps(b, i, len(lam)))
        worst["map_err"] = max(worst["map_err"], rep["map_err"])
        worst["symdiff"] += sum(rep["symdiff"])
    # the autotuned plan (it may move tile boundaries: float rounding only)
    tune = b.autotune(reps=2)
    b.run()
    for i in picks:
        rep = _c_check(imgs[i], lam, _records(b.keypoints(i)), _batch_maps(b, i, len(lam)))
        worst["map_err"] = max(worst["map_err"], rep["map_err"])
        worst["symdiff"] += sum(rep["symdiff"])
    print({"images": 64, "keypoints": n_kp, "checked_against_c": picks, "chosen_plan": tune["chosen"], **worst})
    b.close()


def test_uhd_batch_of_32_frames():
    frames = synth.uhd_frames(32, 1004)
    lam = synth.bank(12)
    b = api.Batch([(3840, 2160)] * 32, lam, kp_capacity=1 << 20)
    b.load(frames)
    b.run()
    counts = b.counts().cpu().numpy()
    assert (counts > 0).all() and (counts <= 1 << 20).all()
    worst = {"map_err": 0.0, "symdiff": 0, "keypoints": 0}
    for i in (0, 31):
        rec = _records(b.keypoints(i))
        rep = _c_check(frames[i], lam, rec, _batch_maps(b, i, len(lam)))
        worst["map_err"] = max(worst["map_err"], rep["map_err"])
        worst["symdiff"] += sum(rep["symdiff"])
        worst["keypoints"] += rep["keypoints"]
    rec0 = _records(b.keypoints(0))
    maps0 = _batch_maps(b, 0, len(lam))
    b.close()
    cs = api.CudaStuff(3840, 2160, lam)
    assert np.array_equal(_records(api.getKeypoints(frames[0], cs, capacity=1 << 20)), rec0)
    for s in range(len(lam)):
        assert np.array_equal(cs.dense_map(s).cpu().numpy(), maps0[s])
    cs.close()
    print({"frames": 32, "checked_against_c": [0, 31], **worst})
