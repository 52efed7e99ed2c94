"""The FP64 reference gradient against central finite differences (CPU).

The loss is piecewise smooth (ReLUs): steps must be small enough not to
cross kinks.  At step 1e-7 the hand-written adjoint agrees with finite
differences to ~1e-8 relative; the test asserts 1e-5.  At the step 1e-4
named for the workload, kink crossings alone move the finite difference by
up to ~1% on this image, which the second test records.

Exactly flat image regions make the complex response e + i o exactly zero,
where |.| has no derivative: the gradient there is the direction of the
rounding noise of z, so it differs between FP64 and FP32 and from finite
differences (on 512x512 images of flat polygons by tens of percent).  The
last test shows that the same picture dequantised (u8 + U(-0.5, 0.5)) / 255
agrees with finite differences at 512x512.
"""
import numpy as np
import pytest

from bimp_b200 import synth
from oracle import bimp_adjoint as A


@pytest.fixture(scope="module")
def case():
    X = synth.synth_image(64, 56, 3, seed=5).astype(np.float64) / 255.0
    lam = [4.0, 5.656854, 8.0]
    M = A.masks_for(X.shape, lam, 7)
    return X, lam, M, A.gradient(X, lam, M)


def test_parameter_gradients_match_fd(case):
    X, lam, M, (L, gX, gth) = case
    h = 1e-7
    for name in ("alpha", "rho", "w_tan", "w_rad"):
        tp, tm = A.Theta(), A.Theta()
        setattr(tp, name, getattr(tp, name) + h)
        setattr(tm, name, getattr(tm, name) - h)
        fd = (A.loss(X, lam, M, tp) - A.loss(X, lam, M, tm)) / (2 * h)
        assert abs(fd - gth[name]) <= 1e-5 * abs(fd), (name, fd, gth[name])


def test_image_gradient_matches_fd(case):
    X, lam, M, (L, gX, gth) = case
    rng = np.random.default_rng(0)
    for _ in range(3):
        v = rng.standard_normal(X.shape)
        h = 1e-7
        fd = (A.loss(X + h * v, lam, M) - A.loss(X - h * v, lam, M)) / (2 * h)
        assert abs(fd - float((gX * v).sum())) <= 1e-5 * abs(fd)


def test_fd_at_step_1e4_is_kink_limited(case):
    X, lam, M, (L, gX, gth) = case
    h = 1e-4
    tp, tm = A.Theta(alpha=1 + h), A.Theta(alpha=1 - h)
    fd = (A.loss(X, lam, M, tp) - A.loss(X, lam, M, tm)) / (2 * h)
    rel = abs(fd - gth["alpha"]) / abs(fd)
    print("alpha: FD(1e-4) vs adjoint relative difference", rel)
    assert rel < 5e-2


def test_dequantised_512_matches_fd():
    X = synth.dequantised(synth.synth_image(512, 512, 20, seed=3), seed=5).astype(np.float64)
    lam = [4.0]
    M = A.masks_for(X.shape, lam, 7)
    L, gX, gth = A.gradient(X, lam, M)
    rng = np.random.default_rng(1)
    v = rng.standard_normal(X.shape)
    h = 1e-8
    fd = (A.loss(X + h * v, lam, M) - A.loss(X - h * v, lam, M)) / (2 * h)
    rel = abs(fd - float((gX * v).sum())) / abs(fd)
    print("512x512 dequantised: FD(1e-8) vs adjoint relative difference", rel)
    # a few hundred ReLU kinks lie within +-1e-8 v of this point
    assert rel < 5e-3
