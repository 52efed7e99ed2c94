"""GPU adjoint of the summed keypoint map against the FP64 CPU reference
gradient (oracle/bimp_adjoint.py), which itself is checked against central
finite differences in tests/test_adjoint_oracle.py.

The loss is piecewise linear in the complex cells (ReLUs), so the gradient is
that of the linear piece the forward lands on.  A float32 forward lands on a
different piece than the FP64 reference wherever a ReLU argument is within
float rounding of zero: at 512x512 there are hundreds of such pixels (and
exact ties along straight image edges, where the loss has no gradient), each
moving the gradient by one pixel's share.  The comparison is therefore made
branch-matched: the reference takes its piecewise choices (ReLU states, the
magnitude floor) from the device's float32 complex cells and computes
everything else in FP64.  Tolerance 1e-3 relative (norm-wise for the image
gradient, per component for the four parameters), the north-star bar.  The
unmatched difference is printed for the record.
"""
import numpy as np
import pytest

from bimp_b200 import api, synth
from oracle import bimp_adjoint as A

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-3


def _run(w, h, n, lam, seed, imgs=None):
    import torch
    if imgs is None:
        imgs = np.stack([synth.synth_image(w, h, max(2, w * h // 3000), seed=seed + i).astype(np.float32) / 255.0
                         for i in range(n)])
    adj = api.Adjoint(w, h, n, lam)
    rng = np.random.default_rng(seed)
    masks = rng.standard_normal(n * adj.mask_stride).astype(np.float32)
    mt = torch.from_numpy(masks).cuda()
    xt = torch.from_numpy(imgs).cuda().contiguous()
    loss = float(adj.forward(xt, mt).item())
    g, gp = adj.backward()
    g = g.cpu().numpy()
    gp = gp.cpu().numpy().copy()
    views = [[masks[i * adj.mask_stride + off:i * adj.mask_stride + off + ww * hh].reshape(hh, ww).astype(np.float64)
              for (off, ww, hh) in adj.layout] for i in range(n)]
    decide = [[np.stack([adj.complex_map(i, s, o).cpu().numpy() for o in range(8)]) for s in range(len(adj.layout))]
              for i in range(n)]
    ref = {"loss": 0.0, "g": [], "p": np.zeros(4), "g_free": [], "p_free": np.zeros(4)}
    for i in range(n):
        x64 = imgs[i].astype(np.float64)
        l_i, g_i, p_i = A.gradient(x64, lam, views[i], decide=decide[i])
        ref["loss"] += l_i
        ref["g"].append(g_i)
        ref["p"] += np.array([p_i["alpha"], p_i["rho"], p_i["w_tan"], p_i["w_rad"]])
        _, gf, pf = A.gradient(x64, lam, views[i])
        ref["g_free"].append(gf)
        ref["p_free"] += np.array([pf["alpha"], pf["rho"], pf["w_tan"], pf["w_rad"]])
    adj.close()
    return loss, g, gp, ref


def _check(loss, g, gp, ref):
    print("loss", loss, ref["loss"], "params", gp, ref["p"])
    assert abs(loss - ref["loss"]) <= 1e-4 * abs(ref["loss"]) + 1e-6
    err = np.linalg.norm(g - np.stack(ref["g"])) / np.linalg.norm(np.stack(ref["g"]))
    free = np.linalg.norm(g - np.stack(ref["g_free"])) / np.linalg.norm(np.stack(ref["g_free"]))
    print(f"image gradient relative error: branch-matched {err:.3e}, FP64 branch {free:.3e}")
    print("parameter relative error (FP64 branch)", np.abs(gp - ref["p_free"]) / np.abs(ref["p_free"]))
    assert err <= GRAD_TOL
    for k in range(4):
        assert abs(gp[k] - ref["p"][k]) <= GRAD_TOL * abs(ref["p"][k]) + 1e-6, (k, gp[k], ref["p"][k])
    return err


@pytest.mark.parametrize("w,h,n,lam", [
    (96, 80, 2, [4.0, 5.656854, 8.0]),          # padded torus, two levels
    (128, 128, 1, [4.0, 8.0]),                  # fftW == dataW and fftH == dataH at every level
])
def test_adjoint_matches_cpu_reference(w, h, n, lam):
    _check(*_run(w, h, n, lam, seed=21))


def test_adjoint_workload_images_match_cpu_reference():
    """Two of the 16 512x512 workload images (uint8 content / 255), 6 scales:
    three pyramid levels, fftW == dataW at each, flat polygons and polygons
    cut by the image border (straight edges on the torus)."""
    imgs, lam = synth.workload("adjoint")
    _check(*_run(512, 512, 2, lam, seed=31, imgs=np.stack(imgs[:2])))


def test_adjoint_is_repeatable():
    """backward() twice after one forward, and forward+backward twice, give
    the same gradient (the accumulators are cleared every call)."""
    import torch
    imgs, lam = synth.workload("adjoint")
    x = torch.from_numpy(np.stack(imgs[:1])).cuda().contiguous()
    adj = api.Adjoint(512, 512, 1, lam)
    m = torch.from_numpy(np.random.default_rng(4).standard_normal(adj.mask_stride).astype(np.float32)).cuda()
    adj.forward(x, m)
    g1, p1 = adj.backward()
    g1, p1 = g1.clone(), p1.clone()
    g2, p2 = adj.backward()
    adj.forward(x, m)
    g3, p3 = adj.backward()
    scale = g1.abs().max().item()
    # float atomics: equal up to summation order
    assert (g1 - g2).abs().max().item() <= 1e-5 * scale and (g1 - g3).abs().max().item() <= 1e-5 * scale
    assert torch.allclose(p1, p2, rtol=1e-6) and torch.allclose(p1, p3, rtol=1e-6)
    adj.close()


def test_adjoint_all_16_workload_images():
    """All 16 images of the 512x512 adjoint workload, 6 scales: branch-matched
    error (the 1e-3 bar) and, for the record, the error against the FP64
    reference's own branch."""
    imgs, lam = synth.workload("adjoint")
    err = _check(*_run(512, 512, 16, lam, seed=37, imgs=np.stack(imgs)))
    print(f"16 images: branch-matched {err:.3e}")


def test_adjoint_uhd_crop_with_12_scales():
    """A 1024x1024 crop of a 3840x2160 frame (uint8 / 255) with the 12-scale
    bank: six pyramid levels down to 32x32, where the coarse scales' kernels
    are wider than their torus (the taps wrap and add)."""
    frame = synth.uhd_frames(1, 1004)[0]
    crop = np.ascontiguousarray(frame[568:1592, 1408:2432]).astype(np.float32) / np.float32(255.0)
    _check(*_run(1024, 1024, 1, synth.bank(12), seed=43, imgs=crop[None]))


def test_autograd_wrapper_matches_finite_differences_on_one_linear_piece():
    """torch.autograd through SummedKeypointMapLoss on two 96x80 images whose
    content has no exactly flat regions (uint8 content plus U(-0.5, 0.5),
    / 255): the directional derivative of the GPU gradient along a seeded
    direction, and the four parameter gradients, against central finite
    differences of the FP64 loss.  The steps (1e-7 along a unit-variance
    direction on the image, 1e-6 on the parameters) keep every ReLU argument
    on its side, so the differences see one linear piece (on the FP64
    reference they match its gradient to about 1e-8; at 1e-6 on the image
    they already cross kinks); tolerance 1e-3 relative."""
    import torch
    from bimp_b200.autograd import summed_map_loss, summed_map_theta
    w, h, n = 96, 80, 2
    lam = [4.0, 5.656854, 8.0]
    imgs = np.stack([synth.dequantised(synth.synth_image(w, h, 4, seed=60 + i), seed=70 + i) for i in range(n)])
    adj = api.Adjoint(w, h, n, lam)
    rng = np.random.default_rng(8)
    masks = rng.standard_normal(n * adj.mask_stride).astype(np.float32)
    x = torch.from_numpy(imgs).cuda().requires_grad_(True)
    theta = summed_map_theta(adj)
    loss = summed_map_loss(x, theta, torch.from_numpy(masks).cuda(), adj)
    gx, gth = torch.autograd.grad(loss, [x, theta])
    gx = gx.cpu().numpy().astype(np.float64)
    gth = gth.cpu().numpy()
    views = [[masks[i * adj.mask_stride + off:i * adj.mask_stride + off + ww * hh].reshape(hh, ww).astype(np.float64)
              for (off, ww, hh) in adj.layout] for i in range(n)]
    adj.close()
    X = imgs.astype(np.float64)

    def L(Xs, th=A.Theta()):
        return sum(A.loss(Xs[i], lam, views[i], th) for i in range(n))

    v = np.random.default_rng(12).standard_normal(X.shape)
    hx = 1e-7
    fd = (L(X + hx * v) - L(X - hx * v)) / (2 * hx)
    dd = float((gx * v).sum())
    print("directional derivative: gpu", dd, "finite difference", fd)
    assert abs(dd - fd) <= 1e-3 * abs(fd)
    base = A.Theta()
    for k, name in enumerate(("alpha", "rho", "w_tan", "w_rad")):
        hp = 1e-6
        up = A.Theta(**{**base.__dict__, name: getattr(base, name) + hp})
        dn = A.Theta(**{**base.__dict__, name: getattr(base, name) - hp})
        fdp = (L(X, up) - L(X, dn)) / (2 * hp)
        print(name, "gpu", gth[k], "finite difference", fdp)
        assert abs(gth[k] - fdp) <= 1e-3 * abs(fdp) + 1e-9


def test_adjoint_chunked_scratch_matches(monkeypatch):
    """The per-cell scratch of one image at a time (BIMP_ADJOINT_CHUNK=1, as
    large batches use automatically) gives the loss and gradients of the
    all-images layout, in less device memory; complex cells remain readable
    for the images of the last chunk only."""
    import torch
    from bimp_b200 import _lib as L
    w, h, n = 96, 80, 3
    lam = [4.0, 5.656854, 8.0]
    imgs = np.stack([synth.synth_image(w, h, 4, seed=80 + i).astype(np.float32) / 255.0 for i in range(n)])
    x = torch.from_numpy(imgs).cuda().contiguous()
    full = api.Adjoint(w, h, n, lam)
    m = torch.from_numpy(np.random.default_rng(3).standard_normal(n * full.mask_stride).astype(np.float32)).cuda()
    l_full = float(full.forward(x, m).item())
    g_full, p_full = full.backward()
    g_full, p_full = g_full.clone(), p_full.clone()
    monkeypatch.setenv("BIMP_ADJOINT_CHUNK", "1")
    ch = api.Adjoint(w, h, n, lam)
    l_ch = float(ch.forward(x, m).item())
    g_ch, p_ch = ch.backward()
    assert ch.device_bytes() < full.device_bytes()
    assert abs(l_ch - l_full) <= 1e-12 * abs(l_full)
    scale = g_full.abs().max().item()
    assert (g_ch - g_full).abs().max().item() <= 1e-5 * scale
    assert torch.allclose(p_ch, p_full, rtol=1e-6, atol=1e-9)
    with pytest.raises(L.BimpError):
        ch.complex_map(0, 0, 0)
    assert torch.equal(ch.complex_map(n - 1, 0, 0), full.complex_map(n - 1, 0, 0))
    full.close()
    ch.close()
