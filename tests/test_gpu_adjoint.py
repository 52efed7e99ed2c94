"""GPU adjoint of the summed keypoint map against the FP64 CPU reference
gradient (oracle/bimp_adjoint.py), which itself is checked against central
finite differences in tests/test_adjoint_oracle.py.

Tolerance: relative 1e-3 (norm-wise for the image gradient, per component
for the four parameters), the north-star bar for the adjoint.
"""
import numpy as np
import pytest

from bimp_b200 import api, synth
from oracle import bimp_adjoint as A

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-3


def _run(w, h, n, lam, seed):
    import torch
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
    gp = gp.cpu().numpy()
    views = [[masks[i * adj.mask_stride + off:i * adj.mask_stride + off + ww * hh].reshape(hh, ww).astype(np.float64)
              for (off, ww, hh) in adj.layout] for i in range(n)]
    ref_loss, ref_g, ref_p = 0.0, [], np.zeros(4)
    for i in range(n):
        l_i, g_i, p_i = A.gradient(imgs[i].astype(np.float64), lam, views[i])
        ref_loss += l_i
        ref_g.append(g_i)
        ref_p += np.array([p_i["alpha"], p_i["rho"], p_i["w_tan"], p_i["w_rad"]])
    return loss, g, gp, ref_loss, np.stack(ref_g), ref_p


@pytest.mark.parametrize("w,h,n,lam", [
    (96, 80, 2, [4.0, 5.656854, 8.0]),          # padded torus, two levels
    (128, 128, 1, [4.0, 8.0]),                  # fftW == dataW and fftH == dataH at every level
])
def test_adjoint_matches_cpu_reference(w, h, n, lam):
    loss, g, gp, ref_loss, ref_g, ref_p = _run(w, h, n, lam, seed=21)
    print("loss", loss, ref_loss, "params", gp, ref_p)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-6
    err = np.linalg.norm(g - ref_g) / np.linalg.norm(ref_g)
    print("image gradient relative error", err)
    assert err <= GRAD_TOL
    for k in range(4):
        assert abs(gp[k] - ref_p[k]) <= GRAD_TOL * abs(ref_p[k]) + 1e-6, (k, gp[k], ref_p[k])
