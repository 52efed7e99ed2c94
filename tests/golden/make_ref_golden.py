"""Regenerate tests/golden/ref_small.npz: outputs of the reference's own BIMP
device kernels (oracle/_ref/libbimpref.so, see oracle/refrun.py) on two small
synthetic images.  Needs a CUDA device and the built reference library.

    python tests/golden/make_ref_golden.py [--out PATH]

Cases: a 128x96 image with wavelengths 4, 5.657, 8 (levels 0 and 1) and a
128x64 image with wavelengths 4, 5.657, whose torus equals its data
(fftW == dataW, fftH == dataH: the stencils' flat reads pass the torus).  Per
scale the summed keypoint map D and the single-stopped map S (float32), and
the keypoint records.  The CPU test tests/test_oracle.py checks the FP64
oracle against these fixtures.
"""
import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "cuda-bimp_b200"))

from bimp_b200 import synth  # noqa: E402
from oracle import refrun  # noqa: E402

CASES = {
    "a": (128, 96, 5, 21, [4.0, float(np.float32(5.656854)), 8.0]),
    "b": (128, 64, 3, 23, [4.0, float(np.float32(5.656854))]),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).parent / "ref_small.npz"))
    args = ap.parse_args()
    out = {}
    for name, (w, h, npoly, seed, lam) in CASES.items():
        img = synth.synth_image(w, h, npoly, seed=seed)
        res = refrun.run(img, lam)
        out[f"{name}_image"] = img
        out[f"{name}_lambdas"] = np.array(lam)
        for i, r in enumerate(res):
            out[f"{name}_D{i}"] = r["D"]
            out[f"{name}_S{i}"] = r["S"]
        rec = refrun.records(res)
        for f in ("x", "y", "size", "response", "octave", "class_id", "angle"):
            out[f"{name}_kp_{f}"] = rec[f]
        print(name, "keypoints", len(rec))
    np.savez_compressed(args.out, **out)


if __name__ == "__main__":
    main()
