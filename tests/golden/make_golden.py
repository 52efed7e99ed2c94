"""Regenerate tests/golden/oracle_small.npz from the FP64 oracle.

    python tests/golden/make_golden.py

A 96x80 synthetic image, wavelengths 4, 5.657, 8: per-scale summed
keypoint maps D and the keypoint table.  The fixture freezes the oracle so
that any later change to its arithmetic shows up in test_oracle.py.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "cuda-bimp_b200"))

from bimp_b200 import synth  # noqa: E402
from oracle import bimp_oracle as O  # noqa: E402


def main():
    img = synth.synth_image(96, 80, 4, seed=11)
    lam = [4.0, float(np.float32(5.656854)), 8.0]
    res = O.run(img, lam)
    tab = O.keypoint_table(res)
    out = {"image": img, "lambdas": np.array(lam)}
    for i, r in enumerate(res):
        out[f"D{i}"] = r["D"]
    out["kp_scale"] = tab["scale"]
    out["kp_ix"] = tab["ix"]
    out["kp_iy"] = tab["iy"]
    out["kp_x"] = tab["x"]
    out["kp_y"] = tab["y"]
    np.savez_compressed(Path(__file__).parent / "oracle_small.npz", **out)
    print("keypoints", len(tab))


if __name__ == "__main__":
    main()
