"""Copy the reference's six real 848x480 IR pairs (article/scenes/*/left.y8, right.y8:
one kitchen at three light levels, projector on and off) into tests/golden/scenes.npz.

They are input fixtures for the full-size parity tests against the reference itself
(tests/test_reference_full_gpu.py); the reference's outputs on them are computed at
test time by oracle/_ref, so only the images are stored.  Needs DOUBLEEYE_REF.

    DOUBLEEYE_REF=<reference root> python tests/golden/make_scenes.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

W, H = 848, 480


def main() -> None:
    root = os.path.join(O.reference_root(), "article", "scenes")
    out = {}
    for name in sorted(os.listdir(root)):
        d = os.path.join(root, name)
        if not os.path.isdir(d):
            continue
        for side, f in (("L", "left.y8"), ("R", "right.y8")):
            img = np.fromfile(os.path.join(d, f), np.uint8)
            assert img.size == W * H, (name, f, img.size)
            out[f"{name}_{side}"] = img.reshape(H, W)
    np.savez_compressed(os.path.join(HERE, "scenes.npz"), **out)
    print("scenes:", sorted({k[:-2] for k in out}))


if __name__ == "__main__":
    main()
