"""Golden vectors for the prior hole fill, from the reference's own ``fill``
(article/coarse_to_fine.py:58-76), imported in place.  Inputs are seeded maps with
holes: scattered, in large blobs, along the edges (the fill wraps around), nearly all
holes, and all holes.  Needs DOUBLEEYE_REF.

    DOUBLEEYE_REF=<reference root> python tests/golden/make_golden_fill.py
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def cases():
    rng = np.random.default_rng(20261204)
    out = []
    for name, (H, W), frac in [("scatter", (48, 64), 0.3), ("dense_holes", (31, 17), 0.9),
                               ("tiny", (5, 3), 0.8), ("one_valid", (20, 24), 1.0)]:
        d = rng.uniform(1, 60, (H, W)).astype(np.float32)
        d[rng.random((H, W)) < frac] = np.nan
        if name == "one_valid":
            d[7, 11] = 17.25
        out.append((name, d))
    d = rng.uniform(5, 40, (96, 120)).astype(np.float32)       # blobs and edge strips
    yy, xx = np.mgrid[:96, :120]
    d[(yy - 40) ** 2 + (xx - 60) ** 2 < 25 ** 2] = np.nan
    d[:, :6] = np.nan
    d[:3, :] = np.nan
    out.append(("blobs_edges", d))
    out.append(("all_holes", np.full((9, 13), np.nan, np.float32)))
    return out


def main() -> None:
    path = os.path.join(O.reference_root(), "article", "coarse_to_fine.py")
    spec = importlib.util.spec_from_file_location("coarse_to_fine", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    data = {}
    for name, d in cases():
        data[name + "_in"] = d
        data[name + "_out"] = mod.fill(d).astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "fill.npz"), **data)
    print("fill cases:", [n for n, _ in cases()])


if __name__ == "__main__":
    main()
