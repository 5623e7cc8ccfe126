"""Golden vectors for the disparity-prior path (--prior), from the reference itself.

The reference's run_dense with a full-resolution prior (core/tools/de_dense.cpp:
738-1608; the mask :797-853, the rectangle filter :438-483, the masked insert
:1166-1297), compiled from its sources into oracle/_ref/ and run at one thread.
Priors: the ground truth plus seeded noise, a constant, and a ramp that leaves part
of the image without candidates.

    python tests/golden/make_golden_prior.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from doubleeye_b200 import synth  # noqa: E402


def cases():
    p = synth.slanted_planes(200, 120, 47, seed=5, tag="prior")
    rng = synth.rng_for("golden:prior")
    noisy = (p.disparity + rng.normal(0, 1.5, p.disparity.shape)).astype(np.float32)
    yield "noisy_b2", p, noisy, 2, dict(dmax=48, iters=8)
    yield "noisy_b4_lrc", p, noisy, 4, dict(dmax=48, iters=4, lrc=1)
    yield "const_b1", p, np.full(p.disparity.shape, 20.3, np.float32), 1, dict(dmax=48)
    q = synth.slanted_planes(160, 96, 63, seed=6, tag="prior-ramp")
    ramp = np.tile(np.linspace(-10, 90, 160, dtype=np.float32), (96, 1))
    yield "ramp_b3", q, ramp, 3, dict(dmax=64, iters=8, dmin=2)


def main() -> None:
    O.build(ref=True)
    ref = O.Reference()
    out = {}
    for name, p, prior, band, kw in cases():
        cfg = O.default_cfg(**kw)
        d, m, c = ref.dense_prior(cfg, p.left, p.right, prior, band)
        out.update({f"{name}_L": p.left, f"{name}_R": p.right, f"{name}_prior": prior,
                    f"{name}_disp": d, f"{name}_margin": m, f"{name}_cand": c,
                    f"{name}_band": np.array(band),
                    f"{name}_cfg": np.array([repr(kw)])})
        print(name, "filled %.3f" % np.isfinite(d).mean())
    np.savez_compressed(os.path.join(HERE, "prior.npz"), **out)


if __name__ == "__main__":
    main()
