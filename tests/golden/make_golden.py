"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs only where the reference tree is present: it builds oracle/_ref/ (the reference
compiled from its own sources by oracle/Makefile) and records the reference's outputs
on small seeded inputs.  The committed .npz files are what the CPU and GPU parity
tests read; nothing at test time needs the reference tree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402
from doubleeye_b200 import synth  # noqa: E402

SCENES = os.path.join(O.reference_root(), "article", "scenes")

# (name, W, H, cfg overrides) -- small enough for the single-threaded oracle to check
# in well under a second each, spread over the configuration space the path supports.
DENSE_CASES = [
    ("dense_a", 97, 41, dict(dmax=16)),
    ("dense_b", 128, 64, dict(dmax=32, iters=8)),
    ("dense_c", 96, 48, dict(dmax=24, iters=3, subpixel=0)),
    ("dense_d", 120, 40, dict(dmax=20, iters=2, lrc=1)),
    ("dense_e", 80, 40, dict(dmax=16, fit_eq=0, min_margin=0.01, iters=1)),
    ("dense_f", 110, 36, dict(dmin=3, dmax=40, iters=4, min_ratio=1.05, ad=0.0)),
    ("dense_g", 64, 64, dict(dmax=64, iters=8, damping=0.0, lambda_=0.05, gamma=-0.2)),
    ("dense_h", 200, 24, dict(dmax=128, iters=8, ad_trunc=30, sigma_s=12.0, sigma_r=0.3)),
]


def cfg_dict(c: O.DeCfg) -> dict:
    return {f: getattr(c, f) for f, _ in c._fields_}


def main() -> None:
    O.build(ref=True)
    ref = O.Reference()
    out = {}

    # --- census / coefficients / filter on a random image and plane ----------------
    rng = synth.rng_for("golden:primitives")
    img = rng.integers(0, 256, (37, 61)).astype(np.uint8)
    img[5:12, 8:20] = 77                      # a flat patch: ties in every compare
    plane = rng.integers(-16384, 16385, (37, 61)).astype(np.int16)
    ax, ay = ref.rf_coeffs(img)
    ax2, ay2 = ref.rf_coeffs(img, 12.0, 0.3)
    np.savez_compressed(
        os.path.join(HERE, "primitives.npz"), img=img, census_7x7=ref.census(img, 3, 3),
        census_9x7=ref.census(img, 4, 3), census_5x5=ref.census(img, 2, 2), ax=ax, ay=ay,
        ax_12_03=ax2, ay_12_03=ay2, plane=plane, filtered=ref.filter_i16(plane, ax, ay))
    out["primitives"] = img.shape

    # --- end-to-end dense runs -------------------------------------------------------
    for name, W, H, kw in DENSE_CASES:
        dmax = kw.get("dmax", 60)
        p = synth.slanted_planes(W, H, min(dmax, 3 * W // 4), tag=f"golden:{name}")
        cfg = O.default_cfg(**kw)
        disp, margin, cand, _ = ref.dense(cfg, p.left, p.right, nthreads=1)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), L=p.left, R=p.right,
                            disp=disp, margin=margin, cand=cand,
                            cfg=np.array([repr(cfg_dict(cfg))]))
        out[name] = (W, H, int(np.isfinite(disp).sum()))

    # --- a real camera pair (reference article/scenes), cropped ----------------------
    for scene, (x0, y0) in (("morning_on", (300, 200)), ("night_off", (200, 150))):
        L = np.fromfile(f"{SCENES}/{scene}/left.y8", np.uint8).reshape(480, 848)
        R = np.fromfile(f"{SCENES}/{scene}/right.y8", np.uint8).reshape(480, 848)
        L = np.ascontiguousarray(L[y0:y0 + 96, x0:x0 + 192])
        R = np.ascontiguousarray(R[y0:y0 + 96, x0:x0 + 192])
        cfg = O.default_cfg(dmax=48, iters=8)
        disp, margin, cand, _ = ref.dense(cfg, L, R, nthreads=1)
        np.savez_compressed(os.path.join(HERE, f"real_{scene}.npz"), L=L, R=R, disp=disp,
                            margin=margin, cand=cand, cfg=np.array([repr(cfg_dict(cfg))]))
        out[f"real_{scene}"] = int(np.isfinite(disp).sum())

    # --- confidence on a grid (the reference test's known answers are in the tests) -
    s1 = np.linspace(-0.2, 1.0, 25, dtype=np.float32)
    s2 = np.linspace(-1.0, 1.0, 21, dtype=np.float32)
    grid = np.array([[ref.confidence(a, b, -0.1, 0.0, 1.0) for b in s2] for a in s1],
                    np.float32)
    grid_cap = np.array([[ref.confidence(a, b, -0.1, 2.0, 1.0) for b in s2] for a in s1],
                        np.float32)
    grid_u8 = np.array([[ref.confidence_u8(a, b, -0.1, 0.0, 1.0) for b in s2] for a in s1],
                       np.uint8)
    np.savez_compressed(os.path.join(HERE, "confidence.npz"), s1=s1, s2=s2, conf=grid,
                        conf_capped=grid_cap, conf_u8=grid_u8)

    for k, v in out.items():
        print(k, v)


if __name__ == "__main__":
    main()
