"""Comparison helpers shared by the parity tests.

Integer stages compare bit for bit.  The row solve orders pixels for the one-to-one
claim by belief; the reference uses std::sort (core/include/doubleeye/dense_solve.hpp:359),
whose order among exactly tied beliefs is unspecified, while this build and the oracle
break ties by x.  ``tie_aware_disp`` therefore accepts a disparity difference only
where it is such a tie: the pixel and at least one other eligible claimant of the same
right pixel have bit-equal beliefs, and both sides award that right pixel to the same
number of claimants.
"""
from __future__ import annotations

import numpy as np


def same_f32(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Elementwise bit-equality for float arrays, NaN equal to NaN."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))


def candidates_from_cand6(cand: np.ndarray, dmin: int):
    """Rebuild cs/cd/cn planes (H, W, 2) from the reference's --out-conf planes."""
    s1, s2, d1, d2 = cand[0], cand[1], cand[2], cand[3]
    H, W = s1.shape
    cs = np.stack([s1, s2], -1).astype(np.float32)
    cd = np.stack([d1, d2], -1)
    cd = np.where(cd > -1e29, cd - dmin, -1).astype(np.int32)
    cn = (s1 > -1e29).astype(np.int32) + (s2 > -1e29).astype(np.int32)
    return cs, cd, cn


def tie_aware_disp(oracle, cfg, cs, cd, cn, cnb, disp_test, disp_ref):
    """Assert disp_test == disp_ref except at exact-tie claim conflicts.
    Returns (n_mismatch, n_pixels)."""
    eq = same_f32(disp_test, disp_ref)
    bad_rows = np.nonzero(~eq.all(axis=1))[0]
    for y in bad_rows:
        _, best, target = oracle.solve_row_debug(
            cfg, cs[y], cd[y], cn[y], cnb[y] if cnb is not None else None)
        for x in np.nonzero(~eq[y])[0]:
            t = target[x]
            assert t >= 0, f"row {y} x {x}: mismatch at a pixel that claims nothing"
            grp = (target == t) & (best == best[x])
            assert grp.sum() >= 2, (
                f"row {y} x {x}: mismatch without an exact tie "
                f"(test {disp_test[y, x]}, ref {disp_ref[y, x]})")
            nt = np.isfinite(disp_test[y][grp]).sum()
            nr = np.isfinite(disp_ref[y][grp]).sum()
            assert nt == nr and nt <= 1, f"row {y} x {x}: tie group winners {nt} vs {nr}"
    return int((~eq).sum()), int(eq.size)
