"""ORACLE -- test infrastructure, not product code.

The error of the fixed-point cost filter against exact arithmetic.

The dense path filters the graded score (Q14 int16) with the reference's integer
recursive filter (Q15 coefficients, int32 carry, int16 store, four passes:
core/tools/de_dense.cpp:411-430,485-508), which the CUDA kernels reproduce bit for
bit.  This module states how far that arithmetic is from the same four passes in
double precision without rounding (or_filter_f64, the exact counterpart of the
reference's float rf_filter, :510-527), per configuration:

  * max and mean |int16 - float64| over every filtered value in the valid window,
    in Q14 least-significant bits (1 LSB = 1/16384 of the score scale);
  * the fraction of pixels whose winning disparity (first maximum over planes in
    ascending order, as the top-2 insert keeps it) is the same under both.

and how far the single-precision row solve (damped max-sum, belief, claim and
sub-pixel fit: core/include/doubleeye/dense_solve.hpp:213-434) is from the same solve
in double precision (or_solve_row_f64):

  * solve only: the float solve and the double solve on the same candidates; the
    fraction of pixels with the same answer (both declined, or disparities within
    0.01 px), the largest disparity difference among them, and the largest belief
    difference;
  * end to end: the int16 filter + float solve (what the GPU computes, bit for bit)
    against the double filter + double solve (exact arithmetic throughout); the
    fraction of pixels with the same answer within 0.5 px and within 1 px.

    python -m oracle.fp64_error            # one JSON line per workload
"""
from __future__ import annotations

import ctypes as C
import json
import sys
import time

import numpy as np

from . import oracle as O


def statement(orc: "O.Oracle", cfg: "O.DeCfg", L: np.ndarray, R: np.ndarray) -> dict:
    L = np.ascontiguousarray(L, np.uint8)
    R = np.ascontiguousarray(R, np.uint8)
    H, W = L.shape
    hw, hh = cfg.census_hw, cfg.census_hh
    cl = orc.census(L, hw, hh)
    cr = orc.census(R, hw, hh)
    ax, ay = orc.rf_coeffs(L, cfg.sigma_s, cfg.sigma_r)
    D = cfg.dmax - cfg.dmin + 1
    best_i = np.full((H, W), -np.inf)
    best_f = np.full((H, W), -np.inf)
    k_i = np.full((H, W), -1, np.int32)
    k_f = np.full((H, W), -1, np.int32)
    emax, esum, n = 0.0, 0.0, 0
    plane = np.zeros((H, W), np.int16)
    for k in range(D):
        d = cfg.dmin + k
        if W - hw <= hw + d:
            break
        orc.lib.or_score_plane(C.byref(cfg), L.ctypes.data, R.ctypes.data, cl.ctypes.data,
                               cr.ctypes.data, W, H, k, plane.ctypes.data)
        f64 = plane.astype(np.float64)
        i16 = plane.copy()
        orc.lib.or_filter_i16(i16.ctypes.data, ax.ctypes.data, ay.ctypes.data, W, H)
        orc.lib.or_filter_f64(f64.ctypes.data, ax.ctypes.data, ay.ctypes.data, W, H)
        win = (slice(hh, H - hh), slice(hw + d, W - hw))
        a = i16[win].astype(np.float64)
        b = f64[win]
        err = np.abs(a - b)
        emax = max(emax, float(err.max()))
        esum += float(err.sum())
        n += err.size
        bi, bf, ki, kf = best_i[win], best_f[win], k_i[win], k_f[win]
        upd = a > bi
        bi[upd] = a[upd]
        ki[upd] = k
        upd = b > bf
        bf[upd] = b[upd]
        kf[upd] = k
    valid = k_i >= 0
    return {"W": W, "H": H, "D": D, "max_err_lsb": emax, "mean_err_lsb": esum / max(n, 1),
            "winner_agreement": float((k_i[valid] == k_f[valid]).mean()), "values": n}


NONE = -1e300


def _same_answer(a: np.ndarray, b: np.ndarray, tol: float) -> np.ndarray:
    fa, fb = np.isfinite(a), np.isfinite(b)
    close = np.zeros(a.shape, bool)
    both = fa & fb
    close[both] = np.abs(a[both].astype(np.float64) - b[both]) <= tol
    return (~fa & ~fb) | close


def solve_statement(orc: "O.Oracle", cfg: "O.DeCfg", L: np.ndarray, R: np.ndarray) -> dict:
    L = np.ascontiguousarray(L, np.uint8)
    R = np.ascontiguousarray(R, np.uint8)
    H, W = L.shape
    cs, cd, cn, cnb = orc.cost_top2(cfg, L, R)
    d32 = np.zeros((H, W), np.float32)
    b32 = np.zeros((H, W), np.float32)
    for y in range(H):
        d, b, _ = orc.solve_row_debug(cfg, cs[y], cd[y], cn[y], cnb[y] if cfg.subpixel else None)
        d32[y], b32[y] = d, b
    nb = np.where(cnb == -32768, NONE, cnb.astype(np.float64) / 16384.0)
    if not cfg.subpixel:
        nb[:] = NONE
    cs64 = np.where(cs > -1e29, cs.astype(np.float64), NONE)
    d64, b64 = orc.solve_f64(cfg, cs64, cd, cn, nb)
    same = _same_answer(d32, d64, 0.01)
    both = np.isfinite(d32) & np.isfinite(d64) & same
    belief = (b32 > -1e29) & (b64 > -1e29)
    fcs, fcd, fcn, fnb = orc.cost_top2_f64(cfg, L, R)
    e64, _ = orc.solve_f64(cfg, fcs, fcd, fcn, fnb)
    return {"solve_agreement": float(same.mean()),
            "solve_max_disp_diff_px": float(np.abs(d32[both] - d64[both]).max()) if both.any() else 0.0,
            "solve_max_belief_err": float(np.abs(b32[belief] - b64[belief]).max()) if belief.any() else 0.0,
            "e2e_agreement_0p5px": float(_same_answer(d32, e64, 0.5).mean()),
            "e2e_agreement_1px": float(_same_answer(d32, e64, 1.0).mean()),
            "filled_f32": float(np.isfinite(d32).mean()),
            "filled_f64": float(np.isfinite(e64).mean()), "iters": int(cfg.iters)}


def workloads():
    from doubleeye_b200 import synth
    yield "C1 848x480 D=64 census 9x7", O.default_cfg(dmax=64, iters=10, census_hw=4), \
        synth.fronto_planes(848, 480)
    yield "C2 848x480 D=128", O.default_cfg(dmax=128, iters=8), \
        synth.slanted_planes(848, 480, 127)
    yield "C3 1500x1000 D=256", O.default_cfg(dmax=256, iters=12), synth.large_scene()
    yield "C4 1280x720 D=256", O.default_cfg(dmax=256, iters=8), \
        synth.slanted_planes(1280, 720, 255, tag="c4-1280")


def main() -> None:
    orc = O.Oracle()
    for name, cfg, p in workloads():
        t = time.perf_counter()
        s = statement(orc, cfg, p.left, p.right)
        s.update(solve_statement(orc, cfg, p.left, p.right))
        s["config"] = name
        s["seconds"] = round(time.perf_counter() - t, 1)
        print(json.dumps(s), flush=True)


if __name__ == "__main__":
    sys.exit(main())
