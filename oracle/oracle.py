"""ORACLE -- test infrastructure, not product code.

ctypes front end for the two CPU checkers built by ``oracle/Makefile``:

* ``Oracle``   -- ``liboracle.so``, this repository's C restatement of the reference
  (``oracle/de_oracle.c``); it travels with the tree and is what the GPU parity tests
  compare against.
* ``Reference`` -- ``_ref/libref.so``, the reference itself (mayio/doubleeye
  ``core/``) compiled from its own sources; present only where it was built.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


class DeCfg(C.Structure):
    """Mirror of ``de_cfg`` in include/doubleeye_b200.h."""
    _fields_ = [("dmin", C.c_int), ("dmax", C.c_int), ("iters", C.c_int),
                ("sigma_s", C.c_float), ("sigma_r", C.c_float), ("ad", C.c_float),
                ("ad_trunc", C.c_int), ("lambda_", C.c_float), ("gamma", C.c_float),
                ("damping", C.c_float), ("min_margin", C.c_float),
                ("min_ratio", C.c_float), ("subpixel", C.c_int), ("fit_eq", C.c_int),
                ("lrc", C.c_int), ("census_hw", C.c_int), ("census_hh", C.c_int)]


class DeKeypoint(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("response", C.c_float),
                ("local_std", C.c_float)]


class DeDetCfg(C.Structure):
    _fields_ = [("grad_window", C.c_int), ("cell", C.c_int), ("per_cell", C.c_int),
                ("min_response", C.c_float), ("min_local_std", C.c_float),
                ("border", C.c_int), ("subpixel", C.c_int),
                ("fast_threshold", C.c_int), ("nms_radius", C.c_int)]


class DeMatchCfg(C.Structure):
    _fields_ = [("max_dy", C.c_float), ("min_disparity", C.c_float),
                ("max_disparity", C.c_float), ("max_candidates", C.c_int),
                ("sigma_y", C.c_float), ("w_y", C.c_float), ("iterations", C.c_int),
                ("damping", C.c_float), ("lambda_", C.c_float), ("gamma", C.c_float),
                ("converge_eps", C.c_float), ("census_bits", C.c_int)]


class DeMatch(C.Structure):
    _fields_ = [("left", C.c_int), ("right", C.c_int), ("score", C.c_float),
                ("belief", C.c_float), ("disparity", C.c_float), ("dy", C.c_float),
                ("margin", C.c_float)]


class DeMatchStats(C.Structure):
    _fields_ = [("left", C.c_int), ("right", C.c_int), ("candidates", C.c_int),
                ("iterations_run", C.c_int), ("converged", C.c_int),
                ("final_max_delta", C.c_float), ("oscillating", C.c_int)]


MATCH_DTYPE = np.dtype([("left", np.int32), ("right", np.int32), ("score", np.float32),
                        ("belief", np.float32), ("disparity", np.float32),
                        ("dy", np.float32), ("margin", np.float32)])


def default_cfg(**kw) -> DeCfg:
    """Reference defaults, core/include/doubleeye/dense_solve.hpp:34-70."""
    c = DeCfg(dmin=1, dmax=60, iters=0, sigma_s=8.0, sigma_r=0.2, ad=0.15, ad_trunc=10,
              lambda_=-0.1, gamma=-0.1, damping=0.4, min_margin=0.0, min_ratio=0.0,
              subpixel=1, fit_eq=1, lrc=0, census_hw=3, census_hh=3)
    for k, v in kw.items():
        setattr(c, "lambda_" if k == "lambda" else k, v)
    return c


def default_det_cfg(**kw) -> DeDetCfg:
    """DetectorConfig defaults, core/include/doubleeye/preproc.hpp:132-145."""
    c = DeDetCfg(grad_window=3, cell=32, per_cell=3, min_response=1.0, min_local_std=2.0,
                 border=8, subpixel=1, fast_threshold=8, nms_radius=3)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def default_match_cfg(**kw) -> DeMatchCfg:
    """MatchConfig defaults, core/include/doubleeye/match.hpp:135-176."""
    c = DeMatchCfg(max_dy=2.0, min_disparity=1.0, max_disparity=220.0, max_candidates=24,
                   sigma_y=1.0, w_y=1.0, iterations=20, damping=0.4, lambda_=0.0,
                   gamma=0.0, converge_eps=1e-4, census_bits=48)
    for k, v in kw.items():
        setattr(c, "lambda_" if k == "lambda" else k, v)
    return c


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


P_U8, P_U16, P_I16, P_I32, P_U64, P_F32 = (C.c_uint8, C.c_uint16, C.c_int16, C.c_int32,
                                           C.c_uint64, C.c_float)


def reference_root() -> str:
    """The reference project's root (the directory holding core/ and article/), from
    the DOUBLEEYE_REF environment variable; only the fixture generators and the
    reference build read the reference tree, and they need it named explicitly."""
    root = os.environ.get("DOUBLEEYE_REF", "")
    if not root or not os.path.isdir(os.path.join(root, "core")):
        raise RuntimeError("set DOUBLEEYE_REF to the reference project's root "
                           "(the directory holding core/ and article/)")
    return root


def fill_prior(dc: np.ndarray, max_sweeps: int = 128) -> np.ndarray:
    """Hole filling of a disparity map before it serves as a prior, restating the
    reference's ``fill`` (article/coarse_to_fine.py:58-76) in float32: each sweep gives
    every non-finite pixel with a finite 4-neighbour (wrapping around the edges) the
    mean of those neighbours, accumulated left, right, up, down; sweeps stop when none
    changes anything or after max_sweeps; non-finite leftovers become 0."""
    d = np.array(dc, np.float32, copy=True)
    for _ in range(max_sweeps):
        hole = ~np.isfinite(d)
        if not hole.any():
            break
        total = np.zeros_like(d)
        count = np.zeros_like(d)
        # (rows, cols) shifts: the neighbour to the left, right, above, below
        for sy, sx in ((0, 1), (0, -1), (1, 0), (-1, 0)):
            nb = np.roll(d, (sy, sx), axis=(0, 1))
            good = np.isfinite(nb)
            total[good] += nb[good]
            count[good] += 1
        upd = hole & (count > 0)
        if not upd.any():
            break
        d[upd] = total[upd] / count[upd]
    d[~np.isfinite(d)] = 0.0
    return d


def build(ref: bool = False) -> None:
    """Build liboracle.so (and _ref/ when asked and the reference tree exists)."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


class Oracle:
    """This repository's C restatement of the reference (liboracle.so)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        L.or_census.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.or_rf_lut.argtypes = [C.c_float, C.c_float, C.c_void_p]
        L.or_rf_coeffs.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.or_score_tables.argtypes = [C.POINTER(DeCfg), C.c_void_p, C.c_void_p]
        L.or_score_tables.restype = C.c_int
        L.or_filter_i16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.or_filter_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.or_score_plane.argtypes = [C.POINTER(DeCfg), C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.or_cost_top2.argtypes = [C.POINTER(DeCfg), C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.or_solve_row.argtypes = [C.POINTER(DeCfg), C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.or_solve_row_debug.argtypes = [C.POINTER(DeCfg), C.c_int] + [C.c_void_p] * 9
        L.or_solve_row_f64.argtypes = [C.POINTER(DeCfg), C.c_int] + [C.c_void_p] * 6
        L.or_cost_top2_f64.argtypes = [C.POINTER(DeCfg), C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_int] + [C.c_void_p] * 4
        L.or_dense.argtypes = [C.POINTER(DeCfg), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                               C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_dense_prior.argtypes = [C.POINTER(DeCfg), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                     C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_confidence.argtypes = [C.c_float] * 5
        L.or_confidence.restype = C.c_float
        L.or_confidence_u8.argtypes = [C.c_float] * 5
        L.or_confidence_u8.restype = C.c_uint
        if hasattr(L, "or_census_at"):
            self._bind_sparse()

    def _bind_sparse(self):
        L = self.lib
        L.or_census_at.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.POINTER(C.c_int)]
        L.or_census_at.restype = C.c_uint64
        L.or_is_fast_corner.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int]
        L.or_shi_tomasi_at.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_shi_tomasi_at.restype = C.c_float
        L.or_local_std_at.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_local_std_at.restype = C.c_float
        L.or_detect_fast.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(DeDetCfg),
                                     C.c_void_p, C.c_int]
        L.or_detect_fast.restype = C.c_int
        L.or_match_masda.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_int, C.POINTER(DeMatchCfg), C.c_void_p, C.c_int,
                                     C.POINTER(DeMatchStats)]
        L.or_match_masda.restype = C.c_int
        L.or_match_edges.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_int, C.POINTER(DeMatchCfg), C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int]
        L.or_match_edges.restype = C.c_int
        L.or_masda_edges.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64,
                                     C.c_int64, C.c_double, C.c_double, C.c_int, C.c_double,
                                     C.c_double, C.c_void_p, C.c_void_p]
        L.or_masda_edges.restype = C.c_int

    # -- sparse --------------------------------------------------------------------
    def census_at(self, img, x, y, hw=3, hh=3):
        img = np.ascontiguousarray(img, np.uint8)
        H, W = img.shape
        ok = C.c_int()
        v = self.lib.or_census_at(img.ctypes.data, W, H, int(x), int(y), hw, hh, C.byref(ok))
        return int(v), bool(ok.value)

    def detect_fast(self, img, det: DeDetCfg | None = None) -> np.ndarray:
        """Keypoints as an (n, 4) float32 array of x, y, response, local_std."""
        img = np.ascontiguousarray(img, np.uint8)
        H, W = img.shape
        det = det or default_det_cfg()
        cap = 1 << 16
        out = np.zeros((cap, 4), np.float32)
        n = self.lib.or_detect_fast(img.ctypes.data, W, H, C.byref(det), out.ctypes.data, cap)
        return out[:min(n, cap)].copy()

    def match_masda(self, kl, dl, kr, dr, cfg: DeMatchCfg | None = None):
        """Matches as a structured array (left, right, score, belief, disparity, dy,
        margin) and the stats."""
        cfg = cfg or default_match_cfg()
        kl = np.ascontiguousarray(kl, np.float32).reshape(-1, 4)
        kr = np.ascontiguousarray(kr, np.float32).reshape(-1, 4)
        dl = np.ascontiguousarray(dl, np.uint64)
        dr = np.ascontiguousarray(dr, np.uint64)
        cap = max(1, len(kl))
        out = np.zeros(cap, MATCH_DTYPE)
        st = DeMatchStats()
        n = self.lib.or_match_masda(kl.ctypes.data, dl.ctypes.data, len(kl), kr.ctypes.data,
                                    dr.ctypes.data, len(kr), C.byref(cfg), out.ctypes.data,
                                    cap, C.byref(st))
        return out[:n].copy(), st

    def match_edges(self, kl, dl, kr, dr, cfg: DeMatchCfg | None = None):
        cfg = cfg or default_match_cfg()
        kl = np.ascontiguousarray(kl, np.float32).reshape(-1, 4)
        kr = np.ascontiguousarray(kr, np.float32).reshape(-1, 4)
        dl = np.ascontiguousarray(dl, np.uint64)
        dr = np.ascontiguousarray(dr, np.uint64)
        cap = max(1, len(kl) * max(1, cfg.max_candidates))
        ei = np.zeros(cap, np.int32)
        ej = np.zeros(cap, np.int32)
        s = np.zeros(cap, np.float32)
        n = self.lib.or_match_edges(kl.ctypes.data, dl.ctypes.data, len(kl), kr.ctypes.data,
                                    dr.ctypes.data, len(kr), C.byref(cfg), ei.ctypes.data,
                                    ej.ctypes.data, s.ctypes.data, cap)
        return ei[:n].copy(), ej[:n].copy(), s[:n].copy()

    def masda_edges(self, ei, ej, se, m, n, lam=-0.1, gam=-0.1, iters=30, damping=0.4,
                    eps=1e-5):
        """masda_sparse in float64 with a stable belief order: (assign[m], hist)."""
        ei = np.ascontiguousarray(ei, np.int64)
        ej = np.ascontiguousarray(ej, np.int64)
        se = np.ascontiguousarray(se, np.float64)
        assign = np.zeros(max(1, m), np.int64)
        hist = np.zeros(max(1, iters), np.float64)
        k = self.lib.or_masda_edges(ei.ctypes.data, ej.ctypes.data, se.ctypes.data, len(se),
                                    m, n, lam, gam, iters, damping, eps, assign.ctypes.data,
                                    hist.ctypes.data)
        return assign[:m].copy(), hist[:k].copy()

    # -- dense ---------------------------------------------------------------------
    def census(self, img: np.ndarray, hw: int = 3, hh: int = 3) -> np.ndarray:
        img = np.ascontiguousarray(img, np.uint8)
        H, W = img.shape
        out = np.zeros((H, W), np.uint64)
        self.lib.or_census(img.ctypes.data, W, H, hw, hh, out.ctypes.data)
        return out

    def rf_lut(self, sigma_s=8.0, sigma_r=0.2) -> np.ndarray:
        lut = np.zeros(256, np.uint16)
        self.lib.or_rf_lut(sigma_s, sigma_r, lut.ctypes.data)
        return lut

    def rf_coeffs(self, L: np.ndarray, sigma_s=8.0, sigma_r=0.2):
        L = np.ascontiguousarray(L, np.uint8)
        H, W = L.shape
        lut = self.rf_lut(sigma_s, sigma_r)
        ax = np.zeros((H, W), np.uint16)
        ay = np.zeros((H, W), np.uint16)
        self.lib.or_rf_coeffs(L.ctypes.data, W, H, lut.ctypes.data, ax.ctypes.data,
                              ay.ctypes.data)
        return ax, ay

    def score_tables(self, cfg: DeCfg):
        tbl = np.zeros(65, np.int16)
        adt = np.zeros(256, np.int16)
        wq = self.lib.or_score_tables(C.byref(cfg), tbl.ctypes.data, adt.ctypes.data)
        return tbl, adt, wq

    def filter_i16(self, plane: np.ndarray, ax, ay) -> np.ndarray:
        p = np.ascontiguousarray(plane, np.int16).copy()
        H, W = p.shape
        self.lib.or_filter_i16(p.ctypes.data, np.ascontiguousarray(ax).ctypes.data,
                               np.ascontiguousarray(ay).ctypes.data, W, H)
        return p

    def filter_f64(self, plane: np.ndarray, ax, ay) -> np.ndarray:
        p = np.ascontiguousarray(plane, np.float64).copy()
        H, W = p.shape
        self.lib.or_filter_f64(p.ctypes.data, np.ascontiguousarray(ax).ctypes.data,
                               np.ascontiguousarray(ay).ctypes.data, W, H)
        return p

    def score_plane(self, cfg: DeCfg, L, R, k: int) -> np.ndarray:
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        H, W = L.shape
        cl = self.census(L, cfg.census_hw, cfg.census_hh)
        cr = self.census(R, cfg.census_hw, cfg.census_hh)
        out = np.zeros((H, W), np.int16)
        self.lib.or_score_plane(C.byref(cfg), L.ctypes.data, R.ctypes.data, cl.ctypes.data,
                                cr.ctypes.data, W, H, k, out.ctypes.data)
        return out

    def cost_top2(self, cfg: DeCfg, L, R, want_rbest: bool = False):
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        H, W = L.shape
        cs = np.zeros((H, W, 2), np.float32)
        cd = np.zeros((H, W, 2), np.int32)
        cn = np.zeros((H, W), np.int32)
        cnb = np.zeros((H, W, 2), np.int16)
        rk = np.zeros((H, W), np.int16) if want_rbest else None
        self.lib.or_cost_top2(C.byref(cfg), L.ctypes.data, R.ctypes.data, W, H, cs.ctypes.data,
                              cd.ctypes.data, cn.ctypes.data, cnb.ctypes.data,
                              rk.ctypes.data if rk is not None else None)
        return (cs, cd, cn, cnb, rk) if want_rbest else (cs, cd, cn, cnb)

    def solve(self, cfg: DeCfg, cs, cd, cn, cnb):
        """Row solve over candidate planes (H, W, 2)."""
        H, W = cn.shape
        cs = np.ascontiguousarray(cs, np.float32)
        cd = np.ascontiguousarray(cd, np.int32)
        cn = np.ascontiguousarray(cn, np.int32)
        cnb = np.ascontiguousarray(cnb, np.int16) if cnb is not None else None
        disp = np.zeros((H, W), np.float32)
        margin = np.zeros((H, W), np.float32)
        lrc2 = np.zeros((H, W), np.float32)
        for y in range(H):
            self.lib.or_solve_row(
                C.byref(cfg), W, cs[y].ctypes.data, cd[y].ctypes.data, cn[y].ctypes.data,
                cnb[y].ctypes.data if cnb is not None else None, disp[y].ctypes.data,
                margin[y].ctypes.data, lrc2[y].ctypes.data)
        return disp, margin, lrc2

    def solve_row_debug(self, cfg: DeCfg, cs, cd, cn, cnb):
        """One row's solve plus each pixel's belief and claim target (-1 = none)."""
        W = cn.shape[0]
        cs = np.ascontiguousarray(cs, np.float32)
        cd = np.ascontiguousarray(cd, np.int32)
        cn = np.ascontiguousarray(cn, np.int32)
        cnb = np.ascontiguousarray(cnb, np.int16) if cnb is not None else None
        disp, margin, lrc2, best = (np.zeros(W, np.float32) for _ in range(4))
        target = np.zeros(W, np.int32)
        self.lib.or_solve_row_debug(
            C.byref(cfg), W, cs.ctypes.data, cd.ctypes.data, cn.ctypes.data,
            cnb.ctypes.data if cnb is not None else None, disp.ctypes.data,
            margin.ctypes.data, lrc2.ctypes.data, best.ctypes.data, target.ctypes.data)
        return disp, best, target

    def solve_f64(self, cfg: DeCfg, cs, cd, cn, nb):
        """The row solve in double precision over candidate planes (H, W, 2): cs and nb
        (the winner's neighbour costs) in score units, -1e300 where missing.
        Returns (disp, belief) as float64."""
        H, W = cn.shape
        cs = np.ascontiguousarray(cs, np.float64)
        cd = np.ascontiguousarray(cd, np.int32)
        cn = np.ascontiguousarray(cn, np.int32)
        nb = np.ascontiguousarray(nb, np.float64)
        disp = np.zeros((H, W), np.float64)
        best = np.zeros((H, W), np.float64)
        for y in range(H):
            self.lib.or_solve_row_f64(C.byref(cfg), W, cs[y].ctypes.data, cd[y].ctypes.data,
                                      cn[y].ctypes.data, nb[y].ctypes.data,
                                      disp[y].ctypes.data, best[y].ctypes.data)
        return disp, best

    def cost_top2_f64(self, cfg: DeCfg, L, R):
        """The cost stage with the filter in double precision, unrounded."""
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        H, W = L.shape
        cs = np.zeros((H, W, 2), np.float64)
        nb = np.zeros((H, W, 2), np.float64)
        cd = np.zeros((H, W, 2), np.int32)
        cn = np.zeros((H, W), np.int32)
        self.lib.or_cost_top2_f64(C.byref(cfg), L.ctypes.data, R.ctypes.data, W, H,
                                  cs.ctypes.data, cd.ctypes.data, cn.ctypes.data, nb.ctypes.data)
        return cs, cd, cn, nb

    def dense(self, cfg: DeCfg, L, R, want_cand: bool = True):
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        H, W = L.shape
        disp = np.zeros((H, W), np.float32)
        margin = np.zeros((H, W), np.float32)
        cand = np.zeros((6, H, W), np.float32) if want_cand else None
        self.lib.or_dense(C.byref(cfg), L.ctypes.data, R.ctypes.data, W, H, disp.ctypes.data,
                          margin.ctypes.data, cand.ctypes.data if cand is not None else None)
        return disp, margin, cand

    def dense_prior(self, cfg: DeCfg, L, R, prior, band=2, want_cand: bool = True):
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        pr = np.ascontiguousarray(prior, np.float32)
        H, W = L.shape
        disp = np.zeros((H, W), np.float32)
        margin = np.zeros((H, W), np.float32)
        cand = np.zeros((6, H, W), np.float32) if want_cand else None
        self.lib.or_dense_prior(C.byref(cfg), L.ctypes.data, R.ctypes.data, W, H,
                                pr.ctypes.data, band, disp.ctypes.data, margin.ctypes.data,
                                cand.ctypes.data if cand is not None else None)
        return disp, margin, cand

    def confidence(self, s1, s2, lam, lrc=0.0, tol=1.0) -> float:
        return self.lib.or_confidence(s1, s2, lam, lrc, tol)

    def confidence_u8(self, s1, s2, lam, lrc=0.0, tol=1.0) -> int:
        return self.lib.or_confidence_u8(s1, s2, lam, lrc, tol)


class Reference:
    """The reference itself, compiled from its sources (oracle/_ref/libref.so)."""

    PATH = os.path.join(HERE, "_ref", "libref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self):
        self.lib = C.CDLL(self.PATH)
        L = self.lib
        L.ref_census_image.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p]
        L.ref_rf_coeffs.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float,
                                    C.c_void_p, C.c_void_p]
        L.ref_rf_filter_i16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.ref_run_dense.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(DeCfg),
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_run_dense_prior.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                          C.POINTER(DeCfg), C.c_int, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_confidence.argtypes = [C.c_float] * 5
        L.ref_confidence.restype = C.c_float
        L.ref_confidence_u8.argtypes = [C.c_float] * 5
        L.ref_confidence_u8.restype = C.c_uint
        L.ref_census_at.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.POINTER(C.c_int)]
        L.ref_census_at.restype = C.c_uint64
        L.ref_detect_fast.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(DeDetCfg),
                                      C.c_void_p, C.c_int]
        L.ref_detect_fast.restype = C.c_int
        L.ref_match_masda.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_int, C.POINTER(DeMatchCfg), C.c_void_p,
                                      C.c_int, C.POINTER(DeMatchStats)]
        L.ref_match_masda.restype = C.c_int
        L.ref_match_brute_force.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                            C.c_void_p, C.c_int, C.POINTER(DeMatchCfg),
                                            C.c_void_p, C.c_int]
        L.ref_match_brute_force.restype = C.c_int

    def census(self, img, hw=3, hh=3):
        img = np.ascontiguousarray(img, np.uint8)
        H, W = img.shape
        out = np.zeros((H, W), np.uint64)
        self.lib.ref_census_image(img.ctypes.data, W, H, hw, hh, out.ctypes.data)
        return out

    def rf_coeffs(self, L, sigma_s=8.0, sigma_r=0.2):
        L = np.ascontiguousarray(L, np.uint8)
        H, W = L.shape
        ax = np.zeros((H, W), np.uint16)
        ay = np.zeros((H, W), np.uint16)
        self.lib.ref_rf_coeffs(L.ctypes.data, W, H, sigma_s, sigma_r, ax.ctypes.data,
                               ay.ctypes.data)
        return ax, ay

    def filter_i16(self, plane, ax, ay):
        p = np.ascontiguousarray(plane, np.int16).copy()
        H, W = p.shape
        self.lib.ref_rf_filter_i16(p.ctypes.data, np.ascontiguousarray(ax).ctypes.data,
                                   np.ascontiguousarray(ay).ctypes.data, W, H)
        return p

    def dense(self, cfg: DeCfg, L, R, nthreads=1, want_cand=True):
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        H, W = L.shape
        disp = np.zeros((H, W), np.float32)
        margin = np.zeros((H, W), np.float32)
        cand = np.zeros((6, H, W), np.float32) if want_cand else None
        t3 = np.zeros(3, np.float64)
        self.lib.ref_run_dense(L.ctypes.data, R.ctypes.data, W, H, C.byref(cfg), nthreads,
                               disp.ctypes.data, margin.ctypes.data,
                               cand.ctypes.data if cand is not None else None, t3.ctypes.data)
        return disp, margin, cand, t3

    def dense_prior(self, cfg: DeCfg, L, R, prior, band=2, nthreads=1, want_cand=True):
        L = np.ascontiguousarray(L, np.uint8)
        R = np.ascontiguousarray(R, np.uint8)
        pr = np.ascontiguousarray(prior, np.float32)
        H, W = L.shape
        disp = np.zeros((H, W), np.float32)
        margin = np.zeros((H, W), np.float32)
        cand = np.zeros((6, H, W), np.float32) if want_cand else None
        self.lib.ref_run_dense_prior(L.ctypes.data, R.ctypes.data, W, H, C.byref(cfg), band,
                                     pr.ctypes.data, nthreads, disp.ctypes.data,
                                     margin.ctypes.data,
                                     cand.ctypes.data if cand is not None else None)
        return disp, margin, cand

    def confidence(self, s1, s2, lam, lrc=0.0, tol=1.0):
        return self.lib.ref_confidence(s1, s2, lam, lrc, tol)

    def census_at(self, img, x, y, hw=3, hh=3):
        img = np.ascontiguousarray(img, np.uint8)
        H, W = img.shape
        ok = C.c_int()
        v = self.lib.ref_census_at(img.ctypes.data, W, H, int(x), int(y), hw, hh, C.byref(ok))
        return int(v), bool(ok.value)

    def detect_fast(self, img, det: DeDetCfg | None = None) -> np.ndarray:
        img = np.ascontiguousarray(img, np.uint8)
        H, W = img.shape
        det = det or default_det_cfg()
        cap = 1 << 16
        out = np.zeros((cap, 4), np.float32)
        n = self.lib.ref_detect_fast(img.ctypes.data, W, H, C.byref(det), out.ctypes.data, cap)
        return out[:min(n, cap)].copy()

    def match_masda(self, kl, dl, kr, dr, cfg: DeMatchCfg | None = None):
        cfg = cfg or default_match_cfg()
        kl = np.ascontiguousarray(kl, np.float32).reshape(-1, 4)
        kr = np.ascontiguousarray(kr, np.float32).reshape(-1, 4)
        dl = np.ascontiguousarray(dl, np.uint64)
        dr = np.ascontiguousarray(dr, np.uint64)
        cap = max(1, len(kl))
        out = np.zeros(cap, MATCH_DTYPE)
        st = DeMatchStats()
        n = self.lib.ref_match_masda(kl.ctypes.data, dl.ctypes.data, len(kl), kr.ctypes.data,
                                     dr.ctypes.data, len(kr), C.byref(cfg), out.ctypes.data,
                                     cap, C.byref(st))
        return out[:n].copy(), st

    def match_brute_force(self, kl, dl, kr, dr, cfg: DeMatchCfg | None = None):
        cfg = cfg or default_match_cfg()
        kl = np.ascontiguousarray(kl, np.float32).reshape(-1, 4)
        kr = np.ascontiguousarray(kr, np.float32).reshape(-1, 4)
        dl = np.ascontiguousarray(dl, np.uint64)
        dr = np.ascontiguousarray(dr, np.uint64)
        cap = max(1, len(kl))
        out = np.zeros(cap, MATCH_DTYPE)
        n = self.lib.ref_match_brute_force(kl.ctypes.data, dl.ctypes.data, len(kl),
                                           kr.ctypes.data, dr.ctypes.data, len(kr),
                                           C.byref(cfg), out.ctypes.data, cap)
        return out[:n].copy()

    def confidence_u8(self, s1, s2, lam, lrc=0.0, tol=1.0):
        return self.lib.ref_confidence_u8(s1, s2, lam, lrc, tol)
