"""ctypes binding of the C ABI (include/doubleeye_b200.h).

The library is the in-tree ``_lib/libdoubleeye_b200.so``.  There is no CPU
fallback: if the library is missing or no CUDA device is present, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libdoubleeye_b200.so")

DE_OK = 0
ERRORS = {-1: "DE_ERR_ARG", -2: "DE_ERR_CUDA", -3: "DE_ERR_OOM", -4: "DE_ERR_TIMEOUT",
          -5: "DE_ERR_UNSUPPORTED", -6: "DE_ERR_BUSY", -7: "DE_ERR_CLOSED"}


class DeError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class DeCfg(C.Structure):
    _fields_ = [("dmin", C.c_int), ("dmax", C.c_int), ("iters", C.c_int),
                ("sigma_s", C.c_float), ("sigma_r", C.c_float), ("ad", C.c_float),
                ("ad_trunc", C.c_int), ("lambda_", C.c_float), ("gamma", C.c_float),
                ("damping", C.c_float), ("min_margin", C.c_float),
                ("min_ratio", C.c_float), ("subpixel", C.c_int), ("fit_eq", C.c_int),
                ("lrc", C.c_int), ("census_hw", C.c_int), ("census_hh", C.c_int)]


class DePair(C.Structure):
    _fields_ = [("L", C.c_void_p), ("R", C.c_void_p), ("W", C.c_int), ("H", C.c_int),
                ("dmax", C.c_int), ("disp", C.c_void_p), ("margin", C.c_void_p),
                ("conf", C.c_void_p), ("cand", C.c_void_p)]


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


vp = C.c_void_p
# name -> (restype, argtypes)
SIGNATURES = {
    "de_cfg_default": (None, [C.POINTER(DeCfg)]),
    "de_det_cfg_default": (None, [C.POINTER(DeDetCfg)]),
    "de_match_cfg_default": (None, [C.POINTER(DeMatchCfg)]),
    "de_last_error": (C.c_char_p, []),
    "de_version": (C.c_char_p, []),
    "de_dense_workspace_bytes": (C.c_int, [C.POINTER(DeCfg), C.POINTER(DePair), C.c_int,
                                           C.POINTER(C.c_size_t)]),
    "de_dense_dev": (C.c_int, [C.POINTER(DeCfg), C.POINTER(DePair), C.c_int, vp, C.c_size_t,
                               vp]),
    "de_dense_noalloc_dev": (C.c_int, [C.POINTER(DeCfg), C.POINTER(DePair), vp]),
    "de_census_dev": (C.c_int, [C.POINTER(DeCfg), vp, vp, C.c_int, C.c_int, vp, vp, vp, vp,
                                vp]),
    "de_cost_workspace_bytes": (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    "de_cost_top2_dev": (C.c_int, [C.POINTER(DeCfg), vp, vp, C.c_int, C.c_int, vp, vp, vp, vp,
                                   vp, C.c_size_t, vp]),
    "de_solve_dev": (C.c_int, [C.POINTER(DeCfg), C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp,
                               vp]),
    "de_confidence": (C.c_float, [C.c_float] * 5),
    "de_stage_timing": (C.c_int, [C.c_int]),
    "de_workspace_status": (C.c_int, [vp, vp, C.POINTER(C.c_int)]),
    "de_set_param": (C.c_int, [C.c_char_p, C.c_int]),
    "de_get_param": (C.c_int, [C.c_char_p, C.POINTER(C.c_int)]),
    "de_stage_times": (C.c_int, [C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "de_ctx_create": (C.c_int, [C.POINTER(DeCfg), C.c_int, C.POINTER(vp)]),
    "de_ctx_destroy": (C.c_int, [vp]),
    "de_ctx_set_cfg": (C.c_int, [vp, C.POINTER(DeCfg)]),
    "de_ctx_dense": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp, vp, vp, vp]),
    "de_ctx_dense_batch": (C.c_int, [vp, C.POINTER(DePair), C.c_int]),
    "de_ctx_dense_prior": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp, C.c_int, vp, vp, vp,
                                     vp]),
    "de_dense_prior_workspace_bytes": (C.c_int, [C.POINTER(DeCfg), C.POINTER(DePair),
                                                 C.POINTER(C.c_size_t)]),
    "de_dense_prior_dev": (C.c_int, [C.POINTER(DeCfg), C.POINTER(DePair), vp, C.c_int, vp,
                                     C.c_size_t, vp]),
    "de_ctx_keypoints": (C.c_int, [vp, vp, C.c_int, C.c_int, C.POINTER(DeDetCfg), vp, vp, vp,
                                   C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "de_census_at_dev": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int,
                                   vp, vp, vp]),
    "de_detect_workspace_bytes": (C.c_int, [C.c_int, C.c_int, C.POINTER(DeDetCfg),
                                            C.POINTER(C.c_size_t)]),
    "de_detect_fast_dev": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(DeDetCfg), vp, C.c_int,
                                     vp, vp, C.c_size_t, vp]),
    "de_keypoint_readout_dev": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_int, C.c_int, vp,
                                          C.c_int, vp, vp]),
    "de_match_workspace_bytes": (C.c_int, [C.c_int, C.c_int, C.POINTER(DeMatchCfg),
                                           C.POINTER(C.c_size_t)]),
    "de_match_masda_dev": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, C.c_int, vp,
                                     C.POINTER(DeMatchCfg), vp, C.c_int, vp, vp, vp,
                                     C.c_size_t, vp]),
    "de_masda_edges_workspace_bytes": (C.c_int, [C.c_longlong, C.c_longlong, C.c_longlong,
                                                 C.POINTER(C.c_size_t)]),
    "de_masda_edges_dev": (C.c_int, [vp, vp, vp, C.c_longlong, C.c_longlong, C.c_longlong,
                                     C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                     vp, vp, vp, vp, vp, C.c_size_t, vp]),
    "de_masda_decide_dev": (C.c_int, [vp, vp, vp, vp, C.c_longlong, C.c_longlong,
                                      C.c_longlong, C.c_double, vp, vp, C.c_size_t, vp]),
    "de_seg_max_excluding_dev": (C.c_int, [vp, vp, C.c_longlong, C.c_longlong, vp, vp,
                                           C.c_size_t, vp]),
    "de_hamming_dev": (C.c_int, [vp, vp, C.c_longlong, vp, vp]),
    "de_census_pts_dev": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_longlong, C.c_int, C.c_int,
                                    vp, vp, vp]),
    "de_build_problem_dev": (C.c_int, [vp, vp, C.c_longlong, vp, vp, C.c_longlong, C.c_float,
                                       C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                       vp, vp]),
    "de_edges_from_matrix_dev": (C.c_int, [vp, C.c_longlong, C.c_longlong, vp, vp, vp,
                                           C.c_longlong, vp, vp, C.c_size_t, vp]),
    "de_dense_problem_edges": (C.c_longlong, [C.c_int] * 6),
    "de_dense_problem_dev": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, vp, vp, vp, C.c_longlong, vp, C.c_size_t, vp]),
    "de_graph_create": (C.c_int, [C.POINTER(DeCfg), C.POINTER(DePair), C.c_int, vp,
                                  C.c_size_t, C.POINTER(vp)]),
    "de_graph_launch": (C.c_int, [vp, vp]),
    "de_graph_destroy": (C.c_int, [vp]),
    "de_server_cfg_default": (None, [vp]),
    "de_server_create": (C.c_int, [C.POINTER(DeCfg), vp, C.POINTER(vp)]),
    "de_server_submit": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int, C.c_uint,
                                   C.POINTER(C.c_ulonglong)]),
    "de_server_wait": (C.c_int, [vp, C.c_ulonglong, C.c_int, vp, vp, vp, vp, vp,
                                 C.POINTER(C.c_double)]),
    "de_server_stats": (C.c_int, [vp, vp]),
    "de_server_reset_stats": (C.c_int, [vp]),
    "de_server_last_disparity": (C.c_int, [vp, C.c_int, vp, C.c_int, C.c_int]),
    "de_server_destroy": (C.c_int, [vp]),
    "de_dedd_encode_dev": (C.c_int, [vp, vp, C.c_int, C.c_int, vp, vp, vp]),
    "de_server_stream_prior": (C.c_int, [vp, C.c_int, C.c_int]),
    "de_match_masda_prior_dev": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, C.c_int, vp,
                                           C.POINTER(DeMatchCfg), vp, vp, C.c_int, vp, vp,
                                           vp, C.c_size_t, vp]),
    "de_ctx_census": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]),
    "de_ctx_census_at": (C.c_int, [vp, vp, C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int,
                                   vp, vp]),
    "de_ctx_detect_fast": (C.c_int, [vp, vp, C.c_int, C.c_int, C.POINTER(DeDetCfg), vp,
                                     C.c_int, C.POINTER(C.c_int)]),
    "de_ctx_match_masda": (C.c_int, [vp, vp, vp, C.c_int, vp, vp, C.c_int,
                                     C.POINTER(DeMatchCfg), vp, vp, C.c_int,
                                     C.POINTER(C.c_int), vp]),
    "de_ctx_solve": (C.c_int, [vp, C.POINTER(DeCfg), C.c_int, C.c_int, vp, vp, vp, vp, vp, vp,
                               vp]),
    "de_prior_fill_workspace_bytes": (C.c_size_t, [C.c_int, C.c_int]),
    "de_prior_fill_dev": (C.c_int, [vp, vp, C.c_int, C.c_int, vp, C.c_size_t, vp]),
}

_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    """Load (once) and return the library; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m doubleeye_b200.build` "
                    "(CUDA path only, no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                if hasattr(L, name):
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
            _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != DE_OK:
        raise DeError(rc, lib().de_last_error().decode(errors="replace"))


def set_param(name: str, value: int) -> None:
    check(lib().de_set_param(name.encode(), int(value)))


def get_param(name: str) -> int:
    v = C.c_int()
    check(lib().de_get_param(name.encode(), C.byref(v)))
    return v.value


PROBE_PATH = os.path.join(PKG, "_lib", "libde_probe.so")
_probe = None


def probe_lib() -> C.CDLL:
    """The bench's integer-pipe probe (de_int_probe), a library of its own outside the
    matcher's C ABI: (op, trips, stream, float* ms, double* lane_ops) -> status."""
    global _probe
    with _lock:
        if _probe is None:
            if not os.path.exists(PROBE_PATH):
                raise RuntimeError(f"{PROBE_PATH} is missing: build with "
                                   "`python -m doubleeye_b200.build`")
            L = C.CDLL(PROBE_PATH)
            L.de_int_probe.restype = C.c_int
            L.de_int_probe.argtypes = [C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_float),
                                       C.POINTER(C.c_double)]
            _probe = L
    return _probe


def exported_symbols() -> list[str]:
    return [n for n in SIGNATURES if hasattr(lib(), n)]
