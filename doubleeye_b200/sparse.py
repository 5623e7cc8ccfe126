"""Keypoint (sparse) MASDA on the GPU: the host-side mirror of the reference's sparse path.

Reference call surface (mayio/doubleeye):
  ``census_at`` (core/src/preproc.cpp:142-162)              -> ``census_at``
  ``detect_keypoints_fast`` (core/src/preproc.cpp:442-545)  -> ``detect_fast``
  ``match_masda`` (core/src/match.cpp:334-417)              -> ``match_masda``
  the de_match tool's per-pair flow, detect both images, census at the rounded
  keypoints, match (core/tools/de_match.cpp:222-240)         -> ``SparseMatcher.match_pair``
  ``DetectorConfig`` / ``MatchConfig`` (preproc.hpp:132-145, match.hpp:135-176)
                                                             -> ``DetCfg`` / ``MatchCfg``

Keypoints are (n, 4) float32 arrays of x, y, response, local_std (``Keypoint``);
matches are structured arrays with the fields of ``Match`` (match.hpp:44-66).
Every call goes through the C ABI into the sm_100a kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import DeDetCfg, DeMatchCfg, DeMatchStats, check, lib

MATCH_DTYPE = np.dtype([("left", np.int32), ("right", np.int32), ("score", np.float32),
                        ("belief", np.float32), ("disparity", np.float32),
                        ("dy", np.float32), ("margin", np.float32)])
STATS_FIELDS = ("left", "right", "candidates", "iterations_run", "converged",
                "final_max_delta", "oscillating")


def DetCfg(**overrides) -> DeDetCfg:
    """A de_det_cfg with DetectorConfig's defaults (grad_window 3, cell 32, per_cell 3,
    min_response 1, min_local_std 2, border 8, sub-pixel on, FAST threshold 8, NMS
    radius 3), fields overridden by keyword."""
    c = DeDetCfg()
    lib().de_det_cfg_default(C.byref(c))
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise TypeError(f"unknown de_det_cfg field {k!r}")
        setattr(c, k, int(v) if isinstance(v, bool) else v)
    return c


def MatchCfg(**overrides) -> DeMatchCfg:
    """A de_match_cfg with MatchConfig's defaults (max_dy 2, disparity 1..220, 24
    candidates, sigma_y = w_y = 1, 20 iterations, damping 0.4, lambda = gamma = 0,
    converge_eps 1e-4, 48-bit descriptor scale)."""
    c = DeMatchCfg()
    lib().de_match_cfg_default(C.byref(c))
    for k, v in overrides.items():
        k = "lambda_" if k == "lambda" else k
        if not hasattr(c, k):
            raise TypeError(f"unknown de_match_cfg field {k!r}")
        setattr(c, k, v)
    return c


def stats_dict(st: DeMatchStats) -> dict:
    return {f: getattr(st, f) for f in STATS_FIELDS}


def _torch():
    import torch
    return torch


def _stream_handle(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _dev_u8(img, device):
    torch = _torch()
    if isinstance(img, np.ndarray):
        img = torch.from_numpy(np.ascontiguousarray(img, np.uint8)).to(device)
    if img.dtype != torch.uint8 or img.dim() != 2:
        raise ValueError("images must be 2-D uint8")
    return img.to(device).contiguous()


class SparseMatcher:
    """Device-resident keypoint matcher.  Detection, descriptors and matching are
    enqueued on the caller's stream with keypoint and match counts kept on the device,
    so ``match_pair`` needs no host round trip; workspaces are kept and grown."""

    def __init__(self, det: Optional[DeDetCfg] = None, cfg: Optional[DeMatchCfg] = None,
                 census: tuple = (3, 3), device: int = 0, kp_cap: int = 16384):
        torch = _torch()
        self.det = det or DetCfg()
        self.cfg = cfg or MatchCfg()
        self.hw, self.hh = census
        self.device = torch.device("cuda", device)
        self.kp_cap = int(kp_cap)
        self._ws = {}

    def _buf(self, key: str, nbytes: int):
        torch = _torch()
        b = self._ws.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)
            self._ws[key] = b
        return b

    # -- stages ---------------------------------------------------------------------------
    def detect(self, img, stream=None, ws_key: str = "det"):
        """-> (keypoints (kp_cap, 4) f32 tensor, count int32 tensor of 1) on the device."""
        torch = _torch()
        img = _dev_u8(img, self.device)
        kp = torch.empty((self.kp_cap, 4), dtype=torch.float32, device=self.device)
        n = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._detect_into(img, kp, n, self._det_ws(img, ws_key), stream)
        return kp, n

    def _det_ws(self, img, ws_key: str):
        H, W = img.shape
        need = C.c_size_t()
        check(lib().de_detect_workspace_bytes(W, H, C.byref(self.det), C.byref(need)))
        return self._buf(ws_key, need.value), need.value

    def _detect_into(self, img, kp, n, ws, stream):
        H, W = img.shape
        buf, nbytes = ws
        check(lib().de_detect_fast_dev(img.data_ptr(), W, H, C.byref(self.det), kp.data_ptr(),
                                       kp.shape[0], n.data_ptr(), buf.data_ptr(), nbytes,
                                       _stream_handle(stream)))

    def census_at(self, img, kp, n=None, stream=None):
        """Descriptors (int64 tensor of uint64 bit patterns) at the keypoints."""
        torch = _torch()
        img = _dev_u8(img, self.device)
        desc = torch.zeros(kp.shape[0], dtype=torch.int64, device=self.device)
        self._census_into(img, kp, n, desc, stream)
        return desc

    def _census_into(self, img, kp, n, desc, stream):
        H, W = img.shape
        check(lib().de_census_at_dev(img.data_ptr(), W, H, kp.data_ptr(), kp.shape[0],
                                     n.data_ptr() if n is not None else None, self.hw,
                                     self.hh, desc.data_ptr(), None, _stream_handle(stream)))

    def match(self, kl, dl, kr, dr, nl=None, nr=None, stream=None):
        """-> (matches (cap, 7) int32 tensor holding de_match records, count tensor,
        stats tensor of 7 int32 holding de_match_stats)."""
        torch = _torch()
        cl, cr = kl.shape[0], kr.shape[0]
        need = C.c_size_t()
        check(lib().de_match_workspace_bytes(cl, cr, C.byref(self.cfg), C.byref(need)))
        ws = self._buf("match", need.value)
        cap = max(1, cl)
        out = torch.empty((cap, 7), dtype=torch.int32, device=self.device)
        n = torch.zeros(1, dtype=torch.int32, device=self.device)
        st = torch.zeros(7, dtype=torch.int32, device=self.device)
        check(lib().de_match_masda_dev(
            kl.data_ptr(), dl.data_ptr(), cl, nl.data_ptr() if nl is not None else None,
            kr.data_ptr(), dr.data_ptr(), cr, nr.data_ptr() if nr is not None else None,
            C.byref(self.cfg), out.data_ptr(), cap, n.data_ptr(), st.data_ptr(),
            ws.data_ptr(), need.value, _stream_handle(stream)))
        return out, n, st

    def match_pair(self, L, R, stream=None) -> dict:
        """Detect both images, describe, match; all on the device, nothing synchronised.
        The right image is detected and described on a second stream beside the left
        one (the two are independent and each is a few small kernels), and the match
        waits for both."""
        torch = _torch()
        main = stream if stream is not None else torch.cuda.current_stream(self.device)
        side = self._side_stream()
        with torch.cuda.stream(main):
            # everything the side stream touches is allocated (and zeroed) on the main
            # stream before the fork, so no tensor crosses the allocator's streams
            L = _dev_u8(L, self.device)
            R = _dev_u8(R, self.device)
            kr = torch.empty((self.kp_cap, 4), dtype=torch.float32, device=self.device)
            nr = torch.zeros(1, dtype=torch.int32, device=self.device)
            dr = torch.zeros(self.kp_cap, dtype=torch.int64, device=self.device)
            wsr = self._det_ws(R, "detR")
            side.wait_stream(main)
            self._detect_into(R, kr, nr, wsr, side)
            self._census_into(R, kr, nr, dr, side)
            kl, nl = self.detect(L, main, "detL")
            dl = self.census_at(L, kl, nl, main)
            main.wait_stream(side)
            m, n, st = self.match(kl, dl, kr, dr, nl, nr, main)
        return dict(kl=kl, nl=nl, kr=kr, nr=nr, dl=dl, dr=dr, matches=m, n=n, stats=st)

    def _side_stream(self):
        torch = _torch()
        s = getattr(self, "_side", None)
        if s is None:
            s = self._side = torch.cuda.Stream(self.device)
        return s

    # -- host results ---------------------------------------------------------------------
    @staticmethod
    def to_host(res: dict) -> dict:
        """Copy a ``match_pair`` result to NumPy: keypoints (n, 4), descriptors,
        matches (structured), stats (dict).  Synchronises the stream."""
        nl = int(res["nl"].item())
        nr = int(res["nr"].item())
        if nl < 0 or nr < 0:
            raise RuntimeError("keypoint suppression did not settle")
        n = int(res["n"].item())
        kl = res["kl"][:min(nl, res["kl"].shape[0])].cpu().numpy()
        kr = res["kr"][:min(nr, res["kr"].shape[0])].cpu().numpy()
        m = res["matches"][:n].cpu().numpy().copy().view(MATCH_DTYPE).reshape(-1)
        st = np.frombuffer(res["stats"].cpu().numpy().tobytes(), dtype=np.uint8)
        s = DeMatchStats.from_buffer_copy(st.tobytes())
        return dict(kl=kl, kr=kr, dl=res["dl"][:len(kl)].cpu().numpy().view(np.uint64),
                    dr=res["dr"][:len(kr)].cpu().numpy().view(np.uint64), matches=m,
                    stats=stats_dict(s))


# -- NumPy conveniences (one call each, synchronous) ------------------------------------

KP_DISPARITY_DTYPE = np.dtype([("x", np.float32), ("y", np.float32),
                               ("disparity", np.float32), ("margin", np.float32)])


def dense_keypoints(left, disp, margin=None, det: Optional[DeDetCfg] = None,
                    device: int = 0) -> tuple:
    """The sparse feature set read out of a dense map (core/tools/de_dense_cuda.cu:
    866-899): FAST keypoints of the left image that carry a positive disparity, with
    the map's disparity and margin there.  Returns (records, number detected)."""
    from .dense import _Ctx
    L = np.ascontiguousarray(left, np.uint8)
    H, W = L.shape
    d = np.ascontiguousarray(disp, np.float32)
    m = np.ascontiguousarray(margin, np.float32) if margin is not None else None
    det = det or DetCfg()
    cap = 1 << 16
    out = np.zeros(cap, KP_DISPARITY_DTYPE)
    n, nd = C.c_int(), C.c_int()
    check(lib().de_ctx_keypoints(_Ctx.get(device), L.ctypes.data, W, H, C.byref(det),
                                 d.ctypes.data, m.ctypes.data if m is not None else None,
                                 out.ctypes.data, cap, C.byref(n), C.byref(nd)))
    return out[:min(n.value, cap)].copy(), nd.value

def detect_fast(img, det: Optional[DeDetCfg] = None, device: int = 0) -> np.ndarray:
    """detect_keypoints_fast on the GPU: (n, 4) float32 x, y, response, local_std."""
    sm = SparseMatcher(det=det, device=device)
    kp, n = sm.detect(img)
    k = int(n.item())
    if k < 0:
        raise RuntimeError("keypoint suppression did not settle")
    return kp[:min(k, sm.kp_cap)].cpu().numpy()


def census_at(img, kp, hw: int = 3, hh: int = 3, device: int = 0) -> np.ndarray:
    """census_at at each keypoint's rounded position: uint64 descriptors."""
    torch = _torch()
    sm = SparseMatcher(census=(hw, hh), device=device)
    k = torch.from_numpy(np.ascontiguousarray(kp, np.float32).reshape(-1, 4)).to(sm.device)
    if k.shape[0] == 0:
        return np.zeros(0, np.uint64)
    return sm.census_at(img, k).cpu().numpy().view(np.uint64)


def match_masda(kl, dl, kr, dr, cfg: Optional[DeMatchCfg] = None, device: int = 0):
    """match_masda on the GPU: (matches structured array, stats dict)."""
    torch = _torch()
    sm = SparseMatcher(cfg=cfg, device=device)
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(sm.device)  # noqa
    kl_t = t(np.asarray(kl, np.float32).reshape(-1, 4), np.float32)
    kr_t = t(np.asarray(kr, np.float32).reshape(-1, 4), np.float32)
    dl_t = t(np.asarray(dl, np.uint64).view(np.int64), np.int64)
    dr_t = t(np.asarray(dr, np.uint64).view(np.int64), np.int64)
    m, n, st = sm.match(kl_t, dl_t, kr_t, dr_t)
    k = int(n.item())
    out = m[:k].cpu().numpy().copy().view(MATCH_DTYPE).reshape(-1)
    s = DeMatchStats.from_buffer_copy(st.cpu().numpy().tobytes())
    return out, stats_dict(s)
