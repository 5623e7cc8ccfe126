"""Dense MASDA stereo on the GPU: the host-side mirror of the reference's dense tools.

Reference call surface (mayio/doubleeye):
  ``run_dense`` (core/tools/de_dense.cpp:738) -> ``run_dense`` here (host arrays, one
  or many pairs), ``DenseMatcher`` (device tensors, caller stream, reusable workspace);
  ``Cfg`` (core/include/doubleeye/dense_solve.hpp:19-97) -> ``Cfg``; the --out-conf
  planes s1,s2,d1,d2,lrc,lrc2 (core/tools/de_dense.cpp:727-737) -> ``cand``.

Every call goes through the C ABI into the sm_100a kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
import weakref
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import DeCfg, DePair, check, lib

CAND_PLANES = ("s1", "s2", "d1", "d2", "lrc", "lrc2")


def Cfg(**overrides) -> DeCfg:
    """A de_cfg with the reference defaults (dmin 1, dmax 60, iters 0, sigma_s 8,
    sigma_r 0.2, ad 0.15, ad_trunc 10, lambda = gamma = -0.1, damping 0.4, sub-pixel
    equiangular fit, 7x7 census) and any field overridden by keyword (``lambda_`` or
    ``lambda`` for the clutter cost)."""
    c = DeCfg()
    lib().de_cfg_default(C.byref(c))
    for k, v in overrides.items():
        k = "lambda_" if k == "lambda" else k
        if not hasattr(c, k):
            raise TypeError(f"unknown de_cfg field {k!r}")
        setattr(c, k, v)
    return c


def cfg_dict(c: DeCfg) -> dict:
    return {f: getattr(c, f) for f, _ in c._fields_}


@dataclasses.dataclass
class DenseResult:
    disp: np.ndarray            # f32 (H, W), NaN where the matcher declined
    margin: np.ndarray          # f32 (H, W)
    conf: np.ndarray            # u8 (H, W)
    cand: Optional[np.ndarray]  # f32 (6, H, W): s1, s2, d1, d2, lrc, lrc2


def pinned_empty(shape, dtype) -> np.ndarray:
    """An uninitialised numpy array in page-locked host memory.  The host-pointer
    entry points move such arrays by DMA directly, with no staging copy; the array
    keeps its allocation alive."""
    torch = _torch()
    dt = np.dtype(dtype)
    n = int(np.prod(shape)) * dt.itemsize
    t = torch.empty(max(n, 1), dtype=torch.uint8, pin_memory=True)
    return t.numpy()[:n].view(dt).reshape(shape)


def new_results(shapes, want_cand: bool = False, pinned: bool = True) -> list[DenseResult]:
    """Output buffers for ``run_dense_batch(..., out=...)``: one DenseResult per
    (H, W), page-locked unless ``pinned`` is False."""
    alloc = pinned_empty if pinned else np.empty
    return [DenseResult(alloc((H, W), np.float32), alloc((H, W), np.float32),
                        alloc((H, W), np.uint8),
                        alloc((6, H, W), np.float32) if want_cand else None)
            for H, W in shapes]


class _Ctx:
    """A de_ctx (host-pointer entry points) per thread and device."""
    _tls = threading.local()

    @classmethod
    def get(cls, device: int = 0):
        cache = getattr(cls._tls, "ctx", None)
        if cache is None:
            cache = cls._tls.ctx = {}
        if device not in cache:
            h = C.c_void_p()
            check(lib().de_ctx_create(C.byref(Cfg()), device, C.byref(h)))
            cache[device] = h
        return cache[device]


def _u8(a) -> np.ndarray:
    if not (isinstance(a, np.ndarray) and a.flags.c_contiguous):
        a = np.ascontiguousarray(a)
    if a.dtype != np.uint8 or a.ndim != 2:
        raise ValueError("images must be 2-D uint8")
    return a


_addr_cache: dict = {}


def _addr(a) -> Optional[int]:
    """Data address of an array.  ``a.ctypes.data`` and ``__array_interface__`` build an
    object per call; five of them per pair were most of a 16-pair call's host time
    (about 100 us of a 3.2 ms call), so addresses are cached per array object while it
    lives.  The cache holds a weak reference, and numpy refuses to resize in place an
    array that has one (``ndarray.resize`` raises; ``np.resize`` returns a new array),
    so a cached address cannot go stale; the size is checked as well."""
    if a is None:
        return None
    e = _addr_cache.get(id(a))
    if e is not None and e[0]() is a and e[1] == a.size:
        return e[2]
    p = a.__array_interface__["data"][0]
    if len(_addr_cache) > 4096:
        _addr_cache.clear()
    _addr_cache[id(a)] = (weakref.ref(a), a.size, p)
    return p


def run_dense(left, right, cfg: Optional[DeCfg] = None, *, want_cand: bool = True,
              device: int = 0) -> DenseResult:
    """One pair, host arrays in and out (uploads, runs every stage, downloads)."""
    return run_dense_batch([(left, right)], cfg, want_cand=want_cand, device=device)[0]


def run_dense_batch(pairs: Sequence, cfg: Optional[DeCfg] = None, *, want_cand=False,
                    device: int = 0, out: Optional[Sequence[DenseResult]] = None
                    ) -> list[DenseResult]:
    """Many pairs of any sizes in one batched launch set.  ``pairs`` holds
    (left, right) or (left, right, dmax) tuples; dmax defaults to the cfg's.  ``out``
    may pass the DenseResult arrays of an earlier call to be overwritten (no new host
    allocation per call)."""
    cfg = cfg or Cfg()
    ctx = _Ctx.get(device)
    check(lib().de_ctx_set_cfg(ctx, C.byref(cfg)))
    keep, outs = [], []
    arr = (DePair * len(pairs))()
    for i, pr in enumerate(pairs):
        L, R = _u8(pr[0]), _u8(pr[1])
        if L.shape != R.shape:
            raise ValueError("left and right differ in shape")
        H, W = L.shape
        if out is not None and out[i].disp.shape == (H, W) and \
                (out[i].cand is not None or not want_cand):
            res = out[i]
        else:
            res = DenseResult(np.empty((H, W), np.float32), np.empty((H, W), np.float32),
                              np.empty((H, W), np.uint8),
                              np.empty((6, H, W), np.float32) if want_cand else None)
        keep += [L, R]
        outs.append(res)
        arr[i] = DePair(_addr(L), _addr(R), W, H, int(pr[2]) if len(pr) > 2 else 0,
                        _addr(res.disp), _addr(res.margin), _addr(res.conf),
                        _addr(res.cand) if want_cand else None)
    check(lib().de_ctx_dense_batch(ctx, arr, len(pairs)))
    return outs


def run_dense_prior(left, right, prior, cfg: Optional[DeCfg] = None, *, band: int = 2,
                    want_cand: bool = True, device: int = 0) -> DenseResult:
    """One pair with a disparity prior as the per-plane mask (the reference's --prior;
    core/tools/de_dense.cpp:797-853): plane d is computed and offered only where the
    prior's band [round(prior) - band, round(prior) + band] admits it.  ``prior`` is a
    W x H float32 map without holes (a previous frame, a coarse pass); sub-pixel
    refinement is off, as the reference sets it."""
    cfg = cfg or Cfg()
    ctx = _Ctx.get(device)
    check(lib().de_ctx_set_cfg(ctx, C.byref(cfg)))
    L, R = _u8(left), _u8(right)
    H, W = L.shape
    pr = np.ascontiguousarray(prior, np.float32)
    if pr.shape != (H, W):
        raise ValueError("the prior must be W x H")
    res = DenseResult(np.empty((H, W), np.float32), np.empty((H, W), np.float32),
                      np.empty((H, W), np.uint8),
                      np.empty((6, H, W), np.float32) if want_cand else None)
    check(lib().de_ctx_dense_prior(ctx, L.ctypes.data, R.ctypes.data, W, H, pr.ctypes.data,
                                   int(band), res.disp.ctypes.data, res.margin.ctypes.data,
                                   res.conf.ctypes.data,
                                   res.cand.ctypes.data if want_cand else None))
    return res


def fill_holes(disp, device: int = 0) -> np.ndarray:
    """A disparity map with its holes filled, ready to serve as a prior: the
    reference's ``fill`` (article/coarse_to_fine.py:58-76; iterated 4-neighbour
    averaging with wrap-around, at most 128 sweeps, what is left becomes 0), run on
    the GPU by de_prior_fill_dev."""
    torch = _torch()
    d = np.ascontiguousarray(disp, np.float32)
    if d.ndim != 2:
        raise ValueError("the map must be 2-D")
    H, W = d.shape
    dev = torch.device("cuda", device)
    with torch.cuda.device(dev):
        src = torch.from_numpy(d).to(dev)
        dst = torch.empty_like(src)
        ws = torch.empty(int(lib().de_prior_fill_workspace_bytes(W, H)), dtype=torch.uint8,
                         device=dev)
        check(lib().de_prior_fill_dev(src.data_ptr(), dst.data_ptr(), W, H, ws.data_ptr(),
                                      ws.numel(), _stream_handle()))
        return dst.cpu().numpy()


# --------------------------------------------------------------------------------------
# Device-tensor API (torch for device memory and streams; the work is the C ABI's)

def _torch():
    import torch
    return torch


def _stream_handle(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


class DenseMatcher:
    """Device-resident matcher: images are CUDA uint8 tensors, outputs are CUDA
    tensors, work is enqueued on the caller's current stream, and the workspace is
    kept and reused across calls (grown when a larger batch needs it).

    ``match`` / ``match_batch`` allocate only their output tensors (through torch's
    caching allocator); ``match_into`` writes caller-provided outputs and allocates
    nothing."""

    def __init__(self, cfg: Optional[DeCfg] = None, device: int = 0, autotune: bool = False):
        torch = _torch()
        self.cfg = cfg or Cfg()
        self.device = torch.device("cuda", device)
        self._ws = None
        self._tuner = None
        if autotune:
            from .autotune import Tuner
            self._tuner = Tuner()

    def tune_for(self, items, stream=None) -> dict:
        """Pick (or recall) the fastest launch shapes for this batch's workload and
        apply them; results are unchanged by the choice."""
        from .autotune import Tuner, signature
        self._tuner = self._tuner or Tuner()
        _, shapes = self._pairs(items)
        return self._tuner.ensure(signature(self.cfg, shapes),
                                  lambda: self._launch(items, stream))

    def workspace_bytes(self, shapes) -> int:
        arr = (DePair * len(shapes))()
        for i, s in enumerate(shapes):
            W, H = s[0], s[1]
            arr[i] = DePair(1, 1, W, H, s[2] if len(s) > 2 else 0, None, None, None, None)
        n = C.c_size_t()
        check(lib().de_dense_workspace_bytes(C.byref(self.cfg), arr, len(shapes), C.byref(n)))
        return n.value

    def _workspace(self, nbytes: int):
        torch = _torch()
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self._ws

    def new_outputs(self, H: int, W: int, cand: bool = False) -> dict:
        torch = _torch()
        d = dict(disp=torch.empty((H, W), dtype=torch.float32, device=self.device),
                 margin=torch.empty((H, W), dtype=torch.float32, device=self.device),
                 conf=torch.empty((H, W), dtype=torch.uint8, device=self.device))
        if cand:
            d["cand"] = torch.empty((6, H, W), dtype=torch.float32, device=self.device)
        return d

    def match_into(self, items, stream=None) -> None:
        """items: list of (L, R, dmax or 0, outputs dict).  Enqueues one batched launch
        set on ``stream`` (default: current)."""
        for L, R, _, _ in items:
            if L.dtype != _torch().uint8 or L.device != self.device or not L.is_contiguous():
                raise ValueError("images must be contiguous CUDA uint8 tensors on the device")
        if self._tuner is not None:
            self.tune_for(items, stream)
        self._launch(items, stream)

    def _launch(self, items, stream=None) -> None:
        arr, shapes = self._pairs(items)
        need = self.workspace_bytes(shapes)
        ws = self._workspace(need)
        check(lib().de_dense_dev(C.byref(self.cfg), arr, len(items), ws.data_ptr(), need,
                                 _stream_handle(stream)))

    def _pairs(self, items):
        arr = (DePair * len(items))()
        shapes = []
        for i, (L, R, dmax, out) in enumerate(items):
            H, W = L.shape
            shapes.append((W, H, dmax))
            ptr = lambda k: out[k].data_ptr() if out.get(k) is not None else None  # noqa
            arr[i] = DePair(L.data_ptr(), R.data_ptr(), W, H, dmax, ptr("disp"),
                            ptr("margin"), ptr("conf"), ptr("cand"))
        return arr, shapes

    def capture(self, items) -> "CapturedBatch":
        """Capture this batch's launch set (fixed buffers) as a CUDA graph; the
        returned object's ``launch(stream)`` replays it, reading the input tensors as
        they are at replay time.  Holds its own workspace."""
        torch = _torch()
        arr, shapes = self._pairs(items)
        need = self.workspace_bytes(shapes)
        ws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)
        g = C.c_void_p()
        check(lib().de_graph_create(C.byref(self.cfg), arr, len(items), ws.data_ptr(), need,
                                    C.byref(g)))
        return CapturedBatch(g, ws, items)

    def match(self, L, R, dmax: int = 0, cand: bool = False, stream=None) -> dict:
        out = self.new_outputs(*L.shape, cand=cand)
        self.match_into([(L, R, dmax, out)], stream)
        return out

    def match_batch(self, pairs, cand: bool = False, stream=None) -> list[dict]:
        outs = [self.new_outputs(*p[0].shape, cand=cand) for p in pairs]
        self.match_into([(p[0], p[1], p[2] if len(p) > 2 else 0, o)
                         for p, o in zip(pairs, outs)], stream)
        return outs


class CapturedBatch:
    """A batch captured as a CUDA graph (``DenseMatcher.capture``)."""

    def __init__(self, handle, workspace, items):
        self._g = handle
        self._keep = (workspace, items)      # buffers the graph reads and writes

    def launch(self, stream=None) -> None:
        check(lib().de_graph_launch(self._g, _stream_handle(stream)))

    def close(self) -> None:
        if self._g:
            check(lib().de_graph_destroy(self._g))
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------------------
# Stage entry points (device tensors), for stage-level parity and custom pipelines

def census(L, R, cfg: Optional[DeCfg] = None, stream=None):
    """Census words of both images (uint64 as int64 tensors) and the left image's
    Q15 coefficient planes ax, ay (int16 tensors holding uint16 bit patterns)."""
    torch = _torch()
    cfg = cfg or Cfg()
    H, W = L.shape
    cl = torch.empty((H, W), dtype=torch.int64, device=L.device)
    cr = torch.empty_like(cl)
    ax = torch.empty((H, W), dtype=torch.int16, device=L.device)
    ay = torch.empty_like(ax)
    check(lib().de_census_dev(C.byref(cfg), L.data_ptr(), R.data_ptr(), W, H, cl.data_ptr(),
                              cr.data_ptr(), ax.data_ptr(), ay.data_ptr(),
                              _stream_handle(stream)))
    return cl, cr, ax, ay


def cost_top2(L, R, cfg: Optional[DeCfg] = None, stream=None):
    """Candidates in the reference layout: cs f32 (H,W,2), cd i32 (H,W,2), cn i32 (H,W),
    cnb i16 (H,W,2)."""
    torch = _torch()
    cfg = cfg or Cfg()
    H, W = L.shape
    D = cfg.dmax - cfg.dmin + 1
    ws_n = lib().de_cost_workspace_bytes(W, H, D)
    ws = torch.empty(ws_n, dtype=torch.uint8, device=L.device)
    cs = torch.empty((H, W, 2), dtype=torch.float32, device=L.device)
    cd = torch.empty((H, W, 2), dtype=torch.int32, device=L.device)
    cn = torch.empty((H, W), dtype=torch.int32, device=L.device)
    cnb = torch.empty((H, W, 2), dtype=torch.int16, device=L.device)
    check(lib().de_cost_top2_dev(C.byref(cfg), L.data_ptr(), R.data_ptr(), W, H, cs.data_ptr(),
                                 cd.data_ptr(), cn.data_ptr(), cnb.data_ptr(), ws.data_ptr(),
                                 ws_n, _stream_handle(stream)))
    return cs, cd, cn, cnb


def solve(cs, cd, cn, cnb, cfg: Optional[DeCfg] = None, stream=None):
    """Row solve over reference-layout candidates: disp, margin, lrc2 (H, W)."""
    torch = _torch()
    cfg = cfg or Cfg()
    H, W = cn.shape
    disp = torch.empty((H, W), dtype=torch.float32, device=cn.device)
    margin = torch.empty_like(disp)
    lrc2 = torch.empty_like(disp)
    check(lib().de_solve_dev(C.byref(cfg), W, H, cs.data_ptr(), cd.data_ptr(), cn.data_ptr(),
                             cnb.data_ptr() if cnb is not None else None, disp.data_ptr(),
                             margin.data_ptr(), lrc2.data_ptr(), _stream_handle(stream)))
    return disp, margin, lrc2


def confidence(s1: float, s2: float, lam: float = -0.1, lrc: float = 0.0,
               lrc_tol: float = 1.0) -> float:
    """confidence() of core/include/doubleeye/dense_solve.hpp:158 (host)."""
    return lib().de_confidence(s1, s2, lam, lrc, lrc_tol)
