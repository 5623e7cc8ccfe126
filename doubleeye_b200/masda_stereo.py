"""The Python entry points of article/masda_stereo.py, on the GPU.

Same names, signatures and return values as the reference module (NumPy in, NumPy
out; torch CUDA tensors are accepted where arrays are):

  census(img, pts, half_w, half_h)          article/masda_stereo.py:264-284
  hamming(a, b)                             :290-295
  build_problem(pl, dl, pr, dr, ...)        :305-326
  masda(S, lam, gam, iters, damping, eps)   :329-389
  decide(S, belief, lam)                    :392-414
  _seg_max_excluding(vals, idx, n)          :417-442
  to_edges(S)                               :445-450
  masda_sparse(ei, ej, se, m, n, ...)       :453-492

All arithmetic is float64 like NumPy and follows the reference's operation order, so
message histories are bit-identical; where NumPy's argsort meets exactly equal
beliefs (its order is unspecified) the lower edge index wins.  Every call runs
through the C ABI; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

BITS = 48


def _torch():
    import torch
    return torch


def _stream() -> int:
    return int(_torch().cuda.current_stream().cuda_stream)


def _dev(a, dtype):
    """A contiguous CUDA tensor of the given numpy dtype holding ``a``."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a.detach()
        want = torch.from_numpy(np.zeros(0, dtype)).dtype
        if t.dtype != want:
            t = t.to(want)
        return t.cuda().contiguous()
    arr = np.ascontiguousarray(np.asarray(a), dtype)
    if arr.dtype == np.uint64:
        return torch.from_numpy(arr.view(np.int64)).cuda()
    return torch.from_numpy(arr).cuda()


def _np(t, dtype=None):
    a = t.cpu().numpy()
    return a.view(dtype) if dtype is not None else a


def _ws(nbytes: int):
    torch = _torch()
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")


def census(img, pts, half_w=3, half_h=3):
    """Census descriptor (uint64) at each point, pts as (x, y) rows truncated to int."""
    torch = _torch()
    img = np.ascontiguousarray(np.asarray(img), np.uint8) if not isinstance(
        img, torch.Tensor) else img
    H, W = img.shape
    xy = np.asarray(pts).astype(int).astype(np.int32).reshape(-1, 2)
    n = len(xy)
    out = torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")
    if n:
        g = _dev(img, np.uint8)
        xy_d = _dev(xy, np.int32)               # kept alive until the kernel has run
        check(lib().de_census_pts_dev(g.data_ptr(), W, H, xy_d.data_ptr(), n, half_w, half_h,
                                      out.data_ptr(), None, _stream()))
    return _np(out[:n], np.uint64)


def hamming(a, b):
    """popcount(a ^ b) per element (int32), NumPy broadcasting."""
    a, b = np.broadcast_arrays(np.asarray(a, np.uint64), np.asarray(b, np.uint64))
    shape = a.shape
    n = a.size
    torch = _torch()
    out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    if n:
        a_d = _dev(a.ravel(), np.uint64)
        b_d = _dev(b.ravel(), np.uint64)
        check(lib().de_hamming_dev(a_d.data_ptr(), b_d.data_ptr(), n, out.data_ptr(),
                                   _stream()))
    return _np(out[:n]).reshape(shape)


def build_problem(pl, dl, pr, dr, max_dy=1.5, dmin=1.0, dmax=60.0, sigma_y=1.0, w_y=1.0):
    """The m x n float32 score matrix, -inf where no candidate edge exists."""
    torch = _torch()
    pl = np.ascontiguousarray(pl, np.float32).reshape(-1, 2)
    pr = np.ascontiguousarray(pr, np.float32).reshape(-1, 2)
    m, n = len(pl), len(pr)
    S = torch.empty((max(m, 1), max(n, 1)), dtype=torch.float32, device="cuda")
    if m and n:
        args = [_dev(pl, np.float32), _dev(dl, np.uint64), _dev(pr, np.float32),
                _dev(dr, np.uint64)]
        check(lib().de_build_problem_dev(
            args[0].data_ptr(), args[1].data_ptr(), m, args[2].data_ptr(), args[3].data_ptr(),
            n, max_dy, dmin, dmax, sigma_y, w_y, BITS, S.data_ptr(), _stream()))
    return _np(S[:m, :n]).copy() if m and n else np.full((m, n), -np.inf, np.float32)


def _to_edges_dev(S):
    """Finite entries of a float32 matrix, row-major, as device tensors."""
    torch = _torch()
    Sd = _dev(S, np.float32)
    m, n = Sd.shape
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = _ws(8 * max(m, 1) + 256)
    check(lib().de_edges_from_matrix_dev(Sd.data_ptr(), m, n, None, None, None, 0,
                                         cnt.data_ptr(), ws.data_ptr(), ws.numel(), _stream()))
    E = int(cnt.item())
    ei = torch.empty(max(E, 1), dtype=torch.int64, device="cuda")
    ej = torch.empty_like(ei)
    se = torch.empty(max(E, 1), dtype=torch.float64, device="cuda")
    check(lib().de_edges_from_matrix_dev(Sd.data_ptr(), m, n, ei.data_ptr(), ej.data_ptr(),
                                         se.data_ptr(), E, cnt.data_ptr(), ws.data_ptr(),
                                         ws.numel(), _stream()))
    return ei[:E], ej[:E], se[:E]


def to_edges(S):
    """Dense score matrix -> (ei, ej, se) edge list, row-major (int64, int64, float64)."""
    ei, ej, se = _to_edges_dev(S)
    return _np(ei), _np(ej), _np(se)


def _seg_max_excluding(vals, idx, n):
    """Per-segment max with each element's own contribution removed."""
    torch = _torch()
    v = _dev(vals, np.float64)
    ix = _dev(idx, np.int64)
    E = v.numel()
    out = torch.empty(max(E, 1), dtype=torch.float64, device="cuda")
    ws = _ws(20 * max(int(n), 1) + 1024)
    check(lib().de_seg_max_excluding_dev(v.data_ptr(), ix.data_ptr(), E, int(n),
                                         out.data_ptr(), ws.data_ptr(), ws.numel(), _stream()))
    return _np(out[:E])


def _solve(ei, ej, se, m, n, lam, gam, iters, damping, eps, want_belief=False):
    torch = _torch()
    E = int(se.numel())
    need = C.c_size_t()
    check(lib().de_masda_edges_workspace_bytes(E, m, n, C.byref(need)))
    ws = _ws(need.value)
    assign = torch.empty(max(m, 1), dtype=torch.int64, device="cuda")
    hist = torch.zeros(max(iters, 1), dtype=torch.float64, device="cuda")
    nh = torch.zeros(1, dtype=torch.int32, device="cuda")
    belief = torch.empty(max(E, 1), dtype=torch.float64, device="cuda") if want_belief else None
    check(lib().de_masda_edges_dev(ei.data_ptr(), ej.data_ptr(), se.data_ptr(), E, m, n,
                                   float(lam), float(gam), int(iters), float(damping),
                                   float(eps), assign.data_ptr(), hist.data_ptr(),
                                   nh.data_ptr(), belief.data_ptr() if belief is not None
                                   else None, ws.data_ptr(), need.value, _stream()))
    k = int(nh.item())
    a = _np(assign[:m])
    out = {int(i): int(j) for i, j in zip(np.nonzero(a >= 0)[0], a[a >= 0])}
    return out, _np(hist[:k]), belief


def masda_sparse(ei, ej, se, m, n, lam=-0.1, gam=-0.1, iters=30, damping=0.4, eps=1e-5):
    """MASDA on an edge list: (dict left -> right, per-iteration max change)."""
    size = se.numel() if hasattr(se, "numel") else np.asarray(se).size
    if size == 0:
        raise ValueError("zero-size array to reduction operation maximum which has no "
                         "identity")
    ei_d, ej_d, se_d = _dev(ei, np.int64), _dev(ej, np.int64), _dev(se, np.float64)
    out, hist, _ = _solve(ei_d, ej_d, se_d, int(m), int(n), lam, gam, iters, damping, eps)
    return out, hist


def masda(S, lam=-0.1, gam=-0.1, iters=30, damping=0.4, eps=1e-5):
    """MASDA on a dense m x n score matrix (-inf = no edge): (dict, hist)."""
    if not hasattr(S, "cuda") and np.asarray(S).dtype != np.float32:
        S = np.asarray(S, np.float64)            # keep float64 scores exact
        m, n = S.shape
        ii, jj = np.nonzero(np.isfinite(S))
        ei, ej, se = _dev(ii, np.int64), _dev(jj, np.int64), _dev(S[ii, jj], np.float64)
    else:
        m, n = S.shape
        ei, ej, se = _to_edges_dev(S)
    if se.numel() == 0:
        return {}, np.array([0.0] if iters > 0 else [])
    out, hist, _ = _solve(ei, ej, se, m, n, lam, gam, iters, damping, eps)
    return out, hist


def decide(S, belief, lam):
    """Greedy one-to-one in belief order over finite beliefs with S > lam."""
    torch = _torch()
    B = np.asarray(belief, np.float64)
    Sm = np.asarray(S)
    m, n = B.shape
    fin = np.isfinite(B)
    ei, ej = np.nonzero(fin)
    E = len(ei)
    need = C.c_size_t()
    check(lib().de_masda_edges_workspace_bytes(E, m, n, C.byref(need)))
    ws = _ws(need.value)
    assign = torch.empty(max(m, 1), dtype=torch.int64, device="cuda")
    if E:
        args = [_dev(ei, np.int64), _dev(ej, np.int64), _dev(Sm[ei, ej], np.float64),
                _dev(B[ei, ej], np.float64)]
        check(lib().de_masda_decide_dev(
            args[0].data_ptr(), args[1].data_ptr(), args[2].data_ptr(), args[3].data_ptr(),
            E, m, n, float(lam), assign.data_ptr(), ws.data_ptr(), need.value, _stream()))
    else:
        assign.fill_(-1)
    a = _np(assign[:m])
    return {int(i): int(j) for i, j in zip(np.nonzero(a >= 0)[0], a[a >= 0])}
