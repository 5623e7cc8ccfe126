"""``torch.ops.doubleeye``: the stereo hot path as torch operators.

Device tensors in, outputs allocated by the operator on the input's device, work
enqueued on the current CUDA stream through the C ABI (the same sm_100a kernels as
``dense`` and ``sparse``; there is no CPU kernel).  Registered on import:

  doubleeye::dense(left, right, dmax, iters, ...) -> (disp, margin, conf)
      the whole dense pipeline, one pair (core/tools/de_dense.cpp:738 run_dense)
  doubleeye::cost_top2(left, right, dmax, ...) -> (cs, cd, cn, cnb)
      census, graded cost, four-pass filter and top-2 candidates in the reference
      layout (core/tools/de_dense_cuda.cu:286-392)
  doubleeye::solve(cs, cd, cn, cnb, dmax, iters, ...) -> (disp, margin, lrc2)
      the row solve over such candidates (core/include/doubleeye/dense_solve.hpp:213)
  doubleeye::match_masda(kl, dl, kr, dr, ...) -> (pairs, values)
      keypoint MASDA (core/src/match.cpp:334): kl/kr (n, 4) float32 keypoints
      (x, y, response, local_std), dl/dr int64 descriptors (uint64 bit patterns);
      pairs (m, 2) int32 (left, right), values (m, 5) float32 (score, belief,
      disparity, dy, margin), in the reference's emission order

Configuration arguments are the de_cfg / de_match_cfg fields with the reference's
defaults.  Each operator has a fake (meta) implementation for shape propagation where
the output shape is known from the inputs.
"""
from __future__ import annotations

import torch

from . import dense, sparse
from ._lib import DeMatchStats

_NS = "doubleeye"


def _cfg(dmax, iters, dmin=1, lambda_=-0.1, gamma=-0.1, damping=0.4, subpixel=True,
         fit_eq=True, lrc=False, min_margin=0.0, min_ratio=0.0, census_hw=3, census_hh=3):
    return dense.Cfg(dmin=int(dmin), dmax=int(dmax), iters=int(iters), lambda_=float(lambda_),
                     gamma=float(gamma), damping=float(damping), subpixel=int(bool(subpixel)),
                     fit_eq=int(bool(fit_eq)), lrc=int(bool(lrc)), min_margin=float(min_margin),
                     min_ratio=float(min_ratio), census_hw=int(census_hw),
                     census_hh=int(census_hh))


def _check_images(left: torch.Tensor, right: torch.Tensor) -> None:
    if left.dtype != torch.uint8 or right.dtype != torch.uint8 or left.dim() != 2 \
            or left.shape != right.shape or not left.is_cuda or not right.is_cuda:
        raise ValueError("left and right must be 2-D uint8 CUDA tensors of one shape")


@torch.library.custom_op(f"{_NS}::dense", mutates_args=())
def dense_op(left: torch.Tensor, right: torch.Tensor, dmax: int = 60, iters: int = 0,
             dmin: int = 1, lambda_: float = -0.1, gamma: float = -0.1,
             damping: float = 0.4, subpixel: bool = True, fit_eq: bool = True,
             lrc: bool = False, min_margin: float = 0.0, min_ratio: float = 0.0,
             census_hw: int = 3, census_hh: int = 3
             ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    _check_images(left, right)
    cfg = _cfg(dmax, iters, dmin, lambda_, gamma, damping, subpixel, fit_eq, lrc, min_margin,
               min_ratio, census_hw, census_hh)
    with torch.cuda.device(left.device):
        m = dense.DenseMatcher(cfg, device=left.device.index or 0)
        out = m.match(left.contiguous(), right.contiguous())
    return out["disp"], out["margin"], out["conf"]


@dense_op.register_fake
def _(left, right, dmax=60, iters=0, dmin=1, lambda_=-0.1, gamma=-0.1, damping=0.4,
      subpixel=True, fit_eq=True, lrc=False, min_margin=0.0, min_ratio=0.0, census_hw=3,
      census_hh=3):
    f = torch.empty(left.shape, dtype=torch.float32, device=left.device)
    return f, torch.empty_like(f), torch.empty(left.shape, dtype=torch.uint8, device=left.device)


@torch.library.custom_op(f"{_NS}::cost_top2", mutates_args=())
def cost_top2_op(left: torch.Tensor, right: torch.Tensor, dmax: int = 60, dmin: int = 1,
                 subpixel: bool = True, census_hw: int = 3, census_hh: int = 3
                 ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    _check_images(left, right)
    cfg = _cfg(dmax, 0, dmin, subpixel=subpixel, census_hw=census_hw, census_hh=census_hh)
    with torch.cuda.device(left.device):
        return dense.cost_top2(left.contiguous(), right.contiguous(), cfg)


@cost_top2_op.register_fake
def _(left, right, dmax=60, dmin=1, subpixel=True, census_hw=3, census_hh=3):
    H, W = left.shape
    dev = left.device
    return (torch.empty((H, W, 2), dtype=torch.float32, device=dev),
            torch.empty((H, W, 2), dtype=torch.int32, device=dev),
            torch.empty((H, W), dtype=torch.int32, device=dev),
            torch.empty((H, W, 2), dtype=torch.int16, device=dev))


@torch.library.custom_op(f"{_NS}::solve", mutates_args=())
def solve_op(cs: torch.Tensor, cd: torch.Tensor, cn: torch.Tensor, cnb: torch.Tensor,
             dmax: int = 60, iters: int = 0, dmin: int = 1, lambda_: float = -0.1,
             gamma: float = -0.1, damping: float = 0.4, subpixel: bool = True,
             fit_eq: bool = True, min_margin: float = 0.0, min_ratio: float = 0.0
             ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    if cs.dtype != torch.float32 or cd.dtype != torch.int32 or cn.dtype != torch.int32 or \
            cnb.dtype != torch.int16 or not cs.is_cuda or cn.dim() != 2 or \
            cs.shape != (*cn.shape, 2) or cd.shape != cs.shape or cnb.shape != cs.shape:
        raise ValueError("candidates: cs f32 (H,W,2), cd i32 (H,W,2), cn i32 (H,W), "
                         "cnb i16 (H,W,2) CUDA tensors")
    cfg = _cfg(dmax, iters, dmin, lambda_, gamma, damping, subpixel, fit_eq,
               min_margin=min_margin, min_ratio=min_ratio)
    with torch.cuda.device(cs.device):
        return dense.solve(cs.contiguous(), cd.contiguous(), cn.contiguous(),
                           cnb.contiguous(), cfg)


@solve_op.register_fake
def _(cs, cd, cn, cnb, dmax=60, iters=0, dmin=1, lambda_=-0.1, gamma=-0.1, damping=0.4,
      subpixel=True, fit_eq=True, min_margin=0.0, min_ratio=0.0):
    f = torch.empty(cn.shape, dtype=torch.float32, device=cn.device)
    return f, torch.empty_like(f), torch.empty_like(f)


@torch.library.custom_op(f"{_NS}::match_masda", mutates_args=())
def match_masda_op(kl: torch.Tensor, dl: torch.Tensor, kr: torch.Tensor, dr: torch.Tensor,
                   max_dy: float = 2.0, min_disparity: float = 1.0,
                   max_disparity: float = 220.0, max_candidates: int = 24,
                   sigma_y: float = 1.0, w_y: float = 1.0, iterations: int = 20,
                   damping: float = 0.4, lambda_: float = 0.0, gamma: float = 0.0,
                   converge_eps: float = 1e-4, census_bits: int = 48
                   ) -> tuple[torch.Tensor, torch.Tensor]:
    for k, ok in ((kl, kl.dim() == 2 and kl.shape[1] == 4 and kl.dtype == torch.float32),
                  (kr, kr.dim() == 2 and kr.shape[1] == 4 and kr.dtype == torch.float32),
                  (dl, dl.dim() == 1 and dl.dtype == torch.int64 and dl.numel() == kl.shape[0]),
                  (dr, dr.dim() == 1 and dr.dtype == torch.int64 and dr.numel() == kr.shape[0])):
        if not ok or not k.is_cuda:
            raise ValueError("kl/kr (n, 4) float32 and dl/dr (n,) int64 CUDA tensors")
    cfg = sparse.MatchCfg(max_dy=max_dy, min_disparity=min_disparity,
                          max_disparity=max_disparity, max_candidates=max_candidates,
                          sigma_y=sigma_y, w_y=w_y, iterations=iterations, damping=damping,
                          lambda_=lambda_, gamma=gamma, converge_eps=converge_eps,
                          census_bits=census_bits)
    sm = sparse.SparseMatcher(cfg=cfg, device=kl.device.index or 0)
    with torch.cuda.device(kl.device):
        out, n, _ = sm.match(kl.contiguous(), dl.contiguous(), kr.contiguous(), dr.contiguous())
        k = int(n.item())                              # the count sizes the outputs
        rec = out[:k]
        return rec[:, :2].contiguous(), rec[:, 2:].contiguous().view(torch.float32)


def stats_of(st: torch.Tensor) -> dict:
    """A de_match_stats record (7 int32 on the device) as a dict."""
    return sparse.stats_dict(DeMatchStats.from_buffer_copy(st.cpu().numpy().tobytes()))


def registered() -> list[str]:
    return [f"{_NS}::{n}" for n in ("dense", "cost_top2", "solve", "match_masda")]
