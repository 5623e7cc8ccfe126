"""dense_problem of article/dense_masda.py:39-79, on the GPU.

``dense_problem(left, right, dmin, dmax, census_cfg=(3, 3)) -> (ei, ej, se, H*W)``:
every interior pixel against every disparity on its row, left index y*W + x, right
index y*W + x - d, se = (24 - Hamming)/24 as float32, in the reference's order
(disparity, then row, then column).  ``device=True`` returns CUDA tensors instead of
NumPy arrays (52 M edges at 848x480, D=128 stay on the GPU for masda_sparse).
"""
from __future__ import annotations

import numpy as np

from ._lib import check, lib
from .masda_stereo import masda_sparse  # noqa: F401  (the solver dense_problem feeds)


def dense_problem(left, right, dmin, dmax, census_cfg=(3, 3), device=False):
    import torch
    L = left if isinstance(left, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(left, np.uint8))
    R = right if isinstance(right, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(right, np.uint8))
    L = L.cuda().contiguous()
    R = R.cuda().contiguous()
    H, W = L.shape
    hw, hh = census_cfg
    E = int(lib().de_dense_problem_edges(W, H, int(dmin), int(dmax), hw, hh))
    ei = torch.empty(max(E, 1), dtype=torch.int64, device="cuda")
    ej = torch.empty_like(ei)
    se = torch.empty(max(E, 1), dtype=torch.float32, device="cuda")
    ws = torch.empty(16 * W * H + 512, dtype=torch.uint8, device="cuda")
    check(lib().de_dense_problem_dev(L.data_ptr(), R.data_ptr(), W, H, int(dmin), int(dmax),
                                     hw, hh, ei.data_ptr(), ej.data_ptr(), se.data_ptr(), E,
                                     ws.data_ptr(), ws.numel(),
                                     int(torch.cuda.current_stream().cuda_stream)))
    ei, ej, se = ei[:E], ej[:E], se[:E]
    if device:
        return ei, ej, se, H * W
    return ei.cpu().numpy(), ej.cpu().numpy(), se.cpu().numpy(), H * W
