"""doubleeye_b200 -- the stereo matching hot path of mayio/doubleeye on B200 (sm_100a).

Census -> graded Census/AD cost -> four-pass recursive edge-aware filter -> per-pixel
top-2 -> MASDA max-sum row solve (dense), and keypoint MASDA (sparse), as hand-written
CUDA behind a C ABI (include/doubleeye_b200.h).  Modules:

  dense        run_dense / DenseMatcher / stage entry points (core/tools/de_dense.cpp)
  synth        seeded synthetic stereo pairs with ground truth
  build        nvcc build of the in-tree library
"""
from .dense import (CAND_PLANES, Cfg, DenseMatcher, DenseResult, census, confidence,
                    cost_top2, run_dense, run_dense_batch, solve)

__all__ = ["CAND_PLANES", "Cfg", "DenseMatcher", "DenseResult", "census", "confidence",
           "cost_top2", "run_dense", "run_dense_batch", "solve"]
