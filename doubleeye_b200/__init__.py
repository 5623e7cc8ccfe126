"""doubleeye_b200 -- the stereo matching hot path of mayio/doubleeye on B200 (sm_100a).

Census -> graded Census/AD cost -> four-pass recursive edge-aware filter -> per-pixel
top-2 -> MASDA max-sum row solve (dense), and keypoint MASDA (sparse), as hand-written
CUDA behind a C ABI (include/doubleeye_b200.h).  Modules:

  dense        run_dense / DenseMatcher / stage entry points (core/tools/de_dense.cpp)
  sparse       FAST detector, census_at, keypoint MASDA (core/src/preproc.cpp, match.cpp)
  masda_stereo the article/masda_stereo.py entry points in float64
  dense_masda  article/dense_masda.py dense_problem
  serve        many-stream server: continuous batching, p50/p99 latency, DEDD planes
  autotune     launch-shape tuner (results unchanged by any setting)
  replicas     multi-GPU replicas: sharding and max-over-ranks
  synth        seeded synthetic stereo pairs with ground truth
  build        nvcc build of the in-tree library and the de_dense_gpu command line
"""
from .dense import (CAND_PLANES, Cfg, DenseMatcher, DenseResult, census, confidence,
                    cost_top2, fill_holes, new_results, pinned_empty, run_dense,
                    run_dense_batch, run_dense_prior, solve)

__all__ = ["CAND_PLANES", "Cfg", "DenseMatcher", "DenseResult", "census", "confidence",
           "cost_top2", "fill_holes", "new_results", "pinned_empty", "run_dense",
           "run_dense_batch", "run_dense_prior", "solve"]
