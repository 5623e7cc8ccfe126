"""The disparity prior as a per-plane mask (--prior): the oracle against the reference's
own outputs (tests/golden/prior.npz, tests/golden/make_golden_prior.py), and the GPU
path against both, bit for bit.  The cases cover a noisy prior at two bands (with and
without left-right reverse matching), a constant prior, and a ramp that leaves most of
the image without candidates."""
import ast
import os

import numpy as np
import pytest

from oracle import oracle as O

CASES = ["noisy_b2", "noisy_b4_lrc", "const_b1", "ramp_b3"]


def same(a, b):
    return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())


@pytest.fixture(scope="module")
def g(golden_dir):
    return np.load(os.path.join(golden_dir, "prior.npz"))


def case(g, name):
    kw = ast.literal_eval(str(g[f"{name}_cfg"][0]))
    return (kw, g[f"{name}_L"], g[f"{name}_R"], g[f"{name}_prior"], int(g[f"{name}_band"]),
            g[f"{name}_disp"], g[f"{name}_margin"], g[f"{name}_cand"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(oracle, g, name):
    kw, L, R, prior, band, disp, margin, cand = case(g, name)
    d, m, c = oracle.dense_prior(O.default_cfg(**kw), L, R, prior, band)
    assert same(d, disp) and same(m, margin) and same(c, cand)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference(g, name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import doubleeye_b200 as de
    kw, L, R, prior, band, disp, margin, cand = case(g, name)
    r = de.run_dense_prior(L, R, prior, de.Cfg(**kw), band=band)
    assert same(r.disp, disp) and same(r.margin, margin) and same(r.cand, cand)


@pytest.mark.gpu
def test_gpu_full_size_previous_frame_prior(oracle):
    """848x480, D=128: the previous frame's disparity as this frame's prior."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import doubleeye_b200 as de
    from doubleeye_b200 import synth
    v = synth.Video(848, 480, 127, stream_id=3)
    f0, f1 = v.frame(0), v.frame(1)
    cfg = dict(dmax=128, iters=8)
    prev = de.run_dense(f0.left, f0.right, de.Cfg(**cfg), want_cand=False).disp
    prior = np.where(np.isfinite(prev), prev, np.float32(64)).astype(np.float32)
    r = de.run_dense_prior(f1.left, f1.right, prior, de.Cfg(**cfg), band=4)
    d, m, c = oracle.dense_prior(O.default_cfg(**cfg), f1.left, f1.right, prior, 4)
    assert same(r.disp, d) and same(r.margin, m) and same(r.cand, c)
    assert np.isfinite(r.disp).mean() > 0.5


@pytest.mark.gpu
def test_gpu_refuses_holes():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import doubleeye_b200 as de
    from doubleeye_b200._lib import DeError
    L = np.zeros((64, 96), np.uint8)
    prior = np.full((64, 96), 10, np.float32)
    prior[5, 5] = np.nan
    with pytest.raises(DeError):
        de.run_dense_prior(L, L, prior, de.Cfg(dmax=32))
