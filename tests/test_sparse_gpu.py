"""Sparse path on the GPU through the C ABI: census_at, the FAST detector and keypoint
MASDA, against the oracle (bit for bit: the CUDA path breaks exact ties the same way)
and against the reference's own golden outputs (tie-aware, see test_oracle_sparse)."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from test_oracle_sparse import (CASES, det_cfg, known_answer_cases, load, match_cfg,
                                objective, same_bits, tie_aware_same)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def sp():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from doubleeye_b200 import build, sparse
    build.build()
    return sparse


def gpu_det(sp, det):
    c = sp.DetCfg()
    for f, _ in c._fields_:
        setattr(c, f, getattr(det, f))
    return c


def gpu_mcfg(sp, cfg):
    c = sp.MatchCfg()
    for f, _ in c._fields_:
        setattr(c, f, getattr(cfg, f))
    return c


def c1(W=848, H=480, seed=5):
    from doubleeye_b200 import synth
    return synth.fronto_planes(W, H, seed=seed)


# -- census_at ------------------------------------------------------------------------

@pytest.mark.parametrize("hw,hh", [(2, 2), (3, 3), (4, 3)])
def test_census_at(sp, oracle, hw, hh):
    p = c1(200, 120)
    rng = np.random.default_rng(hw * 10 + hh)
    kp = np.zeros((500, 4), np.float32)
    kp[:, 0] = rng.uniform(-1, 201, 500)
    kp[:, 1] = rng.uniform(-1, 121, 500)
    got = sp.census_at(p.left, kp, hw, hh)
    want = np.array([oracle.census_at(p.left, int(x + 0.5), int(y + 0.5), hw, hh)[0]
                     for x, y in kp[:, :2]], np.uint64)
    assert np.array_equal(got, want)
    assert (want == 0).sum() < 100


# -- detector -------------------------------------------------------------------------

DET_CASES = [
    ("default", {}),
    ("cell24", dict(cell=24)),
    ("dense_noref", dict(per_cell=6, subpixel=0)),
    ("nms1", dict(nms_radius=1, per_cell=8)),
    ("nms5", dict(nms_radius=5, per_cell=8)),          # the word-fetch suppression up to 7
    ("nms7", dict(nms_radius=7, per_cell=8)),
    ("nms9", dict(nms_radius=9, per_cell=8)),          # the per-pixel suppression above 7
    ("grad5", dict(grad_window=5)),
    ("thr20", dict(fast_threshold=20, min_response=20.0)),
    ("cell128", dict(cell=128, per_cell=40)),
    ("floor", dict(min_local_std=30.0, border=12)),
]


@pytest.mark.parametrize("name,kw", DET_CASES, ids=[c[0] for c in DET_CASES])
def test_detect_fast_bit_exact(sp, oracle, name, kw):
    p = c1(seed=11)
    det = O.default_det_cfg(**kw)
    for img in (p.left, p.right):
        want = oracle.detect_fast(img, det)
        got = sp.detect_fast(img, gpu_det(sp, det))
        assert same_bits(got, want), (name, got.shape, want.shape)
    assert len(want) > 0


def test_detect_odd_sizes_and_empty(sp, oracle):
    from doubleeye_b200 import synth
    for W, H in [(333, 211), (40, 24), (16, 16)]:
        img = synth.fronto_planes(W, H, seed=W).left
        det = O.default_det_cfg(cell=16, border=5)
        assert same_bits(sp.detect_fast(img, gpu_det(sp, det)), oracle.detect_fast(img, det))
    flat = np.full((64, 96), 90, np.uint8)
    assert len(sp.detect_fast(flat, sp.DetCfg())) == 0


def test_detect_real_golden(sp, golden_dir):
    for name in CASES:
        g = load(golden_dir, name)
        det = gpu_det(sp, det_cfg(g["det"]))
        assert same_bits(sp.detect_fast(g["L"], det), g["kl"]), name
        assert same_bits(sp.detect_fast(g["R"], det), g["kr"]), name


# -- matcher --------------------------------------------------------------------------

def described(oracle, p, det, hw=3, hh=3):
    kl = oracle.detect_fast(p.left, det)
    kr = oracle.detect_fast(p.right, det)
    d = lambda img, kp: np.array([oracle.census_at(img, int(x + 0.5), int(y + 0.5), hw, hh)[0]  # noqa
                                  for x, y in kp[:, :2]], np.uint64)
    return kl, d(p.left, kl), kr, d(p.right, kr)


MATCH_CASES = [
    ("default", {}),
    ("lam_neg", dict(lambda_=-0.1, gamma=-0.1, iterations=10)),
    ("cand1", dict(max_candidates=1)),
    ("cand3_band3", dict(max_candidates=3, max_dy=3.0)),
    ("iters0", dict(iterations=0)),
    ("iters1_nodamp", dict(iterations=1, damping=0.0)),
    ("damp099", dict(damping=1.5, iterations=40)),
    ("strict", dict(lambda_=0.5, gamma=0.2)),
    ("bits62", dict(census_bits=62, w_y=0.25, sigma_y=2.0)),
    ("narrow", dict(min_disparity=5.0, max_disparity=30.0)),
]


@pytest.fixture(scope="module")
def c1_problem(oracle):
    p = c1(seed=3)
    return described(oracle, p, O.default_det_cfg(cell=24))


@pytest.mark.parametrize("name,kw", MATCH_CASES, ids=[c[0] for c in MATCH_CASES])
def test_match_masda_bit_exact(sp, oracle, c1_problem, name, kw):
    kl, dl, kr, dr = c1_problem
    assert len(kl) > 1500
    cfg = O.default_match_cfg(**kw)
    want, wst = oracle.match_masda(kl, dl, kr, dr, cfg)
    got, gst = sp.match_masda(kl, dl, kr, dr, gpu_mcfg(sp, cfg))
    assert same_bits(got, want), (name, len(got), len(want))
    assert [gst[f] for f in ("left", "right", "candidates", "iterations_run", "converged",
                             "oscillating")] == [wst.left, wst.right, wst.candidates,
                                                 wst.iterations_run, wst.converged,
                                                 wst.oscillating]
    assert np.float32(gst["final_max_delta"]) == np.float32(wst.final_max_delta)


def test_match_golden_reference(sp, golden_dir):
    for name in CASES:
        g = load(golden_dir, name)
        for k in range(len(g["match_cfgs"])):
            cfg = gpu_mcfg(sp, match_cfg(g["match_cfgs"][k]))
            got, _ = sp.match_masda(g["kl"], g["dl"], g["kr"], g["dr"], cfg)
            assert tie_aware_same(got, g[f"matches_{k}"]), (name, k)


def test_match_bruteforce_problems(sp, oracle, golden_dir):
    g = load(golden_dir, "sparse_bruteforce")
    cfg = match_cfg(g["cfg"][0])
    gcfg = gpu_mcfg(sp, cfg)
    optimal = 0
    for t in range(len(g["off_l"]) - 1):
        sl = slice(g["off_l"][t], g["off_l"][t + 1])
        sr = slice(g["off_r"][t], g["off_r"][t + 1])
        got, _ = sp.match_masda(g["kl"][sl], g["dl"][sl], g["kr"][sr], g["dr"][sr], gcfg)
        want, _ = oracle.match_masda(g["kl"][sl], g["dl"][sl], g["kr"][sr], g["dr"][sr], cfg)
        assert same_bits(got, want), t
        bf = g["brute"][g["off_b"][t]:g["off_b"][t + 1]]
        n, m = sl.stop - sl.start, sr.stop - sr.start
        optimal += objective(got, cfg.lambda_, cfg.gamma, n, m) >= \
            objective(bf, cfg.lambda_, cfg.gamma, n, m) - 1e-4
    assert optimal >= 54


@pytest.mark.parametrize("case", known_answer_cases(), ids=lambda c: c[0])
def test_known_answers(sp, oracle, case):
    name, kl, dl, kr, dr, cfg, want = case
    kl = np.array(kl, np.float32).reshape(-1, 4)
    kr = np.array(kr, np.float32).reshape(-1, 4)
    dl = np.array(dl, np.uint64)
    dr = np.array(dr, np.uint64)
    got, st = sp.match_masda(kl, dl, kr, dr, gpu_mcfg(sp, cfg))
    ref, _ = oracle.match_masda(kl, dl, kr, dr, cfg)
    assert same_bits(got, ref)
    if want is not None:
        assert len(got) == want
    assert st["left"] == len(kl) and st["right"] == len(kr)


def test_match_pair_end_to_end(sp, oracle):
    """Detect both images, describe and match entirely on the device."""
    p = c1(seed=9)
    det = O.default_det_cfg(cell=24)
    cfg = O.default_match_cfg(lambda_=-0.1, gamma=-0.1, iterations=10)
    m = sp.SparseMatcher(det=gpu_det(sp, det), cfg=gpu_mcfg(sp, cfg), census=(4, 3))
    L = torch.from_numpy(p.left).cuda()
    R = torch.from_numpy(p.right).cuda()
    res = m.to_host(m.match_pair(L, R))
    kl, dl, kr, dr = described(oracle, p, det, 4, 3)
    assert same_bits(res["kl"], kl) and same_bits(res["kr"], kr)
    assert np.array_equal(res["dl"], dl) and np.array_equal(res["dr"], dr)
    want, _ = oracle.match_masda(kl, dl, kr, dr, cfg)
    assert same_bits(res["matches"], want)
    good = np.abs(res["matches"]["dy"]) < 1.0
    assert good.mean() > 0.9


def test_bad_arguments(sp):
    from doubleeye_b200._lib import DeError
    with pytest.raises(DeError):
        sp.detect_fast(np.zeros((8, 8), np.uint8))                # below 16x16
    with pytest.raises(DeError):
        sp.detect_fast(np.zeros((64, 64), np.uint8), sp.DetCfg(cell=256))
    kp = np.zeros((16385, 4), np.float32)
    with pytest.raises(DeError):
        sp.match_masda(kp[:2], np.zeros(2, np.uint64), kp, np.zeros(16385, np.uint64))
    with pytest.raises(DeError):
        sp.census_at(np.zeros((32, 32), np.uint8), kp[:4], 5, 5)  # 11x11 > 64 bits


def reference_readout(kp, disp, margin):
    """core/tools/de_dense_cuda.cu:883-891 on NumPy arrays."""
    H, W = disp.shape
    rows = []
    for x, y, _, _ in kp:
        xi = min(max(int(np.float32(x) + np.float32(0.5)), 0), W - 1)
        yi = min(max(int(np.float32(y) + np.float32(0.5)), 0), H - 1)
        d = disp[yi, xi]
        if not d > 0:
            continue
        rows.append((x, y, d, margin[yi, xi]))
    return np.array(rows, np.float32).reshape(-1, 4)


def test_keypoint_readout_from_dense_map(sp, oracle):
    from oracle import oracle as O
    p = c1(424, 240, seed=12)
    d, m, _ = oracle.dense(O.default_cfg(dmax=64, iters=4), p.left, p.right, want_cand=False)
    kp = oracle.detect_fast(p.left, O.default_det_cfg())
    got, detected = sp.dense_keypoints(p.left, d, m)
    want = reference_readout(kp, d, m)
    assert detected == len(kp) and len(want) > 0.5 * len(kp)
    assert got.view(np.float32).reshape(-1, 4).tobytes() == want.tobytes()
    got0, _ = sp.dense_keypoints(p.left, d)                     # no margin plane: zeros
    assert (got0["margin"] == 0).all() and len(got0) == len(got)
