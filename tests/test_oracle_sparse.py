"""The sparse-path oracle against golden vectors made by the reference itself.

Fixtures (tests/golden/make_golden_sparse.py): detect_keypoints_fast, census_at and
match_masda of the reference compiled from its sources, on two synthetic C1-style
crops (7x7 and 9x7 descriptors) and a crop of a real camera pair; 60 small random
problems with the reference's exact brute-force optimum (core/tests/test_match.cpp:
115-168 shape); and the reference's Python masda / masda_sparse / dense_problem /
_seg_max_excluding / hamming (article/masda_stereo.py, article/dense_masda.py).

The reference orders exact ties with std::sort / NumPy argsort, whose tie order is
unspecified; the oracle breaks them by input position.  Match lists are therefore
compared tie-aware: same length, same (left, score, belief, margin) multiset, and a
different right point only where those are equal.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.filterwarnings("ignore::RuntimeWarning")

CASES = ["sparse_c1", "sparse_c1_9x7", "sparse_real"]


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, f"{name}.npz"))


def det_cfg(arr):
    c = O.DeDetCfg()
    for (f, t), v in zip(c._fields_, arr):
        setattr(c, f, int(v) if t is C.c_int else float(v))
    return c


def match_cfg(arr):
    c = O.DeMatchCfg()
    for (f, t), v in zip(c._fields_, arr):
        setattr(c, f, int(v) if t is C.c_int else float(v))
    return c


def same_bits(a, b):
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def tie_aware_same(got, ref, max_flip_frac=0.01):
    """Match lists equal up to choices between exactly tied alternatives."""
    if same_bits(got, ref):
        return True
    if len(got) != len(ref):
        return False
    key = lambda m: np.sort(np.array(  # noqa: E731
        [(r["left"], r["score"], r["belief"], r["margin"]) for r in m],
        dtype=[("l", "i4"), ("s", "f4"), ("b", "f4"), ("g", "f4")]), order=["l", "s", "b"])
    if key(got).tobytes() != key(ref).tobytes():
        return False
    by_left = {int(r["left"]): int(r["right"]) for r in ref}
    flips = sum(by_left[int(r["left"])] != int(r["right"]) for r in got)
    return flips <= max(1, int(max_flip_frac * len(ref)))


@pytest.mark.parametrize("name", CASES)
def test_detector_matches_reference(oracle, golden_dir, name):
    g = load(golden_dir, name)
    det = det_cfg(g["det"])
    assert same_bits(oracle.detect_fast(g["L"], det), g["kl"])
    assert same_bits(oracle.detect_fast(g["R"], det), g["kr"])
    assert len(g["kl"]) > 20


@pytest.mark.parametrize("name", CASES)
def test_census_at_matches_reference(oracle, golden_dir, name):
    g = load(golden_dir, name)
    hw, hh = (int(v) for v in g["census"])
    for img, kp, d in ((g["L"], g["kl"], g["dl"]), (g["R"], g["kr"], g["dr"])):
        got = np.array([oracle.census_at(img, int(x + 0.5), int(y + 0.5), hw, hh)[0]
                        for x, y in kp[:, :2]], np.uint64)
        assert np.array_equal(got, d)


def test_census_at_border_and_window(oracle):
    rng = np.random.default_rng(7)
    img = rng.integers(0, 256, (20, 30)).astype(np.uint8)
    assert oracle.census_at(img, 2, 10, 3, 3) == (0, False)       # window leaves image
    assert oracle.census_at(img, 27, 10, 3, 3) == (0, False)
    v, ok = oracle.census_at(img, 3, 3, 3, 3)
    assert ok and v == int(oracle.census(img, 3, 3)[3, 3])
    v, ok = oracle.census_at(img, 10, 10, 4, 3)                   # 9x7: 62 bits
    assert ok and v == int(oracle.census(img, 4, 3)[10, 10]) and v < (1 << 62)


@pytest.mark.parametrize("name", CASES)
def test_match_matches_reference(oracle, golden_dir, name):
    g = load(golden_dir, name)
    cfgs = g["match_cfgs"]
    for k in range(len(cfgs)):
        cfg = match_cfg(cfgs[k])
        got, st = oracle.match_masda(g["kl"], g["dl"], g["kr"], g["dr"], cfg)
        assert tie_aware_same(got, g[f"matches_{k}"]), (name, k)
        ref_st = g[f"stats_{k}"]
        assert [st.left, st.right, st.candidates, st.iterations_run, st.converged,
                st.oscillating] == [int(v) for v in ref_st[[0, 1, 2, 3, 4, 6]]]
        assert np.float32(st.final_max_delta) == np.float32(ref_st[5])


def objective(matches, lam, gam, n, m):
    return (np.float32(matches["score"].sum(dtype=np.float32)) +
            np.float32(lam) * np.float32(n - len(matches)) +
            np.float32(gam) * np.float32(m - len(matches)))


def test_bruteforce_optimality_and_reference(oracle, golden_dir):
    """core/tests/test_match.cpp:115-168: valid one-to-one matchings, the exact
    optimum on >= 90% of 60 random problems, total objective within 2%."""
    g = load(golden_dir, "sparse_bruteforce")
    cfg = match_cfg(g["cfg"][0])
    optimal = 0
    sm = sb = 0.0
    for t in range(len(g["off_l"]) - 1):
        kl = g["kl"][g["off_l"][t]:g["off_l"][t + 1]]
        kr = g["kr"][g["off_r"][t]:g["off_r"][t + 1]]
        dl = g["dl"][g["off_l"][t]:g["off_l"][t + 1]]
        dr = g["dr"][g["off_r"][t]:g["off_r"][t + 1]]
        ref = g["masda"][g["off_m"][t]:g["off_m"][t + 1]]
        bf = g["brute"][g["off_b"][t]:g["off_b"][t + 1]]
        got, _ = oracle.match_masda(kl, dl, kr, dr, cfg)
        assert tie_aware_same(got, ref, max_flip_frac=1.0), t
        assert len(set(got["left"])) == len(got) and len(set(got["right"])) == len(got)
        va = objective(got, cfg.lambda_, cfg.gamma, len(kl), len(kr))
        vb = objective(bf, cfg.lambda_, cfg.gamma, len(kl), len(kr))
        optimal += va >= vb - 1e-4
        sm += va
        sb += vb
    assert optimal >= 54
    assert sm / sb > 0.98


def kp(x, y):
    return [x, y, 10.0, 10.0]


def desc_with(nbits, off=0):
    d = 0
    for b in range(nbits):
        d |= 1 << ((b + off) % 48)
    return d


def plain(**kw):
    base = dict(max_dy=2.0, min_disparity=1.0, max_disparity=100.0, w_y=0.0, iterations=60,
                damping=0.4, lambda_=0.0, gamma=0.0)
    base.update(kw)
    return O.default_match_cfg(**base)


def known_answer_cases():
    """The unit cases of core/tests/test_match.cpp:61-113,170-211,347-420, as
    (name, kl, dl, kr, dr, cfg, expected match count)."""
    d20 = desc_with(20)
    cases = [
        ("single", [kp(100, 50)], [d20], [kp(80, 50)], [d20], plain(), 1),
        ("dy_gate", [kp(100, 50)], [d20], [kp(80, 60)], [d20], plain(), 0),
        ("negative_disparity", [kp(100, 50)], [d20], [kp(120, 50)], [d20], plain(), 0),
        ("too_far", [kp(100, 50)], [d20], [kp(-50, 50)], [d20], plain(), 0),
        ("y_penalty", [kp(100, 50)], [d20], [kp(80, 51.5)], [d20],
         plain(w_y=1.0, sigma_y=0.5), 0),
        ("exclusivity", [kp(100, 50), kp(101, 50)], [d20, d20], [kp(80, 50)], [d20],
         plain(), 1),
        ("empty_left", [], [], [kp(80, 50)], [d20], plain(), 0),
        ("empty_right", [kp(100, 50)], [d20], [], [], plain(), 0),
        ("empty_both", [], [], [], [], plain(), 0),
    ]
    L = [kp(100 + 10 * i, 50) for i in range(6)]
    R = [kp(80 + 10 * i, 50) for i in range(6)]
    cases.append(("degenerate", L, [d20] * 6, R, [d20] * 6, plain(), None))
    return cases


@pytest.mark.parametrize("case", known_answer_cases(), ids=lambda c: c[0])
def test_known_answers(oracle, case):
    name, kl, dl, kr, dr, cfg, want = case
    kl = np.array(kl, np.float32).reshape(-1, 4)
    kr = np.array(kr, np.float32).reshape(-1, 4)
    got, st = oracle.match_masda(kl, np.array(dl, np.uint64), kr, np.array(dr, np.uint64),
                                 cfg)
    if want is not None:
        assert len(got) == want
    assert len(set(got["left"])) == len(got) and len(set(got["right"])) == len(got)
    if name == "single":
        assert got[0]["left"] == 0 and got[0]["right"] == 0
        assert abs(got[0]["disparity"] - 20.0) < 1e-4 and abs(got[0]["dy"]) < 1e-6
    if name == "degenerate":
        assert len(got) > 0


def test_python_masda_matches_reference(oracle, golden_dir):
    """masda / masda_sparse of article/masda_stereo.py on a keypoint problem: the
    convergence history bit for bit, the assignment exactly."""
    g = load(golden_dir, "py_masda")
    S = g["kp_S"]
    m, n = S.shape
    ei, ej = np.nonzero(np.isfinite(S))
    a, h = oracle.masda_edges(ei, ej, S[ei, ej].astype(np.float64), m, n, -0.1, -0.1, 30,
                              0.4, 1e-5)
    assert np.array_equal(h, g["kp_sparse_hist"]) and np.array_equal(h, g["kp_masda_hist"])
    assert np.array_equal(a, g["kp_sparse"]) and np.array_equal(a, g["kp_masda"])


def test_python_dense_problem_masda_matches_reference(oracle, golden_dir):
    """masda_sparse on dense_problem's edge list (49 distinct scores, so beliefs tie
    often): history bit for bit; assignments agree except at argsort ties."""
    g = load(golden_dir, "py_masda")
    nn = g["dp_L"].size
    a, h = oracle.masda_edges(g["dp_ei"], g["dp_ej"], g["dp_se"].astype(np.float64), nn, nn,
                              -0.1, -0.1, 6, 0.4, 1e-5)
    assert np.array_equal(h, g["dp_hist"])
    ref = g["dp_assign"]
    matched = (ref >= 0) | (a >= 0)
    assert (a[matched] == ref[matched]).mean() >= 0.995
    assert len(np.unique(a[a >= 0])) == (a >= 0).sum()
