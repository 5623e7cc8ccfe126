"""The Python entry points (doubleeye_b200.masda_stereo / dense_masda) on the GPU,
against the reference's own NumPy outputs (tests/golden/py_masda.npz, made by
importing article/masda_stereo.py and article/dense_masda.py) and the oracle.

Float64 like NumPy: histories, scores, edge lists and segment maxima are compared
bit for bit; assignments exactly where beliefs do not tie, and tie-aware on
dense_problem, whose 49 distinct scores make exact belief ties common (NumPy's
argsort order among them is unspecified; both this path and the oracle give ties to
the lower edge index)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ms():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from doubleeye_b200 import build, masda_stereo
    build.build()
    return masda_stereo


@pytest.fixture(scope="module")
def g(golden_dir):
    return np.load(os.path.join(golden_dir, "py_masda.npz"))


def as_arr(d, m):
    return np.array([d.get(i, -1) for i in range(m)], np.int64)


def test_hamming_and_census(ms, g):
    from doubleeye_b200 import synth
    assert np.array_equal(ms.hamming(g["ham_a"], g["ham_b"]), g["ham"])
    p = synth.fronto_planes(256, 160, seed=31, planes=(8, 24, 40))
    assert np.array_equal(ms.census(p.left, g["kp_pl"]), g["kp_dl"])
    assert np.array_equal(ms.census(p.right, g["kp_pr"]), g["kp_dr"])


def test_build_problem_bit_exact(ms, g):
    S = ms.build_problem(g["kp_pl"], g["kp_dl"], g["kp_pr"], g["kp_dr"], max_dy=1.5,
                         dmin=1.0, dmax=60.0)
    assert S.dtype == np.float32 and S.tobytes() == g["kp_S"].tobytes()


def test_seg_max_excluding_bit_exact(ms, g):
    out = ms._seg_max_excluding(g["seg_vals"], g["seg_idx"], 37)
    assert out.tobytes() == g["seg_out"].tobytes()


def test_to_edges_and_masda(ms, g):
    S = g["kp_S"]
    ei, ej, se = ms.to_edges(S)
    ri, rj = np.nonzero(np.isfinite(S))
    assert np.array_equal(ei, ri) and np.array_equal(ej, rj)
    assert se.tobytes() == S[ri, rj].astype(np.float64).tobytes()
    m, n = S.shape
    a, h = ms.masda(S, lam=-0.1, gam=-0.1, iters=30, damping=0.4, eps=1e-5)
    assert h.tobytes() == g["kp_masda_hist"].tobytes()
    assert np.array_equal(as_arr(a, m), g["kp_masda"])
    a2, h2 = ms.masda_sparse(ei, ej, se, m, n, -0.1, -0.1, iters=30, damping=0.4, eps=1e-5)
    assert h2.tobytes() == g["kp_sparse_hist"].tobytes()
    assert np.array_equal(as_arr(a2, m), g["kp_sparse"])


def test_dense_problem_bit_exact(ms, g):
    from doubleeye_b200 import dense_masda as dm
    ei, ej, se, nn = dm.dense_problem(g["dp_L"], g["dp_R"], 1, 12)
    assert nn == g["dp_L"].size
    assert np.array_equal(ei, g["dp_ei"]) and np.array_equal(ej, g["dp_ej"])
    assert se.dtype == np.float32 and se.tobytes() == g["dp_se"].tobytes()


def test_dense_problem_masda_reference_and_oracle(ms, g, oracle):
    nn = g["dp_L"].size
    a, h = ms.masda_sparse(g["dp_ei"], g["dp_ej"], g["dp_se"], nn, nn, -0.1, -0.1, iters=6)
    assert h.tobytes() == g["dp_hist"].tobytes()
    got = as_arr(a, nn)
    want, wh = oracle.masda_edges(g["dp_ei"], g["dp_ej"], g["dp_se"].astype(np.float64), nn,
                                  nn, -0.1, -0.1, 6, 0.4, 1e-5)
    assert np.array_equal(got, want) and np.array_equal(h, wh)
    ref = g["dp_assign"]
    matched = (ref >= 0) | (got >= 0)
    assert (got[matched] == ref[matched]).mean() >= 0.995


@pytest.mark.parametrize("W,H,dmax,iters", [(160, 96, 24, 8), (97, 41, 40, 12)])
def test_dense_problem_masda_vs_oracle(ms, oracle, W, H, dmax, iters):
    from doubleeye_b200 import dense_masda as dm, synth
    p = synth.slanted_planes(W, H, dmax - 1, seed=W + H, tag="py-dense")
    ei, ej, se, nn = dm.dense_problem(p.left, p.right, 1, dmax)
    a, h = ms.masda_sparse(ei, ej, se, nn, nn, -0.1, -0.1, iters=iters)
    want, wh = oracle.masda_edges(ei, ej, se.astype(np.float64), nn, nn, -0.1, -0.1, iters,
                                  0.4, 1e-5)
    assert np.array_equal(h, wh)
    assert np.array_equal(as_arr(a, nn), want)
    assert len(a) > 0.5 * (H - 6) * (W - 6)


def test_decide_with_ties(ms):
    rng = np.random.default_rng(5)
    S = rng.integers(-2, 5, (40, 50)).astype(np.float64) / 4
    S[rng.random(S.shape) < 0.5] = -np.inf
    belief = np.where(np.isfinite(S), rng.integers(-3, 3, S.shape) / 2.0, -np.inf)
    got = ms.decide(S, belief, -0.1)
    # the reference rule with a stable argsort
    order = np.argsort(-belief, axis=None, kind="stable")
    used_i, used_j, want = set(), set(), {}
    for flat in order:
        i, j = divmod(int(flat), S.shape[1])
        if not np.isfinite(belief[i, j]):
            break
        if S[i, j] <= -0.1 or i in used_i or j in used_j:
            continue
        want[i] = j
        used_i.add(i)
        used_j.add(j)
    assert got == want


def test_empty_and_degenerate(ms):
    a, h = ms.masda(np.full((3, 4), -np.inf, np.float32))
    assert a == {} and list(h) == [0.0]
    with pytest.raises(ValueError):
        ms.masda_sparse(np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0), 3, 3)
    a, h = ms.masda_sparse([0, 1], [0, 0], [0.5, 0.5], 2, 1, iters=5)
    assert len(a) == 1 and list(a.values()) == [0]


def test_out_of_range_edges_are_refused(ms):
    from doubleeye_b200._lib import DeError
    with pytest.raises(DeError):
        ms.masda_sparse([0, 1], [0, 5], [0.5, 0.5], 2, 2, iters=3)
    with pytest.raises(DeError):
        ms._seg_max_excluding([1.0, 2.0], [0, 9], 3)
