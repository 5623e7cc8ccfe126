"""Pin the oracle to the reference: every oracle function against the golden vectors
the reference itself produced (tests/golden/make_golden.py), plus the reference's own
known-answer tests (core/tests/test_confidence.cpp:52-60,
core/tests/test_top2_merge.cpp).  CPU only."""
import ast
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle.oracle import DeCfg
from parity import candidates_from_cand6, same_f32, tie_aware_disp


def load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, name + ".npz")))


def cfg_from(z) -> DeCfg:
    d = ast.literal_eval(str(z["cfg"][0]))
    return DeCfg(**d)


def test_census_coeffs_filter(oracle, golden_dir):
    z = load(golden_dir, "primitives")
    img = z["img"]
    assert (oracle.census(img, 3, 3) == z["census_7x7"]).all()
    assert (oracle.census(img, 4, 3) == z["census_9x7"]).all()
    assert (oracle.census(img, 2, 2) == z["census_5x5"]).all()
    ax, ay = oracle.rf_coeffs(img)
    assert (ax == z["ax"]).all() and (ay == z["ay"]).all()
    ax2, ay2 = oracle.rf_coeffs(img, 12.0, 0.3)
    assert (ax2 == z["ax_12_03"]).all() and (ay2 == z["ay_12_03"]).all()
    assert (oracle.filter_i16(z["plane"], ax, ay) == z["filtered"]).all()


def test_census_9x7_is_62_bits(oracle):
    """core/tests/test_preproc.cpp:50-66: a 9x7 window gives 62 bits."""
    img = np.zeros((9, 11), np.uint8)
    img[4, 5] = 255                       # bright centre: every neighbour is darker
    c = oracle.census(img, 4, 3)[4, 5]
    assert int(c) == (1 << 62) - 1


def test_census_monotonic_invariance(oracle):
    """core/tests/test_preproc.cpp:68-93: census ignores a monotonic gain+offset."""
    rng = np.random.default_rng(7)
    img = rng.integers(0, 120, (40, 50)).astype(np.uint8)
    img2 = (img.astype(np.int32) * 2 + 10).astype(np.uint8)
    assert (oracle.census(img) == oracle.census(img2)).all()


DENSE = sorted(os.path.basename(p)[:-4] for p in glob.glob(
    os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
    if os.path.basename(p).startswith(("dense_", "real_")))


@pytest.mark.parametrize("name", DENSE)
def test_dense_end_to_end(oracle, golden_dir, name):
    """Candidate planes bit-exact; disparity bit-exact except exact-tie claims."""
    z = load(golden_dir, name)
    cfg = cfg_from(z)
    disp, margin, cand = oracle.dense(cfg, z["L"], z["R"])
    for p in range(5):
        assert same_f32(cand[p], z["cand"][p]).all(), f"cand plane {p}"
    assert same_f32(margin, z["margin"]).all()
    cs, cd, cn, cnb = oracle.cost_top2(cfg, z["L"], z["R"])
    rcs, rcd, rcn = candidates_from_cand6(z["cand"], cfg.dmin)
    assert (cn == rcn).all()
    m = np.arange(2)[None, None, :] < cn[..., None]
    assert (cs[m] == rcs[m]).all() and (cd[m] == rcd[m]).all()
    nbad, n = tie_aware_disp(oracle, cfg, cs, cd, cn, cnb if cfg.subpixel else None,
                             disp, z["disp"])
    assert nbad <= max(2, n // 500)
    # lrc2 follows disp: equal wherever disp is
    eq = same_f32(disp, z["disp"])
    assert same_f32(cand[5][eq], z["cand"][5][eq]).all()


def test_confidence_known_answers(oracle):
    """The fitted values printed by article/confidence.py, as pinned by
    core/tests/test_confidence.cpp:52-60 (tolerance 1e-5)."""
    lam = -0.1
    for s1, s2, want in [(0.9, 0.3, 1.000000), (0.5, 0.49, 0.700536),
                         (0.682, 0.537, 0.975261), (0.2, -0.5, 0.961586),
                         (0.3, -1e30, 0.986346)]:
        assert abs(oracle.confidence(s1, s2, lam) - want) <= 1e-5
    assert oracle.confidence(-1e30, -1e30, lam) == 0.0
    assert oracle.confidence(0.9, 0.3, lam, 2.0, 1.0) <= 0.35 + 1e-7


def test_confidence_grid(oracle, golden_dir):
    z = load(golden_dir, "confidence")
    for i, a in enumerate(z["s1"]):
        for j, b in enumerate(z["s2"]):
            assert oracle.confidence(a, b, -0.1) == z["conf"][i, j]
            assert oracle.confidence(a, b, -0.1, 2.0, 1.0) == z["conf_capped"][i, j]
            assert oracle.confidence_u8(a, b, -0.1) == z["conf_u8"][i, j]


def _pack(v, k):
    return ((int(v) + 32768) << 8) | (255 - k)


def test_packed_top2_semantics():
    """core/tests/test_top2_merge.cpp: the packed (value+32768)<<8 | (255-k) key makes
    a shfl_down tree merge reproduce the sequential ascending-k strictly-greater scan,
    including exact ties (seeded, tie-saturated and spread values)."""
    rng = np.random.default_rng(20260809)

    def merge(m, o):
        if o[0] > m[0]:
            return (o[0], m[0] if m[0] > o[1] else o[1])
        if o[0] > m[1]:
            return (m[0], o[0])
        return m

    for spread in (3, 12, 30000):
        for _ in range(300):
            D = int(rng.integers(2, 257))
            v = rng.integers(0, spread, D)
            kmax = int(rng.integers(-1, D))
            b0 = b1 = -32768
            i0 = i1 = -1
            for k in range(kmax + 1):
                if v[k] <= b1:
                    continue
                if v[k] > b0:
                    b1, i1, b0, i0 = b0, i0, int(v[k]), k
                else:
                    b1, i1 = int(v[k]), k
            G = (D + 63) // 64
            lanes = []
            for lane in range(32):
                p = (0, 0)
                for g in range(G):
                    for j in range(2):
                        k = g * 64 + lane * 2 + j
                        if k > kmax or k >= D:
                            continue
                        c = _pack(v[k], k)
                        p = (c, p[0]) if c > p[0] else ((p[0], c) if c > p[1] else p)
                lanes.append(p)
            off = 16
            while off:
                lanes = [merge(lanes[l], lanes[l + off] if l + off < 32 else lanes[l])
                         for l in range(32)]
                off //= 2
            r = lanes[0]
            rb0 = (r[0] >> 8) - 32768 if r[0] else -32768
            ri0 = 255 - (r[0] & 255) if r[0] else -1
            rb1 = (r[1] >> 8) - 32768 if r[1] else -32768
            ri1 = 255 - (r[1] & 255) if r[1] else -1
            assert (rb0, ri0, rb1, ri1) == (b0, i0, b1, i1)


def test_fill_prior_matches_reference_fill(golden_dir):
    """The prior hole fill against the reference's own fill
    (article/coarse_to_fine.py:58-76), bit for bit."""
    z = np.load(os.path.join(golden_dir, "fill.npz"))
    names = sorted({k[:-3] for k in z.files if k.endswith("_in")})
    assert len(names) >= 6
    for n in names:
        got = O.fill_prior(z[n + "_in"])
        assert got.tobytes() == z[n + "_out"].tobytes(), n
