"""Parity of the CUDA dense path with the oracle (and, through the golden fixtures,
with the reference itself).  Every call goes through the C ABI.

Integer stages (census, coefficient planes, filtered top-2 candidates and the
winner's neighbour costs) are compared bit for bit.  The row solve is compared bit
for bit too: it uses the same tie rule as the oracle (belief, then x), and its float
arithmetic is uncontracted single precision like the reference's.  Against the
reference's own outputs the disparity is compared tie-aware (tests/parity.py).
The u8 confidence uses CUDA's logf/expf against glibc's: it may differ by 1 level."""
import ast
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from doubleeye_b200 import build
    build.build()


import doubleeye_b200 as de  # noqa: E402
from doubleeye_b200 import synth  # noqa: E402
from oracle.oracle import DeCfg, default_cfg  # noqa: E402
from parity import candidates_from_cand6, same_f32, tie_aware_disp  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def both(**kw):
    return de.Cfg(**kw), default_cfg(**kw)


def rand_pair(W, H, seed, shift=7):
    rng = np.random.default_rng(seed)
    L = rng.integers(0, 256, (H, W)).astype(np.uint8)
    R = np.roll(L, -shift, axis=1)
    R = np.clip(R.astype(int) + rng.integers(-4, 5, R.shape), 0, 255).astype(np.uint8)
    return L, R


@pytest.mark.parametrize("W,H,hw,hh", [(61, 37, 3, 3), (8, 8, 3, 3), (97, 41, 4, 3),
                                       (130, 70, 2, 2), (848, 480, 3, 3), (33, 9, 1, 1)])
def test_census_and_coefficients(oracle, W, H, hw, hh):
    L, R = rand_pair(W, H, W * H)
    L[2:5, 3:9] = 40                              # flat patch: equal compares
    cfg, ocfg = both(census_hw=hw, census_hh=hh, sigma_s=7.0, sigma_r=0.25)
    cl, cr, ax, ay = de.census(dev(L), dev(R), cfg)
    torch.cuda.synchronize()
    assert (cl.cpu().numpy().view(np.uint64) == oracle.census(L, hw, hh)).all()
    assert (cr.cpu().numpy().view(np.uint64) == oracle.census(R, hw, hh)).all()
    oax, oay = oracle.rf_coeffs(L, 7.0, 0.25)
    assert (ax.cpu().numpy().view(np.uint16) == oax).all()
    assert (ay.cpu().numpy().view(np.uint16) == oay).all()


COST_CASES = [
    # (W, H, cfg)
    (97, 41, dict(dmax=16)),
    (128, 64, dict(dmax=64)),
    (200, 50, dict(dmin=3, dmax=130)),                 # D=128, dmin != 1
    (160, 48, dict(dmax=192)),                         # D=192: three k groups
    (300, 40, dict(dmax=256)),                         # D=256, the packing limit
    (90, 30, dict(dmax=33, ad=0.0)),                   # census only
    (120, 36, dict(dmax=40, ad_trunc=40, ad=0.5)),     # wide AD table
    (110, 40, dict(dmax=24, census_hw=4, census_hh=3)),  # 9x7 census, unpacked words
    (64, 20, dict(dmax=70)),                           # D beyond the usable width
    (40, 12, dict(dmax=5, subpixel=0)),
]


@pytest.mark.parametrize("W,H,kw", COST_CASES)
def test_cost_top2_bit_exact(oracle, W, H, kw):
    p = synth.slanted_planes(W, H, min(kw["dmax"], 3 * W // 4), tag=f"cost{W}x{H}")
    cfg, ocfg = both(**kw)
    cs, cd, cn, cnb = (t.cpu().numpy() for t in de.cost_top2(dev(p.left), dev(p.right), cfg))
    ocs, ocd, ocn, ocnb = oracle.cost_top2(ocfg, p.left, p.right)
    assert (cn == ocn).all()
    m = np.arange(2)[None, None, :] < cn[..., None]
    assert (cs[m] == ocs[m]).all()
    assert (cd[m] == ocd[m]).all()
    if ocfg.subpixel:
        win = (cn > 0)[..., None].repeat(2, -1)
        assert (cnb[win] == ocnb[win]).all()


@pytest.mark.parametrize("iters,kw", [(0, {}), (8, {}), (3, dict(fit_eq=0)),
                                      (5, dict(min_margin=0.02)),
                                      (4, dict(min_ratio=1.05, damping=0.0)),
                                      (2, dict(lambda_=0.05, gamma=-0.3, subpixel=0))])
def test_solve_bit_exact(oracle, iters, kw):
    p = synth.slanted_planes(180, 60, 60, tag="solve")
    cfg, ocfg = both(dmax=64, iters=iters, **kw)
    ocs, ocd, ocn, ocnb = oracle.cost_top2(ocfg, p.left, p.right)
    disp, margin, lrc2 = (t.cpu().numpy() for t in de.solve(
        dev(ocs), dev(ocd), dev(ocn), dev(ocnb) if ocfg.subpixel else None, cfg))
    odisp, omargin, olrc2 = oracle.solve(ocfg, ocs, ocd, ocn, ocnb if ocfg.subpixel else None)
    assert same_f32(margin, omargin).all()
    assert same_f32(disp, odisp).all()
    assert same_f32(lrc2, olrc2).all()


FULL_CASES = [
    (97, 41, dict(dmax=16)),
    (128, 64, dict(dmax=32, iters=8)),
    (120, 40, dict(dmax=20, iters=2, lrc=1)),
    (250, 80, dict(dmax=100, iters=8, lrc=1)),
    (64, 64, dict(dmax=64, iters=8, damping=0.0, lambda_=0.05, gamma=-0.2)),
]


@pytest.mark.parametrize("W,H,kw", FULL_CASES)
def test_full_pipeline_bit_exact(oracle, W, H, kw):
    p = synth.slanted_planes(W, H, min(kw["dmax"], 3 * W // 4), tag=f"full{W}x{H}")
    cfg, ocfg = both(**kw)
    r = de.run_dense(p.left, p.right, cfg)
    od, om, oc = oracle.dense(ocfg, p.left, p.right)
    assert same_f32(r.disp, od).all()
    assert same_f32(r.margin, om).all()
    for i in range(6):
        assert same_f32(r.cand[i], oc[i]).all(), f"plane {de.CAND_PLANES[i]}"
    ref_u8 = np.array([[oracle.confidence_u8(oc[0, y, x], oc[1, y, x], ocfg.lambda_,
                                             oc[5, y, x] if np.isfinite(oc[5, y, x]) else 0.0)
                        if np.isfinite(od[y, x]) else 0 for x in range(W)] for y in range(H)])
    assert np.abs(r.conf.astype(int) - ref_u8).max() <= 1


def test_full_size_848x480_d128(oracle):
    """The benchmark configuration itself: 848x480, D=128, 8 iterations."""
    p = synth.slanted_planes(848, 480, 127)
    cfg, ocfg = both(dmax=128, iters=8)
    r = de.run_dense(p.left, p.right, cfg)
    od, om, oc = oracle.dense(ocfg, p.left, p.right)
    assert same_f32(r.disp, od).all()
    assert same_f32(r.margin, om).all()
    for i in range(6):
        assert same_f32(r.cand[i], oc[i]).all()


GOLDEN = sorted(f[:-4] for f in os.listdir(os.path.join(os.path.dirname(__file__), "golden"))
                if f.startswith(("dense_", "real_")))


@pytest.mark.parametrize("name", GOLDEN)
def test_against_reference_golden(oracle, golden_dir, name):
    z = dict(np.load(os.path.join(golden_dir, name + ".npz")))
    ocfg = DeCfg(**ast.literal_eval(str(z["cfg"][0])))
    cfg = de.Cfg(**{f: getattr(ocfg, f) for f, _ in ocfg._fields_})
    r = de.run_dense(z["L"], z["R"], cfg)
    for i in range(5):
        assert same_f32(r.cand[i], z["cand"][i]).all(), f"plane {i}"
    assert same_f32(r.margin, z["margin"]).all()
    cs, cd, cn = candidates_from_cand6(z["cand"], ocfg.dmin)
    _, _, _, cnb = oracle.cost_top2(ocfg, z["L"], z["R"])
    tie_aware_disp(oracle, ocfg, cs, cd, cn, cnb if ocfg.subpixel else None, r.disp, z["disp"])


def test_batch_mixed_shapes_equals_single(oracle):
    """One launch set over uneven pairs gives each pair's single-pair result."""
    shapes = [(96, 48, 32), (160, 64, 64), (64, 40, 16), (200, 30, 128), (96, 48, 48)]
    pairs = [synth.slanted_planes(W, H, D - 1, tag=f"mix{i}") for i, (W, H, D) in
             enumerate(shapes)]
    cfg = de.Cfg(dmax=64, iters=4)
    batch = de.run_dense_batch([(p.left, p.right, D) for p, (_, _, D) in zip(pairs, shapes)],
                               cfg, want_cand=True)
    for p, (_, _, D), b in zip(pairs, shapes, batch):
        s = de.run_dense(p.left, p.right, de.Cfg(dmax=D, iters=4))
        assert same_f32(b.disp, s.disp).all()
        assert same_f32(b.cand, s.cand).all()
        od, _, _ = oracle.dense(default_cfg(dmax=D, iters=4), p.left, p.right)
        assert same_f32(b.disp, od).all()


def test_device_api_matches_host_api():
    p = synth.slanted_planes(200, 100, 60, tag="devapi")
    cfg = de.Cfg(dmax=64, iters=8)
    m = de.DenseMatcher(cfg)
    out = m.match(dev(p.left), dev(p.right), cand=True)
    torch.cuda.synchronize()
    h = de.run_dense(p.left, p.right, cfg)
    assert same_f32(out["disp"].cpu().numpy(), h.disp).all()
    assert same_f32(out["cand"].cpu().numpy(), h.cand).all()


def test_bad_arguments_raise():
    from doubleeye_b200._lib import DeError
    L = np.zeros((4, 4), np.uint8)
    with pytest.raises(DeError):
        de.run_dense(L, L, de.Cfg())                 # below the minimum size
    big = np.zeros((16, 16), np.uint8)
    with pytest.raises(DeError):
        de.run_dense(big, big, de.Cfg(dmax=400))     # D beyond 256


def test_int_probe_rates():
    """The integer-pipe probe behind the integer roofline: every op reports a rate
    per SM clock in a physically possible range (at most 128 lanes, the two
    integer-capable pipes), with POPC on its slower pipe."""
    import ctypes as C
    import torch
    from doubleeye_b200._lib import probe_lib as lib
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    max_hz = 2.2e9                                     # above any B200 boost clock
    for op in range(5):
        ms, n = C.c_float(), C.c_double()
        assert lib().de_int_probe(op, 200, None, C.byref(ms), C.byref(n)) == 0
        assert ms.value > 0 and n.value > 0
        per_clk = n.value / (ms.value * 1e-3) / sms / max_hz
        assert 4.0 < per_clk < 160.0, (op, per_clk)
    assert lib().de_int_probe(7, 10, None, C.byref(ms), C.byref(n)) != 0


COL_SHAPES = [
    (40, 8, dict(dmax=16)),               # two valid rows (the smallest image)
    (97, 9, dict(dmax=16)),               # fewer rows than the prefetch depth
    (130, 12, dict(dmax=64)),
    (200, 50, dict(dmin=3, dmax=130)),
    (160, 21, dict(dmax=192)),            # 24 lanes of 8 padded to 32
    (300, 40, dict(dmax=256)),
    (848, 480, dict(dmax=128)),           # the benchmark shape
]
_COL_ORACLE = {}


@pytest.mark.parametrize("cta", [128, 256])
@pytest.mark.parametrize("kt,pf", [(4, 4), (4, 8), (4, 16), (8, 4), (8, 8), (16, 4)])
@pytest.mark.parametrize("W,H,kw", COL_SHAPES)
def test_column_kernel_shapes_bit_exact(oracle, W, H, kw, kt, pf, cta):
    """Every column-kernel shape (disparities per lane, prefetch depth, CTA size)
    against the oracle, including images shorter than the prefetch depth."""
    from doubleeye_b200 import _lib
    key = (W, H, tuple(sorted(kw.items())))
    p = synth.slanted_planes(W, H, min(kw["dmax"], 3 * W // 4), tag=f"cols{W}x{H}")
    cfg, ocfg = both(**kw)
    if key not in _COL_ORACLE:
        _COL_ORACLE[key] = oracle.cost_top2(ocfg, p.left, p.right)
    ocs, ocd, ocn, ocnb = _COL_ORACLE[key]
    names = ("cols_kt", "cols_pf", "cols_cta")
    saved = [_lib.get_param(n) for n in names]
    try:
        for n, v in zip(names, (kt, pf, cta)):
            _lib.set_param(n, v)
        cs, cd, cn, cnb = (t.cpu().numpy() for t in de.cost_top2(dev(p.left), dev(p.right), cfg))
    finally:
        for n, v in zip(names, saved):
            _lib.set_param(n, v)
    assert (cn == ocn).all()
    m = np.arange(2)[None, None, :] < cn[..., None]
    assert (cs[m] == ocs[m]).all()
    assert (cd[m] == ocd[m]).all()
    win = (cn > 0)[..., None].repeat(2, -1)
    assert (cnb[win] == ocnb[win]).all()
