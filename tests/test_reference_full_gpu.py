"""Full-size parity against the reference itself, and the largest batched shape.

The reference's own run_dense (core/tools/de_dense.cpp:738, compiled from its sources
into oracle/_ref/libref.so, one thread: its deterministic form) is run beside the
CUDA path on
  * the synthetic slanted-plane pair of the benchmark at 848x480, D=128, 8 BP
    iterations;
  * the six real 848x480 IR pairs of the reference's article/scenes (one room at three
    light levels, projector on and off; tests/golden/scenes.npz, copied by
    tests/golden/make_scenes.py), at D=64 and D=128, 8 iterations.
The candidate planes (s1, s2, d1, d2) and the margin must be bit-equal; the disparity
must be bit-equal except where the reference's std::sort and this build's index
tie-break order exactly tied claimants differently (tests/parity.py).  Disparity
agreement counts a pixel as agreeing when its disparity is bit-equal or differs only
by such an exact-tie claim order; it must be at least 99.9%, and the bit-equal
fraction alone at least 99.8% (the reference's own std::sort and std::stable_sort
differ on about 0.1% of pixels of these scenes).  Each case prints both as one JSON
line (run with -s to see them).

The largest shape of the uneven batch, 1920x1080 at D=256, is compared with the
oracle bit for bit.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from parity import candidates_from_cand6, same_f32, tie_aware_disp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SCENES = ["evening_off", "evening_on", "morning_off", "morning_on", "night_off", "night_on"]


@pytest.fixture(scope="module")
def de():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import doubleeye_b200 as de
    from doubleeye_b200 import build
    build.build()
    return de


@pytest.fixture(scope="module")
def ref():
    if not O.Reference.available():
        pytest.skip("oracle/_ref/libref.so (the reference compiled from its sources) "
                    "was not built in this tree")
    return O.Reference()


@pytest.fixture(scope="module")
def scenes(golden_dir):
    return dict(np.load(os.path.join(golden_dir, "scenes.npz")))


def _against_reference(de, ref, oracle, name, L, R, dmax, iters):
    ocfg = O.default_cfg(dmax=dmax, iters=iters)
    cfg = de.Cfg(dmax=dmax, iters=iters)
    r = de.run_dense(L, R, cfg, want_cand=True)
    rd, rm, rc, _ = ref.dense(ocfg, L, R, nthreads=1, want_cand=True)
    for i in range(4):
        assert same_f32(r.cand[i], rc[i]).all(), f"{name}: candidate plane {i}"
    assert same_f32(r.margin, rm).all(), f"{name}: margin"
    cs, cd, cn = candidates_from_cand6(rc, ocfg.dmin)
    # raises on any difference that is not an exact-tie claim order
    nties, npx = tie_aware_disp(oracle, ocfg, cs, cd, cn, None, r.disp, rd)
    agree = 1.0                                   # every difference is an exact tie
    bit_equal = 1.0 - nties / npx
    print(json.dumps({"case": name, "D": dmax, "iters": iters, "pixels": npx,
                      "tie_order_differences": nties, "disparity_agreement": agree,
                      "bit_equal": bit_equal, "filled": float(np.isfinite(r.disp).mean())}))
    assert agree >= 0.999 and bit_equal >= 0.998
    return bit_equal


def test_benchmark_pair_848x480_d128_vs_reference(de, ref, oracle):
    from doubleeye_b200 import synth
    p = synth.slanted_planes(848, 480, 127, seed=0, tag="bench")
    _against_reference(de, ref, oracle, "C2 slanted planes", p.left, p.right, 128, 8)


@pytest.mark.parametrize("dmax", [64, 128])
@pytest.mark.parametrize("scene", SCENES)
def test_real_scene_vs_reference(de, ref, oracle, scenes, scene, dmax):
    _against_reference(de, ref, oracle, scene, scenes[scene + "_L"], scenes[scene + "_R"],
                       dmax, 8)


def test_1920x1080_d256_bit_exact(de, oracle):
    """The largest pair of the uneven batch, against the oracle bit for bit."""
    from doubleeye_b200 import synth
    p = synth.slanted_planes(1920, 1080, 255, tag="c4:1920x1080")
    ocfg = O.default_cfg(dmax=256, iters=8)
    od, om, oc = oracle.dense(ocfg, p.left, p.right)
    r = de.run_dense(p.left, p.right, de.Cfg(dmax=256, iters=8), want_cand=True)
    assert same_f32(r.disp, od).all()
    assert same_f32(r.margin, om).all()
    for i in range(6):
        assert same_f32(r.cand[i], oc[i]).all(), f"plane {i}"
    assert np.isfinite(r.disp).mean() > 0.5
