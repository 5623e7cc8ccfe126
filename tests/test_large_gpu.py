"""The large configuration at full size: 1500x1000, disparities 0-255 (D=256), 12 BP
iterations, thin foreground strips and low-texture regions (synth.large_scene).  The
768 MB filtered volume and every stage at this size against the oracle, bit for bit,
through the host API and the device API."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def de():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import doubleeye_b200 as de
    from doubleeye_b200 import build
    build.build()
    return de


def test_large_config_bit_exact(de, oracle):
    from oracle import oracle as O
    from doubleeye_b200 import synth
    p = synth.large_scene()
    cfg = dict(dmax=256, iters=12)
    od, om, oc = oracle.dense(O.default_cfg(**cfg), p.left, p.right)
    r = de.run_dense(p.left, p.right, de.Cfg(**cfg), want_cand=True)
    assert r.disp.tobytes() == od.tobytes()
    assert r.margin.tobytes() == om.tobytes()
    assert r.cand.tobytes() == oc.tobytes()
    assert np.isfinite(r.disp).mean() > 0.6
    # two at once through the device API (the batch holds 2 x 768 MB of volume)
    m = de.DenseMatcher(de.Cfg(**cfg))
    L = torch.from_numpy(p.left).cuda()
    R = torch.from_numpy(p.right).cuda()
    outs = m.match_batch([(L, R), (R.flip(1).contiguous(), L.flip(1).contiguous())])
    torch.cuda.synchronize()
    assert outs[0]["disp"].cpu().numpy().tobytes() == od.tobytes()
