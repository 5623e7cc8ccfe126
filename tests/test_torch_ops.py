"""torch.ops.doubleeye: the operators are registered without a GPU (with fake
implementations for shape propagation), and on the GPU each operator gives the C-ABI
(ctypes) path's results bit for bit, with outputs allocated on the input's device."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_ops_registered():
    from doubleeye_b200 import ops
    for name in ops.registered():
        ns, op = name.split("::")
        assert hasattr(getattr(torch.ops, ns), op), name


def test_fake_shapes():
    from doubleeye_b200 import ops  # noqa: F401
    from torch._subclasses.fake_tensor import FakeTensorMode
    with FakeTensorMode():
        L = torch.empty((48, 64), dtype=torch.uint8, device="meta")
        d, m, c = torch.ops.doubleeye.dense(L, L, 32, 4)
        assert d.shape == (48, 64) and d.dtype == torch.float32 and c.dtype == torch.uint8
        cs, cd, cn, cnb = torch.ops.doubleeye.cost_top2(L, L, 32)
        assert cs.shape == (48, 64, 2) and cn.shape == (48, 64) and cnb.dtype == torch.int16


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype == np.float32:
        return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())
    return bool((a == b).all())


@pytest.mark.gpu
def test_ops_match_the_ctypes_path():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import doubleeye_b200 as de
    from doubleeye_b200 import build, ops, sparse, synth  # noqa: F401
    build.build()
    p = synth.slanted_planes(256, 160, 47, tag="ops")
    L = torch.from_numpy(p.left).cuda()
    R = torch.from_numpy(p.right).cuda()
    d, m, c = torch.ops.doubleeye.dense(L, R, 48, 8)
    ref = de.run_dense(p.left, p.right, de.Cfg(dmax=48, iters=8), want_cand=False)
    assert d.device == L.device
    assert _same(d.cpu().numpy(), ref.disp) and _same(m.cpu().numpy(), ref.margin)
    assert _same(c.cpu().numpy(), ref.conf)
    cs, cd, cn, cnb = torch.ops.doubleeye.cost_top2(L, R, 48)
    rcs, rcd, rcn, rcnb = de.cost_top2(L, R, de.Cfg(dmax=48))
    for a, b in ((cs, rcs), (cd, rcd), (cn, rcn), (cnb, rcnb)):
        assert torch.equal(a, b)
    sd, sm, sl = torch.ops.doubleeye.solve(cs, cd, cn, cnb, 48, 8)
    rd, rm, rl = de.solve(rcs, rcd, rcn, rcnb, de.Cfg(dmax=48, iters=8))
    assert _same(sd.cpu().numpy(), rd.cpu().numpy()) and _same(sl.cpu().numpy(), rl.cpu().numpy())
    f = synth.fronto_planes(256, 160, seed=3)
    kl = sparse.detect_fast(f.left, sparse.DetCfg(cell=24))
    kr = sparse.detect_fast(f.right, sparse.DetCfg(cell=24))
    dl = sparse.census_at(f.left, kl)
    dr = sparse.census_at(f.right, kr)
    want, _ = sparse.match_masda(kl, dl, kr, dr, sparse.MatchCfg())
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).view(dt)).cuda()  # noqa: E731
    pairs, vals = torch.ops.doubleeye.match_masda(
        t(np.asarray(kl, np.float32).reshape(-1, 4), np.float32), t(dl, np.int64),
        t(np.asarray(kr, np.float32).reshape(-1, 4), np.float32), t(dr, np.int64))
    assert pairs.shape[0] == len(want) > 50
    assert (pairs[:, 0].cpu().numpy() == want["left"]).all()
    assert (pairs[:, 1].cpu().numpy() == want["right"]).all()
    assert _same(vals[:, 1].cpu().numpy(), want["belief"])
    assert _same(vals[:, 2].cpu().numpy(), want["disparity"])
