"""The serving loop (de_server_*): results are the plain pipeline's bit for bit, alone
and in a mix of streams and sizes submitted from several threads; DEDD planes follow
core/tools/de_dense_cuda.cu:729-746; the HBM budget refuses what cannot fit; latency
percentiles are reported; each stream keeps its newest map on the device, also across
a change of size while other lanes are busy; a stream with a temporal prior gets, for
every frame after its first, the prior path's result with its previous served map,
hole-filled as the reference's fill does, as the prior, alone and in the mix."""
import threading

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


def same(a, b):
    if a.dtype == np.float32:
        return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())
    return bool((a == b).all())


def dedd_reference(disp, conf):
    ok = np.isfinite(disp) & (disp > 0)
    with np.errstate(invalid="ignore"):
        q = np.where(ok, np.floor(np.abs(disp) * 16.0 + 0.5) * np.sign(disp), -32768)
    return q.astype(np.int16), np.where(ok, conf, 0).astype(np.uint8)


def test_alone_and_in_the_mix_are_identical(de):
    from doubleeye_b200 import serve, synth
    cfg = de.Cfg(dmax=64, iters=8)
    shapes = [(320, 240, 64), (200, 120, 32), (333, 211, 48), (320, 240, 64)]
    pairs = [(synth.slanted_planes(W, H, D - 1, seed=k, tag="serve"), D)
             for k, (W, H, D) in enumerate(shapes * 3)]
    plain = [de.run_dense(p.left, p.right, de.Cfg(dmax=D, iters=8), want_cand=False)
             for p, D in pairs]
    with serve.Server(cfg, hbm_budget=2 << 30, max_batch=5, lanes=2) as sv:
        alone = []
        for k, (p, D) in enumerate(pairs[:4]):               # one at a time
            alone.append(sv.wait(sv.submit(k, p.left, p.right, D)))
        results = [None] * len(pairs)

        def client(idx):                                     # concurrent submitters
            ts = [(i, sv.submit(i % 4, pairs[i][0].left, pairs[i][0].right, pairs[i][1]))
                  for i in idx]
            for i, t in ts:
                results[i] = sv.wait(t)
        th = [threading.Thread(target=client, args=(list(range(j, len(pairs), 3)),))
              for j in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        st = sv.stats()
        # the stream's newest frame, submitted last: its map is what the stream keeps
        p3, D3 = pairs[7]
        newest = sv.wait(sv.submit(3, p3.left, p3.right, D3))
        last = sv.last_disparity(3, p3.left.shape[1], p3.left.shape[0])
    for k in range(4):
        assert same(alone[k]["disp"], plain[k].disp) and same(alone[k]["conf"], plain[k].conf)
    for k, r in enumerate(results):
        assert same(r["disp"], plain[k].disp), k
        assert same(r["margin"], plain[k].margin), k
        assert same(r["conf"], plain[k].conf), k
        q, qc = dedd_reference(plain[k].disp, plain[k].conf)
        assert same(r["q4"], q) and same(r["qconf"], qc), k
    assert st["completed"] == len(pairs) + 4 and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert same(newest["disp"], plain[7].disp)
    assert same(last, plain[7].disp)


def test_budget_refuses_oversized_pair(de):
    from doubleeye_b200 import serve
    from doubleeye_b200._lib import DeError
    with serve.Server(de.Cfg(dmax=256), hbm_budget=256 << 20, max_batch=4, lanes=2) as sv:
        big = np.zeros((1080, 1920), np.uint8)
        t = sv.submit(0, big, big)
        with pytest.raises(DeError):
            sv.wait(t)
        small = np.random.default_rng(0).integers(0, 255, (64, 96)).astype(np.uint8)
        r = sv.wait(sv.submit(1, small, small, 16))
        assert r["disp"].shape == (64, 96)


def test_simulated_streams_report_latency(de):
    from doubleeye_b200 import serve
    specs = [serve.StreamSpec(320, 240, 64)] * 4 + [serve.StreamSpec(640, 480, 128)] * 2
    frames = serve.make_frames(specs, frames_per_stream=2)
    with serve.Server(de.Cfg(iters=8), hbm_budget=4 << 30, max_batch=8, lanes=2) as sv:
        rep = serve.simulate(sv, specs, frames, duration_s=1.0)
    assert rep["failed"] == 0 and rep["completed"] == rep["requests"]
    assert 0 < rep["p50_ms"] <= rep["p99_ms"] < 1000


def test_stream_changes_size_while_others_run(de):
    """A camera stream switches resolution between frames while other streams' batches
    are in flight on the other lane: every result is the plain pipeline's, and the
    stream's kept map is its newest frame at the new size."""
    from doubleeye_b200 import serve, synth
    small = [synth.slanted_planes(160, 120, 31, seed=k, tag="resize") for k in range(3)]
    big = [synth.slanted_planes(320, 240, 63, seed=10 + k, tag="resize") for k in range(3)]
    other = [synth.slanted_planes(256, 192, 47, seed=20 + k, tag="resize") for k in range(6)]
    with serve.Server(de.Cfg(dmax=64, iters=4), hbm_budget=2 << 30, max_batch=3,
                      lanes=3) as sv:
        tickets = []
        for k in range(3):
            tickets.append((sv.submit(1, other[2 * k].left, other[2 * k].right, 48),
                            other[2 * k], 48))
            tickets.append((sv.submit(0, small[k].left, small[k].right, 32), small[k], 32))
            tickets.append((sv.submit(2, other[2 * k + 1].left, other[2 * k + 1].right, 48),
                            other[2 * k + 1], 48))
            tickets.append((sv.submit(0, big[k].left, big[k].right, 64), big[k], 64))
        for t, p, D in tickets:
            r = sv.wait(t)
            want = de.run_dense(p.left, p.right, de.Cfg(dmax=D, iters=4), want_cand=False)
            assert same(r["disp"], want.disp)
        last = sv.last_disparity(0, 320, 240)
    want = de.run_dense(big[2].left, big[2].right, de.Cfg(dmax=64, iters=4), want_cand=False)
    assert same(last, want.disp)


def _prior_chain(de, frames, D, band):
    """What a prior stream must serve: frame 0 plain, then each frame through the prior
    path with the previous served map, hole-filled by the oracle's restatement of the
    reference's fill, as the prior."""
    from oracle import oracle as O
    cfg = de.Cfg(dmax=D, iters=8)
    out = [de.run_dense(frames[0].left, frames[0].right, cfg, want_cand=False).disp]
    for f in frames[1:]:
        prior = O.fill_prior(out[-1])
        out.append(de.run_dense_prior(f.left, f.right, prior, cfg, band=band,
                                      want_cand=False).disp)
    return out


def test_temporal_prior_alone_and_in_the_mix(de):
    from doubleeye_b200 import serve, synth
    va = synth.Video(320, 240, 63, stream_id=0, seed=5)
    vb = synth.Video(256, 160, 47, stream_id=1, seed=6)
    fa = [va.frame(t) for t in range(4)]
    fb = [vb.frame(t) for t in range(4)]
    plain = [synth.slanted_planes(200, 120, 31, seed=30 + k, tag="mixp") for k in range(4)]
    want_a = _prior_chain(de, fa, 64, 2)
    want_b = _prior_chain(de, fb, 48, 3)
    want_p = [de.run_dense(p.left, p.right, de.Cfg(dmax=32, iters=8), want_cand=False).disp
              for p in plain]
    assert not same(want_a[1], de.run_dense(fa[1].left, fa[1].right, de.Cfg(dmax=64, iters=8),
                                            want_cand=False).disp)
    cfg = de.Cfg(iters=8)
    # alone: one frame at a time
    with serve.Server(cfg, hbm_budget=2 << 30, max_batch=4, lanes=2) as sv:
        sv.stream_prior(0, 2)
        for k, f in enumerate(fa):
            assert same(sv.wait(sv.submit(0, f.left, f.right, 64))["disp"], want_a[k]), k
        assert same(sv.last_disparity(0, 320, 240), want_a[-1])
    # in the mix: two prior streams and a plain one, each from its own thread, all
    # frames submitted without waiting
    res = {}
    with serve.Server(cfg, hbm_budget=2 << 30, max_batch=4, lanes=2) as sv:
        sv.stream_prior(0, 2)
        sv.stream_prior(1, 3)

        def cam(s, frames, D):
            ts = [sv.submit(s, f.left, f.right, D) for f in frames]
            res[s] = [sv.wait(t)["disp"] for t in ts]
        th = [threading.Thread(target=cam, args=a) for a in
              ((0, fa, 64), (1, fb, 48), (2, plain, 32))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert sv.stats()["failed"] == 0
    for k in range(4):
        assert same(res[0][k], want_a[k]), ("a", k)
        assert same(res[1][k], want_b[k]), ("b", k)
        assert same(res[2][k], want_p[k]), ("plain", k)


def test_prior_fill_matches_reference_fill(de, golden_dir):
    """de_prior_fill_dev against the reference's own fill (golden vectors), and
    against the oracle's restatement on a served disparity map."""
    import os
    from oracle import oracle as O
    from doubleeye_b200 import synth
    z = np.load(os.path.join(golden_dir, "fill.npz"))
    for n in sorted({k[:-3] for k in z.files if k.endswith("_in")}):
        assert de.fill_holes(z[n + "_in"]).tobytes() == z[n + "_out"].tobytes(), n
    p = synth.slanted_planes(848, 480, 127, seed=3, tag="fill")
    d = de.run_dense(p.left, p.right, de.Cfg(dmax=128, iters=8), want_cand=False).disp
    assert np.isnan(d).mean() > 0.05
    assert de.fill_holes(d).tobytes() == O.fill_prior(d).tobytes()
