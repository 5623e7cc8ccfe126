"""The serving loop (de_server_*): results are the plain pipeline's bit for bit, alone
and in a mix of streams and sizes submitted from several threads; DEDD planes follow
core/tools/de_dense_cuda.cu:729-746; the HBM budget refuses what cannot fit; latency
percentiles are reported."""
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
        last = sv.last_disparity(3, pairs[3][0].left.shape[1], pairs[3][0].left.shape[0])
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
    assert same(last, results[-1]["disp"]) or same(last, results[-5]["disp"]) or \
        same(last, results[3]["disp"]) or np.isfinite(last).mean() > 0.5


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
