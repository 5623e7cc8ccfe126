"""Batching: uneven pair sizes and disparity ranges in one launch set, the same set
replayed from a captured CUDA graph, and the autotuner's launch-shape knobs, which
must never change a result."""
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
    a, b = a.cpu().numpy(), b.cpu().numpy()
    if a.dtype == np.float32:
        return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())
    return bool((a == b).all())


SHAPES = [(320, 240, 64), (640, 480, 128), (200, 96, 32), (848, 480, 128), (333, 211, 96),
          (1280, 720, 256), (320, 240, 64)]


@pytest.fixture(scope="module")
def batch(de):
    from doubleeye_b200 import synth
    pairs = [synth.slanted_planes(W, H, D - 1, seed=k, tag="batch-gpu") for k, (W, H, D) in
             enumerate(SHAPES)]
    Ls = [torch.from_numpy(p.left).cuda() for p in pairs]
    Rs = [torch.from_numpy(p.right).cuda() for p in pairs]
    return pairs, Ls, Rs


def run(de, m, Ls, Rs, cand=True):
    outs = [m.new_outputs(*L.shape, cand=cand) for L in Ls]
    m.match_into([(L, R, D, o) for L, R, (_, _, D), o in zip(Ls, Rs, SHAPES, outs)])
    torch.cuda.synchronize()
    return outs


def test_mixed_batch_equals_one_pair_at_a_time(de, batch):
    pairs, Ls, Rs = batch
    m = de.DenseMatcher(de.Cfg(iters=8))
    got = run(de, m, Ls, Rs)
    for k, (L, R) in enumerate(zip(Ls, Rs)):
        one = m.new_outputs(*L.shape, cand=True)
        m.match_into([(L, R, SHAPES[k][2], one)])
        torch.cuda.synchronize()
        for key in ("disp", "margin", "conf", "cand"):
            assert same(got[k][key], one[key]), (k, key)


def test_graph_replay_matches_direct_launch(de, batch):
    pairs, Ls, Rs = batch
    m = de.DenseMatcher(de.Cfg(iters=8))
    ref = run(de, m, Ls, Rs)
    Lc = [L.clone() for L in Ls]
    Rc = [R.clone() for R in Rs]
    outs = [m.new_outputs(*L.shape, cand=True) for L in Lc]
    g = m.capture([(L, R, D, o) for L, R, (_, _, D), o in zip(Lc, Rc, SHAPES, outs)])
    for _ in range(2):
        g.launch()
        torch.cuda.synchronize()
        for k in range(len(SHAPES)):
            for key in ("disp", "margin", "conf", "cand"):
                assert same(outs[k][key], ref[k][key]), (k, key)
    # new frames in the captured input buffers: the replay matches a direct launch
    for k in range(len(SHAPES)):
        Lc[k].copy_(Rs[k])
        Rc[k].copy_(Ls[k].roll(-3, dims=1))
    g.launch()
    direct = run(de, m, Lc, Rc)
    for k in range(len(SHAPES)):
        assert same(outs[k]["disp"], direct[k]["disp"]), k
    g.close()


@pytest.mark.parametrize("knob", ["rows_ctas_per_sm", "cols_kt", "cols_pf", "cols_cta",
                                  "solve_threads", "batch_streams", "cols_async"])
def test_knobs_never_change_results(de, batch, knob):
    from doubleeye_b200 import autotune
    pairs, Ls, Rs = batch
    m = de.DenseMatcher(de.Cfg(iters=4))
    saved = autotune.current()
    try:
        ref = run(de, m, Ls, Rs)
        for v in autotune.KNOBS[knob]:
            autotune.apply(dict(saved, **{knob: v}))
            got = run(de, m, Ls, Rs)
            for k in range(len(SHAPES)):
                for key in ("disp", "conf", "cand"):
                    assert same(got[k][key], ref[k][key]), (knob, v, k, key)
    finally:
        autotune.apply(saved)


def test_autotune_picks_and_caches(de, batch, tmp_path):
    from doubleeye_b200 import autotune
    pairs, Ls, Rs = batch
    saved = autotune.current()
    try:
        m = de.DenseMatcher(de.Cfg(iters=4))
        m._tuner = autotune.Tuner(str(tmp_path / "tune.json"))
        items = [(L, R, D, m.new_outputs(*L.shape)) for L, R, (_, _, D) in zip(Ls, Rs, SHAPES)]
        knobs = m.tune_for(items)
        assert set(knobs) == set(autotune.KNOBS)
        for k, v in knobs.items():
            assert v in autotune.KNOBS[k] or v == saved[k]
        again = autotune.Tuner(str(tmp_path / "tune.json"))
        sig = autotune.signature(m.cfg, [(L.shape[1], L.shape[0], D)
                                         for L, (_, _, D) in zip(Ls, SHAPES)])
        assert again.lookup(sig) is not None
    finally:
        autotune.apply(saved)


def test_host_batch_pinned_and_pageable_agree(de, batch):
    """The host-pointer batch moves page-locked buffers by DMA directly and stages
    pageable ones; any mix gives the device path's results."""
    pairs, Ls, Rs = batch
    cfg = de.Cfg(iters=8)
    host = [(p.left, p.right, D) for p, (_, _, D) in zip(pairs, SHAPES)]
    shapes = [p.left.shape for p in pairs]
    pageable = de.run_dense_batch(host, cfg, want_cand=True)
    pinned_in = []
    for k, (L, R, D) in enumerate(host):
        if k % 2 == 0:                                  # every other pair page-locked
            hl, hr = de.pinned_empty(L.shape, np.uint8), de.pinned_empty(R.shape, np.uint8)
            hl[...] = L
            hr[...] = R
            pinned_in.append((hl, hr, D))
        else:
            pinned_in.append((L, R, D))
    outs = de.new_results(shapes, want_cand=True, pinned=True)
    got = de.run_dense_batch(pinned_in, cfg, want_cand=True, out=outs)
    assert all(g is o for g, o in zip(got, outs))       # written in place
    m = de.DenseMatcher(cfg)
    dev = run(de, m, Ls, Rs)
    for k in range(len(SHAPES)):
        for key in ("disp", "margin", "conf", "cand"):
            a, b = getattr(pageable[k], key), getattr(got[k], key)
            assert same(torch.from_numpy(a), torch.from_numpy(b)), (k, key)
            assert same(torch.from_numpy(np.ascontiguousarray(b)), dev[k][key]), (k, key)


def test_host_batch_chunks_equal_single_pairs(de):
    """Ten host pairs run as five chunks (1, 3, 3, 2, 1 pairs), each on its own stream
    and workspace slice, with uploads and downloads overlapping the other chunks'
    compute; every pair's outputs equal a call with that pair alone."""
    from doubleeye_b200 import synth
    pairs = [synth.slanted_planes(640, 480, 63, seed=k, tag="chunks") for k in range(10)]
    cfg = de.Cfg(dmax=64, iters=4)
    shapes = [p.left.shape for p in pairs]
    host = []
    for k, p in enumerate(pairs):                       # a mix of pinned and pageable inputs
        if k % 3 == 0:
            hl, hr = de.pinned_empty(p.left.shape, np.uint8), de.pinned_empty(p.right.shape, np.uint8)
            hl[...] = p.left
            hr[...] = p.right
            host.append((hl, hr))
        else:
            host.append((p.left, p.right))
    outs = de.new_results(shapes, pinned=True)
    for k in range(0, 10, 2):                           # and of pinned and pageable outputs
        outs[k] = de.new_results([shapes[k]], pinned=False)[0]
    got = de.run_dense_batch(host, cfg, out=outs)
    for k, p in enumerate(pairs):
        one = de.run_dense(p.left, p.right, cfg, want_cand=False)
        for key in ("disp", "margin", "conf"):
            a, b = getattr(got[k], key), getattr(one, key)
            assert same(torch.from_numpy(np.ascontiguousarray(a)), torch.from_numpy(b)), (k, key)


def test_batches_on_many_streams_and_a_capture(de, batch):
    """A batch of several pairs runs as parts on streams forked from the caller's; each
    thread keeps a few such sets and hands the least recently used one to a new calling
    stream.  Nine calling streams in turn, then a graph captured on a tenth while the
    others keep launching, all give the one-stream results."""
    pairs, Ls, Rs = batch
    ref = run(de, de.DenseMatcher(de.Cfg(iters=4)), Ls, Rs, cand=False)
    items_for = lambda m: [(L, R, D, m.new_outputs(*L.shape))  # noqa: E731
                           for L, R, (_, _, D) in zip(Ls, Rs, SHAPES)]
    streams = [torch.cuda.Stream() for _ in range(9)]
    mats = [de.DenseMatcher(de.Cfg(iters=4)) for _ in streams]
    items = [items_for(m) for m in mats]
    for rnd in range(2):
        for st, m, it in zip(streams, mats, items):
            st.wait_stream(torch.cuda.current_stream())
            m.match_into(it, stream=st)
    torch.cuda.synchronize()
    for it in items:
        for k in range(len(SHAPES)):
            for key in ("disp", "margin", "conf"):
                assert same(it[k][3][key], ref[k][key]), (k, key)
    mc = de.DenseMatcher(de.Cfg(iters=4))
    cit = items_for(mc)
    g = mc.capture(cit)
    for st, m, it in zip(streams, mats, items):       # other streams launch meanwhile
        m.match_into(it, stream=st)
    g.launch()
    torch.cuda.synchronize()
    for k in range(len(SHAPES)):
        for key in ("disp", "margin", "conf"):
            assert same(cit[k][3][key], ref[k][key]), (k, key)
            assert same(items[0][k][3][key], ref[k][key]), (k, key)
    g.close()
