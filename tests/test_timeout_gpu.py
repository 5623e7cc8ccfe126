"""A device wait that runs out, end to end, without a fault.

Every mbarrier wait in the row kernel is bounded; one that runs out records the
launch set's status word, and the host-pointer context and the server turn that into
DE_ERR_TIMEOUT, while device-pointer callers read it with de_workspace_status.  The
test hook "expire_wait_polls" makes each row-kernel launch end with a bounded wait on
a barrier nothing arrives at, after all its real waits have completed and with no copy
in flight, so that path runs for real.  Afterwards (hook off) the same context,
server and workspace give correct results again: the device stays usable.
"""
import ctypes as C

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


@pytest.fixture
def expire():
    from doubleeye_b200 import _lib
    _lib.set_param("expire_wait_polls", 2000)
    yield
    _lib.set_param("expire_wait_polls", 0)


def _pair():
    from doubleeye_b200 import synth
    return synth.slanted_planes(160, 96, 31, tag="timeout")


def test_host_context_reports_timeout(de, expire, oracle):
    from doubleeye_b200._lib import DeError
    p = _pair()
    with pytest.raises(DeError) as e:
        de.run_dense(p.left, p.right, de.Cfg(dmax=32, iters=4))
    assert e.value.code == -4                       # DE_ERR_TIMEOUT


def test_workspace_status_and_recovery(de, oracle):
    from doubleeye_b200 import _lib
    from oracle import oracle as O
    p = _pair()
    cfg = de.Cfg(dmax=32, iters=4)
    m = de.DenseMatcher(cfg)
    L = torch.from_numpy(p.left).cuda()
    R = torch.from_numpy(p.right).cuda()
    out = m.new_outputs(96, 160)
    stream = torch.cuda.current_stream().cuda_stream
    st = C.c_int(-1)
    _lib.set_param("expire_wait_polls", 2000)
    try:
        m.match_into([(L, R, 0, out)])
        _lib.check(_lib.lib().de_workspace_status(m._ws.data_ptr(), stream, C.byref(st)))
        assert st.value != 0
    finally:
        _lib.set_param("expire_wait_polls", 0)
    m.match_into([(L, R, 0, out)])                   # the same workspace, hook off
    _lib.check(_lib.lib().de_workspace_status(m._ws.data_ptr(), stream, C.byref(st)))
    assert st.value == 0
    od, _, _ = oracle.dense(O.default_cfg(dmax=32, iters=4), p.left, p.right)
    got = out["disp"].cpu().numpy()
    assert ((got.view(np.uint32) == od.view(np.uint32)) | (np.isnan(got) & np.isnan(od))).all()
    r = de.run_dense(p.left, p.right, cfg)           # the host context recovers too
    assert ((r.disp.view(np.uint32) == od.view(np.uint32)) |
            (np.isnan(r.disp) & np.isnan(od))).all()


def test_server_reports_timeout_then_recovers(de):
    from doubleeye_b200 import _lib, serve
    from doubleeye_b200._lib import DeError
    p = _pair()
    with serve.Server(de.Cfg(dmax=32, iters=4), hbm_budget=1 << 30, max_batch=2,
                      lanes=2) as sv:
        _lib.set_param("expire_wait_polls", 2000)
        try:
            t = sv.submit(0, p.left, p.right)
            with pytest.raises(DeError) as e:
                sv.wait(t)
            assert e.value.code == -4
        finally:
            _lib.set_param("expire_wait_polls", 0)
        r = sv.wait(sv.submit(0, p.left, p.right))
        want = de.run_dense(p.left, p.right, de.Cfg(dmax=32, iters=4), want_cand=False)
        assert r["disp"].tobytes() == want.disp.tobytes()
        assert sv.stats()["failed"] == 1
