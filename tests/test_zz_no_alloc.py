"""The dense entry point that allocates nothing, de_dense_noalloc_dev.

It exists for callers that cannot call cudaMalloc: real-time threads that may not
take the driver's allocation locks, hosts that own the device heap, and integrations
whose memory budget is fixed before the process starts.  Its scratch is a fixed
16 MiB device array built into the library, so it takes only the caller's images and
output buffers.  These tests call it through the C ABI, twice in a row on one pair
(with and without the reverse-match plane, which is carved from the same array), and
require each call to give the same bytes as the workspace entry point de_dense_dev
(the dense path is bit-exact, so the tolerance is zero), the device's free memory to
be the same before and after a call, the status word to read 0, and a pair too large
for the array to be refused without running anything.

Kept in a file of its own, collected last, so a failure here leaves every other test
already run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from doubleeye_b200 import _lib, build
    build.build()
    return _lib


def _outputs(H, W):
    return dict(disp=torch.empty((H, W), dtype=torch.float32, device="cuda"),
                margin=torch.empty((H, W), dtype=torch.float32, device="cuda"),
                conf=torch.empty((H, W), dtype=torch.uint8, device="cuda"),
                cand=torch.empty((6, H, W), dtype=torch.float32, device="cuda"))


def _pair(lib, L, R, out):
    H, W = L.shape
    return lib.DePair(L.data_ptr(), R.data_ptr(), W, H, 0, out["disp"].data_ptr(),
                      out["margin"].data_ptr(), out["conf"].data_ptr(), out["cand"].data_ptr())


def _same(a, b):
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    if a.dtype == np.float32:
        return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())
    return bool((a == b).all())


@pytest.mark.parametrize("lrc", [0, 1])
def test_noalloc_matches_workspace_entry_point(lib, lrc):
    import doubleeye_b200 as de
    from doubleeye_b200 import synth
    p = synth.slanted_planes(320, 240, 63, tag="noalloc")
    cfg = de.Cfg(dmax=64, iters=8, lrc=lrc)
    L = torch.from_numpy(p.left).cuda()
    R = torch.from_numpy(p.right).cuda()
    stream = torch.cuda.current_stream().cuda_stream

    # reference result through the caller-workspace entry point
    ref = _outputs(240, 320)
    pr = _pair(lib, L, R, ref)
    need = C.c_size_t()
    lib.check(lib.lib().de_dense_workspace_bytes(C.byref(cfg), C.byref(pr), 1, C.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    lib.check(lib.lib().de_dense_dev(C.byref(cfg), C.byref(pr), 1, ws.data_ptr(), need.value,
                                     stream))
    torch.cuda.synchronize()

    outs = [_outputs(240, 320) for _ in range(2)]
    pairs = [_pair(lib, L, R, o) for o in outs]
    torch.cuda.synchronize()
    for call in range(2):                      # the scratch keeps the last call's contents
        free0 = torch.cuda.mem_get_info()[0]
        held0 = torch.cuda.memory_allocated()
        lib.check(lib.lib().de_dense_noalloc_dev(C.byref(cfg), C.byref(pairs[call]), stream))
        torch.cuda.synchronize()
        if call == 1:                          # after the first call loaded every kernel
            assert torch.cuda.mem_get_info()[0] == free0, "device free memory changed"
        assert torch.cuda.memory_allocated() == held0
        st = C.c_int(-1)
        lib.check(lib.lib().de_workspace_status(None, stream, C.byref(st)))
        assert st.value == 0
        for k in ("disp", "margin", "conf", "cand"):
            assert _same(outs[call][k], ref[k]), f"call {call}: {k} differs from de_dense_dev"
    assert torch.isfinite(ref["disp"]).float().mean().item() > 0.5


def test_noalloc_refuses_pairs_beyond_its_scratch(lib):
    import doubleeye_b200 as de
    cfg = de.Cfg(dmax=128)
    H, W = 480, 848                            # needs ~117 MB of workspace
    L = torch.zeros((H, W), dtype=torch.uint8, device="cuda")
    out = _outputs(H, W)
    rc = lib.lib().de_dense_noalloc_dev(C.byref(cfg), C.byref(_pair(lib, L, L, out)),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == -1                            # DE_ERR_ARG, nothing launched
    assert b"no-allocation scratch" in lib.lib().de_last_error()
