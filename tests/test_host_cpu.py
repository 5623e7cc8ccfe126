"""Host-side helpers of the Python bindings that need no GPU."""
import numpy as np

from doubleeye_b200 import dense


def test_addr_matches_numpy_and_follows_reallocation():
    a = np.zeros((48, 64), np.float32)
    assert dense._addr(a) == a.ctypes.data
    assert dense._addr(a) == a.ctypes.data          # served from the cache
    assert dense._addr(None) is None
    v = a[1:]                                       # a view: its own address
    assert dense._addr(v) == v.ctypes.data
    b = np.zeros(10, np.uint8)
    assert dense._addr(b) == b.ctypes.data
    try:                                            # the only way to move a buffer is
        b.resize(1 << 20, refcheck=False)           # refused while the cache holds b
    except ValueError:
        pass
    assert dense._addr(b) == b.ctypes.data
    for _ in range(100):                            # ids reused by new arrays
        c = np.empty((8, 8), np.uint8)
        assert dense._addr(c) == c.ctypes.data
        del c


def test_u8_accepts_only_2d_uint8():
    img = np.arange(12, dtype=np.uint8).reshape(3, 4)
    assert dense._u8(img) is img
    t = dense._u8(img.T)                            # not contiguous: copied
    assert t.flags.c_contiguous and (t == img.T).all()
    for bad in (img.astype(np.int16), img.reshape(-1)):
        try:
            dense._u8(bad)
        except ValueError:
            continue
        raise AssertionError("accepted a non 2-D uint8 image")
