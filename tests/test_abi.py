"""The C ABI on a machine without a GPU: the library loads, exports every function
include/doubleeye_b200.h declares, and its host-only entry points (defaults,
version, confidence, workspace sizing, argument checks) behave.  No compute call is
made here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "doubleeye_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"DE_API\s+[\w\s\*]+?\b(de_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from doubleeye_b200 import _lib, build
    build.build()
    return _lib


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("de_dense_dev", "de_dense_workspace_bytes", "de_solve_dev",
                 "de_cost_top2_dev", "de_census_dev", "de_detect_fast_dev",
                 "de_match_masda_dev", "de_census_at_dev", "de_ctx_dense",
                 "de_dense_noalloc_dev"):
        assert must in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(lib):
    L = lib.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if n not in lib.SIGNATURES]
    assert not missing, missing


def test_defaults_and_version(lib):
    L = lib.lib()
    c = lib.DeCfg()
    L.de_cfg_default(C.byref(c))
    assert (c.dmin, c.dmax, c.iters, c.census_hw, c.census_hh) == (1, 60, 0, 3, 3)
    assert abs(c.lambda_ + 0.1) < 1e-7 and abs(c.damping - 0.4) < 1e-7
    d = lib.DeDetCfg()
    L.de_det_cfg_default(C.byref(d))
    assert (d.grad_window, d.cell, d.per_cell, d.border, d.fast_threshold,
            d.nms_radius) == (3, 32, 3, 8, 8, 3)
    m = lib.DeMatchCfg()
    L.de_match_cfg_default(C.byref(m))
    assert (m.max_candidates, m.iterations, m.census_bits) == (24, 20, 48)
    assert L.de_version().decode()


def test_confidence_host_matches_oracle(lib, oracle):
    L = lib.lib()
    rng = np.random.default_rng(3)
    for s1, s2 in rng.uniform(-1, 1, (200, 2)).astype(np.float32):
        for lrc in (0.0, 2.0):
            assert np.float32(L.de_confidence(s1, s2, -0.1, lrc, 1.0)) == \
                np.float32(oracle.confidence(float(s1), float(s2), -0.1, lrc, 1.0))


def test_workspace_sizing_and_argument_checks(lib):
    L = lib.lib()
    cfg = lib.DeCfg()
    L.de_cfg_default(C.byref(cfg))
    cfg.dmax = 128
    pair = lib.DePair(1, 1, 848, 480, 0, None, None, None, None)
    n = C.c_size_t()
    assert L.de_dense_workspace_bytes(C.byref(cfg), C.byref(pair), 1, C.byref(n)) == 0
    assert n.value > 848 * 480 * 128 * 2                  # holds the int16 volume
    bad = lib.DePair(1, 1, 4, 480, 0, None, None, None, None)
    assert L.de_dense_workspace_bytes(C.byref(cfg), C.byref(bad), 1, C.byref(n)) == -1
    assert L.de_last_error()
    cfg.dmax = 300                                        # beyond 256 disparities
    assert L.de_dense_workspace_bytes(C.byref(cfg), C.byref(pair), 1, C.byref(n)) == -1
    det = lib.DeDetCfg()
    L.de_det_cfg_default(C.byref(det))
    assert L.de_detect_workspace_bytes(848, 480, C.byref(det), C.byref(n)) == 0
    assert n.value >= 848 * 480 * 13
    det.cell = 1000
    assert L.de_detect_workspace_bytes(848, 480, C.byref(det), C.byref(n)) == -1
    m = lib.DeMatchCfg()
    L.de_match_cfg_default(C.byref(m))
    assert L.de_match_workspace_bytes(2000, 2000, C.byref(m), C.byref(n)) == 0
    assert n.value >= 2000 * 24 * 4 * 8
    m.census_bits = 80
    assert L.de_match_workspace_bytes(2000, 2000, C.byref(m), C.byref(n)) == -1


def test_params_roundtrip(lib):
    for name in ("rows_ctas_per_sm", "cols_kt", "cols_pf", "cols_cta", "solve_threads",
                 "batch_streams", "cols_async"):
        v = lib.get_param(name)
        lib.set_param(name, v)
        assert lib.get_param(name) == v
    with pytest.raises(lib.DeError):
        lib.set_param("no_such_knob", 1)
