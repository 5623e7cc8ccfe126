"""de_dense_gpu, the reference-compatible command line (core/tools/de_dense.cpp argv,
--out / --out-conf bytes; core/tools/de_dense_cuda.cu --stream DEIR/DEDD framing).
Argument handling runs without a GPU; the matching tests are marked gpu and compare
the files it writes with the oracle bit for bit (the oracle against the reference's
golden outputs is test_oracle_golden's job)."""
import ast
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def cli():
    from doubleeye_b200 import build
    build.build()
    return build.CLI


def run(cli, *args, stdin=None):
    return subprocess.run([cli, *map(str, args)], input=stdin, capture_output=True,
                          timeout=300)


def test_usage_and_refused_flags(cli):
    assert run(cli).returncode == 2
    for flag in ("--guided", "--box", "--csct", "--simd", "--c2f", "--dump-vol"):
        r = run(cli, "a", "b", "64", "48", flag)
        assert r.returncode == 2 and b"unsupported" in r.stderr
    assert run(cli, "a", "b", "64", "48", "--topk", "3").returncode == 2


def flags_for(cfg: dict) -> list:
    f = ["--dmax", cfg["dmax"], "--iters", cfg["iters"], "--lambda", cfg["lambda_"],
         "--gamma", cfg["gamma"], "--damping", cfg["damping"], "--sigma-s", cfg["sigma_s"],
         "--sigma-r", cfg["sigma_r"], "--ad", cfg["ad"], "--ad-trunc", cfg["ad_trunc"],
         "--min-margin", cfg["min_margin"], "--min-ratio", cfg["min_ratio"]]
    f.append("--subpixel" if cfg["subpixel"] else "--no-subpixel")
    f.append("--fit-eq" if cfg["fit_eq"] else "--fit-parabola")
    if cfg["lrc"]:
        f.append("--lrc")
    return f


def needs_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["dense_b", "dense_d", "dense_e"])
def test_files_match_oracle(cli, oracle, golden_dir, tmp_path, case):
    needs_gpu()
    g = np.load(os.path.join(golden_dir, f"{case}.npz"))
    cfg = ast.literal_eval(str(g["cfg"][0]))
    assert cfg["dmin"] == 1                      # the reference CLI has no --dmin
    H, W = g["L"].shape
    g["L"].tofile(tmp_path / "l.y8")
    g["R"].tofile(tmp_path / "r.y8")
    r = run(cli, tmp_path / "l.y8", tmp_path / "r.y8", W, H, *flags_for(cfg),
            "--out", tmp_path / "d.f32", "--out-conf", tmp_path / "c.f32")
    assert r.returncode == 0, r.stderr
    last = [ln for ln in r.stdout.decode().splitlines() if "total" in ln][-1]
    assert "census" in last and "solve" in last and "filled" in last
    disp = np.fromfile(tmp_path / "d.f32", np.float32).reshape(H, W)
    cand = np.fromfile(tmp_path / "c.f32", np.float32).reshape(6, H, W)
    oc = O.default_cfg(**{k: v for k, v in cfg.items() if k not in ("census_hw", "census_hh")})
    od, _, ocand = oracle.dense(oc, g["L"], g["R"])
    assert disp.tobytes() == od.tobytes()
    assert cand.tobytes() == ocand.tobytes()


def deir(w, h, stream, frame, img):
    return b"DEIR" + struct.pack("<HHBBI", w, h, stream, 0, frame) + img.tobytes()


@pytest.mark.gpu
def test_stream_framing(cli, oracle, golden_dir):
    needs_gpu()
    g = np.load(os.path.join(golden_dir, "dense_b.npz"))
    H, W = g["L"].shape
    L, R = g["L"], g["R"]
    data = (deir(W, H, 0, 7, R) + deir(W, H, 1, 7, L) +        # right first, then left
            deir(W, H, 1, 8, R) +                             # an unpaired frame
            deir(W, H, 1, 9, L) + deir(W, H, 0, 9, R))
    r = run(cli, "-", "-", W, H, "--stream", "--dmax", 32, "--iters", 8, stdin=data)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    od, _, _ = oracle.dense(O.default_cfg(dmax=32, iters=8), L, R)
    rec = 16 + W * H + 2 * W * H + W * H
    assert len(out) == 2 * rec
    ok = np.isfinite(od) & (od > 0)
    want = np.where(ok, np.floor(np.abs(od) * 16 + 0.5) * np.sign(od), -32768).astype(np.int16)
    for k, frame in enumerate((7, 9)):
        blk = out[k * rec:(k + 1) * rec]
        magic, w, h, num, flags = struct.unpack("<4sHHII", blk[:16])
        assert (magic, w, h, num, flags) == (b"DEDD", W, H, frame, 1)
        assert blk[16:16 + W * H] == L.tobytes()
        q = np.frombuffer(blk[16 + W * H:16 + 3 * W * H], np.int16).reshape(H, W)
        assert np.array_equal(q, want)
        conf = np.frombuffer(blk[16 + 3 * W * H:], np.uint8).reshape(H, W)
        assert (conf[~ok] == 0).all() and conf[ok].max() > 0


@pytest.mark.gpu
def test_keypoints_csv(cli, oracle, golden_dir, tmp_path):
    needs_gpu()
    from doubleeye_b200 import synth
    p = synth.fronto_planes(424, 240, seed=12)
    H, W = p.left.shape
    p.left.tofile(tmp_path / "l.y8")
    p.right.tofile(tmp_path / "r.y8")
    r = run(cli, tmp_path / "l.y8", tmp_path / "r.y8", W, H, "--dmax", 64, "--iters", 4,
            "--keypoints", tmp_path / "kp.csv")
    assert r.returncode == 0, r.stderr
    line = [ln for ln in r.stdout.decode().splitlines() if ln.startswith("keypoints:")][0]
    rows = open(tmp_path / "kp.csv").read().splitlines()
    assert rows[0] == "x,y,disparity,margin"
    od, om, _ = oracle.dense(O.default_cfg(dmax=64, iters=4), p.left, p.right, want_cand=False)
    kp = oracle.detect_fast(p.left, O.default_det_cfg())
    want = []
    for x, y, _, _ in kp:
        xi = min(max(int(np.float32(x) + np.float32(0.5)), 0), W - 1)
        yi = min(max(int(np.float32(y) + np.float32(0.5)), 0), H - 1)
        if od[yi, xi] > 0:
            want.append("%.2f,%.2f,%.4f,%.4f" % (x, y, od[yi, xi], om[yi, xi]))
    assert rows[1:] == want
    assert f"{len(kp)} detected" in line and f"{len(want)} carried" in line


@pytest.mark.gpu
def test_prior_flag(cli, oracle, tmp_path):
    needs_gpu()
    from doubleeye_b200 import synth
    p = synth.slanted_planes(200, 120, 47, seed=5, tag="prior")
    H, W = p.left.shape
    p.left.tofile(tmp_path / "l.y8")
    p.right.tofile(tmp_path / "r.y8")
    half = np.full((H // 2, W // 2), 11.25, np.float32)     # half resolution: doubled
    half.tofile(tmp_path / "p.f32")
    r = run(cli, tmp_path / "l.y8", tmp_path / "r.y8", W, H, "--dmax", 48, "--iters", 8,
            "--prior", tmp_path / "p.f32", "--band", 3, "--out", tmp_path / "d.f32")
    assert r.returncode == 0, r.stderr
    full = np.full((H, W), 22.5, np.float32)
    d, _, _ = oracle.dense_prior(O.default_cfg(dmax=48, iters=8), p.left, p.right, full, 3)
    assert np.fromfile(tmp_path / "d.f32", np.float32).tobytes() == d.tobytes()
    bad = full.copy()
    bad[3, 3] = np.nan
    bad.tofile(tmp_path / "bad.f32")
    r = run(cli, tmp_path / "l.y8", tmp_path / "r.y8", W, H, "--prior", tmp_path / "bad.f32")
    assert r.returncode == 1 and b"holes" in r.stderr
