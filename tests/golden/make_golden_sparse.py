"""Generate the sparse-path golden vectors in tests/golden/ from the reference itself.

Runs only where the reference tree is present.  C++ fixtures come from the
reference compiled from its own sources (oracle/_ref/libref.so: detect_keypoints_fast,
census_at, match_masda, match_brute_force); Python fixtures from the reference's own
article/masda_stereo.py and article/dense_masda.py, imported in place (matplotlib is
absent here and those modules only plot with it, so a stub module stands in).  The
committed .npz files are what the tests read; nothing at test time needs the
reference tree.

    python tests/golden/make_golden_sparse.py
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402
from doubleeye_b200 import synth  # noqa: E402

ARTICLE = os.path.join(O.reference_root(), "article")
SCENES = os.path.join(ARTICLE, "scenes")


def reference_python():
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    plt.__getattr__ = lambda name: (lambda *a, **k: None)
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.path.insert(0, ARTICLE)
    import dense_masda  # noqa: E402
    import masda_stereo  # noqa: E402
    return masda_stereo, dense_masda


def describe(ref, img, kp, hw, hh):
    return np.array([ref.census_at(img, int(x + 0.5), int(y + 0.5), hw, hh)[0]
                     for x, y in kp[:, :2]], np.uint64)


def match_cfg_arrays(cfgs):
    return np.array([[getattr(c, f) for f, _ in c._fields_] for c in cfgs], np.float64)


def stats_array(st):
    return np.array([st.left, st.right, st.candidates, st.iterations_run, st.converged,
                     st.final_max_delta, st.oscillating], np.float64)


def cpp_case(ref, name, L, R, det, cfgs, hw=3, hh=3):
    kl = ref.detect_fast(L, det)
    kr = ref.detect_fast(R, det)
    dl = describe(ref, L, kl, hw, hh)
    dr = describe(ref, R, kr, hw, hh)
    out = dict(L=L, R=R, det=np.array([getattr(det, f) for f, _ in det._fields_], np.float64),
               census=np.array([hw, hh]), kl=kl, kr=kr, dl=dl, dr=dr,
               match_cfgs=match_cfg_arrays(cfgs))
    for k, c in enumerate(cfgs):
        m, st = ref.match_masda(kl, dl, kr, dr, c)
        out[f"matches_{k}"] = m
        out[f"stats_{k}"] = stats_array(st)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return len(kl), len(kr), [len(out[f"matches_{k}"]) for k in range(len(cfgs))]


def small_problems(ref, n_problems=60):
    """Random 3..5 x 3..5 problems shaped like core/tests/test_match.cpp:115-168."""
    rng = synth.rng_for("golden:bruteforce")
    rows = []
    kls, krs, dls, drs, res_m, res_b = [], [], [], [], [], []
    cfg = O.default_match_cfg(max_disparity=100.0, w_y=0.0, iterations=60, lambda_=0.05,
                              gamma=0.0)

    def desc_with(nbits, off):
        d = 0
        for b in range(nbits):
            d |= 1 << ((b + off) % 48)
        return d

    for t in range(n_problems):
        n, m = 3 + t % 3, 3 + (t // 3) % 3
        kl = np.zeros((n, 4), np.float32)
        kr = np.zeros((m, 4), np.float32)
        kl[:, 0] = rng.uniform(20, 120, n).astype(np.float32) + np.float32(60)
        kr[:, 0] = rng.uniform(20, 120, m).astype(np.float32)
        kl[:, 1] = kr[:, 1] = 50.0
        kl[:, 2:] = kr[:, 2:] = 10.0
        dl = np.array([desc_with(int(rng.integers(6, 31)), int(rng.integers(0, 48)))
                       for _ in range(n)], np.uint64)
        dr = np.array([desc_with(int(rng.integers(6, 31)), int(rng.integers(0, 48)))
                       for _ in range(m)], np.uint64)
        a, _ = ref.match_masda(kl, dl, kr, dr, cfg)
        b = ref.match_brute_force(kl, dl, kr, dr, cfg)
        rows.append((n, m, len(a), len(b)))
        kls.append(kl); krs.append(kr); dls.append(dl); drs.append(dr)
        res_m.append(a); res_b.append(b)
    off_l = np.cumsum([0] + [len(k) for k in kls])
    off_r = np.cumsum([0] + [len(k) for k in krs])
    off_m = np.cumsum([0] + [len(k) for k in res_m])
    off_b = np.cumsum([0] + [len(k) for k in res_b])
    np.savez_compressed(os.path.join(HERE, "sparse_bruteforce.npz"),
                        kl=np.concatenate(kls), kr=np.concatenate(krs),
                        dl=np.concatenate(dls), dr=np.concatenate(drs),
                        off_l=off_l, off_r=off_r, off_m=off_m, off_b=off_b,
                        masda=np.concatenate(res_m), brute=np.concatenate(res_b),
                        cfg=match_cfg_arrays([cfg]))
    return len(rows)


def python_cases(ms, dm):
    """build_problem / masda / masda_sparse / dense_problem on small seeded inputs."""
    out = {}
    p = synth.fronto_planes(256, 160, seed=31, planes=(8, 24, 40))
    ref = O.Reference()
    det = O.default_det_cfg(cell=24)
    kl = ref.detect_fast(p.left, det)
    kr = ref.detect_fast(p.right, det)
    pl, pr = kl[:, :2].copy(), kr[:, :2].copy()
    dl = ms.census(p.left, pl)
    dr = ms.census(p.right, pr)
    S = ms.build_problem(pl, dl, pr, dr, max_dy=1.5, dmin=1.0, dmax=60.0)
    a_dense, h_dense = ms.masda(S, lam=-0.1, gam=-0.1, iters=30, damping=0.4, eps=1e-5)
    ei, ej, se = ms.to_edges(S)
    m, n = S.shape
    a_sp, h_sp = ms.masda_sparse(ei, ej, se, m, n, -0.1, -0.1, iters=30, damping=0.4,
                                 eps=1e-5)
    to_arr = lambda d, k: np.array([d.get(i, -1) for i in range(k)], np.int64)  # noqa
    out.update(kp_pl=pl, kp_pr=pr, kp_dl=dl, kp_dr=dr, kp_S=S,
               kp_masda=to_arr(a_dense, m), kp_masda_hist=h_dense,
               kp_sparse=to_arr(a_sp, m), kp_sparse_hist=h_sp)

    q = synth.slanted_planes(72, 40, 15, seed=32, tag="golden-dense-problem")
    ei, ej, se, nn = dm.dense_problem(q.left, q.right, 1, 12)
    a_dp, h_dp = ms.masda_sparse(ei, ej, se, nn, nn, -0.1, -0.1, iters=6)
    out.update(dp_L=q.left, dp_R=q.right, dp_ei=ei, dp_ej=ej, dp_se=se,
               dp_assign=to_arr(a_dp, nn), dp_hist=h_dp)

    rng = synth.rng_for("golden:segmax")
    vals = rng.integers(-3, 4, 400).astype(np.float64)      # many ties on purpose
    idx = rng.integers(0, 37, 400).astype(np.int64)
    out.update(seg_vals=vals, seg_idx=idx, seg_out=ms._seg_max_excluding(vals, idx, 37))
    hx = rng.integers(0, 2**63, 50, dtype=np.int64).astype(np.uint64)
    hy = rng.integers(0, 2**63, 50, dtype=np.int64).astype(np.uint64)
    out.update(ham_a=hx, ham_b=hy, ham=ms.hamming(hx, hy))
    np.savez_compressed(os.path.join(HERE, "py_masda.npz"), **out)
    return {k: v.shape for k, v in out.items() if k in ("kp_S", "dp_ei")}


def main() -> None:
    O.build(ref=True)
    ref = O.Reference()
    cfgs = [O.default_match_cfg(),
            O.default_match_cfg(lambda_=-0.1, gamma=-0.1, iterations=10, max_candidates=8),
            O.default_match_cfg(max_dy=3.0, sigma_y=0.5, damping=0.0, lambda_=0.1)]
    p = synth.fronto_planes(320, 240, seed=21, planes=(8, 24, 52))
    print("sparse_c1", cpp_case(ref, "sparse_c1", p.left, p.right,
                                O.default_det_cfg(cell=24), cfgs))
    q = synth.fronto_planes(256, 192, seed=22, planes=(6, 30))
    print("sparse_c1_9x7", cpp_case(ref, "sparse_c1_9x7", q.left, q.right,
                                    O.default_det_cfg(per_cell=6, subpixel=0), cfgs[:2], 4, 3))
    path = os.path.join(SCENES, "morning_on")
    if os.path.isdir(path):
        L = np.fromfile(os.path.join(path, "left.y8"), np.uint8).reshape(480, 848)
        R = np.fromfile(os.path.join(path, "right.y8"), np.uint8).reshape(480, 848)
        L, R = L[120:360, 200:520].copy(), R[120:360, 200:520].copy()
        print("sparse_real", cpp_case(ref, "sparse_real", L, R, O.default_det_cfg(), cfgs))
    print("bruteforce", small_problems(ref))
    ms, dm = reference_python()
    print("python", python_cases(ms, dm))


if __name__ == "__main__":
    main()
