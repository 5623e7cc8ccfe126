"""Seeded synthetic stereo pairs with exact ground-truth disparity.

The reference measures on Middlebury scenes that are not available here, and its own
article code generates procedural scenes for the same reason
(article/masda_stereo.py:27-39 ``rng_for``, :99-111 ``broadband_texture``, :177-204
``render_pair``).  This module follows that recipe -- per-purpose generators seeded
from a stable crc32 key, a fractal texture, a z-buffered forward warp so occlusions
appear by themselves -- vectorised so a 1920x1080 pair takes well under a second.

Scene families (the workload shapes the benchmarks are quoted on):

* ``fronto_planes``   three fronto-parallel planes at fixed disparities (sparse case)
* ``slanted_planes``  random slanted planes with a gradient bound, occlusion bands
                      refilled with fresh noise, gain/offset on the right image
* ``large_scene``     slanted planes plus thin foreground strips and low-texture
                      regions
* ``video``           a slanted-plane scene translating a few pixels per frame
"""
from __future__ import annotations

import dataclasses
import zlib

import numpy as np

BASE_SEED = 20261203


def rng_for(name: str, seed: int = BASE_SEED) -> np.random.Generator:
    """A generator per purpose, seeded from crc32 so it is stable across processes
    (Python's hash() is salted per process)."""
    return np.random.default_rng(zlib.crc32(f"doubleeye_b200:{seed}:{name}".encode()))


def _bilinear(coarse: np.ndarray, H: int, W: int, scale: float) -> np.ndarray:
    ys = np.arange(H, dtype=np.float64) / scale
    xs = np.arange(W, dtype=np.float64) / scale
    y0 = np.floor(ys).astype(np.int64)
    x0 = np.floor(xs).astype(np.int64)
    wy = (ys - y0)[:, None]
    wx = (xs - x0)[None, :]
    a = coarse[np.ix_(y0, x0)]
    b = coarse[np.ix_(y0, x0 + 1)]
    c = coarse[np.ix_(y0 + 1, x0)]
    d = coarse[np.ix_(y0 + 1, x0 + 1)]
    return (a * (1 - wx) + b * wx) * (1 - wy) + (c * (1 - wx) + d * wx) * wy


def value_noise(H: int, W: int, rng: np.random.Generator, mean=110.0, std=40.0,
                octaves=4, finest=1.5) -> np.ndarray:
    """Fractal value noise: octaves of bilinearly upsampled Gaussian grids, finest
    first, amplitudes halving as the grid coarsens, rescaled to mean/std (float)."""
    img = np.zeros((H, W), np.float64)
    scale, amp = finest, 1.0
    for _ in range(octaves):
        coarse = rng.normal(0.0, 1.0, (int(H / scale) + 3, int(W / scale) + 3))
        img += amp * _bilinear(coarse, H, W, scale)
        scale *= 2.7
        amp *= 0.6
    img = (img - img.mean()) / max(img.std(), 1e-9)
    return mean + std * img


def _voronoi_labels(H, W, seeds_xy: np.ndarray) -> np.ndarray:
    lab = np.zeros((H, W), np.int32)
    best = np.full((H, W), np.inf)
    ys = np.arange(H, dtype=np.float64)[:, None]
    xs = np.arange(W, dtype=np.float64)[None, :]
    for i, (sx, sy) in enumerate(seeds_xy):
        dist = (xs - sx) ** 2 + (ys - sy) ** 2
        m = dist < best
        best[m] = dist[m]
        lab[m] = i
    return lab


def slanted_disparity(H, W, rng, n_planes=12, dlo=0.0, dhi=127.0, max_grad=0.15):
    """Piecewise-planar disparity on a Voronoi partition: each cell a plane
    d = d0 + gx (x - cx) + gy (y - cy), |gx|, |gy| <= max_grad, clipped to [dlo, dhi]."""
    seeds = np.stack([rng.uniform(0, W, n_planes), rng.uniform(0, H, n_planes)], 1)
    d0 = rng.uniform(dlo, dhi, n_planes)
    g = rng.uniform(-max_grad, max_grad, (n_planes, 2))
    lab = _voronoi_labels(H, W, seeds)
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float64)
    d = d0[lab] + g[lab, 0] * (xs - seeds[lab, 0]) + g[lab, 1] * (ys - seeds[lab, 1])
    return np.clip(d, dlo, dhi)


def forward_warp(left: np.ndarray, disp: np.ndarray):
    """Right view by z-buffered forward warp: left pixel x lands at round(x - d); where
    several land on one right pixel the nearest surface (largest d) wins.  Returns the
    warped image and the mask of right pixels that received nothing (disocclusions)."""
    H, W = left.shape
    xs = np.broadcast_to(np.arange(W), (H, W))
    ys = np.broadcast_to(np.arange(H)[:, None], (H, W))
    xr = np.rint(xs - disp).astype(np.int64)
    ok = (xr >= 0) & (xr < W)
    tgt = (ys * W + xr)[ok]
    dv = disp[ok]
    src = left[ok]
    order = np.lexsort((dv, tgt))          # by target, then disparity ascending
    tgt_s = tgt[order][::-1]               # reversed: largest disparity first per target
    first = np.unique(tgt_s, return_index=True)[1]
    right = np.zeros(H * W, np.float64)
    filled = np.zeros(H * W, bool)
    right[tgt_s[first]] = src[order][::-1][first]
    filled[tgt_s[first]] = True
    return right.reshape(H, W), ~filled.reshape(H, W)


def _finish(left_f, right_f, rng, noise, gain=0.0, offset=0.0):
    left = left_f + rng.normal(0.0, noise, left_f.shape) if noise > 0 else left_f
    right = right_f * (1.0 + gain) + offset
    if noise > 0:
        right = right + rng.normal(0.0, noise, right_f.shape)
    return (np.clip(np.rint(left), 0, 255).astype(np.uint8),
            np.clip(np.rint(right), 0, 255).astype(np.uint8))


@dataclasses.dataclass
class Pair:
    left: np.ndarray
    right: np.ndarray
    disparity: np.ndarray     # ground truth for the left view, float32
    visible: np.ndarray       # left pixels whose match is visible in the right view
    dmax: int

    @property
    def shape(self):
        return self.left.shape


def _visible(disp: np.ndarray) -> np.ndarray:
    """Left pixels that won the z-buffer at their landing position."""
    H, W = disp.shape
    xr = np.rint(np.arange(W)[None, :] - disp).astype(np.int64)
    vis = (xr >= 0) & (xr < W)
    best = np.full((H, W), -1.0)
    ys = np.broadcast_to(np.arange(H)[:, None], (H, W))
    np.maximum.at(best, (ys[vis], xr[vis]), disp[vis])
    vis2 = np.zeros_like(vis)
    vis2[vis] = best[ys[vis], xr[vis]] <= disp[vis] + 1e-9
    return vis2


def fronto_planes(W=848, H=480, seed=BASE_SEED, planes=(8, 24, 52), noise=2.0) -> Pair:
    """Value-noise texture (mean 110, std 40) over fronto-parallel planes: the first
    disparity is the background, the others nested rectangles; right = z-buffered
    warp + N(0, noise^2), clipped to u8."""
    rng = rng_for(f"fronto:{W}x{H}", seed)
    tex = value_noise(H, W, rng)
    disp = np.full((H, W), float(planes[0]))
    for i, dv in enumerate(planes[1:], 1):
        x0 = int(W * (0.1 + 0.25 * (i - 1)))
        y0 = int(H * (0.15 + 0.1 * (i - 1)))
        disp[y0:y0 + int(H * 0.45), x0:x0 + int(W * 0.3)] = float(dv)
    right_f, holes = forward_warp(tex, disp)
    right_f[holes] = value_noise(H, W, rng_for(f"fronto:fill:{W}x{H}", seed))[holes]
    left, right = _finish(tex, right_f, rng, noise)
    return Pair(left, right, disp.astype(np.float32), _visible(disp), int(max(planes)) + 1)


def slanted_planes(W=848, H=480, dmax=127, seed=BASE_SEED, n_planes=12, max_grad=0.15,
                   gain_offset=0.05, noise=2.0, tag="slanted") -> Pair:
    """Random slanted planes with disparity in [0, dmax]; disoccluded right pixels
    are refilled with fresh noise; a +-gain_offset gain and offset is applied to the
    right image."""
    rng = rng_for(f"{tag}:{W}x{H}:{dmax}", seed)
    tex = value_noise(H, W, rng)
    disp = slanted_disparity(H, W, rng, n_planes, 0.0, float(dmax), max_grad)
    right_f, holes = forward_warp(tex, disp)
    fresh = value_noise(H, W, rng_for(f"{tag}:fill:{W}x{H}", seed))
    right_f[holes] = fresh[holes]
    gain = rng.uniform(-gain_offset, gain_offset)
    offset = rng.uniform(-gain_offset, gain_offset) * 110.0
    left, right = _finish(tex, right_f, rng, noise, gain, offset)
    return Pair(left, right, disp.astype(np.float32), _visible(disp), dmax)


def large_scene(W=1500, H=1000, dmax=255, seed=BASE_SEED, strips=12, low_texture=0.2,
                noise=2.0) -> Pair:
    """Slanted planes in [0, dmax] plus thin foreground strips 2-6 px wide and
    low-texture regions (texture std 4) covering ~low_texture of the image."""
    rng = rng_for(f"large:{W}x{H}:{dmax}", seed)
    tex = value_noise(H, W, rng)
    # low-texture blobs: large Voronoi cells whose texture is flattened to std 4
    nb = 40
    lab = _voronoi_labels(H, W, np.stack([rng.uniform(0, W, nb), rng.uniform(0, H, nb)], 1))
    sizes = np.bincount(lab.ravel(), minlength=nb) / float(H * W)
    flat = np.zeros(nb, bool)
    acc = 0.0
    for c in rng.permutation(nb):
        if acc >= low_texture:
            break
        flat[c] = True
        acc += sizes[c]
    fm = flat[lab]
    tex[fm] = 110.0 + (tex[fm] - 110.0) * (4.0 / 40.0)
    disp = slanted_disparity(H, W, rng, 12, 0.0, float(dmax) * 0.8, 0.15)
    for _ in range(strips):
        wd = int(rng.integers(2, 7))
        if rng.random() < 0.5:
            x0 = int(rng.integers(0, W - wd))
            y0, y1 = sorted(rng.integers(0, H, 2))
            disp[y0:y1 + 1, x0:x0 + wd] = rng.uniform(0.8 * dmax, dmax)
        else:
            y0 = int(rng.integers(0, H - wd))
            x0, x1 = sorted(rng.integers(0, W, 2))
            disp[y0:y0 + wd, x0:x1 + 1] = rng.uniform(0.8 * dmax, dmax)
    right_f, holes = forward_warp(tex, disp)
    right_f[holes] = value_noise(H, W, rng_for(f"large:fill:{W}x{H}", seed))[holes]
    gain = rng.uniform(-0.05, 0.05)
    left, right = _finish(tex, right_f, rng, noise, gain, rng.uniform(-5, 5))
    return Pair(left, right, disp.astype(np.float32), _visible(disp), dmax)


class Video:
    """A seeded camera stream: one slanted-plane scene, wider than the frame, that
    translates ``speed`` px per frame (1-3) with fresh sensor noise each frame."""

    def __init__(self, W, H, dmax, stream_id: int, seed=BASE_SEED, noise=2.0):
        self.W, self.H, self.dmax, self.noise = W, H, dmax, noise
        rng = rng_for(f"video:{stream_id}:{W}x{H}:{dmax}", seed)
        self.speed = int(rng.integers(1, 4))
        self.pad = 3 * 600 + 8
        WW = W + self.pad
        self.tex = value_noise(H, WW, rng)
        self.disp = slanted_disparity(H, WW, rng, 12, 0.0, float(dmax), 0.15)
        self.gain = rng.uniform(-0.05, 0.05)
        self.stream_id = stream_id
        self.seed = seed

    def frame(self, t: int) -> Pair:
        x0 = (t * self.speed) % (self.pad - 8)
        tex = self.tex[:, x0:x0 + self.W]
        disp = self.disp[:, x0:x0 + self.W]
        right_f, holes = forward_warp(tex, disp)
        right_f[holes] = tex[holes]
        rng = rng_for(f"video:noise:{self.stream_id}:{t}", self.seed)
        left, right = _finish(tex, right_f, rng, self.noise, self.gain, 0.0)
        return Pair(left, right, disp.astype(np.float32), _visible(disp), self.dmax)


# The benchmark's pair shapes for the uneven batch: (W, H) -> D.
BATCH_SHAPES = {(320, 240): 64, (640, 480): 128, (848, 480): 128, (1280, 720): 256,
                (1920, 1080): 256}


def _slanted_job(args):
    W, H, dmax, seed, tag = args
    return slanted_planes(W, H, dmax, seed=seed, tag=tag)


def batch_pairs(n=64, seed=BASE_SEED, shapes=None, workers: int = 0):
    """n distinct pairs with sizes drawn uniformly (seed-fixed) from BATCH_SHAPES, each
    from the slanted-plane generator (its own seed) with disparity range 0..D-1
    matched to its size.  workers > 1 generates them in that many spawned processes
    (the same pairs, in the same order)."""
    shapes = list((shapes or BATCH_SHAPES).items())
    rng = rng_for("batch-draw", seed)
    jobs = []
    for i in range(n):
        (W, H), D = shapes[int(rng.integers(0, len(shapes)))]
        jobs.append((W, H, D - 1, seed + i, f"batch{i}"))
    if workers > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_slanted_job, jobs))
    return [_slanted_job(j) for j in jobs]
