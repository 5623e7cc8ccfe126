"""Serving many camera streams: the Python side of the C-ABI server (de_server_*).

``Server`` admits stereo pairs from any thread (host arrays, any supported size, a
camera-stream id each), batches what is waiting onto the GPU as lanes free up, and
returns each pair's disparity, margin, confidence and DEDD planes (Q4 disparity and
confidence, as core/tools/de_dense_cuda.cu:729-746 encodes them).  Results are the
plain pipeline's bit for bit.

``simulate`` drives a server with camera streams at a frame rate with timing jitter
(the serving workload: 16 streams at 30 Hz, 640x480 / 848x480 plus one 1280x720) and
reports p50/p99 submit-to-result latency and throughput.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
import time
from typing import Optional, Sequence

import numpy as np

from ._lib import DeCfg, check, lib


class DeServerCfg(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_size_t), ("max_batch", C.c_int),
                ("lanes", C.c_int)]


class DeServerReport(C.Structure):
    _fields_ = [("completed", C.c_ulonglong), ("failed", C.c_ulonglong),
                ("batches", C.c_ulonglong), ("mean_batch", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("max_pending", C.c_size_t)]


PLANES = {"disp": 1, "margin": 2, "conf": 4, "q4": 8, "qconf": 16}
PLANE_DTYPES = {"disp": np.float32, "margin": np.float32, "conf": np.uint8, "q4": np.int16,
                "qconf": np.uint8}


def _u8(a) -> np.ndarray:
    a = np.ascontiguousarray(a, np.uint8)
    if a.ndim != 2:
        raise ValueError("images must be 2-D uint8")
    return a


class Server:
    def __init__(self, cfg: Optional[DeCfg] = None, device: int = 0,
                 hbm_budget: int = 8 << 30, max_batch: int = 16, lanes: int = 2):
        from .dense import Cfg
        self.cfg = cfg or Cfg()
        sc = DeServerCfg()
        lib().de_server_cfg_default(C.byref(sc))
        sc.device, sc.hbm_budget, sc.max_batch, sc.lanes = device, hbm_budget, max_batch, lanes
        self._h = C.c_void_p()
        check(lib().de_server_create(C.byref(self.cfg), C.byref(sc), C.byref(self._h)))
        self._shape = {}
        self._mu = threading.Lock()

    def submit(self, stream: int, L, R, dmax: int = 0, planes=None) -> int:
        """Queue a pair; ``planes`` names the outputs that will be read (default all:
        disp, margin, conf, q4, qconf)."""
        L, R = _u8(L), _u8(R)
        H, W = L.shape
        names = tuple(planes) if planes else tuple(PLANES)
        mask = sum(PLANES[n] for n in names)
        t = C.c_ulonglong()
        check(lib().de_server_submit(self._h, int(stream), L.ctypes.data, R.ctypes.data, W, H,
                                     int(dmax), mask, C.byref(t)))
        with self._mu:
            self._shape[t.value] = (H, W, names)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60000, out: dict | None = None) -> dict:
        """Block for a result; ``out`` may supply the arrays to fill (reused across
        calls, no allocation)."""
        with self._mu:
            H, W, names = self._shape[ticket]
        if out is None or any(out.get(n) is None or out[n].shape != (H, W) for n in names):
            out = {n: np.empty((H, W), PLANE_DTYPES[n]) for n in names}
        ptr = lambda n: out[n].ctypes.data if n in names else None  # noqa: E731
        lat = C.c_double()
        check(lib().de_server_wait(self._h, C.c_ulonglong(ticket), int(timeout_ms),
                                   ptr("disp"), ptr("margin"), ptr("conf"), ptr("q4"),
                                   ptr("qconf"), C.byref(lat)))
        with self._mu:
            del self._shape[ticket]
        out["latency_ms"] = lat.value
        return out

    def stream_prior(self, stream: int, band: int = 2) -> None:
        """Match this camera stream's frames with its previous disparity map, hole-
        filled on the device, as the prior (the reference's --prior mask,
        core/tools/de_dense.cpp:797-853); band 0 turns it off.  Frames of such a stream
        run one at a time, in submission order."""
        check(lib().de_server_stream_prior(self._h, int(stream), int(band)))

    def stats(self) -> dict:
        r = DeServerReport()
        check(lib().de_server_stats(self._h, C.byref(r)))
        return {f: getattr(r, f) for f, _ in r._fields_}

    def reset_stats(self) -> None:
        check(lib().de_server_reset_stats(self._h))

    def last_disparity(self, stream: int, W: int, H: int) -> np.ndarray:
        out = np.empty((H, W), np.float32)
        check(lib().de_server_last_disparity(self._h, int(stream), out.ctypes.data, W, H))
        return out

    def close(self) -> None:
        if self._h:
            check(lib().de_server_destroy(self._h))
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class StreamSpec:
    W: int
    H: int
    D: int
    fps: float = 30.0


# The serving workload: 16 camera streams at 30 Hz, mixed 640x480 (D=64) and 848x480
# (D=128), plus one 1280x720 at D=192.
SERVING_STREAMS = ([StreamSpec(640, 480, 64)] * 8 + [StreamSpec(848, 480, 128)] * 7 +
                   [StreamSpec(1280, 720, 192)])


def make_frames(specs: Sequence[StreamSpec], frames_per_stream: int = 3, seed: int = 0):
    """Pre-rendered seeded video frames per stream (the scene translates 1-3 px per
    frame with fresh sensor noise); the simulation cycles through them."""
    from .synth import Video
    out = []
    for s, spec in enumerate(specs):
        v = Video(spec.W, spec.H, spec.D - 1, stream_id=s, seed=seed + 1)
        out.append([v.frame(t) for t in range(frames_per_stream)])
    return out


def simulate(server: Server, specs: Sequence[StreamSpec], frames, duration_s: float = 3.0,
             jitter_ms: float = 3.0, seed: int = 0, collectors: int = 4) -> dict:
    """Submit every stream's frames at its rate (period 1/fps plus Gaussian jitter of
    sigma jitter_ms, random phase per stream) for duration_s, collect all results (the
    live path's DEDD planes: Q4 disparity and confidence), and report the server's
    latency percentiles and the achieved throughput.  Each camera stream has its own
    submitting thread, as separate cameras would, so the offered load does not depend
    on one thread keeping up; ``offered_pairs_per_s`` is what was actually submitted
    per second of the submitting window."""
    import queue
    rng = np.random.default_rng(seed)
    schedules = []
    for s, spec in enumerate(specs):
        t = rng.uniform(0, 1.0 / spec.fps)
        ev = []
        k = 0
        while t < duration_s:
            ev.append((t + rng.normal(0, jitter_ms / 1e3), k))
            t += 1.0 / spec.fps
            k += 1
        schedules.append(sorted(ev))
    done = []
    errors = []
    pending = queue.Queue()
    submitted = [0] * len(specs)
    last_submit = [0.0] * len(specs)

    def collector():
        bufs = {}
        while True:
            item = pending.get()
            if item is None:
                return
            tk, shape = item
            try:
                bufs[shape] = server.wait(tk, out=bufs.get(shape))
                done.append(bufs[shape]["latency_ms"])
            except Exception as e:  # noqa: BLE001 - reported below
                errors.append(str(e))

    def camera(s):
        for at, k in schedules[s]:
            delay = at - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            p = frames[s][k % len(frames[s])]
            try:
                tk = server.submit(s, p.left, p.right, specs[s].D, planes=("q4", "qconf"))
            except Exception as e:  # noqa: BLE001 - reported below
                errors.append(str(e))
                continue
            pending.put((tk, p.left.shape))
            submitted[s] += 1
            last_submit[s] = time.perf_counter() - t0

    cols = [threading.Thread(target=collector) for _ in range(collectors)]
    for th in cols:
        th.start()
    server.reset_stats()
    t0 = time.perf_counter()
    cams = [threading.Thread(target=camera, args=(s,)) for s in range(len(specs))]
    for th in cams:
        th.start()
    for th in cams:
        th.join()
    window = max(max(last_submit), 1e-9)
    for _ in cols:
        pending.put(None)
    for th in cols:
        th.join()
    wall = time.perf_counter() - t0
    st = server.stats()
    requests = sum(len(x) for x in schedules)
    return {"requests": requests, "completed": int(st["completed"]),
            "failed": int(st["failed"]) + len(errors), "wall_s": wall,
            "submit_window_s": window,
            "pairs_per_s": st["completed"] / wall, "p50_ms": st["p50_ms"],
            "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
            "mean_batch": st["mean_batch"], "batches": int(st["batches"]),
            "scheduled_pairs_per_s": requests / duration_s,
            "offered_pairs_per_s": sum(submitted) / window}
