"""Benchmark: dense MASDA stereo at 848x480, D=128, 8 BP iterations (pairs/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--pairs-per-step B]

A step is one batched pass of the whole hot path (census -> cost -> 4-pass filter
-> top-2 -> row solve) over B distinct seeded 848x480 pairs already resident in HBM.
``value`` is whole-job pairs/s (all ranks).  Multi-GPU runs are independent replicas
(pairs need no exchange): each rank matches its own B pairs per step; timing is the
max over ranks of CUDA-event time.  ``e2e`` is the same metric through the public
host API (page-locked host arrays in and out, the copies inside the timed region).

``--impl reference`` times the reference's own CPU implementation of the path
(oracle/_ref, the reference compiled from its sources; else this repository's C
restatement) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

W, H, D, ITERS = 848, 480, 128, 8
METRIC = "stereo pairs/s, dense MASDA 848x480 D=128 8 BP iters"


def disp_evals(n_pairs: int) -> float:
    return float(n_pairs) * W * H * D


# Algorithmic bytes per pair and per stage: compulsory
# traffic of each kernel if every operand is touched once.
WH = W * H
E = WH * D
ALG_BYTES = {
    "census": 2 * WH + 16 * WH + 4 * WH,        # read L,R; write census words, ax, ay
    "rows": 16 * WH + 2 * WH + 2 * E,           # read census words + ax; write volume
    "cols": 2 * E + 2 * WH + 12 * WH,           # read volume + ay; write candidates
    "solve": 12 * WH + 9 * WH,                  # read candidates; write disp, margin, conf
    "pipeline": 2 * WH + 4 * E + 24 * WH + 8 * WH,
}
STAGES = ["census", "rows", "cols", "solve"]

# Algorithmic 32-bit integer operations per pair (the arithmetic roof of the
# integer stages; tensor cores do not apply).  Per disparity evaluation: rows =
# census XOR 2 + POPC 2 + table 1 + |dI| 2 + table 1 + blend 3 (score, 11) + two
# recursive-filter steps 2 x 5 + int16 pack/unpack 2 = 23; cols = two filter steps
# 2 x 5 + top-2 key and insert 4 = 14.  Census: 48 compare-and-set per pixel per
# image.  The solve is latency-bound and has no arithmetic roof here.  Of the row
# stage's ops, 2 per evaluation are POPC (48-bit census words), which run on their
# own, slower pipe: a second, separate bound.
ALG_INT_OPS = {"census": 2 * 48 * 2 * WH, "rows": 23 * E, "cols": 14 * E}
ALG_POPC = {"rows": 2 * E}
# Integer pipe rates are measured on the device at start-up (de_int_probe): the
# integer roof is the rate of add.u32, which issues to both integer-capable pipes
# (the most lane operations per clock any integer mix reaches); POPC has its own.
PROBE_OPS = {"add_u32": 0, "lop3": 1, "shf": 2, "mad_lo": 3, "popc": 4}


def measure_int_rates(device: int) -> dict:
    """Lane operations per SM clock of each probed op (de_int_probe), timed with
    CUDA events; the SM clock is sampled around the probe."""
    import torch
    from doubleeye_b200._lib import probe_lib
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    out = {}
    with ClockSampler(device) as clk:
        for name, op in PROBE_OPS.items():
            ms, n = C.c_float(), C.c_double()
            if probe_lib().de_int_probe(op, 1000 if name == "popc" else 3000, None,
                                  C.byref(ms), C.byref(n)) != 0:
                return {}
            out[name] = n.value / (ms.value * 1e-3) / sms
    mhz = clk.summary().get("sm_mhz") or 1965.0
    return {k: round(v / (mhz * 1e6), 2) for k, v in out.items()} | {"sm_mhz": mhz}


def load_peaks() -> dict:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


def ncu_traffic() -> dict:
    p = os.path.join(REPO, "profiles", "ncu_dram_bytes.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region:
    every 5 ms through NVML in a thread (read-only queries), else nvidia-smi every
    100 ms.  The NVML device is the CUDA device's, matched by PCI bus id."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.samples: list[tuple[float, float, int]] = []      # (sm MHz, max MHz, reasons)
        self.lines: list[str] = []

    def _nvml_handle(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return None

    def __enter__(self):
        h = self._nvml_handle()
        if h is not None:
            self.nvml = h
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nvml
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), mx,
                                     int(get_reasons(h))))
            except Exception:
                break
            self.stop.wait(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            self.t.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        for c, m, r in self.samples:
            sm.append(c)
            mx.append(m)
            reasons |= {n for n, bit in self.REASONS.items() if r & bit}
        names = list(self.REASONS)
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def make_pairs(n: int, seed0: int):
    from doubleeye_b200 import synth
    return [synth.slanted_planes(W, H, D - 1, seed=seed0 + i, tag="bench") for i in range(n)]


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, ws: int) -> float:
    from doubleeye_b200.replicas import max_over_ranks as mor
    return mor(x) if ws > 1 else x


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_sample(reps: int = 5) -> dict:
    """The reference's CPU path (run_dense, core/tools/de_dense.cpp:738) on this host:
    one 848x480 D=128 pair, 8 iterations, timed at all host threads and at one thread
    (the reference's deterministic form), the two interleaved, `reps` times each; the
    minimum is the reported time and the spread is kept."""
    from oracle import oracle as O
    nthreads = os.cpu_count() or 1
    pair = make_pairs(1, 900)[0]
    cfg = O.default_cfg(dmax=D, iters=ITERS)
    if O.Reference.available():
        ref = O.Reference()
        run = lambda nt: ref.dense(cfg, pair.left, pair.right, nthreads=nt, want_cand=False)  # noqa
        kind = "reference"
    else:
        orc = O.Oracle()
        run = lambda nt: orc.dense(cfg, pair.left, pair.right, want_cand=False)  # noqa
        kind, nthreads = "port", 1
    run(nthreads)                                  # warm caches and thread pool
    t_all, t_one = [], []
    for _ in range(reps):
        for nt, acc in ((nthreads, t_all), (1, t_one)):
            t0 = time.perf_counter()
            run(nt)
            acc.append(time.perf_counter() - t0)
    spread = lambda v: {"min_s": min(v), "median_s": sorted(v)[len(v) // 2],  # noqa: E731
                        "max_s": max(v)}
    return {"value": 1.0 / min(t_all), "unit": "pairs/s", "cores": nthreads, "kind": kind,
            "cpu_model": cpu_model(), "python_entry": py_entry_cpu(),
            "single_thread_pairs_per_s": 1.0 / min(t_one),
            "all_threads": spread(t_all), "one_thread": spread(t_one),
            "sample": f"one 848x480 D=128 iters 8 pair, {reps} interleaved repetitions at "
                      f"{nthreads} and 1 thread(s), minimum reported, "
                      f"{'reference run_dense' if kind == 'reference' else 'oracle port'}"}


def py_entry_cpu(iters: int = 3) -> dict:
    """The Python entry points' max-sum (article/masda_stereo.py masda_sparse, float64)
    on one host core: the oracle's C restatement over the same 450x375, disparities
    1..60 edge list the GPU leg solves (built by this build's dense_problem, which is
    bit-exact to the reference's), for `iters` of the 12 iterations, and the 12-iteration
    time scaled from them."""
    import numpy as np
    from doubleeye_b200 import dense_masda, synth
    from oracle import oracle as O
    p = synth.slanted_planes(450, 375, 59, seed=11, tag="py-entry")
    ei, ej, se, n = dense_masda.dense_problem(p.left, p.right, 1, 60)
    se = se.astype(np.float64)
    orc = O.Oracle()
    t0 = time.perf_counter()
    orc.masda_edges(ei, ej, se, n, n, -0.1, -0.1, iters, 0.4, 1e-9)
    t = time.perf_counter() - t0
    return {"kind": "port", "cores": 1, "edges": int(se.shape[0]), "iterations_timed": iters,
            "masda_sparse_ms": t * 1e3, "masda_sparse_12_iterations_ms_scaled": t * 1e3 * 12 / iters}


def run_reference(args) -> None:
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    nthreads = os.cpu_count() or 1
    cfg = O.default_cfg(dmax=D, iters=ITERS)
    pairs = make_pairs(args.ref_sample, 0)
    if O.Reference.available():
        ref = O.Reference()
        run = lambda p: ref.dense(cfg, p.left, p.right, nthreads=nthreads, want_cand=False)  # noqa
        kind, cores, what = "reference", nthreads, "reference run_dense (core/tools/de_dense.cpp)"
    else:
        orc = O.Oracle()
        run = lambda p: orc.dense(cfg, p.left, p.right, want_cand=False)  # noqa
        kind, cores, what = "port", 1, "oracle C restatement"
    for _ in range(args.warmup):
        for p in pairs:
            run(p)
    steps = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ts = time.perf_counter()
        for p in pairs:
            run(p)
        steps.append(time.perf_counter() - ts)
    dt = time.perf_counter() - t0
    steps.sort()
    n = args.steps * len(pairs)
    v = n / dt
    out = {"metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "i16/f32",
           "data": "synthetic (seeded slanted planes)", "impl": "reference",
           "config": {"workload": "dense 848x480 D=128 iters=8", "W": W, "H": H, "D": D,
                      "iters": ITERS, "pairs_per_step": len(pairs), "parallelism": "cpu"},
           "g_disp_evals_per_s": disp_evals(n) / dt / 1e9,
           "step_ms": {"min": steps[0] * 1e3, "median": steps[len(steps) // 2] * 1e3,
                       "max": steps[-1] * 1e3},
           "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": kind,
                            "cpu_model": cpu_model(),
                            "sample": f"{len(pairs)} pairs per step, {what}, "
                                      f"{cores} thread(s)"},
           "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_c4(de, local: int, steps: int, warmup: int, c4_set) -> dict:
    """Batched uneven workload: 64 distinct seeded pairs, sizes drawn uniformly (seed-
    fixed) from {320x240, 640x480, 848x480, 1280x720, 1920x1080} with D in {64, 128,
    256} matched to size, in one launch set (autotuned launch shapes, CUDA-graph
    replay) against one launch set per pair."""
    import torch
    from doubleeye_b200 import autotune, synth
    pairs = [(p, synth.BATCH_SHAPES[(p.left.shape[1], p.left.shape[0])]) for p in c4_set]
    cfg = de.Cfg(iters=ITERS)
    m = de.DenseMatcher(cfg, device=local)
    Ls = [torch.from_numpy(p.left).cuda() for p, _ in pairs]
    Rs = [torch.from_numpy(p.right).cuda() for p, _ in pairs]
    items = [(L, R, D, m.new_outputs(*L.shape)) for L, R, (_, D) in zip(Ls, Rs, pairs)]
    saved = autotune.current()
    knobs = m.tune_for(items)
    evals = sum(float(L.numel()) * D for L, (_, D) in zip(Ls, pairs))

    def timed(fn, reps):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_batch = timed(lambda: m.match_into(items), steps)
    g = m.capture(items)
    ms_graph = timed(g.launch, steps)
    g.close()
    ms_plain = timed(lambda: [m.match_into([it]) for it in items], max(1, steps // 2))
    autotune.apply(saved)
    sizes = {}
    for p, D in pairs:
        key = f"{p.left.shape[1]}x{p.left.shape[0]}/D{D}"
        sizes[key] = sizes.get(key, 0) + 1
    hbm_floor_ms = sum(2 * L.numel() + 4 * L.numel() * D + 32 * L.numel()
                       for L, (_, D) in zip(Ls, pairs)) / (load_peaks()["hbm_gbs"] * 1e6)
    best = min(ms_batch, ms_graph)
    return {"workload": "64 distinct pairs, uneven sizes and D in one launch set",
            "sizes": sizes, "pairs_per_s": 64 / (ms_batch / 1e3),
            "graph_pairs_per_s": 64 / (ms_graph / 1e3),
            "plain_pairs_per_s": 64 / (ms_plain / 1e3),
            "batch_over_plain": ms_plain / best,
            "g_disp_evals_per_s": evals / (best / 1e3) / 1e9,
            "ms_per_batch": best, "hbm_floor_ms": hbm_floor_ms,
            "frac_of_hbm_floor": hbm_floor_ms / best, "knobs": knobs,
            "data": "synthetic, 64 distinct seeded slanted-plane pairs"}


def run_py_entry(local: int) -> dict:
    """The reference's Python entry points on the GPU (float64, as NumPy): the dense
    edge list of a 450x375 pair at disparities 1..60 (article/dense_masda.py
    dense_problem) and max-sum over it, 12 iterations (article/masda_stereo.py
    masda_sparse), the configuration the reference quotes its NumPy time on."""
    import torch
    from doubleeye_b200 import dense_masda, masda_stereo, synth
    p = synth.slanted_planes(450, 375, 59, seed=11, tag="py-entry")
    out = {}
    for rep in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ei, ej, se, n = dense_masda.dense_problem(p.left, p.right, 1, 60, device=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        assign, hist = masda_stereo.masda_sparse(ei, ej, se, n, n, -0.1, -0.1, 12, 0.4, 1e-9)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out = {"workload": "450x375, disparities 1..60, 12 iterations (float64)",
               "edges": int(ei.shape[0]), "dense_problem_ms": (t1 - t0) * 1e3,
               "masda_sparse_ms": (t2 - t1) * 1e3, "total_ms": (t2 - t0) * 1e3}
    return out


def run_c5(de, local: int) -> dict:
    """Serving: 16 camera streams at 30 Hz (640x480 D=64 x8, 848x480 D=128 x7,
    1280x720 D=192 x1, Gaussian arrival jitter sigma 3 ms), then the same streams
    offered at 10x the rate to find the sustained throughput; the plain path is
    one synchronous host-API call per pair over the same frames."""
    from doubleeye_b200 import serve
    specs = serve.SERVING_STREAMS
    frames = serve.make_frames(specs, frames_per_stream=2)
    out = {"streams": "16 at 30 Hz: 640x480/D64 x8, 848x480/D128 x7, 1280x720/D192 x1",
           "outputs": "DEDD planes (Q4 disparity + confidence) per request"}
    with serve.Server(de.Cfg(iters=ITERS), device=local, hbm_budget=24 << 30, max_batch=16,
                      lanes=2) as sv:
        serve.simulate(sv, specs, frames, duration_s=0.5)              # warm-up
        out["at_30hz"] = serve.simulate(sv, specs, frames, duration_s=3.0)
        fast = [serve.StreamSpec(s.W, s.H, s.D, fps=300.0) for s in specs]
        out["at_300hz"] = serve.simulate(sv, fast, frames, duration_s=2.0)
    def plain_pass():
        n = 0
        for s, spec in enumerate(specs):
            for p in frames[s]:
                de.run_dense(p.left, p.right, de.Cfg(dmax=spec.D, iters=ITERS),
                             want_cand=False, device=local)
                n += 1
        return n
    plain_pass()                                       # warm-up: first launches, buffers
    t0 = time.perf_counter()
    n = plain_pass()
    out["plain_pairs_per_s"] = n / (time.perf_counter() - t0)
    out["served_over_plain"] = out["at_300hz"]["pairs_per_s"] / out["plain_pairs_per_s"]
    return out


def run_c1(de, local: int, steps: int, warmup: int) -> dict:
    """The sparse configuration: an 848x480 value-noise scene over fronto-parallel
    planes at 8/24/52 px, 9x7 census.  Keypoint path on the device (FAST detection in
    both images with 24-px cells, about 2100 keypoints each; census descriptors;
    keypoint MASDA, 10 BP iterations), timed as one device-resident pair with CUDA
    events; and the dense cost / filter / top-2 of the same pair at D=64 (no BP)."""
    import torch
    from doubleeye_b200 import sparse, synth
    p = synth.fronto_planes()
    dev = torch.device("cuda", local)
    L = torch.from_numpy(p.left).to(dev)
    R = torch.from_numpy(p.right).to(dev)
    sm = sparse.SparseMatcher(det=sparse.DetCfg(cell=24),
                              cfg=sparse.MatchCfg(iterations=10, census_bits=62),
                              census=(4, 3), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, n):
        for _ in range(warmup):
            r = fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, r

    pair_ms, res = timed(lambda: sm.match_pair(L, R), steps)
    det_ms, _ = timed(lambda: sm.detect(L), steps)
    out = {"workload": "848x480 fronto planes 8/24/52, 9x7 census, ~2100 keypoints, "
                       "keypoint MASDA 10 iterations",
           "sparse_pair_ms": pair_ms, "detect_ms_per_image": det_ms,
           "keypoints_left": int(res["nl"].item()), "keypoints_right": int(res["nr"].item()),
           "matches": int(res["n"].item())}
    m = de.DenseMatcher(de.Cfg(dmax=64, census_hw=4, census_hh=3), device=local)
    for B in (1, 16):
        items = [(L, R, 0, m.new_outputs(480, 848)) for _ in range(B)]
        ms, _ = timed(lambda: m.match_into(items), steps)
        out[f"dense_top2_pairs_per_s_b{B}"] = B / (ms / 1e3)
    return out


def run_c3(de, local: int, steps: int, warmup: int) -> dict:
    """The large configuration: 1500x1000, disparities 0-255, 12 BP iterations, thin
    strips and low-texture regions; device-timed, one pair and four pairs a launch."""
    import torch
    from doubleeye_b200 import synth
    p = synth.large_scene()
    cfg = de.Cfg(dmax=256, iters=12)
    m = de.DenseMatcher(cfg, device=local)
    L = torch.from_numpy(p.left).cuda()
    R = torch.from_numpy(p.right).cuda()
    out = {"workload": "1500x1000 D=256 iters=12 (strips, low texture)"}
    for B in (1, 4):
        items = [(L, R, 0, m.new_outputs(1000, 1500)) for _ in range(B)]
        for _ in range(warmup):
            m.match_into(items)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            m.match_into(items)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[f"pairs_per_s_b{B}"] = B / (ms / 1e3)
        out[f"g_disp_evals_per_s_b{B}"] = B * 1500 * 1000 * 256 / (ms / 1e3) / 1e9
    return out


def launch_sets(n: int) -> int:
    """Census/rows/columns/solve launch sets one batch of n pairs runs as: batches of at
    most 64 pairs, each split into up to `batch_streams` parts on concurrent streams."""
    from doubleeye_b200 import _lib
    parts = _lib.get_param("batch_streams")
    return sum(min(m, parts) for m in
               (min(64, n - first) for first in range(0, n, 64)))


def run_ours(args) -> None:
    import torch
    import doubleeye_b200 as de
    from doubleeye_b200 import build
    from doubleeye_b200._lib import check, lib
    build.build()
    ws, rank, local = dist_setup()
    B, K, Wm = args.pairs_per_step, args.steps, args.warmup
    from doubleeye_b200.replicas import rank_seed
    pairs = make_pairs(B, rank_seed(rank))
    c4_set = None
    if ws == 1 and not args.no_extras:              # 64 distinct pairs, host-generated
        from doubleeye_b200 import synth
        c4_set = synth.batch_pairs(64, seed=4, workers=min(16, os.cpu_count() or 1))
    cfg = de.Cfg(dmax=D, iters=ITERS)
    m = de.DenseMatcher(cfg, device=local)
    Ls = [torch.from_numpy(p.left).cuda() for p in pairs]
    Rs = [torch.from_numpy(p.right).cuda() for p in pairs]
    outs = [m.new_outputs(H, W) for _ in pairs]
    items = [(L, R, 0, o) for L, R, o in zip(Ls, Rs, outs)]
    stream = torch.cuda.current_stream()

    # --- device-timed batched throughput (the headline value) -----------------------
    # No instrumentation inside the timed region beyond one CUDA event per step (the
    # spread of step times); the stage split is taken in a separate pass below.
    for _ in range(Wm):
        m.match_into(items)
    torch.cuda.synchronize()
    barrier(ws)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier(ws)
        ev[0].record(stream)
        for k in range(K):
            m.match_into(items)
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
    barrier(ws)
    ms_local = ev[0].elapsed_time(ev[K])
    step_ms = sorted(ev[k].elapsed_time(ev[k + 1]) for k in range(K))
    ms = max_over_ranks(ms_local, ws)
    total_pairs = ws * B * K
    value = total_pairs / (ms / 1e3)

    # --- stage split (a separate pass with stage events between the kernels) ---------
    lib().de_stage_timing(1)
    Ks = min(K, 20)
    for _ in range(Ks):
        m.match_into(items)
    torch.cuda.synchronize()
    lib().de_stage_timing(0)
    stage = (C.c_float * 4)()
    nl = C.c_int()
    check(lib().de_stage_times(stage, 4, C.byref(nl)))

    # --- plain single-pair path, same device timing -------------------------------
    one = [items[0]]
    for _ in range(Wm):
        m.match_into(one)
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        m.match_into(one)
    e1.record(stream)
    torch.cuda.synchronize()
    plain = ws * K / (max_over_ranks(e0.elapsed_time(e1), ws) / 1e3)

    # --- end to end through the public host API -----------------------------------
    # inputs and outputs in page-locked host memory, moved by DMA inside the timed region
    host = []
    for p in pairs:
        hl, hr = de.pinned_empty(p.left.shape, np.uint8), de.pinned_empty(p.right.shape, np.uint8)
        hl[...] = p.left
        hr[...] = p.right
        host.append((hl, hr))
    res = de.new_results([p.left.shape for p in pairs], pinned=True)
    for _ in range(max(1, Wm // 2)):
        res = de.run_dense_batch(host, cfg, device=local, out=res)
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(K):
        res = de.run_dense_batch(host, cfg, device=local, out=res)
    e2e_s = max_over_ranks(time.perf_counter() - t0, ws)
    filled = float(np.mean([np.isfinite(r.disp).mean() for r in res]))

    # --- roofline of the dominant kernel ------------------------------------------
    per_launch = {st: stage[i] / max(1, nl.value) for i, st in enumerate(STAGES)}
    dom = max(STAGES, key=lambda s: per_launch[s])
    peaks = load_peaks()
    alg = ALG_BYTES[dom] * B                      # one launch processes B pairs
    achieved = alg / (per_launch[dom] / 1e3) / 1e9
    traffic = ncu_traffic().get(dom)
    roof = {"bound": "hbm", "kernel": f"k_{dom}", "achieved": achieved,
            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
            "peak_src": peaks["src"],
            "traffic": traffic * B if traffic is not None else None,
            "alg_bytes_per_launch": alg,
            "pipeline_frac": ALG_BYTES["pipeline"] * B * K / (ms / 1e3) / 1e9
            / peaks["hbm_gbs"] / ws}
    # the integer-arithmetic roof per stage, from the measured pipe rates at the clock
    # sampled during the timed run
    import torch
    clk_mhz = clk.summary().get("sm_mhz") or 1965.0
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    rates = measure_int_rates(local)
    if rates:
        int_peak = sms * rates["add_u32"] * clk_mhz * 1e6 / 1e12       # T ops/s
        popc_peak = sms * rates["popc"] * clk_mhz * 1e6 / 1e12
        roof["int_roof"] = {"lane_ops_per_clk_per_sm": rates}
        for st in ALG_INT_OPS:
            t = per_launch[st] / 1e3
            r = {"achieved_tops": ALG_INT_OPS[st] * B / t / 1e12, "peak_tops": int_peak,
                 "frac": ALG_INT_OPS[st] * B / t / 1e12 / int_peak}
            if st in ALG_POPC:
                r["popc_frac"] = ALG_POPC[st] * B / t / 1e12 / popc_peak
            roof["int_roof"][st] = r
    # the row solve has neither an HBM nor an integer roof worth the name (12 bytes in
    # and 9 out per pixel): it is bound by latency, one CTA per image row holding the
    # row's candidates in shared memory (49 bytes per pixel, five rows per SM at 848
    # pixels), with two block barriers per BP sweep
    roof["solve"] = {"us_per_pair": per_launch["solve"] * 1e3 / B, "bp_sweeps": ITERS,
                     "bound": "latency: shared-memory round trips and 2 block barriers "
                              "per BP sweep, 5 rows per SM"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": K,
               "warmup": Wm, "ms_per_step": ms / K, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "i16/f32",
               "data": "synthetic (seeded slanted planes, 12 planes, grad<=0.15, "
                       "occlusion refill, +-5% gain/offset)",
               "config": {"workload": "dense 848x480 D=128 iters=8", "W": W, "H": H, "D": D,
                          "iters": ITERS, "pairs_per_step": B,
                          "parallelism": f"replicas x{ws}" if ws > 1 else "single",
                          "l2": f"working set > L2 ({B} pairs x "
                                f"{m.workspace_bytes([(W, H, 0)]) / 1e6:.0f} MB)"},
               "g_disp_evals_per_s": disp_evals(total_pairs) / (ms / 1e3) / 1e9,
               "step_ms": {"min": step_ms[0], "median": step_ms[len(step_ms) // 2],
                           "max": step_ms[-1]},
               "plain_pairs_per_s": plain, "batch_over_plain": value / plain,
               "stage_ms_per_launch": per_launch, "filled": filled,
               "roofline": roof,
               "clocks": clk.summary(),
               "e2e": {"value": ws * B * K / e2e_s, "unit": "pairs/s",
                       "h2d_bytes_per_step": B * 2 * WH,
                       "d2h_bytes_per_step": B * 9 * WH},
               "gpu_launches": 4 * K * launch_sets(B)}
        if ws == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline_sample()
        if ws == 1 and not args.no_extras:
            Ke = min(K, 20)
            out["sparse_c1"] = run_c1(de, local, max(3, Ke // 2), Wm)
            out["large_c3"] = run_c3(de, local, max(3, Ke // 4), Wm)
            out["batched_c4"] = run_c4(de, local, Ke, Wm, c4_set)
            out["serving_c5"] = run_c5(de, local)
            out["python_entry"] = run_py_entry(local)
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--pairs-per-step", type=int, default=16)
    ap.add_argument("--ref-sample", type=int, default=2, help="pairs per reference step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched (C4) and serving (C5) sections")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
