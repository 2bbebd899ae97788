"""Benchmark of the batched FFT library on B200.

Output: JSON lines on rank 0.  Every line but the last is a sub-measurement tagged "sub"; the
LAST line is the headline (kept under 2 KB), and the line before it ("sub": "summary") holds the
key figures of every sub-measurement, so both survive a reader that keeps only the end of the
output.

Headline workload (the configuration the metric is quoted on): plain fp32 C2C forward over the
49-point grid N in {64..4096} x batch in {1..4096}, interleaved complex, Re/Im i.i.d. N(0,1)
seeded per point (seed = 1000*log2 N + log2 batch + 1).  One step = one forward transform of
every grid point on inputs resident in HBM, run as ONE ragged launch (k_ragged_flat over the 49
requests: 10,931 tiles of 4096 or 2048 points, one per CTA).  The step touches 355 MB of input
and 355 MB of output, more than the 126 MB L2, so no explicit flush is needed between steps.

  value      algorithmic bytes (16 * N * batch summed over the grid) / device time per step
  e2e        the same metric through the C ABI's synchronous host-pointer entry point with
             pinned host buffers, H2D + kernels + D2H inside the timed step (the whole grid in
             one bfly_plan_run_c2c_many call); `scopes` splits it into event spans
  roofline   the step's only kernel timed with CUDA events on its stream against the measured
             HBM copy bandwidth
  cpu_baseline  the reference's own CPU FFT (its FP64 oracle src/framework/reference.cpp,
             compiled from its sources into oracle/_ref) on a bounded sample of the grid

Sub-measurements (one line each): c2c_grid49_points (every grid point as its own launch, fp32
and split-BF16 tensor cores), ragged_mix256 (the 256-request seed-7 mix, one launch of the
default and of the autotuned work list vs one launch per request, CUDA graphs), real_r2c_c2r (R2C N 128..8192 and C2R N 64..4096 at batch 1, 64, 1024),
long_fwd_bwd, c2c_2d, c2c_any_length, stft, cpu_stdlib (numpy / torch CPU FFT with the
reference's protocol: 3 warm-ups, 20 reps, mean and min).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-extras]
Under torchrun every rank runs the grid on its own GPU (weak scaling; no data-path
collective) and rank 0 prints the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (str(ROOT / "ascend-fft_b200"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "FFT GB/s & %HBM roofline: plain FP32 vs TC split-BF16, fwd+bwd, rel err<=2e-6"
UNIT = "GB/s"
GRID_N = [64, 128, 256, 512, 1024, 2048, 4096]
GRID_B = [1, 4, 16, 64, 256, 1024, 4096]
DOMINANT = (4096, 4096)
WORKLOAD = ("c2c_fwd_grid49: plain fp32 C2C forward over N{64..4096} x batch{1..4096}, "
            "interleaved complex64, N(0,1) seeded per point")


def emit(obj):
    print(json.dumps(obj, separators=(",", ":")), flush=True)


def grid_seed(n, b):
    return 1000 * (n.bit_length() - 1) + (b.bit_length() - 1) + 1


def grid_bytes():
    return sum(16 * n * b for n in GRID_N for b in GRID_B)


def mix256(count: int = 256, seed: int = 7):
    """The ragged request mix: log2 n ~ U{6..12}, batch = round(2^U(0,9)), then the OFDM-like
    2048 x (14*100), radar-like 512 x 4096 and spectral-layer-like 1024 x (8*768) groups of the
    reference's application proxies (scripts/e2e_test.py:94-102)."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count - 3):
        n = 1 << int(rng.integers(6, 13))
        b = max(1, int(round(2.0 ** rng.uniform(0.0, 9.0))))
        reqs.append((n, b))
    return reqs + [(2048, 14 * 100), (512, 4096), (1024, 8 * 768)]


def sample_rows(batch: int, want: int):
    """Evenly spread row indices including the first and the last."""
    if batch <= want:
        return list(range(batch))
    if want == 1:
        return [0]
    return [i * (batch - 1) // (want - 1) for i in range(want)]


def rel_l2_rows(got, ref):
    """Maximum over rows of the relative L2 error against an FP64 result."""
    d = np.linalg.norm(np.asarray(got).astype(np.complex128) - ref, axis=-1)
    r = np.linalg.norm(ref, axis=-1)
    return float((d / np.where(r > 0, r, 1.0)).max()) if d.size else 0.0


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def grid_traffic():
    """DRAM bytes read and written inside one launch of the step's kernel over the full grid,
    from the committed ncu capture (profiles/roofline_traffic.txt), or (None, None)."""
    p = ROOT / "profiles" / "roofline_traffic.txt"
    if not p.exists():
        return None, None
    vals = {}
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and not parts[0].startswith("#"):
            vals[parts[0]] = int(parts[1])
    r, w = vals.get("ragged_grid49_dram_read"), vals.get("ragged_grid49_dram_write")
    if r is None or w is None:
        return None, None
    return r, w


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled every ~1 ms through NVML in a background thread
    while the timed region runs (nvidia-smi -lms 100 as a fallback)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int, bus_id: str | None = None):
        self.index, self.bus_id = index, bus_id
        self.samples, self.times, self.masks, self.reasons, self.max_mhz = [], [], [], set(), None
        self.window = None   # (t0, t1) host time of the timed region
        self._stop = threading.Event()
        self._thread = None
        self._proc = None

    def _nvml_loop(self, nv, h):
        while not self._stop.is_set():
            try:
                t = time.perf_counter()
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.times.append(0.5 * (t + time.perf_counter()))
                self.masks.append(mask)
            except Exception:
                pass
            time.sleep(0.0001)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            if self.bus_id:
                try:
                    h = nv.nvmlDeviceGetHandleByPciBusId(self.bus_id.encode())
                except Exception:
                    h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self._thread.start()
        except Exception:
            try:
                self._proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,"
                     "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                     "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                     "--format=csv,noheader,nounits", "-lms", "100"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._thread = threading.Thread(target=self._smi_loop, daemon=True)
                self._thread.start()
            except Exception:
                self._proc = None
        return self

    def _smi_loop(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            try:
                self.samples.append(float(parts[0]))
                self.times.append(time.perf_counter())
                self.max_mhz = float(parts[1])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, parts[2:6]):
                if val.lower().startswith("active"):
                    self.reasons.add(name)

    def __exit__(self, *exc):
        self._stop.set()
        if self._proc:
            time.sleep(0.15)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._thread:
            self._thread.join(timeout=2)

    def summary(self):
        """Median SM clock over the samples taken inside the timed region (sampling runs from
        before the warm-up, so a short region still gets the samples that fall in it); the
        warm-up's samples stand in when none did."""
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        inside = list(range(len(self.samples)))
        if self.window:
            inside = [i for i, t in enumerate(self.times) if self.window[0] <= t <= self.window[1]]
        use = inside or list(range(len(self.samples)))
        reasons = set(self.reasons)
        for i in use:
            if i < len(self.masks):
                reasons |= {name for bit, name in self.REASONS.items() if self.masks[i] & bit}
        return {"sm_mhz": statistics.median(self.samples[i] for i in use), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "samples_in_timed_region": len(inside) if self.window else len(self.samples)}


# ------------------------------------------------------------------ CPU reference
class CpuReference:
    """The reference's own CPU FFT (oracle/_ref) over the grid with at most rows_cap rows per
    point, on `threads` host threads; falls back to the C restatement when the reference library
    is absent.  Inputs, outputs and the thread pool are set up once, and every output page is
    touched by one untimed pass, so a timed pass holds only the transforms."""

    def __init__(self, rows_cap: int, threads: int):
        from oracle import clib
        self.kind = "reference"
        lib = clib.reference()
        if lib is not None:
            self.fn = lib.ref_fft_rows
        else:
            self.kind = "port"
            rest = clib.restatement()

            def fn(xp, yp, n, rows):
                for r in range(rows):
                    rest.orc_ref_fft(xp + r * 8 * n, yp + r * 8 * n, n)
            self.fn = fn
        self.rows_cap, self.threads = rows_cap, threads
        jobs = []
        for n in GRID_N:
            for b in GRID_B:
                rows = min(b, rows_cap)
                rng = np.random.default_rng(grid_seed(n, b))
                x = rng.standard_normal((rows, 2 * n)).astype(np.float32)
                jobs.append((n, x, np.zeros_like(x)))
        self.chunks = []
        for n, x, y in jobs:
            step = max(1, x.shape[0] // threads)
            for r0 in range(0, x.shape[0], step):
                self.chunks.append((n, x, y, r0, min(x.shape[0], r0 + step)))
        self.nbytes = sum(16 * n * x.shape[0] for n, x, _ in jobs)
        self.pool = ThreadPoolExecutor(max_workers=threads)
        self.passes = 0
        self.run_pass()

    def _work(self, c):
        n, x, y, r0, r1 = c
        self.fn(x[r0:r1].ctypes.data, y[r0:r1].ctypes.data, n, r1 - r0)

    def run_pass(self) -> float:
        """One pass over the sample on the pool; returns its wall time in seconds."""
        t0 = time.perf_counter()
        list(self.pool.map(self._work, self.chunks))
        self.passes += 1
        return time.perf_counter() - t0

    def describe(self, passes: int) -> str:
        return (f"grid49 with <= {self.rows_cap} rows per point ({self.nbytes / 1e6:.1f} MB algorithmic per "
                f"pass), {passes} timed passes, {self.threads} threads, "
                f"{'oracle/_ref refFftF32' if self.kind == 'reference' else 'C restatement'}")

    def close(self):
        self.pool.shutdown()


def cpu_reference_sample(rows_cap: int, budget_s: float, threads: int):
    """Passes of CpuReference for about `budget_s` seconds after one warm-up pass.
    Returns (GB/s, seconds, bytes, kind, sample description)."""
    ref = CpuReference(rows_cap, threads)
    ref.run_pass()
    dt, reps = 0.0, 0
    while True:
        dt += ref.run_pass()
        reps += 1
        if dt >= budget_s:
            break
    ref.close()
    return ref.nbytes * reps / dt / 1e9, dt, ref.nbytes * reps, ref.kind, ref.describe(reps)


def cpu_stdlib(reps: int = 20):
    """The reference's stdlib baseline protocol (scripts/bench_stdlib.py:18-46): numpy.fft.fft
    on complex64 along the last axis and torch.fft.fft on CPU, 3 warm-up calls, then `reps`
    timed calls, mean and min in microseconds; on the config-1 shape (N=1024, B=256, U[-1,1)
    seed 0) and the reference's default grid N {256, 1024, 4096} x B {1, 64, 4096}."""
    import torch

    def bench(fn, x):
        for _ in range(3):
            fn(x)
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            fn(x)
            ts.append(time.perf_counter() - t)
        return round(sum(ts) / len(ts) * 1e6, 1), round(min(ts) * 1e6, 1)

    shapes = [(1024, 256)] + [(n, b) for n in (256, 1024, 4096) for b in (1, 64, 4096)]
    rows = []
    for n, b in shapes:
        rng = np.random.default_rng(0 if (n, b) == (1024, 256) else grid_seed(n, b))
        x = rng.uniform(-1.0, 1.0, size=(b, 2 * n)).astype(np.float32).view(np.complex64)
        nu, nmin = bench(lambda z: np.fft.fft(z, axis=-1), x)
        t = torch.from_numpy(x.copy())
        tu, tmin = bench(lambda z: torch.fft.fft(z), t)
        rows.append([n, b, nu, nmin, tu, tmin])
    return {"sub": "cpu_stdlib", "protocol": "3 warm-ups, 20 reps, mean/min us (scripts/bench_stdlib.py)",
            "cols": ["n", "b", "numpy_us", "numpy_min_us", "torch_us", "torch_min_us"], "rows": rows,
            "numpy": np.__version__, "torch": torch.__version__, "torch_threads": torch.get_num_threads(),
            "cpu_count": os.cpu_count()}


# ------------------------------------------------------------------ distributed helpers
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    ref = CpuReference(256, threads)   # set-up and one page-touching pass, untimed
    for _ in range(args.warmup):
        ref.run_pass()
    per_step = [ref.run_pass() for _ in range(args.steps)]
    ref.close()
    kind, desc, bytes_step = ref.kind, ref.describe(args.steps), ref.nbytes
    ms = statistics.mean(per_step) * 1e3
    value = bytes_step / (ms / 1e3) / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": "rows per grid point capped at 256",
                       "points": len(GRID_N) * len(GRID_B)},
            "same_config": False,
            "same_config_note": ("the reference's CPU FFT runs every grid point with its rows capped at "
                                 "256 (110.9 MB per step against the GPU arm's 710.2 MB); GB/s is per "
                                 "algorithmic byte on both arms"),
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    emit(line)
    return 0


# ------------------------------------------------------------------ sub-measurements
class Subs:
    """Sub-measurements beside the headline (one GPU).  Each figure is device time from CUDA
    events on `stream` around one replay of a CUDA graph holding `reps` launches (after 3 warm-up
    launches outside the capture and at least 20 ms of replays), and the error against an FP64
    numpy FFT on sampled rows."""

    def __init__(self, dev, stream, ctx, plan):
        import torch
        self.torch = torch
        self.dev, self.stream, self.sh = dev, stream, stream.cuda_stream
        self.ctx, self.plan = ctx, plan
        self.peak, _ = load_peaks()
        self.summary = {}

    def timed(self, fn, reps=20):
        torch = self.torch
        for _ in range(3):
            fn()
        self.stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=self.stream):
            for _ in range(reps):
                fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            # replays for at least 20 ms before the timed one: after host-side gaps (input
            # generation, parity checks, the previous sub-measurement) the device runs the first
            # milliseconds of work a few percent slower
            t_w = time.perf_counter()
            while True:
                graph.replay()
                self.stream.synchronize()
                if time.perf_counter() - t_w >= 0.02:
                    break
            e0.record(self.stream)
            graph.replay()
            e1.record(self.stream)
        e1.synchronize()
        del graph
        return e0.elapsed_time(e1) / reps

    def gbs(self, nbytes, ms):
        return nbytes / (ms / 1e3) / 1e9

    def err(self, y, x, inverse=False, rows=4, scale=1.0):
        idx = sample_rows(x.shape[0], rows)
        xs = x[idx].cpu().numpy().astype(np.complex128)
        ref = np.fft.ifft(xs, axis=-1) * xs.shape[-1] * scale if inverse else np.fft.fft(xs, axis=-1)
        return rel_l2_rows(y[idx].cpu().numpy(), ref)

    def check(self, r, what):
        if r:
            raise RuntimeError(f"{what}: status {r}")

    # -- config 2: every grid point as its own launch, fp32 and split-BF16
    def grid_points(self):
        torch, sh, peak = self.torch, self.sh, self.peak
        import bfly
        rows, best = [], None
        for n in GRID_N:
            for b in GRID_B:
                g = torch.Generator(device=self.dev).manual_seed(grid_seed(n, b))
                x = torch.randn(b, n, dtype=torch.complex64, device=self.dev, generator=g)
                y = torch.empty_like(x)
                plan = bfly.plan_for(self.dev, n)
                byts = 16 * n * b
                res = []
                for split in (0, 3, 2):
                    if split:
                        fn = lambda: self.check(plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, split, sh), "tc")
                    else:
                        fn = lambda: self.check(plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh), "c2c")
                    ms = self.timed(fn)
                    res.append((ms, self.gbs(byts, ms), self.err(y, x)))
                (ms0, g0, e0), (_, g3, e3), (_, g2, e2) = res
                # the autotuner's plan for this (n, batch): candidates measured, FP64-checked, best kept
                tuned = self.ctx.select(n, b, 8)
                ms_t = self.timed(lambda: self.check(tuned.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh), "tuned"))
                et = self.err(y, x)
                tuned.close()
                rows.append([n, b, round(ms0 * 1e3, 2), round(g0, 1), round(g0 / peak, 3), float(f"{e0:.3g}"),
                             round(g3, 1), float(f"{e3:.3g}"), round(g2, 1), float(f"{e2:.3g}"),
                             round(ms_t * 1e3, 2), float(f"{et:.3g}")])
                sp = g3 / g0
                if best is None or sp > best[0]:
                    best = (sp, n, b, e3)
                del x, y
        meets = sum(1 for r in rows if r[4] >= 0.70)
        emit({"sub": "c2c_grid49_points", "unit": UNIT, "peak": peak,
              "cols": ["n", "b", "fp32_us", "fp32_gbs", "fp32_frac", "fp32_rel_l2", "tc3_gbs", "tc3_rel_l2",
                       "tc2_gbs", "tc2_rel_l2", "tuned_us", "tuned_rel_l2"], "rows": rows, "fp32_points_at_0.70": meets,
              "tuned": "Context.select(n, batch): the autotuner's plan for the point (fp32 columns: the per-length plan)",
              "l2": "points under 126 MB are L2-warm across the 20 back-to-back launches of the graph"})
        b4096 = [r for r in rows if r[1] == 4096]
        self.summary["grid49_points"] = {
            "fp32_frac_at_b4096": [r[4] for r in b4096], "fp32_points_at_0.70": meets,
            "tc3_vs_fp32_at_b4096": [round(r[6] / r[3], 2) for r in b4096],
            "tc3_best_speedup": [round(best[0], 3), best[1], best[2]],
            "tuned_vs_per_length_time": round(sum(r[10] for r in rows) / sum(r[2] for r in rows), 3),
            "tc3_max_rel_l2": max(r[7] for r in rows), "tc2_max_rel_l2": max(r[9] for r in rows)}

    # -- config 4: the 256-request mix in one launch, against one launch per request
    def ragged_mix(self):
        torch, sh, peak = self.torch, self.sh, self.peak
        reqs = mix256()
        g = torch.Generator(device=self.dev).manual_seed(7)
        bufs = []
        for n, b in reqs:
            x = torch.randn(b, n, dtype=torch.complex64, device=self.dev, generator=g)
            bufs.append((n, b, x, torch.empty_like(x)))
        plan = self.plan
        for n, b, _, _ in bufs:
            self.check(plan.prepare(n, b), "prepare")
        total = sum(16 * n * b for n, b, _, _ in bufs)
        reqs_ptr = [(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0) for n, b, x, y in bufs]
        # the autotuner: launch mode and per-length register radix measured on this very mix
        torch.cuda.synchronize()   # the tuner runs on the plan's stream
        t0 = time.perf_counter()
        ragged, tune_log = self.ctx.tune_ragged(plan, reqs_ptr, want_log=True)
        tune_s = time.perf_counter() - t0
        default = plan.make_ragged(reqs_ptr)
        # default and tuned lists timed in the order D T T D (mean of each pair): the device is a
        # few percent slower for a while after sustained load, which a fixed order would charge
        # to whichever list came second
        run_d = lambda: self.check(default.exec(sh), "ragged")
        run_t = lambda: self.check(ragged.exec(sh), "ragged")
        d0, t0_, t1_, d1 = (self.timed(f, reps=10) for f in (run_d, run_t, run_t, run_d))
        ms_d, ms_r = 0.5 * (d0 + d1), 0.5 * (t0_ + t1_)
        default.close()
        run_t()
        torch.cuda.synchronize()
        worst = 0.0
        for n, b, x, y in bufs[::16] + bufs[-3:]:
            worst = max(worst, self.err(y, x, rows=2))

        import bfly
        plans = {n: bfly.plan_for(self.dev, n) for n, _ in reqs}   # each length's measured best plan

        def per_request():
            for n, b, x, y in bufs:
                self.check(plans[n].exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh), "c2c")
        ms_p = self.timed(per_request, reps=2)
        # the same launches issued one by one from the host (no graph)
        for _ in range(2):
            with torch.cuda.stream(self.stream):
                per_request()
        self.stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(3):
            per_request()
        e1.record(self.stream)
        e1.synchronize()
        ms_e = e0.elapsed_time(e1) / 3
        info = ragged.info()
        ragged.close()
        kernel = {-1: "k_ragged_flat", 0: "k_ragged", 1: "k_ragged_tma<1>", 2: "k_ragged_tma<2>"}[info["stages"]]
        r = {"requests": len(reqs), "bytes": total, "tiles": info["tiles"],
             "tuned": {"kernel": kernel, "mode": info["stages"], "radix8": f"0x{info['radix8']:02x}",
                       "tuning_s": round(tune_s, 2),
                       "candidates": sum(1 for ln in tune_log.splitlines() if ln.startswith("  mode"))},
             "default_gbs": round(self.gbs(total, ms_d), 1),
             "one_launch_gbs": round(self.gbs(total, ms_r), 1), "one_launch_frac": round(self.gbs(total, ms_r) / peak, 3),
             "one_launch_us": round(ms_r * 1e3, 1), "per_request_graph_gbs": round(self.gbs(total, ms_p), 1),
             "per_request_eager_gbs": round(self.gbs(total, ms_e), 1),
             "speedup_vs_per_request_graph": round(ms_p / ms_r, 2),
             "speedup_vs_per_request_eager": round(ms_e / ms_r, 2), "rel_l2_max": float(f"{worst:.3g}")}
        emit({"sub": "ragged_mix256", "unit": UNIT, "seed": 7,
              "mode": "one launch of the autotuned work list replayed from a CUDA graph", **r})
        self.summary["ragged_mix256"] = {k: r[k] for k in ("one_launch_gbs", "one_launch_frac", "default_gbs",
                                                           "speedup_vs_per_request_graph",
                                                           "speedup_vs_per_request_eager", "rel_l2_max")}
        del bufs

    # -- config 3: R2C N 128..8192 and C2R N 64..4096 at batch 1, 64, 1024
    def real_transforms(self):
        torch, sh, peak = self.torch, self.sh, self.peak
        import bfly
        r2c, c2r = [], []
        for kind, ns in (("r2c", [128 << i for i in range(7)]), ("c2r", [64 << i for i in range(7)])):
            for n in ns:
                plan = bfly.plan_for(self.dev, n, "real")
                for b in (1, 64, 1024):
                    rng = np.random.default_rng(n * 7 + b)
                    xr = rng.uniform(-1.0, 1.0, size=(b, n))
                    byts = (8 * n + 8) * b
                    if kind == "r2c":
                        x = torch.from_numpy(xr.astype(np.float32)).to(self.dev)
                        y = torch.empty(b, n // 2 + 1, dtype=torch.complex64, device=self.dev)
                        ms = self.timed(lambda: self.check(plan.exec_r2c(x.data_ptr(), y.data_ptr(), n, b, 1.0, 1.0, sh), "r2c"))
                        idx = sample_rows(b, 4)
                        ref = np.fft.rfft(x[idx].cpu().numpy().astype(np.float64), axis=-1)
                        e = rel_l2_rows(y[idx].cpu().numpy(), ref)
                        r2c.append([n, b, round(ms * 1e3, 2), round(self.gbs(byts, ms), 1), float(f"{e:.3g}")])
                    else:
                        X = np.fft.rfft(xr, axis=-1)
                        X[:, 0] = X[:, 0].real
                        X[:, -1] = X[:, -1].real
                        x = torch.from_numpy(X.astype(np.complex64)).to(self.dev)
                        y = torch.empty(b, n, device=self.dev)
                        ms = self.timed(lambda: self.check(plan.exec_c2r(x.data_ptr(), y.data_ptr(), n, b, 1.0, 1.0, 1.0 / n, sh), "c2r"))
                        idx = sample_rows(b, 4)
                        ref = np.fft.irfft(X[idx].astype(np.complex64).astype(np.complex128), n=n, axis=-1)
                        e = rel_l2_rows(y[idx].cpu().numpy(), ref)
                        c2r.append([n, b, round(ms * 1e3, 2), round(self.gbs(byts, ms), 1), float(f"{e:.3g}")])
                    del x, y
        emit({"sub": "real_r2c_c2r", "unit": UNIT, "bytes": "(8n+8)*batch", "cols": ["n", "b", "us", "gbs", "rel_l2"],
              "r2c": r2c, "c2r": c2r,
              "inputs": "R2C U[-1,1); C2R the rfft of seeded U[-1,1) reals with DC/Nyquist imag zeroed"})
        self.summary["real_r2c_c2r_b1024"] = {
            "r2c_gbs": [r[3] for r in r2c if r[1] == 1024], "c2r_gbs": [r[3] for r in c2r if r[1] == 1024],
            "max_rel_l2": max(r[4] for r in r2c + c2r)}

    # -- config 5: long C2C forward + backward (the conjugate-FFT adjoint), batch * n = 2^26
    def long_fwd_bwd(self):
        torch, sh, peak = self.torch, self.sh, self.peak
        import bfly
        res = {}
        for n in (8192, 16384, 32768, 65536):
            b = (1 << 26) // n
            g = torch.Generator(device=self.dev).manual_seed(11)
            x = torch.randn(b, n, dtype=torch.complex64, device=self.dev, generator=g)
            y = torch.empty_like(x)
            z = torch.empty_like(x)
            plan = bfly.plan_for(self.dev, n)
            byts = 16 * n * b
            ms_f = self.timed(lambda: self.check(plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh), "fwd"))
            ms_b = self.timed(lambda: self.check(plan.exec_c2c(y.data_ptr(), z.data_ptr(), n, b, 1, 1.0, sh), "bwd"))
            res[n] = [round(self.gbs(byts, ms_f), 1), round(self.gbs(byts, ms_b), 1),
                      float(f"{self.err(y, x, rows=2):.3g}"), float(f"{self.err(z, y, inverse=True, rows=2):.3g}")]
            # the same forward on the ring schedule (one launch, intermediate in L2)
            ring = self.ctx.make_plan("r16_cta256_shared_fp32_ring", 8192, 1)
            ms_r = self.timed(lambda: self.check(ring.exec_c2c(x.data_ptr(), z.data_ptr(), n, b, -1, 1.0, sh), "ring"))
            res[n] += [round(self.gbs(byts, ms_r), 1), float(f"{self.err(z, x, rows=2):.3g}")]
            ring.close()
            # context: the GPU's library FFT (cuFFT through torch.fft) forward and inverse, same tensors
            with torch.cuda.stream(self.stream):
                ms_cf = self.timed(lambda: torch.fft.fft(x, out=y))
                ms_cb = self.timed(lambda: torch.fft.ifft(y, out=z))
            res[n] += [round(self.gbs(byts, ms_cf), 1), round(self.gbs(byts, ms_cb), 1)]
            del x, y, z
        emit({"sub": "long_fwd_bwd", "unit": UNIT,
              "cols": ["fwd_gbs", "bwd_gbs", "fwd_rel_l2", "bwd_rel_l2", "ring_fwd_gbs", "ring_rel_l2",
                       "cufft_fwd_gbs", "cufft_inv_gbs"],
              "schedule": "single pass n <= 16384, two-kernel four-step above; ring = one-launch four-step",
              "rows": {f"n{n}_b{(1 << 26) // n}": v for n, v in res.items()}})
        self.summary["long_fwd_bwd_frac"] = {str(n): [round(v[0] / peak, 3), round(v[1] / peak, 3)] for n, v in res.items()}

    # -- 2-D and strided transforms
    def c2c_2d(self):
        torch, sh, peak = self.torch, self.sh, self.peak
        import bfly
        out = {}
        for ny, nx in ((256, 256), (512, 512), (1024, 1024), (2048, 2048), (1024, 128), (128, 1024)):
            b = (1 << 26) // (ny * nx)
            g = torch.Generator(device=self.dev).manual_seed(ny + nx)
            x = torch.randn(b, ny, nx, dtype=torch.complex64, device=self.dev, generator=g)
            y = torch.empty_like(x)
            plan = bfly.plan_for(self.dev, nx)
            ms = self.timed(lambda: self.check(plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, b, -1, 1.0, sh), "2d"))
            ref = np.fft.fft2(x[:1].cpu().numpy().astype(np.complex128)).reshape(1, -1)
            e = rel_l2_rows(y[:1].cpu().numpy().reshape(1, -1), ref)
            out[f"{ny}x{nx}_b{b}"] = [round(self.gbs(16 * ny * nx * b, ms), 1), float(f"{e:.3g}")]
            del x, y
        for n, outer, inner in ((1024, 64, 1024), (256, 1024, 256)):
            g = torch.Generator(device=self.dev).manual_seed(n + inner)
            x = torch.randn(outer, n, inner, dtype=torch.complex64, device=self.dev, generator=g)
            y = torch.empty_like(x)
            plan = bfly.plan_for(self.dev, n)
            ms = self.timed(lambda: self.check(plan.exec_c2c_axis(x.data_ptr(), y.data_ptr(), n, outer, inner, -1, 1.0, sh), "axis"))
            ref = np.fft.fft(x[:1].cpu().numpy().astype(np.complex128), axis=1)
            e = float(np.linalg.norm(y[:1].cpu().numpy() - ref) / np.linalg.norm(ref))
            out[f"axis_n{n}_outer{outer}_inner{inner}"] = [round(self.gbs(16 * n * outer * inner, ms), 1), float(f"{e:.3g}")]
            del x, y
        emit({"sub": "c2c_2d", "unit": UNIT, "cols": ["gbs", "rel_l2"], "rows": out,
              "note": "2-D = row pass + column pass (two HBM round trips) scored on 16 bytes per point"})

    # -- non-power-of-two lengths
    def any_length(self):
        torch, sh = self.torch, self.sh
        import bfly
        out = {}
        for n in (1536, 1920, 6144, 360, 1000, 3000, 6561, 12000, 1001, 1003, 8191):
            b = (1 << 25) // n
            g = torch.Generator(device=self.dev).manual_seed(n)
            x = torch.randn(b, n, dtype=torch.complex64, device=self.dev, generator=g)
            y = torch.empty_like(x)
            plan = bfly.plan_for(self.dev, n)
            ms = self.timed(lambda: self.check(plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh), "c2c"))
            out[f"n{n}_b{b}"] = [round(self.gbs(16 * n * b, ms), 1), float(f"{self.err(y, x):.3g}")]
            del x, y
        emit({"sub": "c2c_any_length", "unit": UNIT, "cols": ["gbs", "rel_l2"], "rows": out})

    # -- STFT / inverse STFT, 4 signals of 2^24 samples, centred, Hann
    def stft(self):
        torch, sh = self.torch, self.sh
        import bfly
        out = {}
        plan = bfly.plan_for(self.dev, 1024, "real")
        for n, hop in ((256, 64), (1024, 256), (4096, 1024), (400, 160)):
            L, S = 1 << 24, 4
            g = torch.Generator(device=self.dev).manual_seed(n)
            x = torch.randn(S, L, device=self.dev, generator=g)
            w = torch.hann_window(n, device=self.dev)
            frames = 1 + L // hop
            y = torch.empty(S, frames, n // 2 + 1, dtype=torch.complex64, device=self.dev)
            ms = self.timed(lambda: self.check(plan.exec_stft(x.data_ptr(), y.data_ptr(), n, S, L, hop, True, w.data_ptr(), sh)[0], "stft"))
            fb = S * frames * (4 * n + 8 * (n // 2 + 1))
            ref = torch.stft(x[:1, :16 * n].double(), n, hop_length=hop, window=w.double(), return_complex=True)[..., :8]
            got = y[:1, :8].transpose(-1, -2).to(torch.complex128)
            e = float((torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item())
            xb = torch.empty(S, L, device=self.dev)
            ms_i = self.timed(lambda: self.check(plan.exec_istft(y.data_ptr(), xb.data_ptr(), n, S, frames, hop, True,
                                                                 w.data_ptr(), L, 1.0, sh), "istft"))
            ib = S * frames * 8 * (n // 2 + 1) + 4 * S * L
            rt = float((torch.linalg.vector_norm(xb - x) / torch.linalg.vector_norm(x)).item())
            row = [round(self.gbs(fb, ms), 1), round(ms, 3), float(f"{e:.3g}"),
                   round(self.gbs(ib, ms_i), 1), round(ms_i, 3), float(f"{rt:.3g}")]
            if n & (n - 1) == 0:   # the fused gradients (one kernel each)
                ms_sb = self.timed(lambda: self.check(plan.exec_stft_backward(y.data_ptr(), xb.data_ptr(), n, S, L, hop,
                                                                             True, w.data_ptr(), sh), "stft_bwd"))
                ms_ib = self.timed(lambda: self.check(plan.exec_istft_backward(x.data_ptr(), y.data_ptr(), n, S, frames,
                                                                              hop, True, w.data_ptr(), L, 1.0, sh),
                                                      "istft_bwd"))
                row += [round(ms_sb, 3), round(ms_ib, 3)]
            out[f"n{n}_hop{hop}"] = row
            del x, y, xb
        emit({"sub": "stft", "unit": UNIT, "signals": "4 x 2^24 samples, centred, Hann",
              "cols": ["stft_frame_gbs", "stft_ms", "stft_rel_l2_vs_torch_f64", "istft_gbs", "istft_ms",
                       "round_trip_rel_l2", "stft_backward_ms", "istft_backward_ms"], "rows": out})


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch
    world, rank, local = dist_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    import bfly

    # clock sampling runs from here to the end of the headline's timed region (which lasts a
    # few ms): the sampler is warm when the region starts, and only its samples inside count
    bus = getattr(torch.cuda.get_device_properties(dev), "pci_bus_id", None)
    clock_sampler = ClockSampler(dev.index, bus).__enter__()
    ctx = bfly.Context()
    rc = ctx.init(device=dev.index)
    if rc:
        raise SystemExit(f"Context.init failed: {rc}")
    plan = ctx.make_plan()
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream

    # resident inputs and outputs for every grid point
    pts = []
    for n in GRID_N:
        for b in GRID_B:
            g = torch.Generator(device=dev).manual_seed(grid_seed(n, b))
            x = torch.randn(b, n, dtype=torch.complex64, device=dev, generator=g)
            pts.append((n, b, x, torch.empty_like(x)))
    torch.cuda.synchronize()
    t_setup = time.perf_counter()
    for n, b, x, y in pts:   # builds twiddle tables outside any capture
        assert plan.prepare(n, b) == 0
    plan_setup_us = (time.perf_counter() - t_setup) * 1e6

    def check(tag):
        worst = 0.0
        for n, b, x, y in pts:
            rows = sample_rows(b, 2)
            ref = np.fft.fft(x[rows].cpu().numpy().astype(np.complex128), axis=-1)
            worst = max(worst, rel_l2_rows(y[rows].cpu().numpy(), ref))
        assert worst <= 1e-6, f"{tag} parity check failed: rel L2 {worst}"
        return worst

    def per_point():
        for n, b, x, y in pts:
            r = plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh)
            if r:
                raise RuntimeError(f"exec_c2c({n},{b}) = {r}")

    # the product path: one ragged launch over all 49 requests
    ragged = plan.make_ragged((x.data_ptr(), y.data_ptr(), n, b, -1, 1.0) for n, b, x, y in pts)

    def ragged_step():
        r = ragged.exec(sh)
        if r:
            raise RuntimeError(f"ragged exec = {r}")

    # parity spot checks of both paths before timing (FP64 numpy FFT on sampled rows)
    with torch.cuda.stream(stream):
        per_point()
    stream.synchronize()
    worst = check("per-point")
    for _, _, _, y in pts:
        y.zero_()
    torch.cuda.synchronize()
    ragged_step()
    stream.synchronize()
    worst = max(worst, check("ragged"))

    warm_runs = {}

    def timed(fn, steps, sample_clocks=False):
        sampler = clock_sampler if sample_clocks else None
        # W warm-up steps, continued until ~20 ms of device work: after the host-side set-up and
        # parity checks the device runs the first milliseconds of work a few percent slower
        done, t_w = 0, time.perf_counter()
        while done < max(3, args.warmup) or time.perf_counter() - t_w < 0.02:
            fn()
            done += 1
            if done % 16 == 0:
                stream.synchronize()
        warm_runs[fn] = done
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.window = (t0, time.perf_counter())
            sampler.__exit__(None, None, None)
        t = e0.elapsed_time(e1) / steps
        torch.cuda.synchronize()
        if dist:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = tt.item()
        return t, sampler

    ms, clocks = timed(ragged_step, args.steps, sample_clocks=True)
    total_bytes = grid_bytes() * world
    value = total_bytes / (ms / 1e3) / 1e9

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        per_point()

    def graph_step():
        with torch.cuda.stream(stream):
            graph.replay()

    ms_graph, _ = timed(graph_step, args.steps)
    per_point_gbs = total_bytes / (ms_graph / 1e3) / 1e9

    # the largest single-size launch timed alone on its stream
    n, b = DOMINANT
    xd = next(x for (nn, bb, x, y) in pts if (nn, bb) == DOMINANT)
    yd = torch.empty_like(xd)
    dom_ms, _ = timed(lambda: plan.exec_c2c(xd.data_ptr(), yd.data_ptr(), n, b, -1, 1.0, sh), 50)
    dom_bytes = 16 * n * b
    peak, peak_kind = load_peaks()
    achieved = grid_bytes() / (ms / 1e3) / 1e9

    # e2e through the C ABI with pinned host buffers: the whole grid in one
    # bfly_plan_run_c2c_many call (H2D, kernels and D2H of different points overlap)
    host = []
    for (nn, bb, x, y) in pts:
        hx = torch.empty((bb, 2 * nn), dtype=torch.float32, pin_memory=True)
        hx.copy_(torch.view_as_real(x).reshape(bb, 2 * nn).cpu())
        hy = torch.empty_like(hx).pin_memory()
        host.append((nn, bb, hx, hy))
    many = [(hx.numpy(), hy.numpy(), nn, bb) for nn, bb, hx, hy in host]
    t0 = time.perf_counter()
    assert plan.run_many(many) == 0   # first use: device buffers grow to the whole grid
    first_use_us = (time.perf_counter() - t0) * 1e6
    e2e_steps = max(3, min(args.steps, 5))

    def e2e_time(step):
        if dist:
            dist.barrier()
        walls = []
        for _ in range(e2e_steps):
            t0 = time.perf_counter()
            step()
            walls.append(time.perf_counter() - t0)
        el = statistics.mean(walls)
        if dist:
            t = torch.tensor([el], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = t.item()
        return el, walls

    def step_many():
        r = plan.run_many(many)
        if r:
            raise RuntimeError(f"run_many = {r}")

    e2e_s, walls = e2e_time(step_many)
    # result check of the host round trip on sampled rows
    for nn, bb, hx, hy in host[::8]:
        rows = sample_rows(bb, 2)
        xs = hx.numpy()[rows].view(np.complex64).astype(np.complex128)
        assert rel_l2_rows(hy.numpy()[rows].view(np.complex64), np.fft.fft(xs, axis=-1)) <= 1e-6
    # event spans of the same bytes, one phase at a time (no overlap): upload of every input,
    # the device chain (the ragged launch), download of every output
    spans = {"h2d": [], "device_chain": [], "d2h": []}
    for _ in range(e2e_steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for (nn, bb, hx, hy), (_, _, x, y) in zip(host, pts):
                torch.view_as_real(x).reshape(bb, 2 * nn).copy_(hx, non_blocking=True)
            ev[1].record(stream)
            ragged_step()
            ev[2].record(stream)
            for (nn, bb, hx, hy), (_, _, x, y) in zip(host, pts):
                hy.copy_(torch.view_as_real(y).reshape(bb, 2 * nn), non_blocking=True)
            ev[3].record(stream)
        ev[3].synchronize()
        spans["h2d"].append(ev[0].elapsed_time(ev[1]) * 1e3)
        spans["device_chain"].append(ev[1].elapsed_time(ev[2]) * 1e3)
        spans["d2h"].append(ev[2].elapsed_time(ev[3]) * 1e3)
    h2d = sum(8 * nn * bb for nn, bb, _, _ in host)
    e2e_value = grid_bytes() * world / e2e_s / 1e9
    scopes = {"plan_setup_us": round(plan_setup_us, 1), "first_use_us": round(first_use_us, 1),
              "host_end_to_end_mean_us": round(statistics.mean(walls) * 1e6, 1),
              "host_end_to_end_min_us": round(min(walls) * 1e6, 1),
              "h2d_us": round(min(spans["h2d"]), 1), "device_chain_us": round(min(spans["device_chain"]), 1),
              "d2h_us": round(min(spans["d2h"]), 1), "reps": e2e_steps,
              "note": "spans: min over reps, phases run one after another; end_to_end overlaps them"}
    info = ragged.info()
    ragged.close()
    del graph

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    summary = {"sub": "summary"}
    if world == 1 and not args.no_extras:
        subs = Subs(dev, stream, ctx, plan)
        for part in (subs.c2c_2d, subs.any_length, subs.stft, subs.long_fwd_bwd, subs.real_transforms,
                     subs.ragged_mix, subs.grid_points):
            part()
        torch.cuda.synchronize()
        summary.update(subs.summary)
    cpu = None
    if world == 1:
        std = cpu_stdlib()
        emit(std)
        c1 = std["rows"][0]
        summary["cpu_stdlib_cfg1_us"] = {"numpy_mean": c1[2], "numpy_min": c1[3], "torch_mean": c1[4],
                                         "torch_min": c1[5], "numpy": std["numpy"],
                                         "torch_threads": std["torch_threads"]}
        threads = os.cpu_count() or 1
        gbs, dt, nb, kind, desc = cpu_reference_sample(256, 10.0, threads)
        cpu = {"value": round(gbs, 4), "unit": UNIT, "cores": threads, "kind": kind, "sample": desc}
    tr, tw = grid_traffic()
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "points": len(pts), "bytes_per_step": total_bytes,
                   "l2": "355 MB in + 355 MB out per step > 126 MB L2; no flush",
                   "launch": "one k_ragged_flat launch per step", "tiles": info["tiles"],
                   "warmup_steps_run": warm_runs.get(ragged_step),
                   "parallelism": f"batch-sharded replicas x{world}", "parity_rel_l2_max": float(f"{worst:.3g}")},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": (tr + tw) if tr is not None else None, "traffic_read": tr,
                     "traffic_note": "ncu dram bytes inside the launch; writes left dirty in L2 drain after it",
                     "kernel": "k_ragged_flat", "peak_kind": peak_kind, "algorithmic_bytes": grid_bytes()},
        "gsamples_per_s": round(sum(n * b for n in GRID_N for b in GRID_B) * world / (ms / 1e3) / 1e9, 1),
        "per_point_graph": {"value": round(per_point_gbs, 1), "launches_per_step": len(pts)},
        "largest_launch": {"kernel": "k_c2c N=4096 batch=4096",
                           "frac": round(dom_bytes / (dom_ms / 1e3) / 1e9 / peak, 4),
                           "launch_us": round(dom_ms * 1e3, 2), "l2": "134 MB in, about the L2 size"},
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d, "path": "bfly_plan_run_c2c_many, pinned host buffers",
                "scopes": scopes},
        "gpu_launches": args.steps,
        "clocks": clocks.summary() if clocks else None,
        "cpu_baseline": cpu,
    }
    if len(summary) > 1:
        emit(summary)
    emit(line)
    return 0


def run_case(spec: str, reps: int):
    """Launch one kernel configuration `reps` times without timing (for ncu captures):
    spec = kind:n:batch with kind in c2c, c2c_inv (any n: non-powers of two run the prime-factor, mixed-radix or Bluestein
    kernel), tc2, tc3 (tensor-core splits), r2c, c2r, cluster (long C2C on the cluster
    schedule), or ragged:grid:CAP or ragged:N:B; or cols:NY:NCOLS:MATS (column kernel), c2d:NY:NX:B (2-D),
    stft:N:HOP:LEN (4 signals, centred, Hann window), istft:N:HOP:LEN (its inverse)."""
    import torch
    import bfly
    parts = spec.split(":")
    kind = parts[0]
    dev = torch.device("cuda", 0)
    ctx = bfly.Context()
    assert ctx.init() == 0
    plan = ctx.make_plan()
    if kind in ("cols", "c2d", "stft", "istft"):
        a, b2, c = (int(v) for v in parts[1:4])
        g = torch.Generator(device=dev).manual_seed(a + b2 + c)
        if kind == "cols":     # NY-point transforms down NCOLS columns of MATS matrices
            x = torch.randn(c, a, b2, dtype=torch.complex64, device=dev, generator=g)
            y = torch.empty_like(x)
            call = lambda: plan.exec_c2c_axis(x.data_ptr(), y.data_ptr(), a, c, b2, -1, 1.0, 0)
        elif kind == "c2d":
            x = torch.randn(c, a, b2, dtype=torch.complex64, device=dev, generator=g)
            y = torch.empty_like(x)
            call = lambda: plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), a, b2, c, -1, 1.0, 0)
        elif kind == "stft":   # stft:N:HOP:LEN
            x = torch.randn(4, c, device=dev, generator=g)
            w = torch.hann_window(a, device=dev)
            y = torch.empty(4, 1 + c // b2, a // 2 + 1, dtype=torch.complex64, device=dev)
            call = lambda: plan.exec_stft(x.data_ptr(), y.data_ptr(), a, 4, c, b2, True, w.data_ptr())[0]
        else:                  # istft:N:HOP:LEN
            fr = 1 + c // b2
            x = torch.randn(4, fr, a // 2 + 1, dtype=torch.complex64, device=dev, generator=g)
            w = torch.hann_window(a, device=dev)
            y = torch.empty(4, c, device=dev)
            call = lambda: plan.exec_istft(x.data_ptr(), y.data_ptr(), a, 4, fr, b2, True, w.data_ptr(), c, 1.0, 0)
        for _ in range(reps):
            r = call()
            if r:
                raise SystemExit(f"{spec}: status {r}")
        torch.cuda.synchronize()
        print(f"case {spec} x{reps} ok")
        return 0
    n, b = parts[1], parts[2]
    if kind == "cluster":
        plan = ctx.make_plan("r16_cta256_shared_fp32_cluster", 8192, 1)
    if kind == "ragged":   # ragged:grid:CAP -> the 49-point grid with batch capped at CAP;
        bufs = []          # ragged:N:B -> one request of B rows of length N
        shapes = ([(nn, min(bb, int(b))) for nn in GRID_N for bb in GRID_B] if n == "grid"
                  else [(int(n), int(b))])
        for nn, bb in shapes:
            x = torch.randn(bb, nn, dtype=torch.complex64, device=dev)
            bufs.append((x, torch.empty_like(x), nn, bb))
        rg = plan.make_ragged((x.data_ptr(), y.data_ptr(), nn, bb, -1, 1.0) for x, y, nn, bb in bufs)
        for _ in range(reps):
            r = rg.exec(0)
            if r:
                raise SystemExit(f"{spec}: status {r}")
        torch.cuda.synchronize()
        print(f"case {spec} x{reps} ok, {sum(16 * nn * bb for _, _, nn, bb in bufs)} bytes per launch")
        return 0
    n, b = int(n), int(b)
    g = torch.Generator(device=dev).manual_seed(grid_seed(n, b))
    if kind in ("c2c", "c2c_inv", "cluster"):
        x = torch.randn(b, n, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        call = lambda: plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, 1 if kind == "c2c_inv" else -1, 1.0, 0)
    elif kind in ("tc2", "tc3"):
        x = torch.randn(b, n, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        call = lambda: plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, int(kind[2]), 0)
    elif kind == "r2c":
        x = torch.randn(b, n, device=dev, generator=g)
        y = torch.empty(b, n // 2 + 1, dtype=torch.complex64, device=dev)
        call = lambda: plan.exec_r2c(x.data_ptr(), y.data_ptr(), n, b, 1.0, 1.0, 0)
    elif kind == "c2r":
        x = torch.randn(b, n // 2 + 1, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty(b, n, device=dev)
        call = lambda: plan.exec_c2r(x.data_ptr(), y.data_ptr(), n, b, 1.0, 1.0, 1.0 / n, 0)
    else:
        raise SystemExit(f"unknown case kind {kind}")
    for _ in range(reps):
        r = call()
        if r:
            raise SystemExit(f"{spec}: status {r}")
    torch.cuda.synchronize()
    print(f"case {spec} x{reps} ok")
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default=None, help="kind:n:batch (see run_case), launch only that kernel (for ncu)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--no-extras", action="store_true", help="skip the sub-measurements beside the headline")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    args = ap.parse_args(argv)
    if args.case:
        return run_case(args.case, args.reps)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
