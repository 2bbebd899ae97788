"""Benchmark of the batched FFT library on B200 (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): plain fp32 C2C forward over
the 49-point grid N in {64..4096} x batch in {1..4096}, interleaved complex, Re/Im i.i.d.
N(0,1) seeded per point (seed = 1000*log2 N + log2 batch + 1).  One step = one forward
transform of every grid point on inputs resident in HBM, run as ONE ragged launch
(k_ragged_flat over the 49 requests: 10,931 tiles of 4096 or 2048 points, one per CTA).  The step touches 355 MB of input and 355 MB of output, more
than the 126 MB L2, so no explicit flush is needed between steps.  The same step as 49
per-point launches replayed from a CUDA graph is reported beside it (per_point_graph).

  value      algorithmic bytes (16 * N * batch summed over the grid) / device time per step
  e2e        the same metric through the C ABI's synchronous host-pointer entry points with
             pinned host buffers, H2D + kernels + D2H inside the timed step: the whole grid in
             one bfly_plan_run_c2c_many call (value), and one bfly_plan_run_c2c call per point
             as the reference calls it (per_call)
  roofline   the step's only kernel (k_ragged_flat over the grid) timed with CUDA events on its
             stream against the measured HBM copy bandwidth; the largest single-size launch
             (N=4096, batch=4096, k_c2c) is reported beside it (largest_launch)
  cpu_baseline  the reference's own CPU FFT (its FP64 oracle src/framework/reference.cpp,
             compiled from its sources into oracle/_ref) on a bounded sample of the grid,
             rows spread over the host's threads

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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


def grid_seed(n, b):
    return 1000 * (n.bit_length() - 1) + (b.bit_length() - 1) + 1


def grid_bytes():
    return sum(16 * n * b for n in GRID_N for b in GRID_B)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dominant_traffic():
    """DRAM bytes of one full-grid launch of the step's kernel: the committed ncu capture of the
    capped grid (profiles/roofline_traffic.txt) scaled by algorithmic bytes, or None."""
    p = ROOT / "profiles" / "roofline_traffic.txt"
    if not p.exists():
        return None
    vals = {}
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and not parts[0].startswith("#"):
            vals[parts[0]] = int(parts[1])
    t, a = vals.get("ragged_grid49_cap1024"), vals.get("ragged_grid49_cap1024_algorithmic")
    if not t or not a:
        return None
    return int(round(t * grid_bytes() / a))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled every ~1 ms through NVML in a background thread
    while the timed region runs (nvidia-smi -lms 100 as a fallback)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int, bus_id: str | None = None):
        self.index, self.bus_id = index, bus_id
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._thread = None
        self._proc = None

    def _nvml_loop(self, nv, h):
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.001)

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
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ CPU reference
def cpu_reference_sample(rows_cap: int, budget_s: float, threads: int):
    """The reference's own CPU FFT (oracle/_ref) over the grid with at most rows_cap rows per
    point; falls back to the C restatement when the reference library is absent.
    Returns (GB/s, seconds, bytes, kind, sample description)."""
    from oracle import clib
    kind = "reference"
    lib = clib.reference()
    if lib is not None:
        fn = lib.ref_fft_rows
    else:
        kind = "port"
        rest = clib.restatement()

        def fn(xp, yp, n, rows):
            for r in range(rows):
                rest.orc_ref_fft(xp + r * 8 * n, yp + r * 8 * n, n)
    jobs = []
    for n in GRID_N:
        for b in GRID_B:
            rows = min(b, rows_cap)
            rng = np.random.default_rng(grid_seed(n, b))
            x = rng.standard_normal((rows, 2 * n)).astype(np.float32)
            jobs.append((n, x, np.empty_like(x)))
    chunks = []
    for n, x, y in jobs:
        step = max(1, x.shape[0] // threads)
        for r0 in range(0, x.shape[0], step):
            r1 = min(x.shape[0], r0 + step)
            chunks.append((n, x, y, r0, r1))
    nbytes = sum(16 * n * x.shape[0] for n, x, _ in jobs)

    def work(c):
        n, x, y, r0, r1 = c
        fn(x[r0:r1].ctypes.data, y[r0:r1].ctypes.data, n, r1 - r0)

    t0 = time.perf_counter()
    reps = 0
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while True:
            list(ex.map(work, chunks))
            reps += 1
            if time.perf_counter() - t0 >= budget_s:
                break
    dt = time.perf_counter() - t0
    desc = (f"grid49 with <= {rows_cap} rows per point ({nbytes / 1e6:.1f} MB algorithmic per pass), "
            f"{reps} passes, {threads} threads, {'oracle/_ref refFftF32' if kind == 'reference' else 'C restatement'}")
    return nbytes * reps / dt / 1e9, dt, nbytes * reps, kind, desc


def stdlib_numpy_sample(budget_s: float):
    """numpy.fft.fft on complex64 (the reference's stdlib baseline, scripts/bench_stdlib.py),
    single-threaded pocketfft, on the grid capped at 64 rows per point."""
    xs = []
    for n in GRID_N:
        for b in GRID_B:
            rng = np.random.default_rng(grid_seed(n, b))
            z = rng.standard_normal((min(b, 64), 2 * n)).astype(np.float32).view(np.complex64)
            xs.append(z)
    nbytes = sum(16 * z.size for z in xs)
    t0 = time.perf_counter()
    reps = 0
    while True:
        for z in xs:
            np.fft.fft(z, axis=-1)
        reps += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return nbytes * reps / dt / 1e9


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
    per_step = []
    bytes_step = 0
    kind = desc = None
    for i in range(args.warmup + args.steps):
        gbs, dt, nb, kind, desc = cpu_reference_sample(256, 0.0, threads)
        if i >= args.warmup:
            per_step.append(dt)
            bytes_step = nb
    ms = statistics.mean(per_step) * 1e3
    value = bytes_step / (ms / 1e3) / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": "rows per grid point capped at 256",
                       "points": len(GRID_N) * len(GRID_B)},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def extra_measurements(dev, stream):
    """Forms beside the plain fp32 grid (single GPU): split-BF16 tensor cores (3 and 2 bf16
    terms) vs fp32 at every point of the 49-point grid; long C2C forward + backward (batch*n =
    2^26; single pass up to n = 16384, four-step above); 2-D C2C at the reference's planned 2-D /
    range-Doppler shapes and transforms along a middle axis; non-power-of-two C2C (prime-factor,
    mixed-radix, Bluestein); STFT and inverse STFT; real transforms forward + adjoint at batch
    1024.  Each figure: algorithmic GB/s from CUDA
    events on `stream` around one replay of a CUDA graph holding 20 launches (after 3 warm-up
    launches), and the error against FP64 on sampled rows."""
    import torch
    import bfly
    import oracle.fft_oracle as O
    sh = stream.cuda_stream
    peak, _ = load_peaks()

    def timed(fn, reps=20):
        # warm-up outside the capture (table builds, workspaces), then `reps` launches captured
        # in one CUDA graph and replayed: the figure is device time, not Python call rate
        for _ in range(3):
            fn()
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            for _ in range(reps):
                fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            graph.replay()
            e0.record(stream)
            graph.replay()
            e1.record(stream)
        e1.synchronize()
        del graph
        return e0.elapsed_time(e1) / reps

    def rel(y, x, inverse=False, rows=4):
        idx = O.sample_batches(x.shape[0], rows)
        xs = x[idx].cpu().numpy().astype(np.complex128)
        ref = np.fft.ifft(xs, axis=-1) * xs.shape[-1] if inverse else np.fft.fft(xs, axis=-1)
        return O.rel_l2_rows(y[idx].cpu().numpy(), ref)

    out = {"split_bf16": {}, "long_fwd_bwd": {}, "real_fwd_adjoint": {}}
    # ---- split-BF16 tensor cores vs plain fp32 at every point of the 49-point grid
    for n, b in ((n, b) for n in GRID_N for b in GRID_B):
        g = torch.Generator(device=dev).manual_seed(grid_seed(n, b))
        x = torch.randn(b, n, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        byts = 16 * n * b
        plan = bfly.plan_for(dev, n)
        res = {}
        for tag, fn in (("fp32", lambda: plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh)),
                        ("tc_split3", lambda: plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, 3, sh)),
                        ("tc_split2", lambda: plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, 2, sh))):
            ms = timed(fn)
            gbs = byts / (ms / 1e3) / 1e9
            res[tag] = {"gbs": round(gbs, 1), "frac": round(gbs / peak, 4), "rel_l2": rel(y, x)}
        res["speedup_split3_vs_fp32"] = round(res["tc_split3"]["gbs"] / res["fp32"]["gbs"], 3)
        res["speedup_split2_vs_fp32"] = round(res["tc_split2"]["gbs"] / res["fp32"]["gbs"], 3)
        out["split_bf16"][f"n{n}_b{b}"] = res
        del x, y
    # ---- long C2C forward + backward (the backward is the conjugate-FFT adjoint)
    for n in (8192, 16384, 32768, 65536):
        b = (1 << 26) // n
        g = torch.Generator(device=dev).manual_seed(11)
        x = torch.randn(b, n, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        z = torch.empty_like(x)
        plan = bfly.plan_for(dev, n)
        byts = 16 * n * b
        ms_f = timed(lambda: plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh))
        ms_b = timed(lambda: plan.exec_c2c(y.data_ptr(), z.data_ptr(), n, b, 1, 1.0, sh))
        out["long_fwd_bwd"][f"n{n}_b{b}"] = {
            "fwd_gbs": round(byts / (ms_f / 1e3) / 1e9, 1), "bwd_gbs": round(byts / (ms_b / 1e3) / 1e9, 1),
            "fwd_bwd_gbs": round(2 * byts / ((ms_f + ms_b) / 1e3) / 1e9, 1),
            "fwd_rel_l2": rel(y, x, rows=2), "bwd_rel_l2": rel(z, y, inverse=True, rows=2),
            "schedule": "single pass" if n <= 16384 else "four-step (2 HBM passes)"}
        del x, y, z
    # ---- 2-D C2C (row pass + column pass) at the reference's planned 2-D / range-Doppler
    # shapes, batch * ny * nx = 2^26; and transforms along the middle axis of [outer][n][inner]
    out["c2c_2d"] = {}
    for ny, nx in ((256, 256), (512, 512), (1024, 1024), (2048, 2048), (1024, 128), (128, 1024)):
        b = (1 << 26) // (ny * nx)
        g = torch.Generator(device=dev).manual_seed(ny + nx)
        x = torch.randn(b, ny, nx, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        plan = bfly.plan_for(dev, nx)
        ms = timed(lambda: plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, b, -1, 1.0, sh))
        xs = x[:1].cpu().numpy().astype(np.complex128)
        ref = np.fft.fft2(xs).reshape(1, -1)
        err = float(np.linalg.norm(y[:1].cpu().numpy().reshape(1, -1) - ref) / np.linalg.norm(ref))
        out["c2c_2d"][f"{ny}x{nx}_b{b}"] = {"gbs": round(16 * ny * nx * b / ms / 1e6, 1),
                                           "frac": round(16 * ny * nx * b / ms / 1e6 / peak, 4),
                                           "rel_l2": err, "passes": 2}
        del x, y
    for n, outer, inner in ((1024, 64, 1024), (256, 1024, 256)):
        g = torch.Generator(device=dev).manual_seed(n + inner)
        x = torch.randn(outer, n, inner, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        plan = bfly.plan_for(dev, n)
        ms = timed(lambda: plan.exec_c2c_axis(x.data_ptr(), y.data_ptr(), n, outer, inner, -1, 1.0, sh))
        xs = x[:1].cpu().numpy().astype(np.complex128)
        ref = np.fft.fft(xs, axis=1)
        err = float(np.linalg.norm(y[:1].cpu().numpy() - ref) / np.linalg.norm(ref))
        out["c2c_2d"][f"axis_n{n}_outer{outer}_inner{inner}"] = {
            "gbs": round(16 * n * outer * inner / ms / 1e6, 1),
            "frac": round(16 * n * outer * inner / ms / 1e6 / peak, 4), "rel_l2": err, "passes": 1}
        del x, y
    # ---- non-power-of-two C2C, batch * n ~ 2^25: prime-factor kernel (n = A * 2^k) and
    # Bluestein (other lengths), one kernel each
    out["c2c_any_length"] = {}
    for n in (1536, 1920, 6144, 360, 1000, 3000, 6561, 12000, 1001, 1003, 8191):
        b = (1 << 25) // n
        g = torch.Generator(device=dev).manual_seed(n)
        x = torch.randn(b, n, dtype=torch.complex64, device=dev, generator=g)
        y = torch.empty_like(x)
        plan = bfly.plan_for(dev, n)
        ms = timed(lambda: plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh))
        gbs = 16 * n * b / ms / 1e6
        pfa = any(n % a == 0 and (n // a) & (n // a - 1) == 0 and n // a >= 16 for a in (3, 5, 9, 15))
        m = n
        for p in (2, 3, 5, 7, 11, 13):
            while m % p == 0:
                m //= p
        kernel = ("prime-factor" if pfa else "mixed-radix" if m == 1 and n <= 12288
                  else f"bluestein (padded length {1 << (2 * n - 2).bit_length()})")
        out["c2c_any_length"][f"n{n}_b{b}"] = {
            "gbs": round(gbs, 1), "frac": round(gbs / peak, 4), "rel_l2": rel(y, x), "kernel": kernel}
        del x, y
    # ---- STFT (frame gather + Hann window + one-sided transform in one kernel), 4 signals of
    # 2^24 samples, centred; bytes counted per frame as the reference's dense-frame R2C proxy
    out["stft"] = {}
    plan = bfly.plan_for(dev, 1024, "real")
    for n, hop in ((256, 64), (1024, 256), (4096, 1024), (400, 160)):
        L, S = 1 << 24, 4
        g = torch.Generator(device=dev).manual_seed(n)
        x = torch.randn(S, L, device=dev, generator=g)
        w = torch.hann_window(n, device=dev)
        frames = 1 + L // hop
        y = torch.empty(S, frames, n // 2 + 1, dtype=torch.complex64, device=dev)
        ms = timed(lambda: plan.exec_stft(x.data_ptr(), y.data_ptr(), n, S, L, hop, True, w.data_ptr(), sh))
        fb = S * frames * (4 * n + 8 * (n // 2 + 1))
        # the first 8 frames depend only on a prefix (left reflect padding + 8 hops + one frame)
        ref = torch.stft(x[:1, :16 * n].double(), n, hop_length=hop, window=w.double(), return_complex=True)[..., :8]
        got = y[:1, :8].transpose(-1, -2).to(torch.complex128)
        err = float((torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item())
        # inverse STFT of the same spectrum back to the 4 signals; bytes = spectrum read + signal
        # written (the two-kernel path also writes and reads every frame once in between)
        xb = torch.empty(S, L, device=dev)
        ms_i = timed(lambda: plan.exec_istft(y.data_ptr(), xb.data_ptr(), n, S, frames, hop, True, w.data_ptr(), L,
                                             1.0, sh))
        ib = S * frames * 8 * (n // 2 + 1) + 4 * S * L
        rt = float((torch.linalg.vector_norm(xb - x) / torch.linalg.vector_norm(x)).item())
        out["stft"][f"n{n}_hop{hop}_S{S}_L{L}"] = {"frame_gbs": round(fb / ms / 1e6, 1),
                                                    "frac": round(fb / ms / 1e6 / peak, 4), "rel_l2": err,
                                                    "frames": S * frames,
                                                    "istft_gbs": round(ib / ms_i / 1e6, 1),
                                                    "istft_ms": round(ms_i, 4), "round_trip_rel_l2": rt}
        del x, y, xb
    # ---- real transforms: R2C forward and its adjoint (weighted C2R), batch 1024
    for n in (128, 1024, 4096, 8192, 400, 1000):
        b = 1024
        g = torch.Generator(device=dev).manual_seed(n)
        x = torch.rand(b, n, device=dev, generator=g) * 2 - 1
        X = torch.empty(b, n // 2 + 1, dtype=torch.complex64, device=dev)
        gx = torch.empty_like(x)
        plan = bfly.plan_for(dev, n, "real")
        byts = (8 * n + 8) * b
        ms_f = timed(lambda: plan.exec_r2c(x.data_ptr(), X.data_ptr(), n, b, 1.0, 1.0, sh))
        ms_b = timed(lambda: plan.exec_c2r(X.data_ptr(), gx.data_ptr(), n, b, 1.0, 0.5, 1.0, sh))
        idx = O.sample_batches(b, 4)
        ref = np.fft.rfft(x[idx].cpu().numpy().astype(np.float64), axis=-1)
        out["real_fwd_adjoint"][f"n{n}_b{b}"] = {
            "r2c_gbs": round(byts / (ms_f / 1e3) / 1e9, 1), "adjoint_c2r_gbs": round(byts / (ms_b / 1e3) / 1e9, 1),
            "r2c_rel_l2": O.rel_l2_rows(X[idx].cpu().numpy(), ref)}
        del x, X, gx
    torch.cuda.synchronize()
    return out


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
    import oracle.fft_oracle as O

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
    for n, b, x, y in pts:   # builds twiddle tables outside any capture
        assert plan.prepare(n, b) == 0

    def check(tag):
        worst = 0.0
        for n, b, x, y in pts:
            rows = O.sample_batches(b, 2)
            ref = np.fft.fft(x[rows].cpu().numpy().astype(np.complex128), axis=-1)
            worst = max(worst, O.rel_l2_rows(y[rows].cpu().numpy(), ref))
        assert worst <= 1e-6, f"{tag} parity check failed: rel L2 {worst}"
        return worst

    def per_point():
        for n, b, x, y in pts:
            r = plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0, sh)
            if r:
                raise RuntimeError(f"exec_c2c({n},{b}) = {r}")

    # the product path: one ragged persistent launch over all 49 requests
    ragged = plan.make_ragged((x.data_ptr(), y.data_ptr(), n, b, -1, 1.0) for n, b, x, y in pts)

    def ragged_step():
        r = ragged.exec(sh)
        if r:
            raise RuntimeError(f"ragged exec = {r}")

    # parity spot checks of both paths before timing
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

    def timed(fn, steps, sample_clocks=False):
        for _ in range(max(3, args.warmup)):
            fn()
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        bus = getattr(torch.cuda.get_device_properties(dev), "pci_bus_id", None)
        sampler = ClockSampler(dev.index, bus) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        if sampler:
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

    # e2e through the C ABI with pinned host buffers: H2D + kernel + D2H per grid point
    host = []
    for (nn, bb, x, y) in pts:
        hx = torch.empty((bb, 2 * nn), dtype=torch.float32, pin_memory=True)
        hx.copy_(torch.view_as_real(x).reshape(bb, 2 * nn).cpu())
        hy = torch.empty_like(hx).pin_memory()
        host.append((nn, bb, hx.numpy(), hy.numpy()))
    e2e_steps = max(1, min(args.steps, 5))
    # (1) the whole grid in one bfly_plan_run_c2c_many call (copies of different points overlap);
    # (2) the reference's per-call pattern, bfly_plan_run_c2c once per point (reported beside it)
    many = [(hx, hy, nn, bb) for nn, bb, hx, hy in host]
    assert plan.run_many(many) == 0   # warm-up: device buffers grow to the whole grid
    for nn, bb, hx, hy in host:
        assert plan.run(hx, hy, nn, bb) == 0

    def e2e_time(step):
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            step()
        el = (time.perf_counter() - t0) / e2e_steps
        if dist:
            t = torch.tensor([el], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = t.item()
        return el

    def step_many():
        r = plan.run_many(many)
        if r:
            raise RuntimeError(f"run_many = {r}")

    def step_per_call():
        for nn, bb, hx, hy in host:
            r = plan.run(hx, hy, nn, bb)
            if r:
                raise RuntimeError(f"run({nn},{bb}) = {r}")

    e2e_s = e2e_time(step_many)
    per_call_s = e2e_time(step_per_call)
    h2d = sum(8 * nn * bb for nn, bb, _, _ in host)
    e2e_value = grid_bytes() * world / e2e_s / 1e9
    per_call_value = grid_bytes() * world / per_call_s / 1e9
    info = ragged.info()
    ragged.close()
    del graph

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    extras = extra_measurements(dev, stream) if world == 1 and not args.no_extras else None
    cpu = None
    if world == 1:
        threads = os.cpu_count() or 1
        gbs, dt, nb, kind, desc = cpu_reference_sample(256, 10.0, threads)
        cpu = {"value": round(gbs, 4), "unit": UNIT, "cores": threads, "kind": kind, "sample": desc,
               "stdlib_numpy_1core_gbs": round(stdlib_numpy_sample(3.0), 4)}
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "points": len(pts), "bytes_per_step": total_bytes,
                   "l2": "355 MB in + 355 MB out per step > 126 MB L2; no flush",
                   "launch": "one ragged launch (k_ragged_flat, one tile per CTA) per step",
                   "parallelism": f"batch-sharded replicas x{world}", "candidate": plan.candidate_id,
                   "ragged": info, "parity_rel_l2_max": worst},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": dominant_traffic(),
                     "kernel": "k_ragged_flat over the 49-point grid", "peak_kind": peak_kind,
                     "launch_us": round(ms * 1e3, 3), "algorithmic_bytes": grid_bytes()},
        "per_point_graph": {"value": round(per_point_gbs, 2), "unit": UNIT,
                            "ms_per_step": round(ms_graph, 5), "launches_per_step": len(pts)},
        "largest_launch": {"kernel": "k_c2c<4096,16,1,fwd> N=4096 batch=4096",
                           "achieved": round(dom_bytes / (dom_ms / 1e3) / 1e9, 2),
                           "frac": round(dom_bytes / (dom_ms / 1e3) / 1e9 / peak, 4),
                           "launch_us": round(dom_ms * 1e3, 3)},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d,
                "path": "bfly_plan_run_c2c_many over the 49 grid points, pinned host buffers",
                "per_call": {"value": round(per_call_value, 3), "unit": UNIT,
                             "path": "bfly_plan_run_c2c once per grid point (the reference's call pattern)"}},
        "gpu_launches": args.steps,
        "clocks": clocks.summary() if clocks else None,
        "cpu_baseline": cpu,
    }
    if extras:
        line.update(extras)
    print(json.dumps(line), flush=True)
    return 0


def run_case(spec: str, reps: int):
    """Launch one kernel configuration `reps` times without timing (for ncu captures):
    spec = kind:n:batch with kind in c2c, c2c_inv (any n: non-powers of two run the prime-factor, mixed-radix or Bluestein
    kernel), tc2, tc3 (tensor-core splits), r2c, c2r, cluster (long C2C on the cluster
    schedule), or ragged:grid:CAP; or cols:NY:NCOLS:MATS (column kernel), c2d:NY:NX:B (2-D),
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
    if kind == "ragged":   # ragged:grid:CAP -> the 49-point grid with batch capped at CAP
        cap = int(b)
        bufs = []
        for nn in GRID_N:
            for bb in GRID_B:
                bb = min(bb, cap)
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
    ap.add_argument("--no-extras", action="store_true", help="skip the split-BF16 / fwd+bwd sub-measurements")
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
