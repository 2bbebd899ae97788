"""Python mirror of the reference's plan API: Context.init(profile, space, kernel), select,
enumerate, make_plan, and Plan.prepare / run / run_r2c / run_c2r / measure with the reference's
integer status codes (TruNcat3/ascend-fft include/butterfly/plan.hpp:26-91).  Host-pointer
calls take numpy float32 arrays; exec_* calls take device pointers (ints) and a CUDA stream
handle and return immediately.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib

PKG_ROOT = Path(__file__).resolve().parents[1]
DEFAULT_PROFILE = PKG_ROOT / "config" / "b200_profile.json"
DEFAULT_SPACE = PKG_ROOT / "config" / "b200_space.json"
DEFAULT_CANDIDATE = "r16_cta256_shared_fp32_stockham"

STATUS = {0: "ok", -1: "kernel unavailable / runtime", -2: "prepare / device", -3: "alloc / stream",
          -4: "H2D / configuration", -5: "launch", -6: "sync", -7: "D2H / acceptance",
          -8: "shape or guard", -9: "already initialised", -10: "null argument",
          -11: "buffer too small"}


class BflyError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} failed with status {code} ({STATUS.get(code, '?')})")
        self.code = code


def _check(what: str, code: int) -> int:
    if code != 0:
        raise BflyError(what, code)
    return code


def _ptr(a: np.ndarray) -> int:
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


class Context:
    """bfly::Context over the C ABI.  init() returns the reference's status code."""

    def __init__(self):
        self._lib = _lib.load()
        h = C.c_void_p()
        _check("bfly_context_create", self._lib.bfly_context_create(C.byref(h)))
        self._h = h

    def init(self, profile=DEFAULT_PROFILE, space=DEFAULT_SPACE, kernel="builtin", device=None) -> int:
        args = (self._h, str(profile).encode(), str(space).encode(), str(kernel).encode())
        if device is None:
            return self._lib.bfly_context_init(*args)
        return self._lib.bfly_context_init_device(*args, int(device))

    def enumerate(self, n: int, batch: int):
        need = C.c_size_t(0)
        cnt = C.c_int(0)
        self._lib.bfly_context_enumerate(self._h, n, batch, None, 0, C.byref(cnt), C.byref(need))
        buf = C.create_string_buffer(need.value + 1)
        _check("enumerate", self._lib.bfly_context_enumerate(self._h, n, batch, buf, len(buf),
                                                               C.byref(cnt), C.byref(need)))
        out = []
        for line in buf.value.decode().splitlines():
            cid, state, reason = (line.split("\t") + ["", ""])[:3]
            out.append({"id": cid, "state": state, "reason": reason})
        return out

    def select(self, n: int, batch: int, top_k: int = 3, want_log: bool = False):
        p = C.c_void_p()
        log = C.create_string_buffer(1 << 16) if want_log else None
        rc = self._lib.bfly_context_select(self._h, n, batch, top_k, C.byref(p), log,
                                           len(log) if log is not None else 0)
        plan = Plan(self, p) if rc == 0 else None
        return (plan, log.value.decode() if log is not None else "") if want_log else plan

    def make_plan(self, candidate_id: str = DEFAULT_CANDIDATE, n: int = 1024, batch: int = 1):
        p = C.c_void_p()
        rc = self._lib.bfly_context_make_plan(self._h, n, batch, candidate_id.encode(), C.byref(p))
        return Plan(self, p) if rc == 0 else None

    def tune_ragged(self, plan, requests, want_log: bool = False):
        """Autotuned ragged work list over `requests` (as Plan.make_ragged) on `plan`: the
        launch mode and per-length radices measured fastest on these requests
        (bfly_context_tune_ragged).  Runs the list many times; outputs are overwritten."""
        arr = _ragged_array(requests)
        h = C.c_void_p()
        log = C.create_string_buffer(1 << 14) if want_log else None
        rc = self._lib.bfly_context_tune_ragged(self._h, plan._h, arr, len(arr), C.byref(h), log,
                                                len(log) if log is not None else 0)
        if rc:
            raise BflyError("bfly_context_tune_ragged", rc)
        rg = Ragged(plan, h)
        return (rg, log.value.decode()) if want_log else rg

    def set_tuning_cache(self, path) -> None:
        self._lib.bfly_context_set_tuning_cache(self._h, str(path).encode() if path else b"")

    @property
    def stream(self) -> int:
        return self._lib.bfly_context_stream(self._h) or 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bfly_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """bfly::Plan over the C ABI.  Methods return the reference's status codes."""

    def __init__(self, ctx: Context, handle: C.c_void_p):
        self._ctx = ctx   # keeps the context (and its stream) alive
        self._lib = ctx._lib
        self._h = handle

    @property
    def candidate_id(self) -> str:
        buf = C.create_string_buffer(256)
        self._lib.bfly_plan_candidate_id(self._h, buf, len(buf))
        return buf.value.decode()

    def prepare(self, n: int, batch: int = 0xFFFFFFFF) -> int:
        return self._lib.bfly_plan_prepare(self._h, n, batch)

    # ---- synchronous host-pointer API (numpy float32 buffers)
    def run(self, x: np.ndarray, out: np.ndarray, n: int, batch: int) -> int:
        return self._lib.bfly_plan_run_c2c(self._h, _ptr(x), _ptr(out), n, batch)

    def run_many(self, requests) -> int:
        """Host-to-host C2C of many requests in one pipelined call.  `requests`: iterable of
        (x, out, n, batch) or (x, out, n, batch, direction, scale) with C-contiguous numpy
        float32 [batch][2n] arrays (pinned memory for full PCIe bandwidth)."""
        reqs = list(requests)
        arr = (_lib.HostRequest * len(reqs))()
        for i, r in enumerate(reqs):
            x, out, n, batch = r[:4]
            direction, scale = (r[4], r[5]) if len(r) > 4 else (-1, 1.0)
            arr[i] = _lib.HostRequest(_ptr(x), _ptr(out), n, batch, direction, scale)
        return self._lib.bfly_plan_run_c2c_many(self._h, arr if reqs else None, len(reqs))

    def run_r2c(self, x: np.ndarray, out: np.ndarray, n: int, batch: int) -> int:
        return self._lib.bfly_plan_run_r2c(self._h, _ptr(x), _ptr(out), n, batch)

    def run_c2r(self, x: np.ndarray, out: np.ndarray, n: int, batch: int) -> int:
        return self._lib.bfly_plan_run_c2r(self._h, _ptr(x), _ptr(out), n, batch)

    def run_inverse(self, x: np.ndarray, out: np.ndarray, n: int, batch: int, scale: float = 1.0) -> int:
        return self._lib.bfly_plan_run_c2c_inverse(self._h, _ptr(x), _ptr(out), n, batch, scale)

    def run_long(self, x: np.ndarray, out: np.ndarray, n: int, batch: int, direction: int = -1) -> int:
        return self._lib.bfly_plan_run_c2c_long(self._h, _ptr(x), _ptr(out), n, batch, direction)

    def measure(self, n: int, batch: int):
        m = _lib.Metric()
        rc = self._lib.bfly_plan_measure(self._h, n, batch, C.byref(m))
        return rc, {"eta_us": m.eta_us, "measured_us": m.measured_us,
                    "max_rel_err": m.max_rel_err, "measured_ok": bool(m.measured_ok)}

    # ---- asynchronous device-pointer API
    def exec_c2c(self, d_in: int, d_out: int, n: int, batch: int, direction: int = -1,
                 scale: float = 1.0, stream: int = 0) -> int:
        return self._lib.bfly_plan_exec_c2c_async(self._h, d_in, d_out, n, batch, direction,
                                                  scale, stream or None)

    def exec_c2c_2d(self, d_in: int, d_out: int, ny: int, nx: int, batch: int, direction: int = -1,
                    scale: float = 1.0, stream: int = 0) -> int:
        """2-D C2C over [batch][ny][nx] complex64 device memory."""
        return self._lib.bfly_plan_exec_c2c_2d_async(self._h, d_in, d_out, ny, nx, batch, direction,
                                                     scale, stream or None)

    def exec_r2c_2d(self, d_in: int, d_out: int, ny: int, nx: int, batch: int, scale: float = 1.0,
                    stream: int = 0) -> int:
        """[batch][ny][nx] float32 -> [batch][ny][nx/2+1] complex64 (rfft2), times scale."""
        return self._lib.bfly_plan_exec_r2c_2d_async(self._h, d_in, d_out, ny, nx, batch, scale, stream or None)

    def exec_c2r_2d(self, d_in: int, d_out: int, ny: int, nx: int, batch: int, scale: float = 1.0,
                    stream: int = 0) -> int:
        """[batch][ny][nx/2+1] complex64 -> [batch][ny][nx] float32 (irfft2 times ny*nx*scale)."""
        return self._lib.bfly_plan_exec_c2r_2d_async(self._h, d_in, d_out, ny, nx, batch, scale, stream or None)

    def exec_c2c_axis(self, d_in: int, d_out: int, n: int, outer: int, inner: int,
                      direction: int = -1, scale: float = 1.0, stream: int = 0) -> int:
        """C2C along the middle axis of a contiguous [outer][n][inner] complex64 array."""
        return self._lib.bfly_plan_exec_c2c_axis_async(self._h, d_in, d_out, n, outer, inner,
                                                       direction, scale, stream or None)

    def exec_stft(self, d_sig: int, d_out: int, n: int, signals: int, sig_len: int, hop: int,
                  center: bool = True, d_window: int = 0, stream: int = 0):
        """STFT into [signals][frames][n/2+1] complex64; returns (status, frames)."""
        frames = C.c_uint64(0)
        rc = self._lib.bfly_plan_exec_stft_async(self._h, d_sig, d_out, n, signals, sig_len, hop,
                                                 1 if center else 0, d_window or None, C.byref(frames),
                                                 stream or None)
        return rc, frames.value

    def exec_istft(self, d_spec: int, d_out: int, n: int, signals: int, frames: int, hop: int,
                   center: bool = True, d_window: int = 0, out_len: int = 0, scale: float = 1.0,
                   stream: int = 0) -> int:
        """Inverse STFT of [signals][frames][n/2+1] complex64 into [signals][out_len] float32."""
        return self._lib.bfly_plan_exec_istft_async(self._h, d_spec, d_out, n, signals, frames, hop,
                                                    1 if center else 0, d_window or None, out_len, scale,
                                                    stream or None)

    def exec_stft_backward(self, d_grad_spec: int, d_grad_sig: int, n: int, signals: int, sig_len: int,
                           hop: int, center: bool = True, d_window: int = 0, stream: int = 0) -> int:
        """Gradient of exec_stft's signal from the gradient of its output, one kernel."""
        return self._lib.bfly_plan_exec_stft_backward_async(self._h, d_grad_spec, d_grad_sig, n, signals, sig_len,
                                                            hop, 1 if center else 0, d_window or None,
                                                            stream or None)

    def exec_istft_backward(self, d_grad_out: int, d_grad_spec: int, n: int, signals: int, frames: int, hop: int,
                            center: bool = True, d_window: int = 0, out_len: int = 0, scale: float = 1.0,
                            stream: int = 0) -> int:
        """Gradient of exec_istft's spectrum from the gradient of its output, one kernel."""
        return self._lib.bfly_plan_exec_istft_backward_async(self._h, d_grad_out, d_grad_spec, n, signals, frames,
                                                             hop, 1 if center else 0, d_window or None, out_len,
                                                             scale, stream or None)

    def exec_r2c(self, d_in: int, d_out: int, n: int, batch: int, s_edge: float = 1.0,
                 s_int: float = 1.0, stream: int = 0) -> int:
        return self._lib.bfly_plan_exec_r2c_async(self._h, d_in, d_out, n, batch, s_edge, s_int,
                                                  stream or None)

    def exec_c2r(self, d_in: int, d_out: int, n: int, batch: int, s_edge: float = 1.0,
                 s_int: float = 1.0, out_scale: float | None = None, stream: int = 0) -> int:
        if out_scale is None:
            out_scale = 1.0 / n
        return self._lib.bfly_plan_exec_c2r_async(self._h, d_in, d_out, n, batch, s_edge, s_int,
                                                  out_scale, stream or None)

    def exec_c2c_tc(self, d_in: int, d_out: int, n: int, batch: int, direction: int = -1,
                    scale: float = 1.0, split_terms: int = 3, stream: int = 0) -> int:
        """Split-BF16 tensor-core C2C (n a power of two in 64..4096; 2 or 3 bf16 terms)."""
        return self._lib.bfly_plan_exec_c2c_tc_async(self._h, d_in, d_out, n, batch, direction, scale,
                                                     split_terms, stream or None)

    def tc_device_status(self) -> int:
        st = C.c_uint()
        rc = self._lib.bfly_tc_device_status(C.byref(st))
        if rc:
            raise BflyError("bfly_tc_device_status", rc)
        return st.value

    def long_device_status(self) -> int:
        """Error word of the single-pass cluster long C2C (0 = clean); reading clears it."""
        st = C.c_uint()
        rc = self._lib.bfly_long_device_status(C.byref(st))
        if rc:
            raise BflyError("bfly_long_device_status", rc)
        return st.value

    def make_ragged(self, requests, mode=None, radix8=None):
        """requests: iterable of (d_in, d_out, n, batch, direction, scale) with device
        pointers; returns a Ragged whose exec(stream) is one persistent kernel launch.
        mode / radix8 give an explicit launch configuration (bfly_ragged_create_config);
        left out, the default applies."""
        arr = _ragged_array(requests)
        h = C.c_void_p()
        if mode is None and radix8 is None:
            rc = self._lib.bfly_ragged_create(self._h, arr, len(arr), C.byref(h))
            what = "bfly_ragged_create"
        else:
            rc = self._lib.bfly_ragged_create_config(self._h, arr, len(arr), -1 if mode is None else mode,
                                                     0x3 if radix8 is None else radix8, C.byref(h))
            what = "bfly_ragged_create_config"
        if rc:
            raise BflyError(what, rc)
        return Ragged(self, h)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bfly_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ragged_array(requests):
    reqs = list(requests)
    arr = (_lib.RaggedRequest * len(reqs))()
    for i, (din, dout, n, b, d, sc) in enumerate(reqs):
        arr[i] = _lib.RaggedRequest(din, dout, n, d, b, sc, 0)
    return arr


class Ragged:
    """One persistent launch over many C2C requests (bfly_ragged_* of the C ABI)."""

    def __init__(self, plan: Plan, handle: C.c_void_p):
        self._plan = plan   # the ragged work list uses the plan's twiddle tables
        self._lib = plan._lib
        self._h = handle

    def exec(self, stream: int = 0) -> int:
        return self._lib.bfly_ragged_exec_async(self._h, stream or None)

    def info(self):
        tiles = C.c_uint64()
        grid = C.c_int()
        stages = C.c_int()
        self._lib.bfly_ragged_info(self._h, C.byref(tiles), C.byref(grid), C.byref(stages))
        radix8 = C.c_uint32()
        self._lib.bfly_ragged_config(self._h, None, C.byref(radix8))
        return {"tiles": tiles.value, "grid": grid.value, "stages": stages.value, "radix8": radix8.value}

    def device_status(self) -> int:
        """0, or 1 when a staged launch gave up on a bounded wait (reading clears it)."""
        st = C.c_uint()
        rc = self._lib.bfly_ragged_device_status(C.byref(st))
        if rc:
            raise BflyError("bfly_ragged_device_status", rc)
        return st.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bfly_ragged_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
