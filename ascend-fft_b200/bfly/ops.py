"""torch.fft-style functions on CUDA tensors backed by the hand-written sm_100a kernels, with
hand-written adjoints behind torch.autograd.Function:

    fft(x)   / ifft(x)      complex64 [..., n], n in 32..65536 (four-step above 16384 points
                            per row, or when the plan schedules it)
    rfft(x)                 float32 [..., n] -> complex64 [..., n/2+1], n in 64..8192
    irfft(X, n)             complex64 [..., n/2+1] -> float32 [..., n]

`norm` follows torch.fft ("backward", "ortho", "forward").  Adjoints:
    fft  : grad_x = s * IFFT_unnormalised(g)          (conjugate FFT)
    ifft : grad_x = s * FFT(g)
    rfft : grad_x = C2R(g) with bins 0 and n/2 weighted 1 and the others 1/2, times s
    irfft: grad_X = R2C(g) with bins 0 and n/2 weighted c and the others 2c  (c = output scale)
Every call enqueues on torch's current stream; nothing runs on the CPU.
"""
from __future__ import annotations

import math
import threading

import torch

from .core import DEFAULT_CANDIDATE, BflyError, Context

_lock = threading.Lock()
_state = {}   # device index -> (Context, Plan)


def plan_for(device: torch.device):
    """Per-device context and default plan (created on first use)."""
    idx = device.index if device.index is not None else torch.cuda.current_device()
    with _lock:
        if idx not in _state:
            ctx = Context()
            rc = ctx.init(device=idx)
            if rc != 0:
                raise BflyError("Context.init", rc)
            plan = ctx.make_plan(DEFAULT_CANDIDATE)
            if plan is None:
                raise BflyError("make_plan", -1)
            _state[idx] = (ctx, plan)
        return _state[idx][1]


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _scale(norm: str | None, n: int, forward: bool) -> float:
    norm = norm or "backward"
    if norm == "ortho":
        return 1.0 / math.sqrt(n)
    if norm == "backward":
        return 1.0 if forward else 1.0 / n
    if norm == "forward":
        return 1.0 / n if forward else 1.0
    raise ValueError(f"invalid norm {norm!r}")


def _need_cuda(t: torch.Tensor, dtype: torch.dtype, what: str):
    if not t.is_cuda:
        raise ValueError(f"{what}: input must be a CUDA tensor (no CPU path)")
    if t.dtype != dtype:
        raise TypeError(f"{what}: expected {dtype}, got {t.dtype}")


def c2c(x: torch.Tensor, direction: int, scale: float, out: torch.Tensor | None = None) -> torch.Tensor:
    _need_cuda(x, torch.complex64, "c2c")
    x = x.contiguous()
    n = x.shape[-1]
    batch = x.numel() // n if n else 0
    y = out if out is not None else torch.empty_like(x)
    if batch == 0:
        return y
    rc = plan_for(x.device).exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, _stream(x))
    if rc:
        raise BflyError(f"exec_c2c(n={n}, batch={batch})", rc)
    return y


def r2c(x: torch.Tensor, s_edge: float = 1.0, s_int: float = 1.0) -> torch.Tensor:
    _need_cuda(x, torch.float32, "r2c")
    x = x.contiguous()
    n = x.shape[-1]
    batch = x.numel() // n if n else 0
    y = torch.empty(*x.shape[:-1], n // 2 + 1, dtype=torch.complex64, device=x.device)
    if batch == 0:
        return y
    rc = plan_for(x.device).exec_r2c(x.data_ptr(), y.data_ptr(), n, batch, s_edge, s_int, _stream(x))
    if rc:
        raise BflyError(f"exec_r2c(n={n}, batch={batch})", rc)
    return y


def c2r(X: torch.Tensor, n: int, s_edge: float = 1.0, s_int: float = 1.0,
        out_scale: float | None = None) -> torch.Tensor:
    _need_cuda(X, torch.complex64, "c2r")
    X = X.contiguous()
    if X.shape[-1] != n // 2 + 1:
        raise ValueError(f"c2r: last dimension {X.shape[-1]} != n/2+1 = {n // 2 + 1}")
    batch = X.numel() // X.shape[-1] if X.shape[-1] else 0
    y = torch.empty(*X.shape[:-1], n, dtype=torch.float32, device=X.device)
    if batch == 0:
        return y
    if out_scale is None:
        out_scale = 1.0 / n
    rc = plan_for(X.device).exec_c2r(X.data_ptr(), y.data_ptr(), n, batch, s_edge, s_int, out_scale,
                                     _stream(X))
    if rc:
        raise BflyError(f"exec_c2r(n={n}, batch={batch})", rc)
    return y


class _FFT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, direction, scale):
        ctx.direction, ctx.scale = direction, scale
        return c2c(x, direction, scale)

    @staticmethod
    def backward(ctx, g):
        return c2c(g.contiguous(), -ctx.direction, ctx.scale), None, None


class _RFFT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, scale):
        ctx.scale, ctx.n = scale, x.shape[-1]
        y = r2c(x)
        return y if scale == 1.0 else y * scale

    @staticmethod
    def backward(ctx, g):
        return c2r(g.contiguous(), ctx.n, 1.0, 0.5, ctx.scale), None


class _IRFFT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, X, n, scale):
        ctx.scale = scale
        return c2r(X, n, 1.0, 1.0, scale)

    @staticmethod
    def backward(ctx, g):
        c = ctx.scale
        return r2c(g.contiguous(), c, 2.0 * c), None, None


def fft(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    return _FFT.apply(x, -1, _scale(norm, x.shape[-1], True))


def ifft(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    return _FFT.apply(x, 1, _scale(norm, x.shape[-1], False))


def rfft(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    return _RFFT.apply(x, _scale(norm, x.shape[-1], True))


def irfft(X: torch.Tensor, n: int | None = None, norm: str | None = None) -> torch.Tensor:
    if n is None:
        n = 2 * (X.shape[-1] - 1)
    return _IRFFT.apply(X, n, _scale(norm, n, False))
