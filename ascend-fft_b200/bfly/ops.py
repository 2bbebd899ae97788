"""torch.fft-style functions on CUDA tensors backed by the hand-written sm_100a kernels, with
hand-written adjoints behind torch.autograd.Function:

    fft(x, dim) / ifft(x, dim)  complex64, n in 32..65536 along the last dim (four-step above
                            16384 points per row), 32..4096 along any other dim (column kernel
                            over the contiguous [outer][n][inner] view)
    fft2(x) / ifft2(x)      complex64 [..., ny, nx]: row pass (nx as fft) + column pass
                            (ny in 32..4096)
    rfft2(x) / irfft2(X)    float32 [..., ny, nx] <-> complex64 [..., ny, nx/2+1] (row R2C + column
                            pass; ny in 32..4096)
    stft(x, n_fft, ...)     float32 [..., L] -> complex64 [..., n_fft/2+1, frames], torch.stft's
                            arguments and defaults (centred reflect padding, hop n_fft/4); framing,
                            window and one-sided transform in one kernel
    istft(X, n_fft, ...)    complex64 [..., n_fft/2+1, frames] -> float32 [..., L], torch.istft's
                            arguments; C2R of every frame, then a windowed overlap-add kernel
    rfft(x)                 float32 [..., n] -> complex64 [..., n/2+1], n in 64..8192 a power of
                            two, or even with n/2 13-smooth (up to 24576)
    irfft(X, n)             complex64 [..., n/2+1] -> float32 [..., n]

`norm` follows torch.fft ("backward", "ortho", "forward").  Adjoints:
    fft  : grad_x = s * IFFT_unnormalised(g)          (conjugate FFT; same for fft2 and any dim)
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
_state = {}   # device index -> {"ctx": Context, "plans": {candidate id: Plan}, "tuned": {...}}

# Kernel variant per length measured fastest on B200 (radix = complex values per thread,
# cta = threads per CTA); lengths not listed use DEFAULT_CANDIDATE.  C2C keys are the transform
# length, real-transform keys the inner complex length n/2.
BEST_C2C = {32: "r8_cta256_shared_fp32_stockham", 64: "r8_cta256_shared_fp32_stockham",
            128: "r16_cta128_shared_fp32_stockham", 256: "r16_cta128_shared_fp32_stockham",
            512: "r16_cta128_shared_fp32_stockham", 1024: "r16_cta256_shared_fp32_stockham",
            2048: "r16_cta128_shared_fp32_stockham", 4096: "r16_cta256_shared_fp32_stockham",
            8192: "r16_cta512_shared_fp32_stockham", 16384: "r16_cta1024_shared_fp32_stockham"}
BEST_REAL = {32: "r8_cta256_shared_fp32_stockham", 64: "r8_cta256_shared_fp32_stockham",
             128: "r16_cta128_shared_fp32_stockham", 256: "r16_cta128_shared_fp32_stockham",
             512: "r16_cta128_shared_fp32_stockham", 1024: "r16_cta128_shared_fp32_stockham",
             2048: "r16_cta128_shared_fp32_stockham"}


def _device_state(device: torch.device):
    idx = device.index if device.index is not None else torch.cuda.current_device()
    with _lock:
        if idx not in _state:
            ctx = Context()
            rc = ctx.init(device=idx)
            if rc != 0:
                raise BflyError("Context.init", rc)
            _state[idx] = {"ctx": ctx, "plans": {}, "tuned": {}}
        return _state[idx]


def _plan_by_id(st, cid: str, n: int):
    with _lock:
        p = st["plans"].get(cid)
        if p is None:
            p = st["ctx"].make_plan(cid, n, 1)
            if p is None:
                raise BflyError(f"make_plan({cid})", -1)
            st["plans"][cid] = p
        return p


def plan_for(device: torch.device, n: int | None = None, kind: str = "c2c"):
    """Plan serving a transform of length n on `device`: an autotuned choice when one was made
    with autotune(), else the measured per-length default, else DEFAULT_CANDIDATE."""
    st = _device_state(device)
    if n is not None and (kind, n) in st["tuned"]:
        return st["tuned"][(kind, n)]
    table = BEST_C2C if kind == "c2c" else BEST_REAL
    key = n if kind == "c2c" else (n // 2 if n else None)
    cid = table.get(key, DEFAULT_CANDIDATE) if key is not None else DEFAULT_CANDIDATE
    # a C2C entry is feasible at its own length (16384 has only the 1024-thread kernel); the
    # real-transform entries, keyed by n/2, and the default are all feasible at 1024
    return _plan_by_id(st, cid, n if kind == "c2c" and n in BEST_C2C else 1024)


def autotune(n: int, batch: int, device: torch.device | None = None, top_k: int = 3,
             cache: str | None = None):
    """Measure candidates for a C2C of length n with the library's autotuner (Context.select)
    and use the fastest for later fft/ifft calls of that length; the choice is persisted in the
    JSON tuning cache `cache` (default $BFLY_TUNING_CACHE, else none).  Returns the log."""
    import os
    device = device or torch.device("cuda", torch.cuda.current_device())
    st = _device_state(device)
    path = cache or os.environ.get("BFLY_TUNING_CACHE")
    if path:
        st["ctx"].set_tuning_cache(path)
    plan, log = st["ctx"].select(n, batch, top_k, want_log=True)
    if plan is None:
        raise BflyError(f"select(n={n}, batch={batch})", -1)
    st["tuned"][("c2c", n)] = plan
    return log


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
    rc = plan_for(x.device, n).exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, _stream(x))
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
    rc = plan_for(x.device, n, "real").exec_r2c(x.data_ptr(), y.data_ptr(), n, batch, s_edge, s_int, _stream(x))
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
    rc = plan_for(X.device, n, "real").exec_c2r(X.data_ptr(), y.data_ptr(), n, batch, s_edge, s_int,
                                                out_scale, _stream(X))
    if rc:
        raise BflyError(f"exec_c2r(n={n}, batch={batch})", rc)
    return y


def _outer_inner(shape, dim: int):
    outer = 1
    for s in shape[:dim]:
        outer *= s
    inner = 1
    for s in shape[dim + 1:]:
        inner *= s
    return outer, inner


def c2c_axis(x: torch.Tensor, dim: int, direction: int, scale: float) -> torch.Tensor:
    """C2C along dimension `dim` of a complex64 CUDA tensor (any dim; contiguous copy made)."""
    _need_cuda(x, torch.complex64, "c2c_axis")
    dim = dim % x.dim()
    if dim == x.dim() - 1:
        return c2c(x, direction, scale)
    x = x.contiguous()
    n = x.shape[dim]
    outer, inner = _outer_inner(x.shape, dim)
    y = torch.empty_like(x)
    if x.numel() == 0:
        return y
    rc = plan_for(x.device, n).exec_c2c_axis(x.data_ptr(), y.data_ptr(), n, outer, inner, direction, scale,
                                             _stream(x))
    if rc:
        raise BflyError(f"exec_c2c_axis(n={n}, outer={outer}, inner={inner})", rc)
    return y


def c2c_2d(x: torch.Tensor, direction: int, scale: float) -> torch.Tensor:
    """2-D C2C over the last two dimensions of a complex64 CUDA tensor."""
    _need_cuda(x, torch.complex64, "c2c_2d")
    _need_2d(x, "c2c_2d")
    x = x.contiguous()
    ny, nx = x.shape[-2], x.shape[-1]
    batch = x.numel() // (ny * nx) if ny * nx else 0
    y = torch.empty_like(x)
    if batch == 0:
        return y
    rc = plan_for(x.device, nx).exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, batch, direction, scale,
                                            _stream(x))
    if rc:
        raise BflyError(f"exec_c2c_2d(ny={ny}, nx={nx}, batch={batch})", rc)
    return y


class _FFTAxis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, dim, direction, scale):
        ctx.dim, ctx.direction, ctx.scale = dim, direction, scale
        return c2c_axis(x, dim, direction, scale)

    @staticmethod
    def backward(ctx, g):
        return c2c_axis(g, ctx.dim, -ctx.direction, ctx.scale), None, None, None


class _FFT2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, direction, scale):
        ctx.direction, ctx.scale = direction, scale
        return c2c_2d(x, direction, scale)

    @staticmethod
    def backward(ctx, g):
        return c2c_2d(g, -ctx.direction, ctx.scale), None, None


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
        return r2c(x, scale, scale)   # the scale rides on the kernel's per-bin weights

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


def c2c_tensor(x: torch.Tensor, direction: int = -1, scale: float = 1.0, split_terms: int = 3) -> torch.Tensor:
    """Split-BF16 tensor-core C2C (n a power of two in 64..4096) on torch's current stream."""
    _need_cuda(x, torch.complex64, "c2c_tensor")
    x = x.contiguous()
    n = x.shape[-1]
    batch = x.numel() // n if n else 0
    y = torch.empty_like(x)
    if batch == 0:
        return y
    rc = plan_for(x.device, n).exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, batch, direction, scale,
                                           split_terms, _stream(x))
    if rc:
        raise BflyError(f"exec_c2c_tc(n={n}, batch={batch})", rc)
    return y


def fft(x: torch.Tensor, norm: str | None = None, dim: int = -1) -> torch.Tensor:
    if dim % max(x.dim(), 1) != x.dim() - 1:
        return _FFTAxis.apply(x, dim, -1, _scale(norm, x.shape[dim], True))
    return _FFT.apply(x, -1, _scale(norm, x.shape[-1], True))


def ifft(x: torch.Tensor, norm: str | None = None, dim: int = -1) -> torch.Tensor:
    if dim % max(x.dim(), 1) != x.dim() - 1:
        return _FFTAxis.apply(x, dim, 1, _scale(norm, x.shape[dim], False))
    return _FFT.apply(x, 1, _scale(norm, x.shape[-1], False))


def _pow2(n: int) -> bool:
    return n >= 64 and n <= 8192 and n & (n - 1) == 0


class _STFT(torch.autograd.Function):
    """Framing + window + R2C in one kernel; the window is a constant (no gradient)."""

    @staticmethod
    def forward(ctx, x, n, hop, center, window):
        signals, length = x.shape
        frames = (1 + length // hop) if center else (1 + (length - n) // hop)
        y = torch.empty(signals, frames, n // 2 + 1, dtype=torch.complex64, device=x.device)
        rc, got = plan_for(x.device, n, "real").exec_stft(
            x.data_ptr(), y.data_ptr(), n, signals, length, hop, center,
            window.data_ptr() if window is not None else 0, _stream(x))
        if rc:
            raise BflyError(f"exec_stft(n={n}, signals={signals}, length={length}, hop={hop})", rc)
        assert got == frames
        ctx.n, ctx.hop, ctx.center, ctx.length = n, hop, center, length
        ctx.save_for_backward(window)
        return y

    @staticmethod
    def backward(ctx, g):
        (window,) = ctx.saved_tensors
        n, hop, length = ctx.n, ctx.hop, ctx.length
        signals, frames = g.shape[0], g.shape[1]
        if _pow2(n) and (length >= n + 2 if ctx.center else length >= n):
            # one kernel: each frame's weighted C2R, the window, the overlap-add and the fold of
            # the reflect padding
            gx = torch.empty(signals, length, dtype=torch.float32, device=g.device)
            rc = plan_for(g.device, n, "real").exec_stft_backward(
                g.contiguous().data_ptr(), gx.data_ptr(), n, signals, length, hop, ctx.center,
                window.data_ptr() if window is not None else 0, _stream(g))
            if rc:
                raise BflyError(f"exec_stft_backward(n={n}, signals={signals}, length={length}, hop={hop})", rc)
            return gx, None, None, None, None
        # other lengths: the adjoint of each frame's one-sided transform (the weighted C2R of
        # rfft's backward), then the window, overlap-add and reflect fold
        fr = c2r(g.contiguous().reshape(signals * frames, n // 2 + 1), n, 1.0, 0.5, 1.0)
        fr = fr.reshape(signals, frames, n)
        if window is not None:
            fr = fr * window
        pad = n // 2 if ctx.center else 0
        padded = length + 2 * pad
        gp = torch.nn.functional.fold(fr.transpose(1, 2), output_size=(1, padded), kernel_size=(1, n),
                                      stride=(1, hop)).reshape(signals, padded)
        gx = gp[:, pad:pad + length].clone()
        if pad:   # reflected samples: x[-i] = x[i], x[L-1+i] = x[L-1-i]
            gx[:, 1:pad + 1] += gp[:, :pad].flip(-1)
            gx[:, length - 1 - pad:length - 1] += gp[:, pad + length:].flip(-1)
        return gx, None, None, None, None


def stft(x: torch.Tensor, n_fft: int, hop_length: int | None = None, win_length: int | None = None,
         window: torch.Tensor | None = None, center: bool = True, pad_mode: str = "reflect",
         normalized: bool = False, onesided: bool | None = None,
         return_complex: bool | None = None) -> torch.Tensor:
    """torch.stft on the fused kernel: float32 [..., L] -> complex64 [..., n_fft/2+1, frames].
    Arguments in torch.stft's order and with its defaults (a window shorter than n_fft is
    centred with zeros)."""
    _need_cuda(x, torch.float32, "stft")
    if return_complex is False or onesided is False:
        raise ValueError("stft: only onesided=True, return_complex=True are supported")
    if center and pad_mode != "reflect":
        raise ValueError("stft: only pad_mode='reflect' is supported")
    hop = hop_length if hop_length is not None else n_fft // 4
    window = _pad_window(window, win_length, n_fft, "stft window", x.device)
    if normalized:
        window = (window if window is not None else torch.ones(n_fft, device=x.device)) * n_fft ** -0.5
    lead = x.shape[:-1]
    y = _STFT.apply(x.contiguous().reshape(-1, x.shape[-1]), n_fft, hop, center, window)
    return y.reshape(*lead, y.shape[-2], y.shape[-1]).transpose(-1, -2)


class _ISTFT(torch.autograd.Function):
    """Inverse transform of every frame + windowed overlap-add divided by the squared-window
    envelope.  Adjoint: h = g / envelope on the padded timeline (zero outside the kept samples),
    then the uncentred windowed STFT of h, weighted like irfft's adjoint (bins 0 and n/2 by c,
    the others by 2c, c = scale / n)."""

    @staticmethod
    def forward(ctx, spec, n, hop, center, window, out_len, scale):
        signals, frames = spec.shape[0], spec.shape[1]
        y = torch.empty(signals, out_len, dtype=torch.float32, device=spec.device)
        rc = plan_for(spec.device, n, "real").exec_istft(
            spec.data_ptr(), y.data_ptr(), n, signals, frames, hop, center,
            window.data_ptr() if window is not None else 0, out_len, scale, _stream(spec))
        if rc:
            raise BflyError(f"exec_istft(n={n}, signals={signals}, frames={frames}, hop={hop})", rc)
        ctx.n, ctx.hop, ctx.center, ctx.scale, ctx.frames = n, hop, center, scale, frames
        ctx.save_for_backward(window)
        return y

    @staticmethod
    def backward(ctx, g):
        (window,) = ctx.saved_tensors
        n, hop, frames = ctx.n, ctx.hop, ctx.frames
        if _pow2(n):
            # one kernel: the frames of g / envelope, windowed, transformed and weighted
            gs = torch.empty(g.shape[0], frames, n // 2 + 1, dtype=torch.complex64, device=g.device)
            rc = plan_for(g.device, n, "real").exec_istft_backward(
                g.contiguous().data_ptr(), gs.data_ptr(), n, g.shape[0], frames, hop, ctx.center,
                window.data_ptr() if window is not None else 0, g.shape[1], ctx.scale, _stream(g))
            if rc:
                raise BflyError(f"exec_istft_backward(n={n}, frames={frames}, hop={hop})", rc)
            return gs, None, None, None, None, None, None
        padded = n + hop * (frames - 1)
        start = n // 2 if ctx.center else 0
        env = _envelope(window, n, hop, frames, g.device)
        keep = max(0, min(g.shape[1], padded - start))
        h = torch.zeros(g.shape[0], padded, dtype=torch.float32, device=g.device)
        e = env[start:start + keep]
        h[:, start:start + keep] = torch.where(e > 0, g[:, :keep] / torch.where(e > 0, e, 1.0), 0.0)
        gs = torch.empty(g.shape[0], frames, n // 2 + 1, dtype=torch.complex64, device=g.device)
        rc, got = plan_for(g.device, n, "real").exec_stft(
            h.data_ptr(), gs.data_ptr(), n, g.shape[0], padded, hop, False,
            window.data_ptr() if window is not None else 0, _stream(g))
        if rc or got != frames:
            raise BflyError(f"exec_stft (istft adjoint, n={n}, frames={frames})", rc or -1)
        c = ctx.scale / n
        wt = torch.full((n // 2 + 1,), 2.0 * c, dtype=torch.float32, device=g.device)
        wt[0] = wt[-1] = c
        return gs * wt, None, None, None, None, None, None


def _envelope(window, n: int, hop: int, frames: int, device) -> torch.Tensor:
    """Overlap-added squared window over the padded timeline, n + hop*(frames-1) samples."""
    w2 = (window * window) if window is not None else torch.ones(n, device=device)
    cols = w2.reshape(1, n, 1).expand(1, n, frames)
    padded = n + hop * (frames - 1)
    return torch.nn.functional.fold(cols, output_size=(1, padded), kernel_size=(1, n),
                                    stride=(1, hop)).reshape(padded)


_envelope_checked = {}   # (window ptr, version, n, hop, frames, start, length) already verified


def _pad_window(window, win_length, n_fft, what, device):
    """torch.stft / torch.istft window handling: shape (win_length,), centred in n_fft with zeros."""
    if window is None:
        if win_length is None or win_length == n_fft:
            return None
        window = torch.ones(win_length, dtype=torch.float32, device=device)
    _need_cuda(window, torch.float32, what)
    wl = win_length if win_length is not None else n_fft
    if window.shape != (wl,) or wl > n_fft or wl < 1:
        raise ValueError(f"{what}: window must have shape ({wl},) with win_length <= n_fft")
    if wl < n_fft:
        left = (n_fft - wl) // 2
        window = torch.nn.functional.pad(window, (left, n_fft - wl - left))
    return window.contiguous()


def istft(X: torch.Tensor, n_fft: int, hop_length: int | None = None, win_length: int | None = None,
          window: torch.Tensor | None = None, center: bool = True, normalized: bool = False,
          onesided: bool | None = None, length: int | None = None,
          return_complex: bool = False) -> torch.Tensor:
    """torch.istft on the device kernels: complex64 [..., n_fft/2+1, frames] -> float32 [..., L].

    Every frame is inverse-transformed (irfft, 1/n_fft), multiplied by the window and overlap-
    added; each sample is divided by the overlap-added squared window, as torch.istft does, and
    a window envelope below 1e-11 inside the kept samples raises like torch.istft."""
    _need_cuda(X, torch.complex64, "istft")
    if return_complex or onesided is False:
        raise ValueError("istft: only onesided input and real output are supported")
    if X.dim() < 2 or X.shape[-2] != n_fft // 2 + 1:
        raise ValueError(f"istft: expected [..., {n_fft // 2 + 1}, frames], got {tuple(X.shape)}")
    hop = hop_length if hop_length is not None else n_fft // 4
    if hop <= 0 or hop > n_fft:
        raise ValueError(f"istft: hop_length must be in [1, n_fft], got {hop}")
    window = _pad_window(window, win_length, n_fft, "istft window", X.device)
    frames = X.shape[-1]
    padded = n_fft + hop * (frames - 1)
    start = n_fft // 2 if center else 0
    out_len = length if length is not None else padded - 2 * start
    if out_len <= 0:
        raise ValueError("istft: empty output")
    # the envelope of the kept samples must not vanish (torch.istft's check); verified once per
    # window contents and geometry
    key = (window.data_ptr() if window is not None else 0, window._version if window is not None else 0,
           X.device.index, n_fft, hop, frames, start, out_len)
    if key not in _envelope_checked:
        env = _envelope(window, n_fft, hop, frames, X.device)[start:start + out_len]
        if env.numel() and float(env.min()) < 1e-11:
            raise RuntimeError("istft: window overlap-add envelope is zero inside the output "
                               "(the window and hop do not satisfy the NOLA condition)")
        if len(_envelope_checked) > 256:
            _envelope_checked.clear()
        _envelope_checked[key] = True
    lead = X.shape[:-2]
    spec = X.reshape(-1, X.shape[-2], frames).transpose(-1, -2).contiguous()
    scale = n_fft ** 0.5 if normalized else 1.0
    y = _ISTFT.apply(spec, n_fft, hop, center, window, out_len, scale)
    return y.reshape(*lead, out_len)


class _RFFT2(torch.autograd.Function):
    """rfft2 = column FFT o row R2C; adjoint = row R2C^T (weighted C2R) o conjugate column FFT."""

    @staticmethod
    def forward(ctx, x, scale):
        _need_cuda(x, torch.float32, "rfft2")
        x = x.contiguous()
        ny, nx = x.shape[-2], x.shape[-1]
        batch = x.numel() // (ny * nx) if ny * nx else 0
        y = torch.empty(*x.shape[:-1], nx // 2 + 1, dtype=torch.complex64, device=x.device)
        ctx.scale, ctx.nx = scale, nx
        if batch == 0:
            return y
        rc = plan_for(x.device, nx, "real").exec_r2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, batch, scale, _stream(x))
        if rc:
            raise BflyError(f"exec_r2c_2d(ny={ny}, nx={nx}, batch={batch})", rc)
        return y

    @staticmethod
    def backward(ctx, g):
        gc = c2c_axis(g.contiguous(), -2, 1, 1.0)
        return c2r(gc, ctx.nx, 1.0, 0.5, ctx.scale), None


class _IRFFT2(torch.autograd.Function):
    """irfft2 = row C2R o inverse column FFT; adjoint = forward column FFT o row C2R^T (weighted R2C)."""

    @staticmethod
    def forward(ctx, X, nx, scale):
        _need_cuda(X, torch.complex64, "irfft2")
        X = X.contiguous()
        ny = X.shape[-2]
        if X.shape[-1] != nx // 2 + 1:
            raise ValueError(f"irfft2: last dimension {X.shape[-1]} != nx/2+1 = {nx // 2 + 1}")
        batch = X.numel() // (ny * X.shape[-1]) if X.numel() else 0
        y = torch.empty(*X.shape[:-1], nx, dtype=torch.float32, device=X.device)
        ctx.scale = scale
        if batch == 0:
            return y
        rc = plan_for(X.device, nx, "real").exec_c2r_2d(X.data_ptr(), y.data_ptr(), ny, nx, batch, scale, _stream(X))
        if rc:
            raise BflyError(f"exec_c2r_2d(ny={ny}, nx={nx}, batch={batch})", rc)
        return y

    @staticmethod
    def backward(ctx, g):
        c = ctx.scale
        return c2c_axis(r2c(g.contiguous(), c, 2.0 * c), -2, -1, 1.0), None, None


def _need_2d(x: torch.Tensor, what: str):
    if x.dim() < 2:
        raise ValueError(f"{what}: input needs at least two dimensions")


def fft2(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    """2-D FFT over the last two dimensions (torch.fft.fft2 with dim=(-2, -1))."""
    _need_2d(x, "fft2")
    return _FFT2.apply(x, -1, _scale(norm, x.shape[-2] * x.shape[-1], True))


def ifft2(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    _need_2d(x, "ifft2")
    return _FFT2.apply(x, 1, _scale(norm, x.shape[-2] * x.shape[-1], False))


def rfft2(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    """torch.fft.rfft2 over the last two dimensions: float32 [..., ny, nx] -> [..., ny, nx/2+1]."""
    _need_2d(x, "rfft2")
    return _RFFT2.apply(x, _scale(norm, x.shape[-2] * x.shape[-1], True))


def irfft2(X: torch.Tensor, s: tuple | None = None, norm: str | None = None) -> torch.Tensor:
    """torch.fft.irfft2 over the last two dimensions; s = (ny, nx) output size (default
    (X.shape[-2], 2*(X.shape[-1]-1)))."""
    _need_2d(X, "irfft2")
    ny = X.shape[-2]
    nx = s[-1] if s is not None else 2 * (X.shape[-1] - 1)
    if s is not None and s[-2] != ny:
        raise ValueError("irfft2: s[-2] must equal X.shape[-2] (no cropping or padding)")
    return _IRFFT2.apply(X, nx, _scale(norm, ny * nx, False))


def rfft(x: torch.Tensor, norm: str | None = None) -> torch.Tensor:
    return _RFFT.apply(x, _scale(norm, x.shape[-1], True))


def irfft(X: torch.Tensor, n: int | None = None, norm: str | None = None) -> torch.Tensor:
    if n is None:
        n = 2 * (X.shape[-1] - 1)
    return _IRFFT.apply(X, n, _scale(norm, n, False))
