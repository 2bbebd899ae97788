"""Gradients of the STFT and of the inverse STFT, each one kernel through the C ABI
(bfly_plan_exec_stft_backward_async, bfly_plan_exec_istft_backward_async), against torch
autograd of torch.stft / torch.istft in float64 on the same inputs.

The STFT gradient folds the centred reflect padding back onto the signal: the cases include
the shortest signal it serves (n + 2 samples, every output in a fold region or next to one),
hops that do not divide the length, no window, and signals long enough to be split over many
CTAs (the first and the last segment own the fold outputs).  The inverse STFT's gradient divides
by the window envelope inside the kernel, including the edges where fewer frames overlap.
Tolerance: rel L2 <= 1e-5 (the gradient tolerance of the other autograd tests)."""
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    import torch
    return (torch.linalg.vector_norm(a.double() - b.double()) / torch.linalg.vector_norm(b.double())).item()


STFT_CASES = [
    # n, hop, center, length, windowed
    (256, 64, True, 258, True),          # n + 2: both folds, nothing in between
    (256, 64, True, 259, False),
    (256, 100, True, 5001, True),        # hop not dividing the length
    (64, 16, True, 1000, True),
    (1024, 256, True, 1 << 18, True),    # many segments
    (4096, 1024, True, 100003, True),
    (8192, 2048, True, 40000, False),
    (512, 128, False, 4096, True),       # uncentred: no fold
    (2048, 512, False, 10000, True),
]


@pytest.mark.parametrize("n,hop,center,length,windowed", STFT_CASES)
def test_stft_backward_matches_torch(plan, cuda, n, hop, center, length, windowed):
    import torch
    g = torch.Generator(device=cuda).manual_seed(n + hop + length)
    signals = 3
    x = torch.rand(signals, length, device=cuda, generator=g, dtype=torch.float64) * 2 - 1
    w = torch.hann_window(n, device=cuda, dtype=torch.float64) if windowed else None
    frames = 1 + length // hop if center else 1 + (length - n) // hop
    gy = torch.randn(signals, frames, n // 2 + 1, dtype=torch.complex128, device=cuda, generator=g)
    # reference: torch autograd through torch.stft in float64 ([..., bins, frames] layout)
    xr = x.clone().requires_grad_(True)
    y = torch.stft(xr, n, hop_length=hop, window=w, center=center, pad_mode="reflect", return_complex=True)
    (y * gy.transpose(-1, -2).conj()).real.sum().backward()
    want = xr.grad
    got = torch.empty(signals, length, device=cuda)
    g32 = gy.to(torch.complex64).contiguous()
    w32 = w.float().contiguous() if windowed else None
    assert plan.exec_stft_backward(g32.data_ptr(), got.data_ptr(), n, signals, length, hop, center,
                                   w32.data_ptr() if windowed else 0) == 0
    torch.cuda.synchronize()
    assert _rel(got, want) <= 1e-5


ISTFT_CASES = [
    # n, hop, center, frames, out_len (0: the full length), window
    (256, 64, True, 20, 0, "hann"),
    (256, 64, True, 20, 500, "hann"),      # shorter output: the gradient is zero past it
    (1024, 256, True, 300, 0, "hann"),
    (1024, 250, False, 40, 0, "raised"),   # uncentred (a window without zeros), hop not dividing n
    (4096, 1024, True, 64, 0, "hann"),
    (8192, 2048, True, 16, 0, "hann"),
    (64, 16, True, 200, 0, "none"),
]


@pytest.mark.parametrize("n,hop,center,frames,out_len,win", ISTFT_CASES)
def test_istft_backward_matches_torch(plan, cuda, n, hop, center, frames, out_len, win):
    import torch
    g = torch.Generator(device=cuda).manual_seed(n + hop + frames)
    signals = 2
    spec = torch.randn(signals, frames, n // 2 + 1, dtype=torch.complex128, device=cuda, generator=g)
    spec[..., 0] = spec[..., 0].real
    spec[..., -1] = spec[..., -1].real
    windowed = win != "none"
    w = torch.hann_window(n, device=cuda, dtype=torch.float64) if windowed else None
    if win == "raised":
        w = 0.9 * w + 0.1
    full = n + hop * (frames - 1) - (n if center else 0)
    length = out_len or full
    scale = 0.75
    gy = torch.randn(signals, length, dtype=torch.float64, device=cuda, generator=g)
    sr = spec.clone().requires_grad_(True)
    y = torch.istft(sr.transpose(-1, -2), n, hop_length=hop, window=w, center=center, length=length) * scale
    (y * gy).sum().backward()
    want = sr.grad
    got = torch.empty(signals, frames, n // 2 + 1, dtype=torch.complex64, device=cuda)
    gy32 = gy.float().contiguous()
    w32 = w.float().contiguous() if windowed else None
    assert plan.exec_istft_backward(gy32.data_ptr(), got.data_ptr(), n, signals, frames, hop, center,
                                    w32.data_ptr() if windowed else 0, length, scale) == 0
    torch.cuda.synchronize()
    assert _rel(torch.view_as_real(got), torch.view_as_real(want)) <= 1e-5


def test_backward_entry_points_reject_unsupported(plan, cuda):
    import torch
    buf = torch.empty(1 << 16, device=cuda)
    p = buf.data_ptr()
    assert plan.exec_stft_backward(p, p, 256, 1, 257, 64, True) == -8      # centred needs n + 2 samples
    assert plan.exec_stft_backward(p, p, 400, 1, 4000, 100, True) == -8    # powers of two only
    assert plan.exec_stft_backward(p, p, 256, 1, 4000, 0, True) == -8
    assert plan.exec_istft_backward(p, p, 256, 1, 0, 64, True, 0, 100) == -8
    assert plan.exec_istft_backward(p, p, 256, 1, 4, 300, True, 0, 100) == -8   # hop > n
    assert plan.exec_istft_backward(p, p + 4, 256, 1, 4, 64, True, p + 4, 100) == -8   # window not 8-byte aligned
