"""STFT (frame gather + window + one-sided transform in one kernel) against FP64 numpy and
torch.stft.

Shapes follow the reference's STFT application case (docs/testing.md:118,
config/test_matrix.json: R2C n = 256..8192 with 1, 8, 64, 256 frames), with overlapping
frames (hop < n), odd hops, centred reflect padding and a Hann window.  Tolerance: rel L2
<= 1e-6 per frame against FP64 (the R2C tolerance); gradients against torch.stft's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stft_fp64(x, n, hop, center, window):
    x = np.asarray(x, dtype=np.float64)
    if center:
        x = np.pad(x, [(0, 0)] * (x.ndim - 1) + [(n // 2, n // 2)], mode="reflect")
    frames = 1 + (x.shape[-1] - n) // hop
    idx = np.arange(frames)[:, None] * hop + np.arange(n)[None, :]
    fr = x[..., idx] * (np.asarray(window, dtype=np.float64) if window is not None else 1.0)
    return np.fft.rfft(fr, axis=-1)   # [..., frames, n/2+1]


def _rel_frames(got, ref):
    d = np.linalg.norm(got.astype(np.complex128) - ref, axis=-1)
    r = np.maximum(np.linalg.norm(ref, axis=-1), 1e-30)
    return float((d / r).max())


@pytest.mark.parametrize("n", [256, 512, 1024, 2048, 4096, 8192])
@pytest.mark.parametrize("frames", [1, 8, 64, 256])
def test_stft_reference_grid(plan, cuda, n, frames):
    import torch
    hop = n // 4
    length = n + (frames - 1) * hop            # uncentred: exactly `frames` frames
    g = torch.Generator(device=cuda).manual_seed(n + frames)
    x = torch.rand(2, length, device=cuda, generator=g) * 2 - 1
    w = torch.hann_window(n, device=cuda)
    out = torch.empty(2, frames, n // 2 + 1, dtype=torch.complex64, device=cuda)
    rc, got = plan.exec_stft(x.data_ptr(), out.data_ptr(), n, 2, length, hop, False, w.data_ptr())
    assert rc == 0 and got == frames
    torch.cuda.synchronize()
    ref = _stft_fp64(x.cpu().numpy(), n, hop, False, w.cpu().numpy())
    assert _rel_frames(out.cpu().numpy(), ref) <= 1e-6


@pytest.mark.parametrize("n,hop", [(64, 16), (512, 100), (1024, 333), (4096, 1024), (2048, 2048)])
@pytest.mark.parametrize("center", [True, False])
@pytest.mark.parametrize("windowed", [True, False])
def test_stft_hops_padding_window(plan, cuda, n, hop, center, windowed):
    import torch
    length = 5 * n + 37
    g = torch.Generator(device=cuda).manual_seed(n + hop)
    x = torch.randn(3, length, device=cuda, generator=g)
    w = torch.hann_window(n, device=cuda) if windowed else None
    frames = 1 + length // hop if center else 1 + (length - n) // hop
    out = torch.empty(3, frames, n // 2 + 1, dtype=torch.complex64, device=cuda)
    rc, got = plan.exec_stft(x.data_ptr(), out.data_ptr(), n, 3, length, hop, center,
                             w.data_ptr() if windowed else 0)
    assert rc == 0 and got == frames
    torch.cuda.synchronize()
    ref = _stft_fp64(x.cpu().numpy(), n, hop, center, w.cpu().numpy() if windowed else None)
    assert _rel_frames(out.cpu().numpy(), ref) <= 1e-6


def test_stft_matches_torch_stft(cuda):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(1)
    x = torch.randn(4, 48000, device=cuda, generator=g)
    w = torch.hann_window(1024, device=cuda)
    for kwargs in ({}, {"hop_length": 160}, {"center": False}, {"normalized": True}, {"window": w},
                   {"window": w, "hop_length": 441, "center": False}):
        ref = torch.stft(x, 1024, return_complex=True, **kwargs)
        got = bfly.stft(x, 1024, **kwargs)
        assert got.shape == ref.shape, (kwargs, got.shape, ref.shape)
        rel = (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item()
        assert rel <= 2e-6, (kwargs, rel)
    one = torch.randn(8000, device=cuda, generator=g)   # 1-D input
    assert torch.allclose(bfly.stft(one, 256), torch.stft(one, 256, return_complex=True), rtol=0, atol=2e-4)


@pytest.mark.parametrize("center", [True, False])
def test_stft_autograd(cuda, center):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(5)
    x0 = torch.randn(2, 3000, device=cuda, generator=g)
    w = torch.hann_window(256, device=cuda)
    xa = x0.clone().requires_grad_(True)
    xb = x0.clone().requires_grad_(True)
    ya = bfly.stft(xa, 256, hop_length=100, window=w, center=center)
    yb = torch.stft(xb, 256, hop_length=100, window=w, center=center, return_complex=True)
    wt = torch.rand(ya.shape, device=cuda, generator=g)
    (wt * ya.abs() ** 2).sum().backward()
    (wt * yb.abs() ** 2).sum().backward()
    rel = (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item()
    assert rel <= 1e-5, rel


def test_stft_rejects_unsupported(cuda):
    import torch
    import bfly
    x = torch.randn(1000, device=cuda)
    with pytest.raises(bfly.BflyError):
        bfly.stft(x, 34)                       # even, but 17 is not 13-smooth
    with pytest.raises(ValueError):
        bfly.stft(x, 256, pad_mode="constant")
    with pytest.raises(ValueError):
        bfly.stft(x, 256, return_complex=False)
    with pytest.raises(TypeError):
        bfly.stft(x.double(), 256)
