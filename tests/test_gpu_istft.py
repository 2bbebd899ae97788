"""Inverse STFT (C2R of every frame + windowed overlap-add kernel) against FP64 numpy and
torch.istft.

The FP64 restatement follows torch.istft's definition: irfft of every frame (1/n_fft, sqrt(n_fft)
more when normalized), times the window, overlap-added every hop samples, divided by the
overlap-added squared window, trimmed by n_fft/2 when centred and zero-padded (or cut) to
`length`.  Tolerance: rel L2 <= 2e-6 per signal against FP64 (fp32 irfft error ~1e-7 plus the
envelope division), 5e-6 against torch.istft, 1e-5 for gradients against torch's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _istft_fp64(spec, n, hop, center, window, length, normalized=False):
    """spec: [..., n/2+1, frames] complex."""
    spec = np.asarray(spec, dtype=np.complex128)
    frames = spec.shape[-1]
    fr = np.fft.irfft(np.swapaxes(spec, -1, -2), n, axis=-1)   # [..., frames, n]
    if normalized:
        fr = fr * np.sqrt(n)
    w = np.ones(n) if window is None else np.asarray(window, dtype=np.float64)
    padded = n + hop * (frames - 1)
    y = np.zeros(spec.shape[:-2] + (padded,))
    env = np.zeros(padded)
    for f in range(frames):
        y[..., f * hop:f * hop + n] += fr[..., f, :] * w
        env[f * hop:f * hop + n] += w * w
    start = n // 2 if center else 0
    end = start + length if length is not None else padded - start
    y = y[..., start:min(end, padded)] / env[start:min(end, padded)]
    if end > padded:
        y = np.concatenate([y, np.zeros(y.shape[:-1] + (end - padded,))], axis=-1)
    return y


def _rel(got, ref):
    got = np.asarray(got, dtype=np.float64)
    d = np.linalg.norm((got - ref).reshape(-1, ref.shape[-1]), axis=-1)
    r = np.maximum(np.linalg.norm(ref.reshape(-1, ref.shape[-1]), axis=-1), 1e-30)
    return float((d / r).max())


def _spec(cuda, n, hop, signals, length, seed, window=None):
    import torch
    g = torch.Generator(device=cuda).manual_seed(seed)
    x = torch.randn(signals, length, device=cuda, generator=g)
    return x, torch.stft(x, n, hop_length=hop, window=window, return_complex=True)


@pytest.mark.parametrize("n,hop", [(64, 16), (256, 64), (512, 100), (1024, 256), (2048, 2048), (4096, 1024),
                                   (8192, 2048)])
@pytest.mark.parametrize("center", [True, False])
@pytest.mark.parametrize("windowed", [True, False])
@pytest.mark.parametrize("tail", [7, 8])
def test_istft_against_fp64(plan, cuda, n, hop, center, windowed, tail):
    """Through the plan entry point: [signals][frames][n/2+1] -> [signals][out_len], random
    (non-Hermitian-consistent) spectra, out_len past the last frame to check the zero tail
    (tail 8 keeps out_len a multiple of 4: the float4 overlap-add; tail 7 the scalar one)."""
    import torch
    if windowed and not center and hop == n:
        pytest.skip("Hann window with hop = n_fft violates NOLA at the frame edges")
    frames, signals = 9, 3
    g = torch.Generator(device=cuda).manual_seed(n + hop + center + tail)
    spec = torch.randn(signals, frames, n // 2 + 1, dtype=torch.complex64, device=cuda, generator=g)
    # a Hann window shifted off zero keeps the uncentred envelope away from 0 at the ends
    w = (torch.hann_window(n, device=cuda) + 0.1) if windowed else None
    padded = n + hop * (frames - 1)
    start = n // 2 if center else 0
    out_len = padded - 2 * start + tail
    y = torch.full((signals, out_len), float("nan"), device=cuda)
    assert plan.exec_istft(spec.data_ptr(), y.data_ptr(), n, signals, frames, hop, center,
                           w.data_ptr() if windowed else 0, out_len, 1.0) == 0
    torch.cuda.synchronize()
    ref = _istft_fp64(spec.cpu().numpy().transpose(0, 2, 1), n, hop, center,
                      w.cpu().numpy() if windowed else None, out_len)
    got = y.cpu().numpy()
    assert np.isfinite(got).all()
    assert _rel(got, ref) <= 2e-6


@pytest.mark.parametrize("kwargs", [{}, {"hop_length": 160}, {"center": False, "window": "hann+"},
                                    {"normalized": True}, {"window": "hann"}, {"length": 47000},
                                    {"length": 48500}, {"win_length": 800, "window": "hann800"},
                                    {"hop_length": 441, "window": "hann"}])
def test_istft_matches_torch_istft(cuda, kwargs):
    import torch
    import bfly
    n = 1024
    kw = dict(kwargs)
    win = kw.pop("window", None)
    if win == "hann":
        kw["window"] = torch.hann_window(n, device=cuda)
    elif win == "hann+":
        kw["window"] = torch.hann_window(n, device=cuda) + 0.05
    elif win == "hann800":
        kw["window"] = torch.hann_window(800, device=cuda)
    stft_kw = {k: v for k, v in kw.items() if k != "length"}
    x, spec = (lambda g: (g, torch.stft(g, n, return_complex=True, **stft_kw)))(
        torch.randn(2, 48000, device=cuda, generator=torch.Generator(device=cuda).manual_seed(11)))
    ref = torch.istft(spec, n, **kw)
    got = bfly.istft(spec, n, **kw)
    assert got.shape == ref.shape, (kwargs, got.shape, ref.shape)
    rel = (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item()
    assert rel <= 5e-6, (kwargs, rel)


@pytest.mark.parametrize("n", [256, 1024, 4096])
def test_stft_istft_round_trip(cuda, n):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(n)
    x = torch.randn(4, 20 * n + 3, device=cuda, generator=g)
    w = torch.hann_window(n, device=cuda)
    back = bfly.istft(bfly.stft(x, n, window=w), n, window=w, length=x.shape[-1])
    rel = (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item()
    assert rel <= 2e-6, rel
    one = torch.randn(5000, device=cuda, generator=g)   # 1-D signal <-> 2-D spectrum
    assert bfly.istft(bfly.stft(one, 256), 256, length=5000).shape == (5000,)


@pytest.mark.parametrize("center", [True, False])
def test_istft_autograd(cuda, center):
    import torch
    import bfly
    n, hop = 256, 100
    w = torch.hann_window(n, device=cuda) + 0.1
    _, spec0 = _spec(cuda, n, hop, 2, 3000, 21, w)
    sa = spec0.clone().requires_grad_(True)
    sb = spec0.clone().requires_grad_(True)
    ya = bfly.istft(sa, n, hop_length=hop, window=w, center=center, length=2900)
    yb = torch.istft(sb, n, hop_length=hop, window=w, center=center, length=2900)
    wt = torch.rand(ya.shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(3))
    (wt * ya * ya).sum().backward()
    (wt * yb * yb).sum().backward()
    rel = (torch.linalg.vector_norm(sa.grad - sb.grad) / torch.linalg.vector_norm(sb.grad)).item()
    assert rel <= 1e-5, rel


def test_istft_rejects_unsupported(cuda):
    import torch
    import bfly
    spec = torch.randn(129, 40, dtype=torch.complex64, device=cuda)
    with pytest.raises(RuntimeError):   # Hann window, hop = n_fft, uncentred: zero envelope (NOLA)
        bfly.istft(spec, 256, hop_length=256, window=torch.hann_window(256, device=cuda), center=False)
    with pytest.raises(ValueError):
        bfly.istft(spec, 256, onesided=False)
    with pytest.raises(ValueError):
        bfly.istft(spec, 512)                      # bins do not match n_fft
    with pytest.raises(ValueError):
        bfly.istft(spec, 256, hop_length=300)      # hop above n_fft
    with pytest.raises(TypeError):
        bfly.istft(spec.to(torch.complex128), 256)
    with pytest.raises(bfly.BflyError):
        bfly.istft(torch.randn(18, 40, dtype=torch.complex64, device=cuda), 34)   # 17 is not 13-smooth
