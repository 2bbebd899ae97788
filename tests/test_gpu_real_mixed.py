"""Real transforms of even non-power-of-two lengths (n = 2M, M 13-smooth) on the mixed-radix
passes: R2C / C2R against FP64 numpy.rfft / irfft, their adjoints against torch.fft's
gradients, STFT and inverse STFT against torch.stft / torch.istft (n_fft = 400 with hop 160 is
the common speech front-end), and the 2-D real transforms whose rows take this path.  Tolerance: rel L2 <= 1e-6 per row (the
R2C / C2R gate), 2e-6 against torch, 1e-5 for gradients."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

LENGTHS = [6, 10, 12, 20, 22, 26, 96, 100, 160, 320, 400, 480, 640, 1000, 1536, 2000, 2002, 6000, 10000, 24000]


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("batch", [1, 37])
def test_rfft_irfft_match_fp64(plan, cuda, n, batch):
    import torch
    g = torch.Generator(device=cuda).manual_seed(n + batch)
    x = torch.rand(batch, n, device=cuda, generator=g) * 2 - 1
    X = torch.empty(batch, n // 2 + 1, dtype=torch.complex64, device=cuda)
    assert plan.exec_r2c(x.data_ptr(), X.data_ptr(), n, batch, 1.0, 1.0, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.rfft(x.cpu().numpy().astype(np.float64), axis=-1)
    assert O.rel_l2_rows(X.cpu().numpy(), ref) <= 1e-6, n
    # irfft of a spectrum whose DC / Nyquist carry imaginary parts (numpy ignores them)
    S = torch.randn(batch, n // 2 + 1, dtype=torch.complex64, device=cuda, generator=g)
    y = torch.empty(batch, n, device=cuda)
    assert plan.exec_c2r(S.data_ptr(), y.data_ptr(), n, batch, 1.0, 1.0, 1.0 / n, 0) == 0
    torch.cuda.synchronize()
    ref2 = np.fft.irfft(S.cpu().numpy().astype(np.complex128), n, axis=-1)
    d = np.linalg.norm(y.cpu().numpy() - ref2, axis=-1) / np.linalg.norm(ref2, axis=-1)
    assert float(d.max()) <= 1e-6, n


@pytest.mark.parametrize("n", [400, 1000, 6000])
def test_real_mixed_large_batch_and_torch_layer(cuda, n):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(n)
    x = torch.randn((1 << 22) // n + 3, n, device=cuda, generator=g)
    ref = torch.fft.rfft(x)
    got = bfly.rfft(x)
    assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 2e-6
    back = bfly.irfft(got, n)
    assert (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item() <= 2e-6


@pytest.mark.parametrize("n", [400, 1000])
def test_real_mixed_autograd(cuda, n):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(7 + n)
    x0 = torch.randn(5, n, device=cuda, generator=g)
    w = torch.rand(5, n // 2 + 1, device=cuda, generator=g)
    xa = x0.clone().requires_grad_(True)
    xb = x0.clone().requires_grad_(True)
    (w * bfly.rfft(xa).abs() ** 2).sum().backward()
    (w * torch.fft.rfft(xb).abs() ** 2).sum().backward()
    assert (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item() <= 1e-5
    X0 = torch.fft.rfft(x0)
    Xa = X0.clone().requires_grad_(True)
    Xb = X0.clone().requires_grad_(True)
    v = torch.rand(5, n, device=cuda, generator=g)
    (v * bfly.irfft(Xa, n) ** 2).sum().backward()
    (v * torch.fft.irfft(Xb, n) ** 2).sum().backward()
    assert (torch.linalg.vector_norm(Xa.grad - Xb.grad) / torch.linalg.vector_norm(Xb.grad)).item() <= 1e-5


@pytest.mark.parametrize("n_fft,hop", [(400, 160), (480, 120), (1000, 250), (96, 24), (2000, 333)])
@pytest.mark.parametrize("center", [True, False])
def test_stft_mixed_matches_torch(cuda, n_fft, hop, center):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(n_fft + hop)
    x = torch.randn(3, 16000, device=cuda, generator=g)
    w = torch.hann_window(n_fft, device=cuda)
    ref = torch.stft(x, n_fft, hop_length=hop, window=w, center=center, return_complex=True)
    got = bfly.stft(x, n_fft, hop_length=hop, window=w, center=center)
    assert got.shape == ref.shape
    assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 2e-6


def test_stft_mixed_autograd(cuda):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(3)
    x0 = torch.randn(2, 8000, device=cuda, generator=g)
    w = torch.hann_window(400, device=cuda)
    xa = x0.clone().requires_grad_(True)
    xb = x0.clone().requires_grad_(True)
    ya = bfly.stft(xa, 400, hop_length=160, window=w)
    yb = torch.stft(xb, 400, hop_length=160, window=w, return_complex=True)
    wt = torch.rand(ya.shape, device=cuda, generator=g)
    (wt * ya.abs() ** 2).sum().backward()
    (wt * yb.abs() ** 2).sum().backward()
    assert (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item() <= 1e-5


def test_real_2d_mixed_rows(plan, cuda):
    import torch
    ny, nx, batch = 64, 96, 3
    g = torch.Generator(device=cuda).manual_seed(11)
    x = torch.randn(batch, ny, nx, device=cuda, generator=g)
    X = torch.empty(batch, ny, nx // 2 + 1, dtype=torch.complex64, device=cuda)
    assert plan.exec_r2c_2d(x.data_ptr(), X.data_ptr(), ny, nx, batch, 1.0, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.rfft2(x.cpu().numpy().astype(np.float64))
    d = np.linalg.norm((X.cpu().numpy() - ref).reshape(batch, -1), axis=-1)
    assert float((d / np.linalg.norm(ref.reshape(batch, -1), axis=-1)).max()) <= 2e-6
    y = torch.empty_like(x)
    assert plan.exec_c2r_2d(X.data_ptr(), y.data_ptr(), ny, nx, batch, 1.0 / (ny * nx), 0) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)).item() <= 4e-6


@pytest.mark.parametrize("n_fft,hop,center,length", [(400, 160, True, None), (480, 120, True, 15000), (150, 37, True, None),
                                                     (1000, 250, False, None), (6000, 1500, True, None), (400, 100, True, 16003)])
def test_istft_mixed_matches_torch(cuda, n_fft, hop, center, length):
    """One kernel for even non-power-of-two n_fft: float4 overlap-add where n_fft, hop and the
    output length are multiples of 4, scalar otherwise (150 and hop 37)."""
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(n_fft + hop)
    x = torch.randn(2, 16000, device=cuda, generator=g)
    w = torch.hann_window(n_fft, device=cuda) + (0.0 if center else 0.1)
    spec = torch.stft(x, n_fft, hop_length=hop, window=w, center=center, return_complex=True)
    ref = torch.istft(spec, n_fft, hop_length=hop, window=w, center=center, length=length)
    got = bfly.istft(spec, n_fft, hop_length=hop, window=w, center=center, length=length)
    assert got.shape == ref.shape
    assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 5e-6
    back = bfly.istft(bfly.stft(x, n_fft, hop_length=hop, window=w, center=center), n_fft, hop_length=hop,
                      window=w, center=center, length=x.shape[-1] if center else None)
    if center:
        assert (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item() <= 4e-6


def test_istft_mixed_autograd(cuda):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(21)
    w = torch.hann_window(400, device=cuda) + 0.1
    spec0 = torch.stft(torch.randn(2, 6000, device=cuda, generator=g), 400, hop_length=160, window=w,
                       return_complex=True)
    sa = spec0.clone().requires_grad_(True)
    sb = spec0.clone().requires_grad_(True)
    ya = bfly.istft(sa, 400, hop_length=160, window=w, length=5900)
    yb = torch.istft(sb, 400, hop_length=160, window=w, length=5900)
    wt = torch.rand(ya.shape, device=cuda, generator=g)
    (wt * ya * ya).sum().backward()
    (wt * yb * yb).sum().backward()
    assert (torch.linalg.vector_norm(sa.grad - sb.grad) / torch.linalg.vector_norm(sb.grad)).item() <= 1e-5
