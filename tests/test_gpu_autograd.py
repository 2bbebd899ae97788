"""torch-level ops and hand-written adjoints against torch.fft (values and gradients) and
FP64 finite differences of the loss sum(w * |X|^2)."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("n", [64, 1024, 4096, 8192, 65536])
@pytest.mark.parametrize("norm", ["backward", "ortho", "forward"])
def test_fft_ifft_values_and_grads(cuda, n, norm):
    torch = _torch()
    import bfly
    batch = 4 if n <= 8192 else 2
    g = torch.Generator(device=cuda).manual_seed(n)
    x = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    w = torch.rand(batch, n, device=cuda, generator=g)
    tol = 1e-6 if n <= 4096 else 2e-6
    for ours, theirs in ((bfly.fft, torch.fft.fft), (bfly.ifft, torch.fft.ifft)):
        a = x.clone().requires_grad_(True)
        b = x.clone().requires_grad_(True)
        ya = ours(a, norm=norm)
        yb = theirs(b, norm=norm)
        ref = (np.fft.fft if ours is bfly.fft else np.fft.ifft)(
            x.cpu().numpy().astype(np.complex128), axis=-1, norm=norm)
        assert O.rel_l2(ya.detach().cpu().numpy(), ref) <= tol
        (w * ya.abs() ** 2).sum().backward()
        (w * yb.abs() ** 2).sum().backward()
        rel = (torch.linalg.vector_norm(a.grad - b.grad) / torch.linalg.vector_norm(b.grad)).item()
        assert rel <= 1e-5


@pytest.mark.parametrize("n", [128, 1024, 8192])
def test_rfft_grad(cuda, n):
    torch = _torch()
    import bfly
    batch = 3
    g = torch.Generator(device=cuda).manual_seed(7)
    x = (torch.rand(batch, n, device=cuda, generator=g) * 2 - 1)
    w = torch.rand(batch, n // 2 + 1, device=cuda, generator=g)
    for norm in ("backward", "ortho", "forward"):
        a = x.clone().requires_grad_(True)
        b = x.clone().requires_grad_(True)
        (w * bfly.rfft(a, norm=norm).abs() ** 2).sum().backward()
        (w * torch.fft.rfft(b, norm=norm).abs() ** 2).sum().backward()
        rel = (torch.linalg.vector_norm(a.grad - b.grad) / torch.linalg.vector_norm(b.grad)).item()
        assert rel <= 1e-5, norm


@pytest.mark.parametrize("n", [64, 1024, 4096])
def test_irfft_grad(cuda, n):
    torch = _torch()
    import bfly
    batch = 3
    X = torch.from_numpy(O.to_complex(O.half_spectrum_input(n, batch, 5)).astype(np.complex64)).to(cuda)
    g = torch.Generator(device=cuda).manual_seed(8)
    w = torch.rand(batch, n, device=cuda, generator=g)
    for norm in ("backward", "ortho", "forward"):
        a = X.clone().requires_grad_(True)
        b = X.clone().requires_grad_(True)
        ya = bfly.irfft(a, n, norm=norm)
        yb = torch.fft.irfft(b, n, norm=norm)
        assert (torch.linalg.vector_norm(ya - yb) / torch.linalg.vector_norm(yb)).item() <= 1e-6
        (w * ya ** 2).sum().backward()
        (w * yb ** 2).sum().backward()
        # torch leaves a nonzero imaginary gradient on DC/Nyquist bins is impossible: compare all
        rel = (torch.linalg.vector_norm(a.grad - b.grad) / torch.linalg.vector_norm(b.grad)).item()
        assert rel <= 1e-5, norm


def test_rfft_grad_vs_fp64_finite_differences(cuda):
    """Loss = sum(w * |rfft(x)|^2): analytic adjoint vs central differences in float64."""
    torch = _torch()
    import bfly
    n, batch = 128, 2
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (batch, n))
    w = rng.uniform(0, 1, (batch, n // 2 + 1))

    def loss64(xx):
        return float((w * np.abs(np.fft.rfft(xx, axis=-1)) ** 2).sum())

    xt = torch.tensor(x, dtype=torch.float32, device=cuda, requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float32, device=cuda)
    (wt * bfly.rfft(xt).abs() ** 2).sum().backward()
    grad = xt.grad.double().cpu().numpy()
    h = 1e-5
    idx = [(0, 0), (0, 1), (0, n // 2), (1, 17), (1, n - 1)]
    for (i, j) in idx:
        xp = x.copy(); xp[i, j] += h
        xm = x.copy(); xm[i, j] -= h
        fd = (loss64(xp) - loss64(xm)) / (2 * h)
        assert abs(grad[i, j] - fd) <= 1e-3 * max(1.0, abs(fd)), (i, j, grad[i, j], fd)


@pytest.mark.parametrize("n,batch,seed", [(64, 2, 3), (1024, 2, 4), (8192, 2, 11), (65536, 1, 11)])
@pytest.mark.parametrize("op", ["fft", "ifft"])
def test_c2c_grad_vs_fp64_finite_differences(cuda, n, batch, seed, op):
    """Loss = sum(w * |F(x)|^2) with F = fft or ifft on complex x (the long lengths under the
    long-transform loss: x ~ N(0,1), w ~ U(0,1), seeded): the conjugate-FFT adjoint against FP64
    central differences of the real and imaginary part of sampled entries.  torch's gradient of
    a real loss in a complex input is dL/dRe + i dL/dIm.  The loss is quadratic, so the central
    difference is exact up to FP64 rounding."""
    torch = _torch()
    import bfly
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    x = x.astype(np.complex64).astype(np.complex128)
    w = rng.uniform(0, 1, (batch, n))
    f64 = np.fft.fft if op == "fft" else np.fft.ifft

    def loss64(xx):
        return float((w * np.abs(f64(xx, axis=-1)) ** 2).sum())

    xt = torch.tensor(x, dtype=torch.complex64, device=cuda, requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float32, device=cuda)
    (wt * getattr(bfly, op)(xt).abs() ** 2).sum().backward()
    grad = xt.grad.cpu().numpy().astype(np.complex128)
    idx = [(0, 0), (0, 1), (0, n // 2), (batch - 1, n // 3), (batch - 1, n - 1)]
    h = 1e-3
    got, want = [], []
    for (i, j) in idx:
        for unit in (1.0, 1j):
            xp = x.copy(); xp[i, j] += h * unit
            xm = x.copy(); xm[i, j] -= h * unit
            want.append((loss64(xp) - loss64(xm)) / (2 * h))
            got.append(grad[i, j].real if unit == 1.0 else grad[i, j].imag)
    got, want = np.array(got), np.array(want)
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel <= 1e-5, (op, n, rel)
