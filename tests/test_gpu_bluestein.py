"""Any-length C2C (Bluestein's chirp-z algorithm in one kernel) against FP64 numpy.

The reference supports power-of-two lengths only (docs/reference/support.md:14,
docs/testing.md:16-17 list non-power-of-two lengths as missing).  A Bluestein transform of
length n runs two fp32 FFTs of the padded length M >= 2n-1 and three chirp/filter products, so
its error is gated at rel L2 <= 2e-6 per row (the tolerance of the two-pass long transforms);
the measured error is asserted, not assumed."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

# lengths with a prime factor above 13 (13-smooth lengths run the mixed-radix kernel)
LENGTHS = [17, 19, 23, 34, 38, 97, 127, 209, 1003, 1023, 2047, 3001, 4097, 5003, 6553, 8191]


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("direction", [-1, 1])
def test_bluestein_matches_fp64(plan, cuda, n, direction):
    import torch
    batch = 3 if n > 1000 else 65
    x = torch.from_numpy(O.normal_input(n, batch, 50 + n)).to(cuda).view(torch.complex64)
    y = torch.empty_like(x)
    scale = 1.0 if direction < 0 else 1.0 / n
    assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=-1) if direction < 0 else np.fft.ifft(xd, axis=-1)
    err = O.rel_l2_rows(y.cpu().numpy(), ref)
    assert err <= 2e-6, (n, direction, err)
    assert O.max_rel_scaled_rows(O.to_interleaved(y.cpu().numpy()), O.to_interleaved(ref)) <= 1e-4


def test_bluestein_known_answers(plan, cuda):
    """Impulse at p -> exp(-2*pi*i*p*k/n); constant -> n at bin 0; in place equals out of place."""
    import torch
    n = 1003
    pos = [0, 1, 7, 499, 1002]
    x = torch.zeros(len(pos) + 1, n, dtype=torch.complex64, device=cuda)
    for r, p in enumerate(pos):
        x[r, p] = 1.0
    x[len(pos)] = 1.0
    y = torch.empty_like(x)
    assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, x.shape[0], -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    k = np.arange(n)
    ref = np.stack([np.exp(-2j * np.pi * ((p * k) % n) / n) for p in pos] + [np.eye(1, n)[0] * n])
    got = y.cpu().numpy()
    assert np.max(np.abs(got[:-1] - ref[:-1])) <= 5e-6
    assert np.max(np.abs(got[-1] - ref[-1])) <= 5e-6 * n
    z = x.clone()
    assert plan.exec_c2c(z.data_ptr(), z.data_ptr(), n, z.shape[0], -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(z, y)


def test_bluestein_large_batch_round_trip(plan, cuda):
    import torch
    n, batch = 3001, 1 << 14
    g = torch.Generator(device=cuda).manual_seed(3)
    a = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    fa = torch.empty_like(a)
    back = torch.empty_like(a)
    assert plan.exec_c2c(a.data_ptr(), fa.data_ptr(), n, batch, -1, 1.0, 0) == 0
    assert plan.exec_c2c(fa.data_ptr(), back.data_ptr(), n, batch, 1, 1.0 / n, 0) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(back - a) / torch.linalg.vector_norm(a)).item() <= 4e-6
    rows = O.sample_batches(batch, 4)
    ref = np.fft.fft(a[rows].cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(fa[rows].cpu().numpy(), ref) <= 2e-6


def test_bluestein_torch_layer_and_autograd(cuda):
    import torch
    import bfly
    x0 = torch.randn(4, 374, dtype=torch.complex64, device=cuda)
    for norm in (None, "ortho", "forward"):
        ref = torch.fft.fft(x0, norm=norm)
        got = bfly.fft(x0, norm=norm)
        assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 3e-6
        back = bfly.ifft(got, norm=norm)
        assert (torch.linalg.vector_norm(back - x0) / torch.linalg.vector_norm(x0)).item() <= 4e-6
    w = torch.rand(4, 374, device=cuda)
    xa = x0.clone().requires_grad_(True)
    xb = x0.clone().requires_grad_(True)
    (w * bfly.fft(xa).abs() ** 2).sum().backward()
    (w * torch.fft.fft(xb).abs() ** 2).sum().backward()
    assert (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item() <= 1e-5


def test_bluestein_in_2d_rows(plan, cuda):
    """A 2-D transform whose rows have a non-power-of-two length (columns stay power of two)."""
    import torch
    ny, nx = 64, 170
    x = torch.randn(2, ny, nx, dtype=torch.complex64, device=cuda)
    y = torch.empty_like(x)
    assert plan.exec_c2c_2d(x.data_ptr(), y.data_ptr(), ny, nx, 2, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.fft2(x.cpu().numpy().astype(np.complex128)).reshape(2, -1)
    assert O.rel_l2_rows(y.cpu().numpy().reshape(2, -1), ref) <= 3e-6


def test_bluestein_guards(plan, cuda):
    import torch
    x = torch.zeros(2, 9001, dtype=torch.complex64, device=cuda)
    assert plan.exec_c2c(x.data_ptr(), x.data_ptr(), 9001, 1, -1, 1.0, 0) == -8   # prime, above 8192
    assert plan.exec_c2c(x.data_ptr(), x.data_ptr(), 1, 1, -1, 1.0, 0) == -8
