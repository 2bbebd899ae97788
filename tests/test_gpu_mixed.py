"""Mixed-radix C2C (Stockham passes of radix 2..16, odd primes up to 13 and composites, through
shared memory) against FP64 numpy, for every length the kernel serves.

The reference supports power-of-two lengths only (docs/testing.md:16-17 lists radix-3/5/7 as
missing).  The kernel takes n = 2^a 3^b 5^c 7^d 11^e 13^f up to 12288 that is neither a power of
two >= 32 (Stockham team kernels) nor A*2^k with A in {3, 5, 9, 15} (prime-factor kernel).  Tolerance:
rel L2 <= 1e-6 per row against FP64, the single-pass C2C gate, plus the reference's
maxRelScaled <= 1e-4."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


def _smooth(n):
    for p in (2, 3, 5, 7, 11, 13):
        while n % p == 0:
            n //= p
    return n == 1


def _pfa(n):
    return any(n % a == 0 and (n // a) >= 16 and (n // a) & (n // a - 1) == 0 for a in (3, 5, 9, 15))


MIXED = [n for n in range(2, 12289) if _smooth(n) and not (n & (n - 1) == 0 and n >= 32) and not _pfa(n)]


def _check(plan, cuda, n, batch, direction, seed):
    import torch
    x = torch.from_numpy(O.normal_input(n, batch, seed)).to(cuda).view(torch.complex64)
    y = torch.empty_like(x)
    scale = 1.0 if direction < 0 else 1.0 / n
    assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=-1) if direction < 0 else np.fft.ifft(xd, axis=-1)
    got = y.cpu().numpy()
    return O.rel_l2_rows(got, ref), O.max_rel_scaled_rows(O.to_interleaved(got), O.to_interleaved(ref))


def test_every_mixed_length(plan, cuda):
    """All 760 lengths, forward and inverse, 3 rows each."""
    assert len(MIXED) > 700
    worst = (0.0, None)
    for n in MIXED:
        for direction in (-1, 1):
            err, mrs = _check(plan, cuda, n, 3, direction, 7000 + n)
            assert err <= 1e-6 and mrs <= 1e-4, (n, direction, err, mrs)
            worst = max(worst, (err, n))
    print("worst rel L2", worst)


@pytest.mark.parametrize("n", [6, 60, 100, 360, 1000, 2401, 3000, 5000, 6561, 10935, 12000, 12250, 11, 143, 1001,
                               4095, 1331, 2197, 9152, 441, 882, 1764, 2205, 3600])
@pytest.mark.parametrize("direction", [-1, 1])
def test_mixed_large_batches(plan, cuda, n, direction):
    """Many rows per launch, batch not a multiple of the rows per CTA."""
    batch = max(3, (1 << 21) // n + 1)
    err, mrs = _check(plan, cuda, n, batch, direction, 900 + n)
    assert err <= 1e-6 and mrs <= 1e-4, (n, err, mrs)


def test_mixed_known_answers_and_in_place(plan, cuda):
    """Impulse at p -> exp(-2 pi i p k / n); constant -> n at bin 0; in place equals out of place."""
    import torch
    for n in (7, 13, 49, 1000, 1001, 2401, 11025):
        pos = [0, 1, 3, n // 2, n - 1]
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
        assert np.max(np.abs(got[:-1] - ref[:-1])) <= 2e-6, n
        assert np.max(np.abs(got[-1] - ref[-1])) <= 2e-6 * n, n
        z = x.clone()
        assert plan.exec_c2c(z.data_ptr(), z.data_ptr(), n, z.shape[0], -1, 1.0, 0) == 0
        torch.cuda.synchronize()
        assert torch.equal(z, y), n


def test_mixed_torch_layer_2d_and_autograd(cuda):
    import torch
    import bfly
    x0 = torch.randn(6, 1000, dtype=torch.complex64, device=cuda)
    for norm in (None, "ortho", "forward"):
        ref = torch.fft.fft(x0, norm=norm)
        got = bfly.fft(x0, norm=norm)
        assert (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item() <= 2e-6
    xa = x0.clone().requires_grad_(True)
    xb = x0.clone().requires_grad_(True)
    w = torch.rand(6, 1000, device=cuda)
    (w * bfly.fft(xa).abs() ** 2).sum().backward()
    (w * torch.fft.fft(xb).abs() ** 2).sum().backward()
    assert (torch.linalg.vector_norm(xa.grad - xb.grad) / torch.linalg.vector_norm(xb.grad)).item() <= 1e-5
    img = torch.randn(3, 64, 360, dtype=torch.complex64, device=cuda)   # 2-D: mixed-radix rows
    ref = torch.fft.fft2(img)
    assert (torch.linalg.vector_norm(bfly.fft2(img) - ref) / torch.linalg.vector_norm(ref)).item() <= 2e-6
