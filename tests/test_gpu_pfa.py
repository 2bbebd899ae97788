"""C2C of n = A * 2^k (A in {3, 5, 9, 15}) by the prime-factor (Good-Thomas) kernel, against
FP64 numpy.

These lengths are not powers of two, which the reference does not support
(docs/reference/support.md:14).  The kernel is one B-point fp32 Stockham FFT plus a direct
A-point DFT per element, so it is gated like the power-of-two path: rel L2 <= 1e-6 per row."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(a, b) for a in (3, 5, 9, 15) for b in (16, 32, 64, 128, 256, 512, 1024, 2048, 4096)
          if a * b <= 12288]


@pytest.mark.parametrize("a,b", SHAPES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_pfa_matches_fp64(plan, cuda, a, b, direction):
    import torch
    n = a * b
    batch = 3 if n > 2048 else 37
    x = torch.from_numpy(O.normal_input(n, batch, 90 + n)).to(cuda).view(torch.complex64)
    y = torch.empty_like(x)
    scale = 1.0 if direction < 0 else 1.0 / n
    assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=-1) if direction < 0 else np.fft.ifft(xd, axis=-1)
    err = O.rel_l2_rows(y.cpu().numpy(), ref)
    assert err <= 1e-6, (n, direction, err)


@pytest.mark.parametrize("n", [48, 1280, 1536, 7680, 9216, 12288])
def test_pfa_known_answers_and_in_place(plan, cuda, n):
    import torch
    pos = [0, 1, 3, n // 2 + 1, n - 1]
    x = torch.zeros(len(pos), n, dtype=torch.complex64, device=cuda)
    for r, p in enumerate(pos):
        x[r, p] = 1.0
    y = torch.empty_like(x)
    assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, len(pos), -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    k = np.arange(n)
    ref = np.stack([np.exp(-2j * np.pi * ((p * k) % n) / n) for p in pos])
    assert np.max(np.abs(y.cpu().numpy() - ref)) <= 2e-6
    z = x.clone()
    assert plan.exec_c2c(z.data_ptr(), z.data_ptr(), n, len(pos), -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(z, y)


def test_pfa_large_batch_and_torch_layer(cuda):
    import torch
    import bfly
    g = torch.Generator(device=cuda).manual_seed(4)
    x = torch.randn(1 << 14, 1536, dtype=torch.complex64, device=cuda, generator=g)
    y = bfly.fft(x)
    ref = torch.fft.fft(x)
    assert (torch.linalg.vector_norm(y - ref) / torch.linalg.vector_norm(ref)).item() <= 2e-6
    back = bfly.ifft(y)
    assert (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item() <= 2e-6


def test_lengths_outside_every_kernel(plan, cuda):
    import torch
    x = torch.zeros(1, 15360, dtype=torch.complex64, device=cuda)
    assert plan.exec_c2c(x.data_ptr(), x.data_ptr(), 15360, 1, -1, 1.0, 0) == -8   # 15*1024 > 12288, > 8192
