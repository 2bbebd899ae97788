"""Long C2C (n = 8192 .. 65536) on one thread-block cluster per row, through the C ABI.

The cluster schedule computes the same four-step decomposition as the two-kernel schedule
(column FFTs of N1 = n/256 points, twiddle W_n^(n2*k1), row FFTs of 256 points) with the
transpose done in distributed shared memory.  Both schedules are checked against the FP64
oracle (rel L2 <= 2e-6 per row, the long-C2C tolerance) and against each other (rel L2 <= 1e-6:
they perform the same fp32 operations, so any larger difference is an indexing error)."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

CLUSTER = "r16_cta256_shared_fp32_cluster"
FOUR_STEP = "r16_cta256_shared_fp32_four_step"
LONG = [8192, 16384, 32768, 65536]


def _plans(ctx):
    pc = ctx.make_plan(CLUSTER, 8192, 1)
    pf = ctx.make_plan(FOUR_STEP, 8192, 1)
    assert pc is not None and pf is not None
    return pc, pf


@pytest.mark.parametrize("n", LONG)
@pytest.mark.parametrize("batch", [1, 5, 33])
@pytest.mark.parametrize("direction", [-1, 1])
def test_cluster_matches_oracle_and_four_step(ctx, cuda, n, batch, direction):
    import torch
    pc, pf = _plans(ctx)
    x = torch.from_numpy(O.normal_input(n, batch, 7 + n % 97 + batch)).to(cuda).view(torch.complex64)
    yc = torch.empty_like(x)
    yf = torch.empty_like(x)
    scale = 1.0 if direction < 0 else 1.0 / n
    assert pc.exec_c2c(x.data_ptr(), yc.data_ptr(), n, batch, direction, scale, 0) == 0
    assert pf.exec_c2c(x.data_ptr(), yf.data_ptr(), n, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=-1) if direction < 0 else np.fft.ifft(xd, axis=-1)
    assert O.rel_l2_rows(yc.cpu().numpy(), ref) <= 2e-6
    assert O.rel_l2_rows(yf.cpu().numpy(), ref) <= 2e-6
    assert O.max_rel_scaled_rows(O.to_interleaved(yc.cpu().numpy()), O.to_interleaved(ref)) <= 1e-4
    diff = (torch.linalg.vector_norm(yc - yf) / torch.linalg.vector_norm(yf)).item()
    assert diff <= 1e-6, diff
    assert pc.long_device_status() == 0


@pytest.mark.parametrize("n", LONG)
def test_cluster_impulses_and_in_place(ctx, cuda, n):
    """A unit impulse at position p transforms to W_n^(p*k): this pins the output permutation
    exactly; the in-place call (in == out) must give the same result as out-of-place."""
    import torch
    pc, _ = _plans(ctx)
    pos = [0, 1, 255, 256, n // 2 + 3, n - 1]
    x = torch.zeros(len(pos), n, dtype=torch.complex64, device=cuda)
    for r, p in enumerate(pos):
        x[r, p] = 1.0
    y = torch.empty_like(x)
    assert pc.exec_c2c(x.data_ptr(), y.data_ptr(), n, len(pos), -1, 1.0, 0) == 0
    k = np.arange(n)
    ref = np.stack([np.exp(-2j * np.pi * ((p * k) % n) / n) for p in pos])
    torch.cuda.synchronize()
    assert np.max(np.abs(y.cpu().numpy() - ref)) <= 2e-6
    assert pc.exec_c2c(x.data_ptr(), x.data_ptr(), n, len(pos), -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(x, y)


def test_cluster_large_batch_round_trip(ctx, cuda):
    """batch * n = 2^26 at n = 32768: forward then inverse returns the input."""
    import torch
    pc, _ = _plans(ctx)
    n = 32768
    batch = O.long_batch(n)
    g = torch.Generator(device=cuda).manual_seed(5)
    a = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    fa = torch.empty_like(a)
    back = torch.empty_like(a)
    assert pc.exec_c2c(a.data_ptr(), fa.data_ptr(), n, batch, -1, 1.0, 0) == 0
    assert pc.exec_c2c(fa.data_ptr(), back.data_ptr(), n, batch, 1, 1.0 / n, 0) == 0
    torch.cuda.synchronize()
    assert (torch.linalg.vector_norm(back - a) / torch.linalg.vector_norm(a)).item() <= 4e-6
    rows = O.sample_batches(batch, 4)
    ref = np.fft.fft(a[rows].cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(fa[rows].cpu().numpy(), ref) <= 2e-6


@pytest.mark.parametrize("n", [8192, 65536])
def test_cluster_unaligned_input_uses_four_step(ctx, cuda, n):
    """An input that is only 8-byte aligned cannot be described by the TMA tensor map; the plan
    must still return the right transform (through the four-step kernels)."""
    import torch
    pc, _ = _plans(ctx)
    batch = 3
    buf = torch.from_numpy(O.normal_input(n, batch + 1, 21)).to(cuda).view(torch.complex64).reshape(-1)
    x = buf[1:1 + batch * n].view(batch, n)            # offset by one complex value: 8-byte aligned
    assert x.data_ptr() % 16 == 8
    y = torch.empty(batch, n, dtype=torch.complex64, device=cuda)
    assert pc.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(y.cpu().numpy(), ref) <= 2e-6
    assert pc.long_device_status() == 0


@pytest.mark.parametrize("n", [16384, 32768, 65536])
@pytest.mark.parametrize("direction", [-1, 1])
def test_cluster_512_thread_ctas(ctx, cuda, n, direction):
    """The 512-thread-CTA cluster kernels (half the cluster size) give the same transform."""
    import torch
    p512 = ctx.make_plan("r16_cta512_shared_fp32_cluster", n, 1)
    _, pf = _plans(ctx)
    assert p512 is not None
    batch = 7
    x = torch.from_numpy(O.normal_input(n, batch, 3 + n % 89)).to(cuda).view(torch.complex64)
    y = torch.empty_like(x)
    yf = torch.empty_like(x)
    scale = 1.0 if direction < 0 else 1.0 / n
    assert p512.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, 0) == 0
    assert pf.exec_c2c(x.data_ptr(), yf.data_ptr(), n, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=-1) if direction < 0 else np.fft.ifft(xd, axis=-1)
    assert O.rel_l2_rows(y.cpu().numpy(), ref) <= 2e-6
    assert (torch.linalg.vector_norm(y - yf) / torch.linalg.vector_norm(yf)).item() <= 1e-6
    assert p512.long_device_status() == 0
