"""Transforms over more than 2^31 complex values in one call (about 17 GB per buffer): every
offset in the kernels is 64-bit, so rows on both sides of element 2^31 and the last row must be
right.  Checked against FP64 numpy on sampled rows for the single-pass team kernel, the
mixed-radix and prime-factor kernels and the four-step long transform (whose workspace is
another 17 GB).  Each case frees its buffers before the next; the plan is private to this file
so its workspace is released at the end."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

BIG = 1 << 31


@pytest.fixture(scope="module")
def big_plan(ctx):
    import torch
    free, _ = torch.cuda.mem_get_info()
    if free < 60 * (1 << 30):
        pytest.skip("needs ~55 GB of free device memory")
    p = ctx.make_plan()
    yield p
    del p
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n", [4096, 1000, 1536, 65536])
def test_more_than_2_31_values(big_plan, cuda, n):
    import torch
    batch = BIG // n + 3
    g = torch.Generator(device=cuda).manual_seed(n)
    x = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    y = torch.empty_like(x)
    assert x.numel() > BIG
    assert big_plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    edge = BIG // n   # first row holding elements at or past 2^31
    rows = [0, edge - 1, edge, edge + 1, batch - 1]
    xs = x[rows].cpu().numpy().astype(np.complex128)
    got = y[rows].cpu().numpy()
    tol = 2e-6 if n > 16384 else 1e-6
    assert O.rel_l2_rows(got, np.fft.fft(xs, axis=-1)) <= tol, n
    del x, y
    torch.cuda.empty_cache()
