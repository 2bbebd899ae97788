"""R2C / C2R / long C2C parity on the GPU through the C ABI against the FP64 oracle.
Tolerances: rel L2 <= 1e-6 for inner lengths <= 4096, <= 2e-6 for the four-step long C2C,
and the reference's maxRelScaled <= 1e-4 gate."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [128, 256, 512, 1024, 2048, 4096, 8192])
@pytest.mark.parametrize("batch", [1, 3, 64])
def test_r2c(plan, n, batch):
    x = O.real_input(n, batch, 100 + n + batch)
    out = np.empty((batch, n + 2), np.float32)
    assert plan.run_r2c(x, out, n, batch) == 0
    ref = O.r2c(x)
    assert O.rel_l2_rows(out, ref) <= 1e-6
    assert O.max_rel_scaled_rows(out, O.to_interleaved(ref)) <= 1e-4
    # DC and Nyquist bins of a real signal are real
    assert np.all(out[:, 1] == 0) and np.all(out[:, n + 1] == 0)


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("batch", [1, 5, 64])
def test_c2r(plan, n, batch):
    X = O.half_spectrum_input(n, batch, 200 + n)
    # non-zero DC/Nyquist imaginary parts must be ignored (reference.cpp:64-79)
    X[:, 1] = 0.75
    X[:, n + 1] = -0.5
    out = np.empty((batch, n), np.float32)
    assert plan.run_c2r(X, out, n, batch) == 0
    ref = O.c2r(X, n)
    assert O.rel_l2_rows(out, ref) <= 1e-6
    assert O.max_rel_scaled_rows(out, ref) <= 1e-4


@pytest.mark.parametrize("n", [128, 1024, 4096])
def test_r2c_c2r_round_trip(plan, n):
    batch = 3
    x = np.stack([O.pattern_at(np.arange(n) + b * n) for b in range(batch)]).astype(np.float32)
    spec = np.empty((batch, n + 2), np.float32)
    back = np.empty((batch, n), np.float32)
    assert plan.run_r2c(x, spec, n, batch) == 0
    assert plan.run_c2r(spec, back, n, batch) == 0
    assert O.max_rel_scaled_rows(back, x) <= 1e-4
    assert np.linalg.norm(back - x) / np.linalg.norm(x) <= 1e-6


def test_real_guards(plan):
    x = np.zeros(8192 * 2, np.float32)
    out = np.zeros(8192 * 2 + 4, np.float32)
    assert plan.run_r2c(x, out, 64, 1) == -8
    assert plan.run_c2r(x, out, 8192, 1) == -8
    assert plan.run_r2c(x, out, 16384, 1) == -8
    assert plan.run_c2r(x, out, 32, 1) == -8


@pytest.mark.parametrize("n", [8192, 16384, 32768, 65536])
def test_long_c2c(plan, n):
    batch = 3
    x = O.normal_input(n, batch, 11)
    out = np.empty_like(x)
    assert plan.run_long(x, out, n, batch, -1) == 0
    ref = O.c2c(x)
    assert O.rel_l2_rows(out, ref) <= 2e-6
    assert O.max_rel_scaled_rows(out, O.to_interleaved(ref)) <= 1e-4
    back = np.empty_like(x)
    assert plan.run_long(out, back, n, batch, 1) == 0
    assert O.rel_l2_rows(back / n, O.to_complex(x)) <= 4e-6


@pytest.mark.parametrize("n", [8192, 65536])
def test_long_full_size_property(ctx, cuda, n):
    """batch * n = 2^26: forward then inverse returns the input; sampled rows vs FP64."""
    import torch
    batch = O.long_batch(n)
    g = torch.Generator(device=cuda).manual_seed(11)
    a = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    p = ctx.make_plan()
    fa = torch.empty_like(a)
    back = torch.empty_like(a)
    assert p.exec_c2c(a.data_ptr(), fa.data_ptr(), n, batch, -1, 1.0) == 0
    assert p.exec_c2c(fa.data_ptr(), back.data_ptr(), n, batch, 1, 1.0 / n) == 0
    torch.cuda.synchronize()
    rt = torch.linalg.vector_norm(back - a) / torch.linalg.vector_norm(a)
    assert rt.item() <= 4e-6
    rows = O.sample_batches(batch, 4)
    ref = np.fft.fft(a[rows].cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(fa[rows].cpu().numpy(), ref) <= 2e-6
