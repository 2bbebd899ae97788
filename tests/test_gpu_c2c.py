"""C2C parity on the GPU through the C ABI against the FP64 oracle.

Tolerances: relative L2 <= 1e-6 per row for n <= 4096 (the project target) and the reference's
acceptance gate maxRelScaled <= 1e-4 (src/host/fft_check.cpp:1313), plus the reference's
published error level <= 2.41e-7 maxRelScaled on its C2C grid
(results/published/ascend910_9382-migration-20261013/matrix.csv, max_rel column) as a bound
the GPU must not exceed by more than 2x.
"""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6
REF_GATE = 1e-4


def run_c2c(plan, x, n, batch):
    out = np.empty_like(x)
    assert plan.run(x, out, n, batch) == 0
    return out


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("batch", [1, 3, 47, 148, 149, 256])
def test_c2c_grid_normal(plan, n, batch):
    x = O.normal_input(n, batch, O.grid_seed(n, max(1, batch)))
    got = run_c2c(plan, x, n, batch)
    ref = O.c2c(x)
    assert O.rel_l2_rows(got, ref) <= REL_L2
    assert O.max_rel_scaled_rows(got, O.to_interleaved(ref)) <= REF_GATE


def test_c2c_config1_uniform(plan):
    x = O.cfg1_input(1024, 256, 0)
    got = run_c2c(plan, x, 1024, 256)
    ref = O.c2c(x)
    assert O.rel_l2(got, ref) <= REL_L2
    # published reference error at this shape: maxRel 2.33e-7 (matrix.md:45)
    assert O.max_rel_scaled_rows(got, O.to_interleaved(ref)) <= 2 * 2.41e-7


@pytest.mark.parametrize("mode", ["sin", "impulse", "constant", "tone", "alternating", "random",
                                  "dynamic", "near-cancellation", "ofdm", "radar", "dl", "zero"])
@pytest.mark.parametrize("n", [64, 1024, 4096])
def test_c2c_harness_modes(plan, mode, n):
    batch = 9
    x = O.harness_input(mode, n, batch, seed=42)
    got = run_c2c(plan, x, n, batch)
    ref = O.c2c(x)
    assert O.max_rel_scaled_rows(got, O.to_interleaved(ref)) <= REF_GATE
    if mode == "zero":
        assert not np.any(got)
    elif mode == "impulse":
        # impulse at k = b: |X| == 1 everywhere
        mag = np.abs(O.to_complex(got))
        assert np.allclose(mag, 1.0, atol=1e-6)
    else:
        assert O.rel_l2_rows(got, ref) <= 5 * REL_L2 if mode in ("dynamic", "near-cancellation") else REL_L2


@pytest.mark.parametrize("n", [32, 64, 512, 4096])
def test_exec_all_variants(ctx, cuda, n):
    """Every compiled (radix, cta) candidate that is feasible for n gives the same answer."""
    import torch
    batch = 37
    x = O.normal_input(n, batch, 5)
    ref = O.c2c(x)
    xd = torch.from_numpy(x).to(cuda)
    for c in ctx.enumerate(n, batch):
        if c["state"] == "Infeasible":
            continue
        p = ctx.make_plan(c["id"], n, batch)
        assert p is not None, c
        yd = torch.empty_like(xd)
        assert p.exec_c2c(xd.data_ptr(), yd.data_ptr(), n, batch, -1, 1.0) == 0
        torch.cuda.synchronize()
        assert O.rel_l2_rows(yd.cpu().numpy(), ref) <= REL_L2, c["id"]


@pytest.mark.parametrize("n", [64, 256, 4096])
def test_inverse_and_scale(plan, n):
    batch = 11
    x = O.normal_input(n, batch, 9)
    out = np.empty_like(x)
    assert plan.run_inverse(x, out, n, batch, 1.0 / n) == 0
    ref = O.c2c_inverse(x, 1.0 / n)
    assert O.rel_l2_rows(out, ref) <= REL_L2
    # round trip
    y = run_c2c(plan, x, n, batch)
    back = np.empty_like(y)
    assert plan.run_inverse(y, back, n, batch, 1.0 / n) == 0
    assert O.rel_l2_rows(back, O.to_complex(x)) <= 2 * REL_L2


def test_large_batch_properties(ctx, cuda):
    """Full-size property check: n=4096, batch=4096 (128 MiB per tensor): linearity and the
    inverse round trip, with a sampled-row oracle comparison."""
    import torch
    n, batch = 4096, 4096
    g = torch.Generator(device=cuda).manual_seed(3)
    a = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    b = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    p = ctx.make_plan()
    fa, fb, fab = (torch.empty_like(a) for _ in range(3))
    s = a + 2 * b
    for src, dst in ((a, fa), (b, fb), (s, fab)):
        assert p.exec_c2c(src.data_ptr(), dst.data_ptr(), n, batch, -1, 1.0) == 0
    torch.cuda.synchronize()
    lin = torch.linalg.vector_norm(fab - (fa + 2 * fb)) / torch.linalg.vector_norm(fab)
    assert lin.item() <= 2e-6
    back = torch.empty_like(a)
    assert p.exec_c2c(fa.data_ptr(), back.data_ptr(), n, batch, 1, 1.0 / n) == 0
    torch.cuda.synchronize()
    rt = torch.linalg.vector_norm(back - a) / torch.linalg.vector_norm(a)
    assert rt.item() <= 2e-6
    rows = O.sample_batches(batch, 8)
    ah = a[rows].cpu().numpy()
    ref = np.fft.fft(ah.astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(fa[rows].cpu().numpy(), ref) <= REL_L2


def test_guards(plan):
    x = np.zeros(2 * 128, np.float32)
    out = np.zeros_like(x)
    for n in (0, 1, 32, 100, 192, 8192, 16384):
        assert plan.run(x, out, n, 1) == -8
    assert plan.run(x, out, 128, 0) == -8
    assert plan.run(x, out, 128, 0xFFFFFFFF) == -8
