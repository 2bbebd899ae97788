"""Plan reuse, stale-output detection and lifecycle checks, after the reference's harness and
test profiles: the A/B/A re-execution under one plan with a stale-output detector
(src/host/fft_check.cpp:1294-1301), the smoke profile's batches {1, 3, 47, 48, 49} at
n in {64, 256, 1024, 4096} (docs/testing.md:30-54, config/test_matrix.json), and the stress
profile's plan reuse with device-memory leak checks."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 1024, 4096, 8192, 1536, 1000])
def test_aba_sequence_no_stale_output(ctx, cuda, n):
    """Transform A, then B, then A again under one plan (device and host entry points): the
    second A must equal the first bit for bit, B must differ and match its own oracle."""
    import torch
    plan = ctx.make_plan()
    batch = 9
    a = torch.from_numpy(O.normal_input(n, batch, 1)).to(cuda).view(torch.complex64)
    b = torch.from_numpy(O.normal_input(n, batch, 2)).to(cuda).view(torch.complex64)
    y = torch.empty_like(a)
    outs = []
    for x in (a, b, a):
        assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, 0) == 0
        torch.cuda.synchronize()
        outs.append(y.clone())
    assert torch.equal(outs[0], outs[2])
    assert not torch.equal(outs[0], outs[1])
    ref_b = np.fft.fft(b.cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(outs[1].cpu().numpy(), ref_b) <= 2e-6
    if n <= 4096 and n & (n - 1) == 0 and n >= 64:   # the reference's host-pointer envelope
        ha = O.normal_input(n, batch, 1)
        hb = O.normal_input(n, batch, 2)
        hy = np.empty_like(ha)
        host = []
        for hx in (ha, hb, ha):
            assert plan.run(hx, hy, n, batch) == 0
            host.append(hy.copy())
        assert np.array_equal(host[0], host[2]) and not np.array_equal(host[0], host[1])
        assert np.array_equal(host[0], outs[0].cpu().numpy().view(np.float32).reshape(batch, 2 * n))


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
@pytest.mark.parametrize("batch", [1, 3, 47, 48, 49])
def test_smoke_profile(plan, n, batch):
    """select -> run on the reference's pattern input, every row against its FP64 oracle with
    the reference's acceptance metric and the relative-L2 gate."""
    x = O.pattern_at(np.arange(batch * 2 * n)).reshape(batch, 2 * n)   # patternAt over the buffer
    y = np.empty_like(x)
    assert plan.run(x, y, n, batch) == 0
    ref = O.c2c(x)
    assert O.max_rel_scaled_rows(y, O.to_interleaved(ref)) <= 1e-4
    assert O.rel_l2_rows(y, ref) <= 1e-6


def test_plan_lifecycle_releases_device_memory(cuda):
    """Contexts and plans that build tables and workspaces for many kinds of transform give all
    their device memory back when destroyed; one plan reused for 10,000 launches stays correct."""
    import gc
    import torch
    import bfly

    x = torch.randn(64, 8192, dtype=torch.complex64, device=cuda)
    y = torch.empty_like(x)
    r = torch.randn(64, 8192, device=cuda)
    R = torch.empty(64, 4097, dtype=torch.complex64, device=cuda)

    def cycle():
        ctx = bfly.Context()
        assert ctx.init(device=cuda.index or 0) == 0
        plans = [ctx.make_plan(), ctx.make_plan("r16_cta256_shared_fp32_four_step", 8192, 1)]
        for n in (64, 4096, 8192, 1536, 1000, 32768):      # single pass, prime-factor, Bluestein
            assert plans[0].exec_c2c(x.data_ptr(), y.data_ptr(), n, 4, -1, 1.0, 0) == 0
        assert plans[0].exec_r2c(r.data_ptr(), R.data_ptr(), 8192, 4, 1.0, 1.0, 0) == 0
        assert plans[0].exec_c2c_2d(x.data_ptr(), y.data_ptr(), 64, 8192, 1, -1, 1.0, 0) == 0
        for n in (8192, 32768):                            # four-step workspace
            assert plans[1].exec_c2c(x.data_ptr(), y.data_ptr(), n, 4, -1, 1.0, 0) == 0
        torch.cuda.synchronize()
        del plans
        ctx.close()
        gc.collect()
        torch.cuda.synchronize()

    cycle()                      # module loads and first-use allocations of the process
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(20):
        cycle()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 <= 8 << 20, (free0, free1)   # nothing retained beyond driver slack

    ctx = bfly.Context()
    assert ctx.init(device=cuda.index or 0) == 0
    plan = ctx.make_plan()
    small = torch.randn(3, 256, dtype=torch.complex64, device=cuda)
    out = torch.empty_like(small)
    assert plan.exec_c2c(small.data_ptr(), out.data_ptr(), 256, 3, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    first = out.clone()
    for _ in range(10000):
        assert plan.exec_c2c(small.data_ptr(), out.data_ptr(), 256, 3, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    assert torch.equal(out, first)
    del plan
    ctx.close()
