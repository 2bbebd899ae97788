"""Split-BF16 tensor-core C2C (tcgen05) through the C ABI, against the FP64 oracle.

The error of every configuration is measured and bounded: three bf16 terms (6 products) must
meet the project tolerance of the fp32 path (rel L2 <= 1e-6 per row); two terms (3 products)
keep ~16-17 bits per factor and are gated at rel L2 <= 3e-5 (they are reported, not sold as
fp32-accurate).  The tensor-core result must also agree with the CUDA-core fp32 path to the
same bounds, and the device status word must stay clear."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

TOL = {3: 1e-6, 2: 3e-5}


LENGTHS = [64, 128, 256, 512, 1024, 2048, 4096]   # radix-16 passes on tcgen05, the rest in fp32


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("split", [3, 2])
@pytest.mark.parametrize("batch", [1, 3, 37])
def test_tc_c2c_forward(ctx, cuda, n, split, batch):
    import torch
    plan = ctx.make_plan()
    x = torch.from_numpy(O.normal_input(n, batch, 17 + n + batch)).to(cuda).view(torch.complex64)
    y = torch.empty_like(x)
    assert plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, split, 0) == 0
    torch.cuda.synchronize()
    assert plan.tc_device_status() == 0
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=-1)
    err = O.rel_l2_rows(y.cpu().numpy(), ref)
    assert err <= TOL[split], (n, split, batch, err)
    assert O.max_rel_scaled_rows(O.to_interleaved(y.cpu().numpy()), O.to_interleaved(ref)) <= 1e-4
    fp32 = torch.empty_like(x)
    assert plan.exec_c2c(x.data_ptr(), fp32.data_ptr(), n, batch, -1, 1.0, 0) == 0
    torch.cuda.synchronize()
    rel = (torch.linalg.vector_norm(y - fp32) / torch.linalg.vector_norm(fp32)).item()
    assert rel <= 2 * TOL[split]


@pytest.mark.parametrize("n", LENGTHS)
def test_tc_inverse_and_round_trip(ctx, cuda, n):
    import torch
    plan = ctx.make_plan()
    batch = 5
    x = torch.from_numpy(O.normal_input(n, batch, 3)).to(cuda).view(torch.complex64)
    y = torch.empty_like(x)
    back = torch.empty_like(x)
    assert plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, 3, 0) == 0
    assert plan.exec_c2c_tc(y.data_ptr(), back.data_ptr(), n, batch, 1, 1.0 / n, 3, 0) == 0
    torch.cuda.synchronize()
    ref = np.fft.ifft(y.cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(back.cpu().numpy(), ref) <= 1e-6
    assert (torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)).item() <= 2e-6


def test_tc_large_batch_and_guards(ctx, cuda):
    import torch
    plan = ctx.make_plan()
    n, batch = 4096, 2048
    g = torch.Generator(device=cuda).manual_seed(9)
    x = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    y = torch.empty_like(x)
    assert plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, 3, 0) == 0
    torch.cuda.synchronize()
    rows = O.sample_batches(batch, 4)
    ref = np.fft.fft(x[rows].cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(y[rows].cpu().numpy(), ref) <= 1e-6
    for bad_n in (32, 96, 8192):
        assert plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), bad_n, 1, -1, 1.0, 3, 0) == -8
    assert plan.exec_c2c_tc(x.data_ptr(), y.data_ptr(), 4096, 1, -1, 1.0, 4, 0) == -8
