"""The B200 kernels against the reference's own fp32 output on identical seeded inputs.

The reference's device output needs an Ascend NPU, so its stand-in is the C restatement of the
fp32 arithmetic of its AscendC kernels (oracle/kfft_fp32.c: kfft_fwd, kfft_r2c_post,
kfft_c2r_prep/post, src/ascendc/fft_radix2.cpp and fft_real.cpp), which the CPU tests hold
within the reference's published device error of the FP64 oracle.  Here the GPU result must
agree with it at the tolerance the reference's path is held to against FP64: rel L2 <= 1e-6 per
row and the reference's maxRelScaled <= 1e-4 (src/host/fft_check.cpp:1313); both are also
checked against FP64 to show neither side drifts."""
import numpy as np
import pytest

import oracle.clib as clib
import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("batch", [1, 7])
def test_c2c_against_reference_fp32(plan, n, batch):
    x = O.normal_input(n, batch, 500 + n + batch)
    y = np.empty_like(x)
    assert plan.run(x, y, n, batch) == 0
    ref32 = clib.kfft_fwd(x, n)
    ref64 = O.c2c(x)
    assert O.rel_l2_rows(y, O.to_complex(ref32)) <= 1e-6
    assert O.max_rel_scaled_rows(y, ref32) <= 1e-4
    assert O.rel_l2_rows(ref32, ref64) <= 1e-6 and O.rel_l2_rows(y, ref64) <= 1e-6


@pytest.mark.parametrize("n", [128, 256, 1024, 4096, 8192])
def test_r2c_against_reference_fp32(plan, n):
    batch = 5
    x = np.random.default_rng(n).uniform(-1, 1, (batch, n)).astype(np.float32)
    y = np.empty((batch, n + 2), np.float32)
    assert plan.run_r2c(x, y, n, batch) == 0
    ref32 = clib.kfft_r2c(x, n)
    ref64 = np.fft.rfft(x.astype(np.float64), axis=-1)
    assert O.rel_l2_rows(y, O.to_complex(ref32)) <= 1e-6
    assert O.max_rel_scaled_rows(y, ref32) <= 1e-4
    assert O.rel_l2_rows(y, ref64) <= 1e-6


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
def test_c2r_against_reference_fp32(plan, n):
    batch = 5
    r = np.random.default_rng(n + 1).uniform(-1, 1, (batch, n))
    X = np.fft.rfft(r, axis=-1)
    X[:, 0] = X[:, 0].real
    X[:, -1] = X[:, -1].real
    h = O.to_interleaved(X.astype(np.complex64))
    y = np.empty((batch, n), np.float32)
    assert plan.run_c2r(h, y, n, batch) == 0
    ref32 = clib.kfft_c2r(h, n)
    ref64 = np.fft.irfft(X, n, axis=-1)
    d = np.linalg.norm(y - ref32, axis=-1) / np.linalg.norm(ref32, axis=-1)
    assert float(d.max()) <= 1e-6
    d64 = np.linalg.norm(y - ref64, axis=-1) / np.linalg.norm(ref64, axis=-1)
    assert float(d64.max()) <= 1e-6
