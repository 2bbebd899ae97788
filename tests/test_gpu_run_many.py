"""Batched host-to-host round trip (bfly_plan_run_c2c_many) against the device entry point.

Every request must produce exactly what exec_c2c produces for the same rows: the batched call
only reorders copies and launches across streams, never the arithmetic.  Requests mix
single-pass, Bluestein, long (single-pass and four-step) lengths and sizes that split into
several pipeline chunks."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

REQS = [(64, 1, -1, 1.0), (4096, 700, -1, 1.0), (1000, 33, 1, 1e-3), (8192, 300, -1, 1.0),
        (32768, 40, 1, 1.0 / 32768), (256, 5000, -1, 0.5), (16384, 2, -1, 1.0)]


def _pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()


def test_run_many_matches_exec(plan, cuda):
    import torch
    host = []
    for i, (n, b, d, s) in enumerate(REQS):
        x = _pinned((b, 2 * n))
        x[:] = O.normal_input(n, b, 80 + i)
        host.append((x, _pinned((b, 2 * n)), n, b, d, s))
    for _ in range(2):   # twice in a row: device buffers reused
        for _, y, _, _, _, _ in host:
            y[:] = np.nan
        assert plan.run_many(host) == 0
        for x, y, n, b, d, s in host:
            xd = torch.from_numpy(x).to(cuda)
            yd = torch.empty_like(xd)
            assert plan.exec_c2c(xd.data_ptr(), yd.data_ptr(), n, b, d, s, 0) == 0
            torch.cuda.synchronize()
            assert np.array_equal(y, yd.cpu().numpy()), (n, b)
    x, y, n, b, d, s = host[1]
    ref = np.fft.fft(O.to_complex(x).astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(y, ref) <= 1e-6


def test_run_many_guards(plan):
    x = np.zeros((2, 128), dtype=np.float32)
    y = np.zeros_like(x)
    assert plan.run_many([]) == -8
    assert plan.run_many([(x, y, 64, 2), (x, y, 9001, 1)]) == -8
    assert plan.run_many([(x, y, 64, 2, 0, 1.0)]) == -8


@pytest.mark.parametrize("kind", ["c2c", "r2c", "c2r"])
def test_pageable_round_trip_matches_exec(plan, cuda, kind):
    """Large transfers from ordinary (pageable) host memory go through the plan's pinned staging
    slots; results must equal the device entry point's bit for bit."""
    import torch
    n, batch = (4096, 3000) if kind == "c2c" else (2048, 6000)
    rng = np.random.default_rng(3)
    if kind == "c2c":
        x = rng.standard_normal((batch, 2 * n)).astype(np.float32)
        y = np.empty_like(x)
        assert plan.run(x, y, n, batch) == 0
        xd = torch.from_numpy(x).to(cuda)
        yd = torch.empty_like(xd)
        assert plan.exec_c2c(xd.data_ptr(), yd.data_ptr(), n, batch, -1, 1.0, 0) == 0
    elif kind == "r2c":
        x = rng.standard_normal((batch, n)).astype(np.float32)
        y = np.empty((batch, n + 2), np.float32)
        assert plan.run_r2c(x, y, n, batch) == 0
        xd = torch.from_numpy(x).to(cuda)
        yd = torch.empty(batch, n + 2, device=cuda)
        assert plan.exec_r2c(xd.data_ptr(), yd.data_ptr(), n, batch, 1.0, 1.0, 0) == 0
    else:
        x = rng.standard_normal((batch, n + 2)).astype(np.float32)
        y = np.empty((batch, n), np.float32)
        assert plan.run_c2r(x, y, n, batch) == 0
        xd = torch.from_numpy(x).to(cuda)
        yd = torch.empty(batch, n, device=cuda)
        assert plan.exec_c2r(xd.data_ptr(), yd.data_ptr(), n, batch, 1.0, 1.0, 1.0 / n, 0) == 0
    torch.cuda.synchronize()
    assert np.array_equal(y, yd.cpu().numpy())
