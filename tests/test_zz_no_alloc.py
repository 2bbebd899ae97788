"""The allocation-free long C2C entry point (bfly_exec_c2c_long_noalloc).

It exists for callers that cannot call cudaMalloc when they need a transform (graph capture
in progress, real-time loops, memory owned by another allocator), so it keeps its workspace in
a fixed 32 MiB array of the library instead of growing a plan-owned one.  This file runs last
(pytest collects it after the other test files) so that a failure here leaves every other test
already run; it also passes alone in a fresh process.

Checks, through the C ABI: two calls in a row (a forward at the workspace limit, then an
inverse with a scale) agree with the regular plan entry point within the long-transform
tolerance (relative L2 <= 2e-6), the second call (a length and direction nothing in the
process has run before) leaves the device's free memory unchanged, and sizes past the limit,
including a batch whose product with n wraps in 64 bits, are rejected with -12.
"""
import ctypes as C

import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

MAX_ELEMS = 4194304


def _rel(a, b):
    import torch
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def test_noalloc_long_matches_plan_entry_point(cuda):
    import torch
    import bfly

    lib = bfly.load()
    ctx = bfly.Context()
    assert ctx.init(device=cuda.index or 0) == 0
    plan = ctx.make_plan()
    stream = torch.cuda.current_stream(cuda).cuda_stream
    g = torch.Generator(device=cuda).manual_seed(11)

    # call 1: forward at the workspace limit (65536 x 64), before the plan runs that length
    n, batch = 65536, MAX_ELEMS // 65536
    x = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    want = torch.empty_like(x)
    got = torch.empty_like(x)
    assert lib.bfly_exec_c2c_long_noalloc(x.data_ptr(), got.data_ptr(), n, batch, -1, 1.0, stream) == 0
    assert plan.exec_c2c(x.data_ptr(), want.data_ptr(), n, batch, -1, 1.0, stream) == 0
    torch.cuda.synchronize()
    assert _rel(got, want) <= 2e-6
    rows = O.sample_batches(batch, 2)
    ref = np.fft.fft(x[rows].cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(got[rows].cpu().numpy(), ref) <= 2e-6

    # call 2: inverse with a scale at another length.  Neither the plan nor the first call has
    # run this (length, direction), so a call that loaded device code or allocated a workspace
    # here would show in the free device memory; the plan's result is computed afterwards.
    n2, batch2 = 8192, 37
    y = torch.randn(batch2, n2, dtype=torch.complex64, device=cuda, generator=g)
    want2 = torch.empty_like(y)
    got2 = torch.empty_like(y)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(cuda)[0]
    assert lib.bfly_exec_c2c_long_noalloc(y.data_ptr(), got2.data_ptr(), n2, batch2, 1, 1.0 / n2,
                                          stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(cuda)[0] == free_before
    assert plan.exec_c2c(y.data_ptr(), want2.data_ptr(), n2, batch2, 1, 1.0 / n2, stream) == 0
    torch.cuda.synchronize()
    assert _rel(got2, want2) <= 2e-6


def test_noalloc_long_rejects_bad_sizes(cuda):
    import bfly
    lib = bfly.load()
    p = C.c_void_p(16)   # never dereferenced: every call below is rejected before GPU work
    assert lib.bfly_exec_c2c_long_noalloc(p, p, 65536, MAX_ELEMS // 65536 + 1, -1, 1.0, None) == -12
    assert lib.bfly_exec_c2c_long_noalloc(p, p, 8192, MAX_ELEMS // 8192 + 1, -1, 1.0, None) == -12
    # n * batch wraps to 65536 in 64 bits: still too large
    assert lib.bfly_exec_c2c_long_noalloc(p, p, 65536, (1 << 48) + 1, -1, 1.0, None) == -12
    assert lib.bfly_exec_c2c_long_noalloc(p, p, 4096, 1, -1, 1.0, None) == -8
    assert lib.bfly_exec_c2c_long_noalloc(p, p, 8192, 1, 0, 1.0, None) == -8
    assert lib.bfly_exec_c2c_long_noalloc(None, p, 8192, 1, -1, 1.0, None) == -10
