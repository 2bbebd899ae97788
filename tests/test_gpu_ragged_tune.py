"""Ragged launch configurations and the ragged autotuner on the GPU through the C ABI.

Every (length, register radix) variant of the ragged kernels -- n = 32..2048 with 8 or 16
values per thread, n = 4096 with 16 -- under every launch mode (-1 one tile per CTA, 0
persistent plain loads, 1 and 2 persistent bulk-copy staged tiles), with batch counts that leave
partial tiles, every row checked against FP64 (rel L2 <= 1e-6 per row).  Then
bfly_context_tune_ragged on the 256-request benchmark mix (seed 7): the tuned work list computes
the same transform, its choice is written to the tuning cache and a second call on the same
shapes reuses it without measuring."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

LENGTHS = (32, 64, 128, 256, 512, 1024, 2048, 4096)


def _buffers(cuda, reqs, seed):
    import torch
    g = torch.Generator(device=cuda).manual_seed(seed)
    bufs = []
    for i, (n, b) in enumerate(reqs):
        x = torch.randn(b, n, dtype=torch.complex64, device=cuda, generator=g)
        bufs.append((n, b, x, torch.empty_like(x), -1 if i % 3 else 1, 1.0 if i % 3 else 1.0 / n))
    return bufs


def _requests(bufs):
    return [(x.data_ptr(), y.data_ptr(), n, b, d, s) for n, b, x, y, d, s in bufs]


def _check(bufs, rows_per_request=None, tol=1e-6):
    for n, b, x, y, d, s in bufs:
        rows = list(range(b)) if rows_per_request is None else O.sample_batches(b, rows_per_request)
        xs = x[rows].cpu().numpy().astype(np.complex128)
        ref = np.fft.fft(xs, axis=-1) if d < 0 else np.fft.ifft(xs, axis=-1) * n * s
        err = O.rel_l2_rows(y[rows].cpu().numpy(), ref)
        assert err <= tol, (n, b, d, err)


def _tiles(reqs, radix8):
    total = 0
    for n, b in reqs:
        logn = n.bit_length() - 1
        e = 8 if (radix8 >> (logn - 5)) & 1 else 16
        rows = 256 // (n // e)
        total += (b + rows - 1) // rows
    return total


@pytest.mark.parametrize("mode", [-1, 0, 1, 2])
@pytest.mark.parametrize("radix8", [0x00, 0x7F, 0x55, 0x2A])
def test_every_variant_every_mode(ctx, cuda, mode, radix8):
    import torch
    plan = ctx.make_plan()
    reqs = [(n, b) for n in LENGTHS for b in (1, 3, 65, 129)]
    bufs = _buffers(cuda, reqs, seed=radix8 + 4 * (mode + 1))
    rg = plan.make_ragged(_requests(bufs), mode=mode, radix8=radix8)
    info = rg.info()
    assert info["stages"] == mode and info["radix8"] == radix8
    assert info["tiles"] == _tiles(reqs, radix8)
    assert rg.exec(torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert rg.device_status() == 0
    _check(bufs)
    rg.close()


def test_invalid_configurations_rejected(ctx, cuda):
    import torch
    plan = ctx.make_plan()
    x = torch.randn(4, 4096, dtype=torch.complex64, device=cuda)
    y = torch.empty_like(x)
    req = [(x.data_ptr(), y.data_ptr(), 4096, 4, -1, 1.0)]
    for mode, radix8 in ((-1, 0x80), (3, 0x3), (-2, 0x3)):
        with pytest.raises(Exception) as e:
            plan.make_ragged(req, mode=mode, radix8=radix8)
        assert "-8" in str(e.value)
    base = torch.randn(257, dtype=torch.complex64, device=cuda)
    odd = [(base[1:].data_ptr(), y.data_ptr(), 256, 1, -1, 1.0)]   # 8-byte aligned input
    with pytest.raises(Exception):
        plan.make_ragged(odd, mode=1, radix8=0x3)
    assert plan.make_ragged(odd, mode=0, radix8=0x3).info()["stages"] == 0


def test_tune_ragged_mix_and_cache(ctx, cuda, tmp_path):
    import torch
    plan = ctx.make_plan()
    reqs = O.ragged_requests(256, 7)
    bufs = _buffers(cuda, reqs, seed=7)
    cache = tmp_path / "tune.json"
    ctx.set_tuning_cache(cache)
    try:
        rg, log = ctx.tune_ragged(plan, _requests(bufs), want_log=True)
        assert "(default)" in log and "selected:" in log, log
        info = rg.info()
        assert info["stages"] in (-1, 0, 1, 2) and info["radix8"] & 0x80 == 0
        assert '"kind": "ragged"' in cache.read_text()
        for _, _, _, y, _, _ in bufs:
            y.zero_()
        assert rg.exec(0) == 0
        torch.cuda.synchronize()
        assert rg.device_status() == 0
        _check(bufs, rows_per_request=3)
        rg2, log2 = ctx.tune_ragged(plan, _requests(bufs), want_log=True)
        assert "tuning cache" in log2, log2
        assert rg2.info()["stages"] == info["stages"] and rg2.info()["radix8"] == info["radix8"]
    finally:
        ctx.set_tuning_cache("")


def test_tune_ragged_graph_capture(ctx, cuda):
    """The tuned work list is an ordinary one: captured in a CUDA graph and replayed."""
    import torch
    plan = ctx.make_plan()
    reqs = [(64, 4096), (1024, 300), (4096, 17), (256, 1), (2048, 1400)]
    bufs = _buffers(cuda, reqs, seed=9)
    rg = ctx.tune_ragged(plan, _requests(bufs))
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        assert rg.exec(s.cuda_stream) == 0
    for _, _, _, y, _, _ in bufs:
        y.zero_()
    graph.replay()
    torch.cuda.synchronize()
    _check(bufs, rows_per_request=4)
    del graph
