"""Ragged persistent launch (one kernel for many lengths and batch counts) on the GPU through
the C ABI: the 256-request mix of the benchmark configuration (seed 7), forward and inverse
requests mixed, checked per request against the FP64 oracle on sampled rows, plus CUDA graph
capture and replay."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu


def _build(ctx, cuda, reqs, seed=7):
    import torch
    plan = ctx.make_plan()
    bufs = []
    g = torch.Generator(device=cuda).manual_seed(seed)
    for i, (n, b) in enumerate(reqs):
        x = torch.randn(b, n, dtype=torch.complex64, device=cuda, generator=g)
        bufs.append((n, b, x, torch.empty_like(x), -1 if i % 3 else 1, 1.0 if i % 3 else 1.0 / n))
    ragged = plan.make_ragged((x.data_ptr(), y.data_ptr(), n, b, d, s) for n, b, x, y, d, s in bufs)
    return plan, ragged, bufs


def _check(bufs, tol=1e-6):
    worst = 0.0
    for n, b, x, y, d, s in bufs:
        rows = O.sample_batches(b, 3)
        xs = x[rows].cpu().numpy().astype(np.complex128)
        ref = np.fft.fft(xs, axis=-1) if d < 0 else np.fft.ifft(xs, axis=-1) * n * s
        err = O.rel_l2_rows(y[rows].cpu().numpy(), ref)
        worst = max(worst, err)
        assert err <= tol, (n, b, d, err)
    return worst


@pytest.mark.parametrize("stages", ["-1", "0", "1", "2"])
def test_ragged_config_mix(ctx, cuda, stages, monkeypatch):
    """The 256-request mix: one tile per CTA (-1), persistent CTAs with plain loads (0) and with
    bulk-copy staged tiles (1, 2)."""
    import torch
    monkeypatch.setenv("BFLY_RAGGED_STAGES", stages)
    reqs = O.ragged_requests(256, 7)
    plan, ragged, bufs = _build(ctx, cuda, reqs)
    info = ragged.info()
    assert info["tiles"] > 0 and info["grid"] > 0 and info["stages"] == int(stages)
    assert ragged.exec(torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert ragged.device_status() == 0
    _check(bufs)
    ragged.close()


def test_ragged_unaligned_inputs_use_plain_loads(ctx, cuda):
    """An input that is only 8-byte aligned cannot be bulk-copied: asking for staged tiles
    falls back to the plain persistent kernel."""
    import torch
    plan = ctx.make_plan()
    n, b = 256, 33
    base = torch.randn(b * n + 1, dtype=torch.complex64, device=cuda)
    x = base[1:].view(b, n)                      # 8-byte offset
    y = torch.empty(b, n, dtype=torch.complex64, device=cuda)
    os = __import__("os")
    os.environ["BFLY_RAGGED_STAGES"] = "1"
    try:
        rg = plan.make_ragged([(x.data_ptr(), y.data_ptr(), n, b, -1, 1.0)])
    finally:
        del os.environ["BFLY_RAGGED_STAGES"]
    assert x.data_ptr() % 16 == 8 and rg.info()["stages"] == 0
    assert rg.exec(0) == 0
    torch.cuda.synchronize()
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(y.cpu().numpy(), ref) <= 1e-6


def test_ragged_every_length_and_partial_tiles(ctx, cuda):
    import torch
    reqs = [(n, b) for n in (32, 64, 128, 256, 512, 1024, 2048, 4096) for b in (1, 3, 65, 129)]
    plan, ragged, bufs = _build(ctx, cuda, reqs, seed=3)
    assert ragged.exec(0) == 0
    torch.cuda.synchronize()
    _check(bufs)


def test_ragged_graph_capture_replay(ctx, cuda):
    import torch
    reqs = [(64, 4096), (1024, 300), (4096, 17), (256, 1)]
    plan, ragged, bufs = _build(ctx, cuda, reqs, seed=5)
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        assert ragged.exec(s.cuda_stream) == 0
    for _, _, _, y, _, _ in bufs:
        y.zero_()
    graph.replay()
    torch.cuda.synchronize()
    _check(bufs)
    # replay again after changing the inputs in place: the graph reads the new values
    for _, _, x, _, _, _ in bufs:
        x.mul_(2)
    graph.replay()
    torch.cuda.synchronize()
    _check(bufs)
