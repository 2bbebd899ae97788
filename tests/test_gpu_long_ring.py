"""Long C2C (n = 8192 .. 65536) on the "ring" schedule: one persistent launch with its four-step
intermediate in an L2-resident ring of row slots (k_long_ring), through the C ABI.

The ring kernel runs the same per-element arithmetic as the two-kernel four-step (N1-point
column FFTs, W_n^(n2*k1), 256-point row FFTs), so the two are compared with each other (rel L2
<= 1e-7: any larger difference is an indexing or ordering error) and both against the FP64
oracle at the long-C2C tolerance (rel L2 <= 2e-6 per row).  Small slots (1 MB) make the ring
wrap many times within one launch, exercising the waits on the slot counters; batches that are
not a multiple of the slot rows leave a partial last chunk.  The autotuner can choose the ring
schedule; the default long C2C plan stays the two-kernel four-step, measured faster on B200."""
import numpy as np
import pytest

import oracle.fft_oracle as O

pytestmark = pytest.mark.gpu

LONG = [8192, 16384, 32768, 65536]


RING = "r16_cta256_shared_fp32_ring"
FOUR_STEP = "r16_cta256_shared_fp32_four_step"


def _run(plan, x, n, batch, direction, scale, monkeypatch, slot_mb="8"):
    import torch
    monkeypatch.setenv("BFLY_LONG_RING_MB", slot_mb)
    y = torch.empty_like(x)
    assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, direction, scale, 0) == 0
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("n", LONG)
@pytest.mark.parametrize("batch", [1, 5, 37])
@pytest.mark.parametrize("direction", [-1, 1])
@pytest.mark.parametrize("slot_mb", ["1", "8"])
def test_ring_matches_oracle_and_two_kernel(ctx, cuda, monkeypatch, n, batch, direction, slot_mb):
    import torch
    plan = ctx.make_plan(RING, 8192, 1)
    four = ctx.make_plan(FOUR_STEP, 8192, 1)
    x = torch.from_numpy(O.normal_input(n, batch, 3 + n % 89 + batch)).to(cuda).view(torch.complex64)
    scale = 1.0 if direction < 0 else 1.0 / n
    yr = _run(plan, x, n, batch, direction, scale, monkeypatch, slot_mb)
    assert plan.long_device_status() == 0
    y2 = _run(four, x, n, batch, direction, scale, monkeypatch)
    xd = x.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(xd, axis=-1) if direction < 0 else np.fft.ifft(xd, axis=-1)
    assert O.rel_l2_rows(yr.cpu().numpy(), ref) <= 2e-6
    assert O.rel_l2_rows(y2.cpu().numpy(), ref) <= 2e-6
    assert O.max_rel_scaled_rows(O.to_interleaved(yr.cpu().numpy()), O.to_interleaved(ref)) <= 1e-4
    diff = (torch.linalg.vector_norm(yr - y2) / torch.linalg.vector_norm(y2)).item()
    assert diff <= 1e-7, diff


@pytest.mark.parametrize("n,batch", [(8192, 130), (65536, 19)])
def test_ring_many_chunks(ctx, cuda, monkeypatch, n, batch):
    """1 MB slots: 2 rows (n = 65536) or 16 rows (n = 8192) per chunk, the ring reused 3-4 times
    per slot in one launch; every row checked against FP64."""
    import torch
    plan = ctx.make_plan(RING, 8192, 1)
    g = torch.Generator(device=cuda).manual_seed(n + batch)
    x = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    y = _run(plan, x, n, batch, -1, 1.0, monkeypatch, "1")
    assert plan.long_device_status() == 0
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_l2_rows(y.cpu().numpy(), ref) <= 2e-6


def test_ring_graph_capture_and_replay(ctx, cuda, monkeypatch):
    """The launch (counter reset + cooperative kernel) captured in a CUDA graph and replayed on
    new input gives the eager result."""
    import torch
    monkeypatch.setenv("BFLY_LONG_RING_MB", "4")
    n, batch = 32768, 45
    plan = ctx.make_plan(RING, 8192, 1)
    assert plan.prepare(n, batch) == 0
    g = torch.Generator(device=cuda).manual_seed(5)
    x = torch.randn(batch, n, dtype=torch.complex64, device=cuda, generator=g)
    y = torch.empty_like(x)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):   # warm-up: workspace and counters are allocated outside the capture
        assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, s.cuda_stream) == 0
    s.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        assert plan.exec_c2c(x.data_ptr(), y.data_ptr(), n, batch, -1, 1.0, s.cuda_stream) == 0
    for seed in (6, 7):
        x.copy_(torch.randn(batch, n, dtype=torch.complex64, device=cuda,
                            generator=torch.Generator(device=cuda).manual_seed(seed)))
        y.zero_()
        graph.replay()
        torch.cuda.synchronize()
        rows = O.sample_batches(batch, 4)
        ref = np.fft.fft(x[rows].cpu().numpy().astype(np.complex128), axis=-1)
        assert O.rel_l2_rows(y[rows].cpu().numpy(), ref) <= 2e-6
    del graph
    assert plan.long_device_status() == 0
