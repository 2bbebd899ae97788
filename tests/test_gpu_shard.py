"""Batch sharding with the library's kernels: two gloo ranks, each transforming its contiguous
row range with bfly.fft on cuda:0 and all-gathering the shards (the multi-GPU path of
bfly.shard; on this one-GPU runner both ranks share the device, which is valid because the
ranks' kernels never wait on one another).  The gathered result must equal the unsharded
bfly.fft bit for bit (the same kernel on the same rows) and the FP64 FFT to rel L2 <= 1e-6."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    for p in (str(root / "ascend-fft_b200"), str(root)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import torch
    import torch.distributed as dist
    import bfly
    from bfly.shard import shard_rows, sharded_fft
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dev = torch.device("cuda", 0)
        g = torch.Generator().manual_seed(3)
        batch, n = 1001, 1024
        x = torch.randn(batch, n, dtype=torch.complex64, generator=g)
        fn = lambda t: bfly.fft(t.to(dev)).cpu()
        local, full = sharded_fft(x, fn, gather=True)
        whole = bfly.fft(x.to(dev)).cpu()
        a, b = shard_rows(batch, world, rank)
        ref = np.fft.fft(x.numpy().astype(np.complex128), axis=-1)
        err = float(np.max(np.linalg.norm(full.numpy() - ref, axis=-1) / np.linalg.norm(ref, axis=-1)))
        ok = torch.equal(local, whole[a:b]) and torch.equal(full, whole) and err <= 1e-6
        q.put((rank, bool(ok), err))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_bfly_fft(cuda):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[:2] for r in res] == [(0, True), (1, True)], res
