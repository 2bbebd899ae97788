"""CPU, world size 2 over gloo: batch sharding covers every row exactly once and the gathered
result equals the unsharded transform (the row transform here is numpy's FFT standing in for
the GPU kernel; the sharding logic is what is under test)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from bfly.shard import shard_rows, sharded_fft


def test_shard_rows_partition():
    for batch in (0, 1, 2, 3, 7, 148, 4097):
        for world in (1, 2, 3, 4, 8):
            covered = []
            sizes = []
            for r in range(world):
                a, b = shard_rows(batch, world, r)
                covered += list(range(a, b))
                sizes.append(b - a)
            assert covered == list(range(batch))
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_rows(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(0)
        x = torch.randn(13, 64, dtype=torch.complex64, generator=g)
        fn = lambda t: torch.from_numpy(np.fft.fft(t.numpy(), axis=-1).astype(np.complex64))
        local, full = sharded_fft(x, fn, gather=True)
        ref = torch.from_numpy(np.fft.fft(x.numpy(), axis=-1).astype(np.complex64))
        a, b = shard_rows(13, world, rank)
        ok = torch.allclose(local, ref[a:b]) and torch.allclose(full, ref)
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, True), (1, True)]
