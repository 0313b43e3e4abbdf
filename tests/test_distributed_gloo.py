"""Multi-process host logic of the sharded path on CPU (gloo, world size 2):
trial sharding and the cross-rank reduction of the average and PRTF sums."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_shard_balances_and_covers():
    from als_speckle_b200.distributed import shard
    costs = [256 ** 2 * 1000] * 64 + [512 ** 2 * 1000] * 32 + [1024 ** 2 * 1000] * 8 + [2048 ** 2 * 1000] * 2
    for world in (1, 2, 4, 8):
        parts = shard(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, frames, phasors, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from als_speckle_b200.distributed import shard, reduce_sums, finish_average
        parts = shard([1.0] * frames.shape[0], world)
        mine = parts[rank]
        fsum = torch.from_numpy(frames[mine].sum(axis=0)).to(torch.complex64)
        psum = torch.from_numpy(phasors[mine].sum(axis=0)).to(torch.complex64)
        count = reduce_sums(fsum, psum, len(mine))
        q.put((rank, count, finish_average(fsum, count).numpy(), psum.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_equals_single_process():
    rng = np.random.default_rng(0)
    F = 7
    frames = (rng.standard_normal((F, 6, 5)) + 1j * rng.standard_normal((F, 6, 5))).astype(np.complex64)
    ph = rng.standard_normal((F, 8, 8)) + 1j * rng.standard_normal((F, 8, 8))
    phasors = (ph / np.abs(ph)).astype(np.complex64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, frames, phasors, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, count, avg, psum in out:
        assert count == F
        assert np.allclose(avg, frames.mean(axis=0), atol=1e-6)
        assert np.allclose(psum, phasors.sum(axis=0), atol=1e-5)
