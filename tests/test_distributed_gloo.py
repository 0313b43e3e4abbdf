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


class FakeOps:
    """The per-rank steps of solve_sharded on the CPU: trial k's "solve"
    writes a known frame (a fixed object moved by a trial-specific shift on
    the 1/16 grid, times a trial-specific phase); alignment, registration,
    sums and PRTF run through the oracle's numpy restatements."""

    def __init__(self, base):
        self.base = base

    @staticmethod
    def frame_for(base, k):
        from oracle import phasing_oracle as O
        rng = np.random.default_rng(100 + k)
        dy, dx = rng.integers(-24, 25, 2) / 16.0
        return O.fourier_shift(base, dy, dx, N=32) * np.exp(1j * rng.uniform(-3, 3))

    def solve(self, specs):
        for s in specs:
            s.save.copy_(torch.from_numpy(self.frame_for(self.base, s.trial).astype(np.complex64)))

    def align_phase(self, frames):
        from oracle import phasing_oracle as O
        if frames.shape[0]:
            frames.copy_(torch.from_numpy(O.align_global_phase(frames.numpy().astype(np.complex128))
                                          .astype(np.complex64)))
        return frames

    def register(self, frames, ref, upsample):
        from oracle import phasing_oracle as O
        if frames.shape[0]:
            _, al = O.register_subpixel(frames.numpy().astype(np.complex128),
                                        ref.numpy().astype(np.complex128), N=32, upsample=upsample)
            frames.copy_(torch.from_numpy(al.astype(np.complex64)))
        return frames

    def sums(self, frames, N):
        f = frames.numpy().astype(np.complex128)
        emb = np.zeros((f.shape[0], N, N), np.complex128)
        emb[:, :f.shape[1], :f.shape[2]] = f
        F = np.fft.fft2(emb)
        with np.errstate(divide="ignore", invalid="ignore"):
            ph = np.nan_to_num(F / np.abs(F))
        return (torch.from_numpy(f.sum(axis=0).astype(np.complex64)),
                torch.from_numpy(ph.sum(axis=0).astype(np.complex64)))

    def finish_prtf(self, psum, count):
        return torch.from_numpy(np.fft.fftshift(np.abs(psum.numpy() / count)).astype(np.float32))


def _job_inputs():
    N = 64
    S = np.zeros((N, N), np.float32)
    S[22:42, 22:42] = 1
    M = np.ones((N, N), np.float32)
    rng = np.random.default_rng(1)
    base = np.zeros((30, 30), np.complex128)
    base[5:25, 5:25] = rng.random((20, 20)) * np.exp(1j * rng.uniform(-1, 1, (20, 20)))
    return torch.from_numpy(M), torch.from_numpy(S), base


def _sharded_worker(rank, world, port, n_trials, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from als_speckle_b200.distributed import solve_sharded
        M, S, base = _job_inputs()
        avg, prtf, count, mine = solve_sharded(M, S, n_trials, 10, order=(("hio", 10),), seed=4,
                                               box=(17, 17, 30, 30), N_prtf=32, upsample=16,
                                               ops=FakeOps(base))
        q.put((rank, count, mine, avg.numpy(), prtf.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_trials", [7, 1])
def test_solve_sharded_two_ranks_equals_one_process(n_trials):
    """The whole sharded pipeline (shard, solve, phase alignment, broadcast
    of trial 0's crop, registration, sums, all-reduce, finish) on two gloo
    ranks gives the single-process result; with one trial, rank 1 has none
    and still takes part in every collective."""
    from als_speckle_b200.distributed import solve_sharded
    M, S, base = _job_inputs()
    avg1, prtf1, count1, mine1 = solve_sharded(M, S, n_trials, 10, order=(("hio", 10),), seed=4,
                                               box=(17, 17, 30, 30), N_prtf=32, upsample=16,
                                               ops=FakeOps(base))
    assert count1 == n_trials and mine1 == list(range(n_trials))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, n_trials, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=120) for _ in range(2)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(out[0][2] + out[1][2]) == list(range(n_trials))
    for rank, count, mine, avg, prtf in out:
        assert count == n_trials
        assert np.allclose(avg, avg1.numpy(), atol=1e-5)
        assert np.allclose(prtf, prtf1.numpy(), atol=1e-5)
    # the registration did its job: every trial lines up with trial 0, so the
    # average is trial 0's phase-aligned crop, not a blur of shifted copies
    from oracle import phasing_oracle as O
    ref = O.align_global_phase(FakeOps.frame_for(base, 0))
    assert np.linalg.norm(avg1.numpy() - ref) / np.linalg.norm(ref) < 0.02
