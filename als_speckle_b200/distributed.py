"""Multi-GPU trial sharding: one process per GPU, no collective on the data path.

Trials are independent, so each rank iterates its own share of them.  The
only exchanges happen after the iterations: the owner of trial 0 broadcasts
its phase-aligned crop (every rank registers its trials to it), then the sum
of the aligned reconstructions (for the average) and the sum of unit Fourier
phasors (for the PRTF) are added across ranks with one all-reduce each
(NCCL over NVLink between GPUs; gloo on the CPU in the tests).
``solve_sharded`` runs that whole pipeline for one reconstruction.  The
reference has no multi-device path (``speckle/gpu.py:491-493``).
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import torch
import torch.distributed as dist


def shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Indices of the trials each rank runs: greedy longest-first onto the
    least-loaded rank, balancing sum(cost) (cost ~ N^2 * iterations)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += costs[i]
    for o in out:
        o.sort()
    return out


def reduce_sums(frame_sum: torch.Tensor, phasor_sum: torch.Tensor, count: int, group=None):
    """All-reduce (in place) the aligned-frame sum and the PRTF phasor sum of
    the local trials; returns the global trial count."""
    c = torch.tensor([float(count)], dtype=torch.float64, device=frame_sum.device)
    for t in (frame_sum, phasor_sum):
        if torch.is_complex(t):
            v = torch.view_as_real(t)
            dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
        else:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
    return int(c.item())


def finish_average(frame_sum: torch.Tensor, count: int) -> torch.Tensor:
    return frame_sum / count


def local_sums(aligned_frames: torch.Tensor, N: int):
    """(sum of aligned frames, sum of unit Fourier phasors) of this rank's
    frames, on the device through libspeckle_b200."""
    from ._lib import call, ptr, stream_ptr
    F, r, c = aligned_frames.shape
    frames = aligned_frames.to(torch.complex64).contiguous()
    fsum = torch.zeros((r, c), dtype=torch.complex64, device=frames.device)
    acc = torch.zeros((N, N), dtype=torch.complex64, device=frames.device)
    if F:
        call("sp_mean_frames", ptr(frames), F, r * c, ptr(fsum), stream_ptr())
        fsum *= F
        work = torch.empty((F, N, N), dtype=torch.complex64, device=frames.device)
        call("sp_prtf_phasors", ptr(frames), F, r, c, N, ptr(work), ptr(acc), stream_ptr())
    return fsum, acc


def finish_prtf(phasor_sum: torch.Tensor, count: int) -> torch.Tensor:
    from ._lib import call, ptr, stream_ptr
    N = phasor_sum.shape[-1]
    out = torch.empty((N, N), dtype=torch.float32, device=phasor_sum.device)
    call("sp_prtf_finish", ptr(phasor_sum.contiguous()), int(count), N, ptr(out), stream_ptr())
    return out


class DeviceOps:
    """The per-rank steps of ``solve_sharded`` on this rank's GPU, through
    libspeckle_b200: the engine solve, the global-phase alignment
    (``phasing.py:1355-1404``), the subpixel registration to a reference
    frame, the local sums and the PRTF finish."""

    def __init__(self, engine=None, device=None):
        from .engine import Engine
        self.engine = engine or Engine(device=device)

    def solve(self, specs):
        self.engine.solve(specs)

    def align_phase(self, frames):
        from ._lib import call, ptr, stream_ptr
        F = frames.shape[0]
        if F == 0:
            return frames
        sums = torch.empty(5 * F, dtype=torch.float64, device=frames.device)
        angles = torch.empty(F, dtype=torch.float64, device=frames.device)
        call("sp_align_global_phase", ptr(frames), F, frames[0].numel(), ptr(angles), ptr(sums),
             stream_ptr())
        return frames

    def register(self, frames, ref, upsample):
        import ctypes
        from ._lib import call, ptr, stream_ptr
        F, rows, cols = frames.shape
        if F == 0:
            return frames
        n = max(8, 1 << (max(rows, cols) - 1).bit_length())
        nb = ctypes.c_size_t(0)
        call("sp_register_workspace_size", F, n, int(upsample), ctypes.byref(nb))
        work = torch.empty(nb.value, dtype=torch.uint8, device=frames.device)
        shifts = torch.empty((F, 3), dtype=torch.float64, device=frames.device)
        call("sp_register_subpixel", ptr(frames), F, rows, cols, ptr(ref.contiguous()), n,
             int(upsample), ptr(work), nb.value, ptr(shifts), ptr(frames), stream_ptr())
        return frames

    def sums(self, frames, N):
        return local_sums(frames, N)

    def finish_prtf(self, phasor_sum, count):
        return finish_prtf(phasor_sum, count)


def _owner(parts, trial):
    for r, p in enumerate(parts):
        if trial in p:
            return r
    raise ValueError("trial %d is in no shard" % trial)


def solve_sharded(modulus, support, n_trials, iterations, order=None, beta=0.9, seed=0,
                  box=None, N_prtf=None, upsample=64, ops=None, group=None,
                  costs: Optional[Sequence[float]] = None):
    """One reconstruction of ``n_trials`` random-phase trials spread over the
    ranks of ``group``: shard (longest-first) -> each rank's engine solve ->
    global-phase alignment -> broadcast of trial 0's aligned crop from its
    owner -> subpixel registration of every local trial to it -> local sums
    of frames and PRTF phasors -> all-reduce -> average and PRTF.  Trial k
    starts from the same random phase (seed, k) on whichever rank runs it, so
    the result matches a single-process run of the same job.  Returns
    (average (rows, cols), prtf (N_prtf, N_prtf), trial count, this rank's
    trial indices).  Every rank must call it with the same arguments."""
    from .engine import TrialSpec
    from .masking import bounding_box
    import numpy as np
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    ops = ops or DeviceOps(device=modulus.device)
    N = int(modulus.shape[-1])
    if box is None:
        bb = bounding_box(support.detach().cpu().numpy(), pad=10)
        box = (int(bb[0]), int(bb[2]), int(bb[1] - bb[0]), int(bb[3] - bb[2]))
    r0, c0, rows, cols = box
    parts = shard(costs if costs is not None else [float(N * N * iterations)] * n_trials, world)
    mine = parts[rank]
    dev = modulus.device
    psis = torch.zeros((len(mine), N, N), dtype=torch.complex64, device=dev)
    saves = torch.zeros((len(mine), rows, cols), dtype=torch.complex64, device=dev)
    specs = [TrialSpec(psi=psis[j], modulus=modulus, support=support, iterations=iterations,
                       order=order, beta=beta, random_phase=True, seed=seed, trial=k, box=box,
                       save=saves[j]) for j, k in enumerate(mine)]
    if specs:
        ops.solve(specs)
    ops.align_phase(saves)
    owner = _owner(parts, 0)
    ref = saves[mine.index(0)].clone() if rank == owner else \
        torch.zeros((rows, cols), dtype=torch.complex64, device=dev)
    if world > 1:
        dist.broadcast(torch.view_as_real(ref), src=dist.get_global_rank(group, owner)
                       if group is not None else owner, group=group)
    ops.register(saves, ref, upsample)
    fsum, psum = ops.sums(saves, N_prtf or N)
    count = reduce_sums(fsum, psum, len(mine), group) if world > 1 else len(mine)
    return finish_average(fsum, count), ops.finish_prtf(psum, count), count, mine
