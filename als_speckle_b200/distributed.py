"""Multi-GPU trial sharding: one process per GPU, no collective on the data path.

Trials are independent, so each rank iterates its own share of them.  The
only exchange happens after the iterations: the sum of the globally
phase-aligned reconstructions (for the average) and the sum of unit Fourier
phasors (for the PRTF) are added across ranks with one all-reduce each
(NCCL over NVLink between GPUs; gloo on the CPU in the tests).  The
reference has no multi-device path (``speckle/gpu.py:491-493``).
"""
from __future__ import annotations

from typing import List, Sequence

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
