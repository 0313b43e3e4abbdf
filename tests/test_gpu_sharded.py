"""distributed.solve_sharded on one GPU (a single rank, no process group):
the whole pipeline -- engine solve, global-phase alignment, registration to
trial 0, frame and PRTF-phasor sums, average and PRTF -- through the device
operators, against the same steps called one by one.  Tolerance 1e-6
relative (the sharded form adds frames and phasors and divides once; the
direct form averages and normalises in its own kernels)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_single_rank_sharded_solve_equals_direct_pipeline():
    from als_speckle_b200 import synth
    from als_speckle_b200.distributed import DeviceOps, solve_sharded
    from als_speckle_b200.engine import Engine, TrialSpec
    from als_speckle_b200.masking import bounding_box
    from als_speckle_b200.phasing import align_frames_subpixel, align_global_phase, mean_frames, prtf
    _, M, S = synth.pattern(128, n_ellipses=6, box=32, peak=1e6, seed=4, support_edge=40)
    Md, Sd = torch.from_numpy(M).cuda(), torch.from_numpy(S).cuda()
    bb = bounding_box(S, pad=10)
    box = (int(bb[0]), int(bb[2]), int(bb[1] - bb[0]), int(bb[3] - bb[2]))
    order = (("hio", 20), ("er", 5))
    avg, p, count, mine = solve_sharded(Md, Sd, 6, 25, order=order, beta=0.9, seed=11, box=box,
                                        N_prtf=128, upsample=32, ops=DeviceOps(Engine(e_per_n={})))
    torch.cuda.synchronize()
    assert count == 6 and mine == list(range(6))

    eng = Engine(e_per_n={})
    r0, c0, rows, cols = box
    psis = torch.zeros((6, 128, 128), dtype=torch.complex64, device="cuda")
    saves = torch.zeros((6, rows, cols), dtype=torch.complex64, device="cuda")
    eng.solve([TrialSpec(psi=psis[k], modulus=Md, support=Sd, iterations=25, order=order, beta=0.9,
                         random_phase=True, seed=11, trial=k, box=box, save=saves[k])
               for k in range(6)])
    al = align_frames_subpixel(align_global_phase(saves), upsample=32)
    want_avg = mean_frames(al).cpu().numpy()
    want_p = prtf(al, N=128).cpu().numpy()
    got_avg, got_p = avg.cpu().numpy(), p.cpu().numpy()
    assert np.linalg.norm(got_avg - want_avg) / np.linalg.norm(want_avg) < 1e-6
    assert np.max(np.abs(got_p - want_p)) < 1e-6
    eng.close()
