"""Statistical parity over 32 seeds.

Projection iterations are chaotic, so long runs are compared by distribution:
32 seeded random-phase starts (identical starts on both sides) iterated on
the GPU and in the FP64 oracle — 100 HIO (beta 0.9) + 20 ER at N = 128, and
the plain 256^2 configuration (20 ellipses, 1e5 photons, 80^2 support,
200 HIO + 20 ER), and the benchmark's 512^2 configuration (40 ellipses,
1e6 photons, 160^2 support, 500 HIO + 50 ER).  The final R-factors must agree in mean to 1% and pass a
two-sample Kolmogorov-Smirnov test, and the annular PRTFs of the two sets of
reconstructions must agree to 0.05 per annulus.  The oracle's trials run in
a spawned process pool (the test process has already initialised CUDA).
"""
import multiprocessing as mp
import os

import numpy as np
import pytest
import torch

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu

N, SEEDS, ORDER, ITERS, BETA = 128, 32, (("hio", 100), ("er", 20)), 120, 0.9

CASES = {
    "small128": dict(N=128, pattern=dict(n_ellipses=10, box=32, peak=1e5, seed=3, support_edge=40),
                     order=(("hio", 100), ("er", 20))),
    "plain256": dict(N=256, pattern=dict(n_ellipses=20, box=64, peak=1e5, seed=0, support_edge=80),
                     order=(("hio", 200), ("er", 20))),
    "hio512": dict(N=512, pattern=dict(n_ellipses=40, box=128, peak=1e6, seed=0, support_edge=160),
                   order=(("hio", 500), ("er", 50))),
}


def _oracle_trial(args):
    """One FP64 oracle trial from the seeded random-phase start (pool worker)."""
    M, S, k, order, iters, box = args
    psi = O.seed_random_phase(M, S, 77, k)
    psi, e = O.iterate(psi, M, S, iters, order=order, beta=BETA, mode="f64", errors=True)
    return e[-1, 1], O.crop(psi, box[0], box[1], box[2], box[3])


def _annular(p):
    n = p.shape[0]
    y, x = np.indices(p.shape)
    r = np.floor(np.hypot(y - n // 2, x - n // 2)).astype(int)
    keep = r < n // 2
    return np.bincount(r[keep], weights=p[keep]) / np.maximum(np.bincount(r[keep]), 1)


@pytest.mark.parametrize("case", sorted(CASES))
def test_final_r_factor_and_prtf_distributions_match_oracle(case):
    from scipy.stats import ks_2samp
    from als_speckle_b200 import synth
    from als_speckle_b200.engine import Engine, TrialSpec
    from als_speckle_b200.masking import bounding_box
    c = CASES[case]
    n, order = c["N"], c["order"]
    iters = sum(k for _, k in order)
    _, M, S = synth.pattern(n, **c["pattern"])
    bb = bounding_box(S, pad=10)
    box = (int(bb[0]), int(bb[2]), int(bb[1] - bb[0]), int(bb[3] - bb[2]))
    m = M.astype(np.float64)

    # GPU
    Md, Sd = torch.from_numpy(M).cuda(), torch.from_numpy(S).cuda()
    psis = torch.zeros((SEEDS, n, n), dtype=torch.complex64, device="cuda")
    saves = torch.zeros((SEEDS, box[2], box[3]), dtype=torch.complex64, device="cuda")
    errs = torch.zeros((SEEDS, iters, 2), dtype=torch.float64, device="cuda")
    eng = Engine(use_graph=False)
    eng.solve([TrialSpec(psi=psis[k], modulus=Md, support=Sd, iterations=iters, order=order,
                         beta=BETA, random_phase=True, seed=77, trial=k, box=box, save=saves[k],
                         errors=errs[k]) for k in range(SEEDS)])
    torch.cuda.synchronize()
    r_gpu = errs[:, -1, 1].cpu().numpy() / np.sum(m)

    # FP64 oracle from the same starts, one trial per worker
    workers = max(1, min(16, len(os.sched_getaffinity(0))))
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(_oracle_trial, [(M, S, k, order, iters, box) for k in range(SEEDS)])
    r_ref = np.array([r for r, _ in res])
    crops = [cr for _, cr in res]

    assert abs(r_gpu.mean() - r_ref.mean()) / r_ref.mean() < 0.01
    assert ks_2samp(r_gpu, r_ref).pvalue > 0.01

    from als_speckle_b200.phasing import align_global_phase, prtf
    p_gpu = prtf(align_global_phase(saves), N=n).cpu().numpy()
    p_ref = O.prtf(O.align_global_phase(np.array(crops)), N=n)
    assert np.max(np.abs(_annular(p_gpu) - _annular(p_ref))) < 0.05
    eng.close()


def test_checkpoint_resume_is_bit_exact():
    """Stopping after k iterations and resuming from psi (the whole state)
    reproduces the uninterrupted run bit for bit."""
    from als_speckle_b200 import synth
    from als_speckle_b200.engine import Engine, TrialSpec
    from als_speckle_b200.serving import rotated_order
    from als_speckle_b200.engine import expand_runs
    _, M, S = synth.pattern(N, n_ellipses=10, box=32, peak=1e5, seed=4, support_edge=40)
    Md, Sd = torch.from_numpy(M).cuda(), torch.from_numpy(S).cuda()
    order = (("hio", 7), ("dm", 2), ("er", 1))
    eng = Engine(use_graph=False)
    a = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    eng.solve([TrialSpec(psi=a, modulus=Md, support=Sd, iterations=40, order=order, beta=0.9,
                         random_phase=True, seed=5, trial=1)])
    b = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    eng.solve([TrialSpec(psi=b, modulus=Md, support=Sd, iterations=13, order=order, beta=0.9,
                         random_phase=True, seed=5, trial=1)])
    saved = b.cpu().clone()  # the checkpoint: psi and the iteration count
    c = saved.cuda()
    algs, counts = expand_runs(order)
    flat = [x for x, n in zip(algs, counts) for _ in range(n)]
    eng.solve([TrialSpec(psi=c, modulus=Md, support=Sd, iterations=27,
                         order=rotated_order(flat, 13), beta=0.9)])
    torch.cuda.synchronize()
    assert torch.equal(a, c)
    eng.close()
