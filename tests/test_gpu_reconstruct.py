"""``phasing.reconstruct`` (``phasing.py:932-988``): seed and iterate every
trial, align the global phases, average, refine the support.

The reference's method cannot run as written (it loops over the integer
``rounds`` and reads an undefined ``self.trials``), so its parity rests on its
parts, each pinned elsewhere: ``seed`` (numpy's global RNG), ``iterate``,
``align_global_phase``, the mean over the savebuffer's slots and
``refine_support``.  Here the composition is checked against the FP64 oracle
run step by step from the same seeds (a short run, before FP32 rounding is
amplified), and the support refinement against the module function applied
to the average."""
import numpy as np
import pytest

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu

N, TRIALS, ITERS = 64, 3, 12


def _inputs():
    from als_speckle_b200 import synth
    _, M, S = synth.pattern(N, n_ellipses=5, box=16, peak=1e5, seed=21, support_edge=22)
    return M, S


def test_reconstruct_equals_seed_iterate_align_mean():
    from als_speckle_b200.phasing import phasing
    M, S = _inputs()
    r = phasing()
    r.load(modulus=M, support=S, numtrials=TRIALS)
    np.random.seed(11)
    r.reconstruct(iterations=ITERS, rounds=1, refine_support=False)
    assert r.numtrial == TRIALS
    got = r.reconstruction
    assert got.shape == (r.rows, r.cols)

    np.random.seed(11)
    frames = np.zeros((TRIALS + 1, r.rows, r.cols), np.complex128)
    for k in range(TRIALS):
        start = O.seed_reference(N, S.astype(np.float32) / S.max())
        psi = O.iterate(start.astype(np.complex128), M, S / S.max(), ITERS, order=None, beta=0.8,
                        mode="f64")
        frames[k] = O.crop(psi, r.r0, r.c0, r.rows, r.cols)
    frames = O.align_global_phase(frames)
    want = frames.mean(axis=0)  # the last (empty) slot is part of the mean, as in the reference
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel < 1e-4, rel
    # psi_in holds the last trial's iterate
    assert np.allclose(r.get(r.psi_in)[r.r0:r.r0 + r.rows, r.c0:r.c0 + r.cols],
                       r.get(r.savebuffer)[TRIALS - 1])


def test_reconstruct_refines_and_reloads_the_support():
    from als_speckle_b200.phasing import phasing, refine_support
    M, S = _inputs()
    r = phasing()
    r.load(modulus=M, support=S, numtrials=TRIALS)
    crop = r._support_host[r.r0:r.r0 + r.rows, r.c0:r.c0 + r.cols].copy()
    np.random.seed(5)
    r.reconstruct(iterations=ITERS, rounds=1, refinement_parameters={"local_threshold": 0.1})
    refined, _ = refine_support(crop, r.reconstruction, blur=3, local_threshold=0.1,
                                global_threshold=0.0)
    want = np.zeros((N, N), np.float32)
    want[:refined.shape[0], :refined.shape[1]] = refined
    want /= want.max()
    assert np.array_equal(r.get(r.support), want)
    # the reload restarted the trial count and resized the savebuffer to the new box
    assert r.numtrial == 0
    assert tuple(r.savebuffer.shape) == (TRIALS + 1, r.rows, r.cols)
    # a second round runs on the refined support
    r.reconstruct(iterations=ITERS, rounds=1, refine_support=False)
    assert np.all(np.isfinite(r.reconstruction)) and np.abs(r.reconstruction).max() > 0


def test_reconstruct_rejects_bad_parameters():
    from als_speckle_b200.phasing import phasing
    M, S = _inputs()
    r = phasing()
    r.load(modulus=M, support=S, numtrials=2)
    with pytest.raises(TypeError):
        r.reconstruct(iterations=2, refinement_parameters=[("blur_sigma", 2)])
    r.numtrial = 2  # one free slot left for two trials
    with pytest.raises(IndexError):
        r.reconstruct(iterations=2, refine_support=False)
