"""Size-independent properties of the engine on the benchmark's full
configuration: 128 random-phase trials of the 512^2 pattern (40 ellipses in a
128^2 box, 1e6 photons, Poisson, 160^2 support), checked on every trial.

* Error reduction does not increase the Fourier-domain error: with
  E_k = sum(|FFT(psi_k)| - M)^2 taken before projection k, each ER step from
  an iterate that satisfies the support gives E_{k+1} <= E_k (Fienup, "Phase
  retrieval algorithms: a comparison", Appl. Opt. 21, 2758 (1982):
  E_F(k+1) <= E_O(k) <= E_F(k)); in FP32 the sums may rise by rounding near
  convergence, so a relative 1e-5 is allowed.
* After an ER step psi is exactly zero outside the support (the update is
  psi = S * psi_out with S in {0, 1}), and the savebuffer crop equals psi's.
* Every trial of the 128-trial call equals the same trial run alone, bit for
  bit (psi and crop), so batching changes nothing at this size either.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRIALS, HIO, ER = 128, 30, 20


@pytest.fixture(scope="module")
def job():
    import torch
    from als_speckle_b200 import synth
    from als_speckle_b200.engine import Engine, TrialSpec
    from als_speckle_b200.masking import bounding_box
    _, M, S = synth.config_pattern("hio_512x128", seed=0)
    N = M.shape[0]
    assert N == 512
    bb = bounding_box(S, pad=10)
    box = (int(bb[0]), int(bb[2]), int(bb[1] - bb[0]), int(bb[3] - bb[2]))
    Md, Sd = torch.from_numpy(M).cuda(), torch.from_numpy(S).cuda()
    eng = Engine(use_graph=True)

    def run(ks):
        psi = torch.zeros((len(ks), N, N), dtype=torch.complex64, device="cuda")
        save = torch.zeros((len(ks), box[2], box[3]), dtype=torch.complex64, device="cuda")
        err = torch.zeros((len(ks), HIO + ER, 2), dtype=torch.float64, device="cuda")
        eng.solve([TrialSpec(psi=psi[j], modulus=Md, support=Sd, iterations=HIO + ER,
                             order=(("hio", HIO), ("er", ER)), beta=0.9, random_phase=True,
                             seed=31, trial=k, box=box, save=save[j], errors=err[j])
                   for j, k in enumerate(ks)])
        torch.cuda.synchronize()
        return psi.cpu().numpy(), save.cpu().numpy(), err.cpu().numpy()

    psi, save, err = run(list(range(TRIALS)))
    yield dict(M=M, S=S, box=box, psi=psi, save=save, err=err, run=run)
    eng.close()


def test_er_does_not_increase_the_fourier_error(job):
    e = job["err"][:, :, 0]
    assert np.all(np.isfinite(e)) and np.all(e > 0)
    # from the second ER projection on, the iterate satisfies the support
    # (the first starts from the last HIO update, which need not)
    er = e[:, HIO + 1:]
    rise = er[:, 1:] / er[:, :-1] - 1.0
    assert rise.max() < 1e-5, (rise.max(), np.unravel_index(rise.argmax(), rise.shape))


def test_er_leaves_nothing_outside_the_support_and_the_crop_is_psi(job):
    S, psi, save = job["S"], job["psi"], job["save"]
    outside = S == 0
    assert outside.sum() > 0
    assert np.count_nonzero(psi[:, outside]) == 0
    r0, c0, rows, cols = job["box"]
    assert np.array_equal(save, psi[:, r0:r0 + rows, c0:c0 + cols])


def test_every_trial_equals_itself_alone(job):
    for k in (0, 1, 63, 127):
        p, s, e = job["run"]([k])
        assert np.array_equal(p[0], job["psi"][k]), k
        assert np.array_equal(s[0], job["save"][k]), k
        assert np.allclose(e[0], job["err"][k], rtol=1e-12, atol=0), k
