"""Longitudinally partially coherent projection (load(spectrum=...)) on the GPU.

The divisor is sqrt(radial_rescale(div^2)) (phasing.py:1139-1156,
kernels/phasing_radial_rescale.cl), after the ipsf blur when both are given.
The reference runs it only on OpenCL, so the checks are against the FP64
oracle's restatement of the kernel (itself pinned to a line-by-line
restatement); one projection to 1e-5 relative L2 norm (2e-5 with an ipsf as
well, see test_gpu_coherence.py), three iterations to 1e-4."""
import numpy as np
import pytest
import torch

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu

SPEC = np.array([np.linspace(0.95, 1.05, 7) * 778.0,
                 np.exp(-0.5 * np.linspace(-2, 2, 7) ** 2)])


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, complex) - b) / np.linalg.norm(b))


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def gaussian_ipsf(N, sigma):
    q = np.fft.fftfreq(N) * N
    g = np.exp(-0.5 * (q[:, None] ** 2 + q[None, :] ** 2) / sigma ** 2)
    return np.fft.fft2(g / g.sum()).astype(np.complex64)


@pytest.fixture(scope="module")
def engine():
    from als_speckle_b200.engine import Engine
    e = Engine(use_graph=False)
    yield e
    e.close()


def _case(N, seed=0):
    from als_speckle_b200 import synth
    _, M, S = synth.pattern(N, n_ellipses=6, box=N // 4, peak=1e6, seed=N + seed,
                            support_edge=N // 4 + N // 16)
    rng = np.random.default_rng(seed)
    psi0 = ((rng.random((N, N)) + 1j * rng.random((N, N))) * S).astype(np.complex64)
    return M, S, psi0


def _spectrum_dev(spec=SPEC):
    r, w = O.spectrum_rescales(spec)
    return dev(r), dev(w)


@pytest.mark.parametrize("N", [64, 256, 512])
@pytest.mark.parametrize("alg", ["hio", "dm"])
@pytest.mark.parametrize("with_ipsf", [False, True])
def test_spectrum_projection_vs_fp64_oracle(engine, N, alg, with_ipsf):
    from als_speckle_b200.engine import TrialSpec
    M, S, psi0 = _case(N)
    ipsf = gaussian_ipsf(N, 1.5) if with_ipsf else None
    want, _ = O.iteration(psi0, M, S, alg, 0.9, mode="f64", ipsf=ipsf, spectrum=SPEC)
    psi = dev(psi0)
    err = torch.zeros((1, 2), dtype=torch.float64, device="cuda")
    engine.solve([TrialSpec(psi=psi, modulus=dev(M), support=dev(S), iterations=1,
                            order=((alg, 1),), beta=0.9, errors=err, spectrum=_spectrum_dev(),
                            ipsf=dev(ipsf) if with_ipsf else None)])
    assert rel(psi.cpu().numpy(), want) < (2e-5 if with_ipsf else 1e-5)
    plain, _ = O.iteration(psi0, M, S, alg, 0.9, mode="f64", ipsf=ipsf)
    assert rel(plain, want) > 1e-3  # the spectrum changes the result


# 21 samples (more than the 16 the rescale kernel tabulates per pass), and
# factors from 0.4 to 2.5: taps far outside (-N/2, N/2) (weight 0, read at
# their coordinate modulo N) and strongly magnified ones.
SPEC_WIDE = np.array([np.concatenate([np.linspace(0.4, 0.9, 10), [1.0], np.linspace(1.1, 2.5, 10)]),
                      np.concatenate([np.linspace(0.1, 0.9, 10), [1.0], np.linspace(0.9, 0.1, 10)])])


@pytest.mark.parametrize("N", [256, 2048])
def test_spectrum_many_wide_samples_vs_fp64_oracle(engine, N):
    from als_speckle_b200.engine import TrialSpec
    M, S, psi0 = _case(N, seed=3)
    want, _ = O.iteration(psi0, M, S, "hio", 0.9, mode="f64", spectrum=SPEC_WIDE)
    psi = dev(psi0)
    engine.solve([TrialSpec(psi=psi, modulus=dev(M), support=dev(S), iterations=1,
                            order=(("hio", 1),), beta=0.9, spectrum=_spectrum_dev(SPEC_WIDE))])
    assert rel(psi.cpu().numpy(), want) < 1e-5


def test_spectrum_batch_equals_alone(engine):
    """Spectrum, ipsf and coherent trials together give the same bits as alone."""
    from als_speckle_b200.engine import TrialSpec
    cases = []
    for k, (N, alg, mode) in enumerate([(128, "hio", "spec"), (128, "raar", "both"),
                                        (256, "dm", "spec"), (128, "hio", None)]):
        M, S, _ = _case(N, seed=k)
        cases.append((N, alg, dev(M), dev(S), mode, k))

    def run(sel):
        out, specs = [], []
        for (N, alg, M, S, mode, k) in sel:
            psi = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
            err = torch.zeros((5, 2), dtype=torch.float64, device="cuda")
            specs.append(TrialSpec(psi=psi, modulus=M, support=S, iterations=5, order=((alg, 5),),
                                   beta=0.9, random_phase=True, seed=2, trial=k, errors=err,
                                   spectrum=_spectrum_dev() if mode else None,
                                   ipsf=dev(gaussian_ipsf(N, 1.2)) if mode == "both" else None))
            out.append((psi, err))
        engine.solve(specs)
        torch.cuda.synchronize()
        return [(p.cpu().numpy(), e.cpu().numpy()) for p, e in out]

    together = run(cases)
    for c, (p, e) in zip(cases, together):
        (pa, ea), = run([c])
        assert np.array_equal(pa, p)
        assert np.allclose(ea, e, rtol=1e-12, atol=0)


def test_phasing_class_with_spectrum():
    from als_speckle_b200.phasing import phasing
    N = 128
    M, S, psi0 = _case(N, seed=7)
    r = phasing()
    r.load(modulus=M, support=S, spectrum=SPEC, numtrials=1)
    assert r.spectrum_state == 2
    r.psi_in.copy_(torch.from_numpy(psi0))
    r.iterate(3, order=(("hio", 2), ("er", 1)), beta=0.9)
    want = O.iterate(psi0, M, S, 3, order=(("hio", 2), ("er", 1)), beta=0.9, mode="f64", spectrum=SPEC)
    assert rel(r.get(r.psi_in), want) < 1e-4
