"""Partially coherent projection (load(ipsf=...)) on the GPU, through the C ABI.

The divisor sqrt(|IFFT2(FFT2(|F|^2) * ipsf)|) replaces |F| in the modulus
replacement (phasing.py:1109-1137).  Checked against the reference's own
numpy path (golden vectors made by tests/golden/make_golden.py), against the
FP64 oracle at larger sizes, over a short mixed trajectory, in a batch mixed
with coherent trials, and through the phasing class.  Tolerances as in
test_gpu_engine.py: one projection 1e-5 relative L2 norm, trajectories 1e-4;
against the FP64 oracle at large N, max(1e-5, twice the reference's own
single-precision error on the same input): the divisor transforms |F|^2,
whose dynamic range (~1e12 for a 1e6-photon pattern) makes the reference's
complex64 arithmetic itself deviate by ~2e-5 at 2048^2.
"""
import os

import numpy as np
import pytest
import torch

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


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


@pytest.fixture(scope="module")
def coh():
    return np.load(os.path.join(G, "coherence.npz"))


def _spec(psi, M, S, iters, order, beta, **kw):
    from als_speckle_b200.engine import TrialSpec
    return TrialSpec(psi=psi, modulus=M, support=S, iterations=iters, order=order, beta=beta, **kw)


@pytest.mark.parametrize("N", [32, 64])
@pytest.mark.parametrize("alg", ["hio", "er", "raar", "sf", "dm"])
def test_coherent_projection_vs_reference_golden(engine, coh, N, alg):
    psi = dev(coh["N%d_psi" % N])
    M, S, ip = (dev(coh["N%d_%s" % (N, k)]) for k in ("modulus", "support", "ipsf"))
    beta = float(coh["N%d_%s_beta" % (N, alg)])
    engine.solve([_spec(psi, M, S, 1, ((alg, 1),), beta, quirks="cpu", ipsf=ip)])
    assert rel(psi.cpu().numpy(), coh["N%d_%s_psi_in" % (N, alg)]) < 1e-5


def test_coherent_trajectory_vs_reference_golden(engine, coh):
    psi = dev(coh["traj_psi0"])
    M, S, ip = (dev(coh["traj_%s" % k]) for k in ("modulus", "support", "ipsf"))
    engine.solve([_spec(psi, M, S, 8, (("hio", 3), ("dm", 2), ("er", 1)), 0.9, quirks="cpu", ipsf=ip)])
    assert rel(psi.cpu().numpy(), coh["traj_psi_in"]) < 1e-4


@pytest.mark.parametrize("N", [128, 512, 2048])
@pytest.mark.parametrize("alg", ["hio", "raar", "dm"])
def test_coherent_projection_vs_fp64_oracle(engine, N, alg):
    """One partially coherent iteration against the FP64 oracle, with the
    FP64 error sums (of |F| against M, before the projection)."""
    from als_speckle_b200 import synth
    _, M, S = synth.pattern(N, n_ellipses=6, box=N // 4, peak=1e6, seed=N, support_edge=N // 4 + N // 16)
    rng = np.random.default_rng(2)
    psi0 = ((rng.random((N, N)) + 1j * rng.random((N, N))) * S).astype(np.complex64)
    ipsf = gaussian_ipsf(N, 2.0)
    beta = 0.87 if alg == "raar" else 0.9
    want, _ = O.iteration(psi0, M, S, alg, beta, mode="f64", ipsf=ipsf)
    ref32, _ = O.iteration(psi0, M, S, alg, beta, mode="ref64", ipsf=ipsf)
    tol = max(1e-5, 2 * rel(ref32, want))
    psi = dev(psi0)
    err = torch.zeros((1, 2), dtype=torch.float64, device="cuda")
    engine.solve([_spec(psi, dev(M), dev(S), 1, ((alg, 1),), beta, ipsf=dev(ipsf), errors=err)])
    assert rel(psi.cpu().numpy(), want) < tol
    f = np.abs(np.fft.fft2(psi0.astype(np.complex128)))
    e2 = np.sum((f - M) ** 2)
    assert abs(err[0, 0].item() - e2) / e2 < 1e-5


def test_mixed_batch_equals_alone(engine):
    """Coherent and partially coherent trials of two sizes in one call give
    the same bits as each alone, random-phase starts and error sums included."""
    from als_speckle_b200 import synth
    cases = []
    for k, (N, alg, pc) in enumerate([(128, "hio", True), (128, "hio", False), (256, "dm", True),
                                      (256, "raar", False), (128, "er", True)]):
        _, M, S = synth.pattern(N, n_ellipses=5, box=N // 4, peak=1e6, seed=10 + k, support_edge=N // 4 + 8)
        cases.append((N, alg, dev(M), dev(S), dev(gaussian_ipsf(N, 1.5)) if pc else None, k))

    def run(sel):
        out = []
        specs = []
        for (N, alg, M, S, ip, k) in sel:
            psi = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
            err = torch.zeros((6, 2), dtype=torch.float64, device="cuda")
            specs.append(_spec(psi, M, S, 6, ((alg, 4), ("er", 2)), 0.9, random_phase=True, seed=3,
                               trial=k, ipsf=ip, errors=err))
            out.append((psi, err))
        engine.solve(specs)
        torch.cuda.synchronize()
        return [(p.cpu().numpy(), e.cpu().numpy()) for p, e in out]

    together = run(cases)
    for c, (p, e) in zip(cases, together):
        (pa, ea), = run([c])
        assert np.array_equal(pa, p)
        assert np.allclose(ea, e, rtol=1e-12, atol=0)


def test_phasing_class_with_ipsf(coh):
    """load(ipsf=...) then iterate, as a user of the reference would."""
    from als_speckle_b200.phasing import phasing
    N = 64
    psi0 = coh["N%d_psi" % N]
    M, S, ip = (coh["N%d_%s" % (N, k)] for k in ("modulus", "support", "ipsf"))
    r = phasing()
    r.load(modulus=M, support=S, ipsf=ip, numtrials=1)
    assert r.ipsf_state == 2
    r.psi_in.copy_(torch.from_numpy(psi0))
    r.iterate(3, order=(("hio", 2), ("raar", 1)), beta=0.9)
    want = O.iterate(psi0, M, S, 3, order=(("hio", 2), ("raar", 1)), beta=0.9, mode="f64", ipsf=ip)
    assert rel(r.get(r.psi_in), want) < 1e-4


# ------------------------------------------------ optimize_coherence
@pytest.fixture(scope="module")
def copt():
    return np.load(os.path.join(G, "coherence_opt.npz"))


def test_optimize_coherence_rl_vs_reference_golden(copt):
    """Richardson-Lucy on one frame: the reference's numpy branch keeps the
    real part of the (complex) estimate; compare that part to 1e-4."""
    from als_speckle_b200.phasing import phasing
    r = phasing()
    out = r.optimize_coherence(copt["est1"], modulus=copt["modulus"], load=False, silent=True,
                               iterations=int(copt["rl_iterations"]))
    want = copt["rl_ipsf"]
    assert np.linalg.norm(out.real - want) / np.linalg.norm(want) < 1e-4


def test_optimize_coherence_rl_frames_are_independent(copt):
    """Batched over frames, the result (the last frame's estimate) equals the
    last frame run alone, and loading it sets the ipsf."""
    from als_speckle_b200.phasing import phasing
    r = phasing()
    M = copt["modulus"]
    both = r.optimize_coherence(copt["est2"], modulus=M, load=True, silent=True, iterations=5)
    assert r.ipsf_state == 1  # no modulus loaded yet: waiting for it
    alone = r.optimize_coherence(copt["est2"][1:], modulus=M, load=False, silent=True, iterations=5)
    assert np.array_equal(both, alone)
    assert abs(abs(np.fft.ifftshift(both)[0, 0]) - 1) < 1e-6  # divided by its magnitude there


def test_optimize_coherence_gaussian_vs_reference_golden(copt):
    """Gaussian fit: lengths agree with the reference's to the optimiser's
    own tolerance (xtol 0.1); the objective runs on the device."""
    from als_speckle_b200.phasing import phasing
    r = phasing()
    out = r.optimize_coherence(copt["est2"], modulus=copt["modulus"], load=False, silent=True,
                               method="gaussian")
    assert out.shape == (2, 2)
    assert np.max(np.abs(out - copt["gaussian_lengths"])) < 0.15
