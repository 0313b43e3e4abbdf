"""Edge cases of the engine on the GPU: the largest supported size, an
iterate whose transform is zero everywhere, an empty batch, and sizes the
engine rejects.  Oracle comparisons use the FP64 oracle at 1e-5 relative L2
norm (||a-b||/||b||), as the other projection tests do.
"""
import numpy as np
import pytest
import torch

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _inputs(N, seed):
    rng = np.random.default_rng(seed)
    B = N // 4
    obj = np.zeros((N, N), np.complex128)
    c = N // 2
    obj[c - B // 2:c + B // 2, c - B // 2:c + B // 2] = rng.random((B, B)) * np.exp(
        1j * rng.uniform(-0.7, 0.7, (B, B)))
    M = np.abs(np.fft.fft2(obj)).astype(np.float32)
    S = np.zeros((N, N), np.float32)
    s = B + N // 8
    S[c - s // 2:c + s // 2, c - s // 2:c + s // 2] = 1
    psi = ((rng.random((N, N)) + 1j * rng.random((N, N))) * S).astype(np.complex64)
    return psi, M, S


def _solve(psi, M, S, alg, beta, iters=1, **kw):
    from als_speckle_b200.engine import Engine, TrialSpec
    e = Engine(use_graph=False)
    try:
        p = torch.from_numpy(psi).cuda()
        e.solve([TrialSpec(psi=p, modulus=torch.from_numpy(M).cuda(), support=torch.from_numpy(S).cuda(),
                           iterations=iters, order=((alg, iters),), beta=beta, **kw)])
        return p.cpu().numpy()
    finally:
        e.close()


@pytest.mark.parametrize("alg", ["hio", "dm"])
def test_largest_size_projection_vs_fp64_oracle(alg):
    """N = 4096, the largest size the engine takes (2 GiB of FP64 oracle planes)."""
    N = 4096
    psi, M, S = _inputs(N, 11)
    got = _solve(psi, M, S, alg, 0.9)
    want, _ = O.iteration(psi, M, S, alg, 0.9, mode="f64")
    assert rel(got, want) < 1e-5


@pytest.mark.parametrize("alg", ["hio", "er", "raar", "dm"])
def test_zero_iterate_keeps_the_modulus_with_zero_phase(alg):
    """psi = 0: |F| = 0 at every pixel, where the reference divides by zero;
    the engine (and the oracle) replace F by the modulus with zero phase."""
    N = 256
    _, M, S = _inputs(N, 12)
    psi = np.zeros((N, N), np.complex64)
    got = _solve(psi, M, S, alg, 0.9)
    want, _ = O.iteration(psi, M, S, alg, 0.9, mode="f64")
    assert np.all(np.isfinite(got))
    assert rel(got, want) < 1e-5


def test_zero_modulus_pixels():
    """A modulus with zeros (a beamstop-like disc and a blank quadrant of
    frequencies) projects those frequencies to zero, as the oracle does."""
    N = 512
    psi, M, S = _inputs(N, 13)
    M = M.copy()
    M[:N // 2, N // 2:] = 0
    yy, xx = np.mgrid[:N, :N]
    M[(np.minimum(yy, N - yy) ** 2 + np.minimum(xx, N - xx) ** 2) < 36] = 0
    got = _solve(psi, M, S, "hio", 0.9)
    want, _ = O.iteration(psi, M, S, "hio", 0.9, mode="f64")
    assert rel(got, want) < 1e-5


def test_empty_batch_is_a_no_op():
    from als_speckle_b200.engine import Engine
    from als_speckle_b200 import _lib
    e = Engine(use_graph=False)
    try:
        e.solve([])
    finally:
        e.close()
    assert _lib.lib.sp_engine_run(None, 0, None, 0, None, None) == 0


@pytest.mark.parametrize("N", [4, 48, 8192])
def test_rejected_sizes(N):
    """Sizes that are not a power of two in [8, 4096] fail with an error
    before anything is launched."""
    from als_speckle_b200.engine import Engine, TrialSpec
    from als_speckle_b200._lib import SpeckleError
    e = Engine(use_graph=False)
    try:
        z = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
        m = torch.ones((N, N), dtype=torch.float32, device="cuda")
        with pytest.raises((SpeckleError, ValueError)):
            e.solve([TrialSpec(psi=z, modulus=m, support=m, iterations=1)])
    finally:
        e.close()
