"""Seeded inputs shared by the fixture generator and the tests.

``projection_inputs(N, seed)`` builds a fixed iterate, modulus and support:
a random complex object in a centred B x B box (B = N/4), the modulus of its
transform, a centred square support slightly larger than the box, and a
random start U[0,1) + i U[0,1) inside the support.  The large-N golden
fixture stores reference outputs for these inputs (sampled at fixed pixels)
instead of the inputs themselves, so the tests rebuild them here; the fixture
also stores FP64 sums of the inputs so that a change in numpy's generator or
FFT shows up as a failed input check rather than a silent mismatch.
"""
import numpy as np


def projection_inputs(N, seed):
    rng = np.random.default_rng(seed)
    B = max(2, N // 4)
    obj = np.zeros((N, N), np.complex128)
    c = N // 2
    box = rng.random((B, B)) * np.exp(1j * rng.uniform(-0.7, 0.7, (B, B)))
    obj[c - B // 2:c - B // 2 + B, c - B // 2:c - B // 2 + B] = box
    modulus = np.abs(np.fft.fft2(obj)).astype(np.float32)
    support = np.zeros((N, N), np.float32)
    S = min(N, B + max(2, N // 8))
    support[c - S // 2:c - S // 2 + S, c - S // 2:c - S // 2 + S] = 1
    psi = (rng.random((N, N)) + 1j * rng.random((N, N))).astype(np.complex64) * support
    return psi.astype(np.complex64), modulus, support


def input_sums(psi, modulus, support):
    """FP64 fingerprints of the inputs: sum |psi|^2, sum M, sum S."""
    return np.array([np.sum(np.abs(psi.astype(np.complex128)) ** 2),
                     np.sum(modulus.astype(np.float64)), np.sum(support.astype(np.float64))])


def prtf_estimates(N, frames, seed):
    """``frames`` N x N reconstructions of one object (a random complex box
    of edge N/4 at the centre) with independent noise and phase offsets, as a
    set of aligned trials looks: the PRTF input of the unwrap fixtures."""
    rng = np.random.default_rng(seed)
    B = max(2, N // 4)
    c = N // 2
    obj = rng.random((B, B)) * np.exp(1j * rng.uniform(-0.6, 0.6, (B, B)))
    out = np.zeros((frames, N, N), np.complex64)
    for f in range(frames):
        noisy = obj + 0.15 * (rng.standard_normal((B, B)) + 1j * rng.standard_normal((B, B)))
        out[f, c - B // 2:c - B // 2 + B, c - B // 2:c - B // 2 + B] = noisy * np.exp(1j * rng.uniform(-0.2, 0.2))
    return out


def smooth_map(N, seed):
    """A smooth float32 N x N map (a few Gaussian bumps and a radial falloff
    plus mild noise) with structure at every radius: the input of the
    large-N unwrap fixture."""
    rng = np.random.default_rng(seed)
    y, x = np.indices((N, N)).astype(np.float64)
    r = np.hypot(y - N // 2, x - N // 2)
    m = np.exp(-r / (0.35 * N))
    for _ in range(6):
        cy, cx = rng.uniform(0.1 * N, 0.9 * N, 2)
        s = rng.uniform(0.02, 0.08) * N
        m += rng.uniform(0.2, 0.8) * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * s * s))
    m += 0.02 * rng.random((N, N))
    return m.astype(np.float32)
