"""Trial-quality measures on the GPU: rftf against the reference's own numpy
output (golden vectors), remove_hot_pixels bit for bit, gpu_rftf and
covar_results against the oracle's restatements (their reference versions
need OpenCL, and covar_results cannot run in the reference at all).
Tolerances: RFTF values (in [0, 1]) to 1e-4 absolute, cross-correlation
maxima to 1e-5 relative, covariances to 1e-5 absolute."""
import os

import numpy as np
import pytest

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def qual():
    return np.load(os.path.join(G, "quality.npz"))


@pytest.mark.parametrize("N", [32, 64])
@pytest.mark.parametrize("case", ["plain", "centred", "ipsf_out", "scale", "hot"])
def test_rftf_vs_reference_golden(qual, N, case):
    from als_speckle_b200.phasing import rftf
    g, e, ip = qual["N%d_goal" % N], qual["N%d_est" % N], qual["N%d_ipsf" % N]
    kw = {"ipsf_out": {"ipsf": ip}, "scale": {"scale": True}, "hot": {"hot_pixels": True}}.get(case, {})
    goal = np.fft.fftshift(g) if case == "centred" else g
    out = rftf(e, goal, **kw)
    assert out.shape == (N, N)
    assert np.max(np.abs(out - qual["N%d_%s" % (N, case)])) < 1e-4


@pytest.mark.parametrize("N", [32, 64])
def test_remove_hot_pixels_vs_reference_golden(qual, N):
    from als_speckle_b200.phasing import remove_hot_pixels
    out = remove_hot_pixels(qual["N%d_hp_in" % N], iterations=2)
    assert np.array_equal(out, qual["N%d_hp_out" % N])


@pytest.mark.parametrize("with_ipsf", [False, True])
def test_gpu_rftf_vs_oracle(qual, with_ipsf):
    from als_speckle_b200.phasing import gpu_rftf
    g, e, ip = qual["N64_goal"], qual["N64_est"], qual["N64_ipsf"]
    rng = np.random.default_rng(4)
    ests = np.stack([e + 0.02 * (rng.standard_normal(e.shape) + 1j * rng.standard_normal(e.shape))
                     for _ in range(4)]).astype(np.complex64)
    out, q = gpu_rftf(None, ests, g, ipsf=ip if with_ipsf else None, rftfq=True)
    want = O.gpu_rftf(ests, g, ipsf=ip if with_ipsf else None)
    assert np.max(np.abs(out - want)) < 1e-4
    assert np.allclose(q, O.unwrap_average(want), atol=1e-4)


def test_covar_results_vs_oracle():
    from als_speckle_b200.phasing import covar_results
    rng = np.random.default_rng(5)
    obj = rng.random((40, 40)) * np.exp(1j * rng.random((40, 40)))
    data = np.zeros((6, 48, 48), np.complex64)
    for k in range(6):
        if k < 4:  # four copies of one object at different positions, with noise
            data[k, k:k + 40, 2 * k:2 * k + 40] = obj + 0.05 * rng.standard_normal((40, 40))
        else:
            data[k, :40, :40] = rng.random((40, 40))
    mask = np.ones((6, 6))
    mask[0, 5] = 0  # a pair left out
    cc, cov, stats, dft = covar_results(None, data, threshold=0.8, mask=mask)
    wcc, wcov, wstats, wdft = O.covar_results(data.astype(np.complex128), threshold=0.8, mask=mask)
    assert dft.shape == wdft.shape == (6, 128, 128)
    sel = wcc > 0
    assert np.array_equal(cc > 0, sel)
    assert np.max(np.abs(cc[sel] - wcc[sel]) / wcc[sel]) < 1e-5
    assert np.max(np.abs(cov - wcov)) < 1e-5
    assert np.array_equal(stats[:, 2], wstats[:, 2])
    assert np.allclose(stats[:, 1], wstats[:, 1], atol=1e-5)
