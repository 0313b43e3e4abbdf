"""Post-processing on the GPU against the reference's own outputs and the
FP64 oracle: the polar unwrap behind ``prtfq`` / ``rftfq`` (golden vectors
made by running the reference), the average of aligned frames against an
FP64 numpy mean, and the device PRTF at the benchmark's size (512^2, 32
frames) against the oracle.

Tolerances: unwrapped samples and their row means 1e-5 relative (float32
outputs of an FP64 interpolation, the reference rounds each sample to float32
as well); PRTF values (in [0, 1]) 2e-5 absolute; the mean of frames 1e-6
relative L2 against FP64."""
import os
import sys

import numpy as np
import pytest

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, G)
import golden_inputs  # noqa: E402


@pytest.fixture(scope="module")
def unw():
    return np.load(os.path.join(G, "unwrap.npz"))


def _rel(a, b):
    a, b = np.asarray(a, np.complex128), np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_unwrap_512_matches_reference(unw):
    """sp_unwrap through the C ABI on the reference's 512^2 unwrap case."""
    import torch
    from als_speckle_b200._lib import call, ptr, stream_ptr
    m = golden_inputs.smooth_map(512, 77)
    rows, cols = (int(x) for x in unw["map512_shape"])
    a = torch.from_numpy(m).cuda()
    work = torch.empty((512, 512), dtype=torch.float64, device="cuda")
    uw = torch.empty((rows, cols), dtype=torch.float32, device="cuda")
    mean = torch.empty(rows, dtype=torch.float32, device="cuda")
    call("sp_unwrap", ptr(a), 512, 0, 256, 256.0, 256.0, 0, ptr(work), ptr(uw), ptr(mean),
         stream_ptr())
    got = uw.cpu().numpy().ravel()[unw["map512_idx"]]
    assert np.allclose(got, unw["map512_samples"], rtol=1e-5, atol=1e-7)
    assert np.allclose(mean.cpu().numpy(), unw["map512_mean"], rtol=1e-5, atol=1e-7)


def test_unwrap_rejects_grid_outside_map():
    import torch
    from als_speckle_b200._lib import SpeckleError, call, ptr, stream_ptr
    a = torch.zeros((64, 64), dtype=torch.float32, device="cuda")
    work = torch.empty((64, 64), dtype=torch.float64, device="cuda")
    mean = torch.empty(40, dtype=torch.float32, device="cuda")
    with pytest.raises(SpeckleError):
        call("sp_unwrap", ptr(a), 64, 0, 40, 32.0, 32.0, 0, ptr(work), None, ptr(mean), stream_ptr())


@pytest.mark.parametrize("N", [32, 64])
def test_prtfq_matches_reference(unw, N):
    from als_speckle_b200.phasing import prtf
    arr, q = prtf(unw["prtf%d_in" % N], prtfq=True)
    assert np.max(np.abs(arr - unw["prtf%d_array" % N])) < 2e-5
    assert np.allclose(q, unw["prtf%d_q" % N], rtol=1e-5, atol=2e-6)


@pytest.mark.parametrize("N", [32, 64])
@pytest.mark.parametrize("case", ["plain", "scale"])
def test_rftfq_matches_reference(unw, N, case):
    from als_speckle_b200.phasing import rftf
    qual = np.load(os.path.join(G, "quality.npz"))
    arr, q = rftf(qual["N%d_est" % N], qual["N%d_goal" % N], rftfq=True, scale=(case == "scale"))
    assert np.allclose(q, unw["rftf%d_%s_q" % (N, case)], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("shape", [(1, 7, 9), (5, 20, 24), (128, 180, 180)])
def test_mean_frames_vs_numpy_fp64(shape):
    """sp_mean_frames against numpy's FP64 mean of the same frames."""
    import torch
    from als_speckle_b200.phasing import mean_frames
    rng = np.random.default_rng(sum(shape))
    f = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    got = mean_frames(torch.from_numpy(f).cuda()).cpu().numpy()
    want = f.astype(np.complex128).mean(axis=0)
    assert got.shape == want.shape
    assert _rel(got, want) < 1e-6


def test_prtf_512_32_frames_vs_oracle():
    """The device PRTF at the benchmark's size against the FP64 oracle, and
    its polar average against the oracle's unwrap of the same map."""
    import torch
    from als_speckle_b200.phasing import prtf
    est = golden_inputs.prtf_estimates(512, 32, 9)
    arr, q = prtf(torch.from_numpy(est).cuda(), prtfq=True)
    want = O.prtf(est.astype(np.complex128))
    assert np.max(np.abs(arr.cpu().numpy() - want)) < 2e-5
    want_q = O.unwrap_average(arr.cpu().numpy())
    assert np.allclose(q.cpu().numpy(), want_q, rtol=1e-5, atol=1e-6)


def test_unwrap_general_grid_vs_oracle():
    """sp_unwrap on an inner radius, an off-centre centre and an explicit
    column count against the oracle's restatement of wrapping.unwrap (which
    makes scipy's map_coordinates call)."""
    import torch
    from als_speckle_b200._lib import call, ptr, stream_ptr
    m = golden_inputs.smooth_map(128, 5)
    r_in, r_out, cy, cx, cols = 5, 40, 60.0, 70.0, 150
    a = torch.from_numpy(m).cuda()
    work = torch.empty((128, 128), dtype=torch.float64, device="cuda")
    uw = torch.empty((r_out - r_in, cols), dtype=torch.float32, device="cuda")
    mean = torch.empty(r_out - r_in, dtype=torch.float32, device="cuda")
    call("sp_unwrap", ptr(a), 128, r_in, r_out, cy, cx, cols, ptr(work), ptr(uw), ptr(mean),
         stream_ptr())
    want = O.unwrap(m, r_in, r_out, (cy, cx), columns=cols)
    assert np.allclose(uw.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
    assert np.allclose(mean.cpu().numpy(), want.mean(axis=1), rtol=1e-5, atol=1e-6)
