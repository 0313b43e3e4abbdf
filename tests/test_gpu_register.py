"""Subpixel registration (``sp_register_subpixel`` through the C ABI, via
``phasing.align_frames_subpixel``) against the reference's whole-pixel
alignment answers and the FP64 oracle.

* Whole-pixel shifts: the reference's own ``align_frames`` coordinates
  (golden vectors in the semantics of ``test/test_conditioning.py:34-52``)
  must come back exactly, as d = -coordinates, and the aligned frames must
  equal the reference frame (1e-5 relative).
* Fractional shifts on the 1/U grid and a global phase: recovered exactly
  (1e-9), aligned frames within 1e-5 relative of the FP64 oracle's.
* Crops that are not a power of two (the batched workload's 180 x 180 crops in
  a 256 x 256 transform), many frames: shifts equal to the oracle's, aligned
  frames within 1e-5 relative."""
import os

import numpy as np
import pytest

from oracle import phasing_oracle as O

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _object(n, box, seed):
    rng = np.random.default_rng(seed)
    ref = np.zeros((n, n), np.complex128)
    o = (n - box) // 2
    ref[o:o + box, o:o + box] = rng.random((box, box)) * np.exp(1j * rng.uniform(-1, 1, (box, box)))
    return ref


def test_whole_pixel_shifts_match_reference_align_frames():
    from als_speckle_b200.phasing import align_frames_subpixel
    h = np.load(os.path.join(G, "helpers.npz"))
    ref = h["af_ref"].astype(np.complex64)
    for k in range(3):
        rolled = h["af%d_rolled" % k].astype(np.complex64)
        want = np.asarray(h["af%d_coords" % k]).reshape(-1)  # the reference's roll amounts
        aligned, d = align_frames_subpixel(rolled[None], align_to=ref, upsample=20, return_type="both")
        assert np.array_equal(d[0, :2], -want.astype(np.float64))
        assert _rel(aligned[0], ref) < 1e-5


@pytest.mark.parametrize("U", [1, 16, 64])
def test_fractional_shifts_and_phase(U):
    from als_speckle_b200.phasing import align_frames_subpixel
    ref = _object(64, 24, 1)
    true = [(0.0, 0.0, 0.0), (3.0, -5.0, 0.3), (1.25, -2.5, -1.1), (-4.0 + 5 / 16, 0.5, 2.0)]
    frames = []
    for dy, dx, th in true:
        dy, dx = round(dy * U) / U, round(dx * U) / U
        frames.append(O.fourier_shift(ref, dy, dx) * np.exp(1j * th))
    frames = np.stack(frames).astype(np.complex64)
    aligned, d = align_frames_subpixel(frames, align_to=ref.astype(np.complex64), upsample=U,
                                       return_type="both")
    wd, wal = O.register_subpixel(frames.astype(np.complex128), ref.astype(np.complex64).astype(np.complex128),
                                  upsample=U)
    for k, (dy, dx, th) in enumerate(true):
        assert abs(d[k, 0] - round(dy * U) / U) < 1e-9 and abs(d[k, 1] - round(dx * U) / U) < 1e-9
        assert abs(np.angle(np.exp(1j * (d[k, 2] - th)))) < 1e-4
    assert np.array_equal(d[:, :2], wd[:, :2])
    assert _rel(aligned, wal) < 1e-5


def test_crops_in_larger_transform_many_frames():
    """180 x 180 crops (the batched workload's savebuffer) in 256 x 256."""
    from als_speckle_b200.phasing import align_frames_subpixel
    rng = np.random.default_rng(5)
    base = _object(180, 120, 7)
    frames = []
    for k in range(24):
        # shifts on the 1/64 grid: the noise moves the peak far less than
        # half a grid step, so FP32 and FP64 pick the same grid point
        dy, dx = rng.integers(-192, 193, 2) / 64.0
        f = O.fourier_shift(base, dy, dx, N=256) * np.exp(1j * rng.uniform(-np.pi, np.pi))
        frames.append(f + 0.01 * (rng.standard_normal(f.shape) + 1j * rng.standard_normal(f.shape)))
    frames = np.stack(frames).astype(np.complex64)
    aligned, d = align_frames_subpixel(frames, upsample=64, return_type="both")
    wd, wal = O.register_subpixel(frames.astype(np.complex128), frames[0].astype(np.complex128),
                                  N=256, upsample=64)
    assert np.array_equal(d[:, :2], wd[:, :2])
    assert np.max(np.abs(d[:, 2] - wd[:, 2])) < 1e-4
    assert _rel(aligned, wal) < 1e-5
    # aligned to frame 0: each frame now matches it up to the added noise
    # (1% per pixel on both frames) and the edge ripple of the band-limited shift
    for k in range(1, 24):
        assert _rel(aligned[k], aligned[0]) < 0.1


def test_device_tensors_in_place_shape():
    import torch
    from als_speckle_b200.phasing import align_frames_subpixel
    ref = _object(32, 12, 3).astype(np.complex64)
    t = torch.from_numpy(np.stack([ref, np.roll(ref, 2, 1)])).cuda()
    out = align_frames_subpixel(t)
    assert out.is_cuda and tuple(out.shape) == (2, 32, 32)
    assert _rel(out.cpu().numpy()[1], ref) < 1e-5
    c = align_frames_subpixel(t, return_type="coordinates")
    assert tuple(c.shape) == (2, 3) and float(c[1, 1]) == 2.0  # frame 1 = ref rolled by +2
