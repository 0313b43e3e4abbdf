"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's numpy phasing path (dhparks/als_speckle, Python 2 source
loaded unmodified through ``refshim``) on fixed, seeded inputs and stores
inputs and outputs as ``.npz`` files.  Run it from the repository root in a
container that has the reference checkout:

    python tests/golden/make_golden.py <reference_root> [fixture ...]

The tests read only the ``.npz`` files; they never need the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
if len(sys.argv) > 1:
    os.environ["SPECKLE_REF_ROOT"] = sys.argv[1]
import golden_inputs as inputs  # noqa: E402
from oracle import refshim  # noqa: E402

ref = refshim.load_reference()


def _quiet(fn, *a, **k):
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def _inputs(N, seed):
    return inputs.projection_inputs(N, seed)


def projections():
    """One reference iteration of each algorithm from a fixed state."""
    out = {}
    for N in (8, 32, 64):
        psi, modulus, support = _inputs(N, 100 + N)
        out["N%d_psi" % N] = psi
        out["N%d_modulus" % N] = modulus
        out["N%d_support" % N] = support
        for alg in ("hio", "er", "raar", "sf", "dm"):
            beta = 0.9 if alg != "raar" else 0.87
            r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
            _quiet(r.load, modulus=modulus, support=support, numtrials=1)
            r.psi_in = psi.copy()
            _quiet(r.iterate, 1, order=((alg, 1),), beta=beta)
            out["N%d_%s_psi_in" % (N, alg)] = np.asarray(r.psi_in)
            out["N%d_%s_psi_out" % (N, alg)] = np.asarray(r.psi_out)
            out["N%d_%s_beta" % (N, alg)] = np.float64(beta)
            out["N%d_%s_savebuffer" % (N, alg)] = np.asarray(r.savebuffer)
            out["N%d_%s_box" % (N, alg)] = np.array([r.r0, r.rows, r.c0, r.cols])
    np.savez_compressed(os.path.join(HERE, "projections.npz"), **out)


def projections_large(samples=4096):
    """One reference iteration of each algorithm at 256^2 and 512^2.  The
    inputs are rebuilt by the tests from ``inputs.projection_inputs``; the
    outputs are stored at ``samples`` fixed pixels (the same for every
    algorithm) plus FP64 whole-plane sums, which keeps the fixture small."""
    out = {}
    for N in (256, 512):
        seed = 100 + N
        psi, modulus, support = _inputs(N, seed)
        out["N%d_seed" % N] = np.int64(seed)
        out["N%d_input_sums" % N] = inputs.input_sums(psi, modulus, support)
        idx = np.random.default_rng(7 + N).choice(N * N, samples, replace=False)
        # half of the samples inside the support, where the update keeps the projection
        inside = np.flatnonzero(support.ravel() > 0)
        idx[: samples // 2] = np.random.default_rng(8 + N).choice(inside, samples // 2, replace=False)
        out["N%d_idx" % N] = idx.astype(np.int64)
        for alg in ("hio", "er", "raar", "sf", "dm"):
            beta = 0.9 if alg != "raar" else 0.87
            r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
            _quiet(r.load, modulus=modulus, support=support, numtrials=1)
            r.psi_in = psi.copy()
            _quiet(r.iterate, 1, order=((alg, 1),), beta=beta)
            res = np.asarray(r.psi_in).astype(np.complex128)
            out["N%d_%s_beta" % (N, alg)] = np.float64(beta)
            out["N%d_%s_samples" % (N, alg)] = res.ravel()[idx].astype(np.complex64)
            out["N%d_%s_sums" % (N, alg)] = np.array(
                [np.sum(np.abs(res) ** 2), np.sum(res).real, np.sum(res).imag])
    np.savez_compressed(os.path.join(HERE, "projections_large.npz"), **out)


def trajectories():
    """Short multi-iteration runs of the reference (default order, beta 0.8,
    and a RAAR/DM schedule) from a seeded start."""
    out = {}
    N = 32
    psi, modulus, support = _inputs(N, 7)
    out["modulus"], out["support"], out["psi0"] = modulus, support, psi
    for name, order, beta, iters in (("default", None, 0.8, 12),
                                     ("hio_er", (("hio", 8), ("er", 2)), 0.9, 10),
                                     ("raar_dm", (("raar", 3), ("dm", 2)), 0.87, 10)):
        r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
        _quiet(r.load, modulus=modulus, support=support, numtrials=2)
        r.psi_in = psi.copy()
        _quiet(r.iterate, iters, order=order, beta=beta)
        out[name + "_final"] = np.asarray(r.psi_in)
        out[name + "_iters"] = np.int64(iters)
        out[name + "_beta"] = np.float64(beta)
    np.savez_compressed(os.path.join(HERE, "trajectories.npz"), **out)


def seeds():
    """``phasing.seed(val)`` output for a fixed val."""
    N = 16
    _, modulus, support = _inputs(N, 3)
    r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
    _quiet(r.load, modulus=modulus, support=support, numtrials=1)
    r.seed(1234)
    np.savez_compressed(os.path.join(HERE, "seed.npz"), support=support,
                        val=np.int64(1234), psi=np.asarray(r.psi_in))


def helpers():
    """bounding_box, refine_support, align_global_phase, prtf, align_frames,
    center_of_mass_average on fixed inputs."""
    out = {}
    rng = np.random.default_rng(11)
    # bounding boxes (including the test_mask.py known answer)
    box = np.zeros((256, 256))
    box[18:90, 45:63] = 1
    cases = [(box, 0, False), (box, 14, False), (box, 10, False), (box, 4, True)]
    blob = np.zeros((64, 64)); blob[3:20, 50:63] = 1
    cases += [(blob, 10, False), (blob, 4, True), (blob, 0, True)]
    for i, (d, pad, sq) in enumerate(cases):
        out["bb%d_data" % i] = d.astype(np.float32)
        out["bb%d_pad" % i] = np.int64(pad)
        out["bb%d_square" % i] = np.int64(sq)
        out["bb%d_box" % i] = ref.masking.bounding_box(d, pad=pad, force_to_square=sq)
    # refine_support: two-part support, random magnitudes
    N = 48
    sup = np.zeros((N, N)); sup[6:20, 8:22] = 1; sup[28:44, 26:40] = 1
    avg = (rng.random((N, N)) * sup + 0.05 * rng.random((N, N))) * np.exp(1j * rng.random((N, N)))
    for j, (blur, lt, gt) in enumerate(((3, 0.2, 0.0), (1.5, 0.15, 0.05), (0.7, 0.3, 0.0))):
        refined, blurred = _quiet(ref.phasing.refine_support, sup.copy(), avg, blur=blur,
                                  local_threshold=lt, global_threshold=gt)
        out["rs%d_support" % j] = sup
        out["rs%d_avg" % j] = avg
        out["rs%d_params" % j] = np.array([blur, lt, gt])
        out["rs%d_refined" % j] = refined
        out["rs%d_blurred" % j] = blurred
    # align_global_phase on frames with random global phases
    frames = (rng.random((5, 20, 24)) + 0.2j * rng.random((5, 20, 24)))
    frames *= np.exp(1j * rng.uniform(0, 2 * np.pi, (5, 1, 1)))
    frames = frames.astype(np.complex64)
    out["agp_in"] = frames
    out["agp_out"] = _quiet(ref.phasing.align_global_phase, frames)
    # prtf
    est = (rng.random((6, 12, 12)) * np.exp(1j * rng.normal(0, 0.3, (6, 12, 12)))).astype(np.complex64)
    out["prtf_in"] = est
    # prtf(N > rows) raises a broadcast error in the reference (phasing.py:1446-1448)
    out["prtf_N12"] = _quiet(ref.phasing.prtf, est)
    # align_frames (integer rolls), conditioning.py:316-430
    data = rng.random((32, 32))
    for k, (ry, rx) in enumerate(((3, 5), (0, 11), (15, 2))):
        rolled = np.roll(np.roll(data, rx, axis=1), ry, axis=0)
        out["af%d_rolled" % k] = rolled
        out["af%d_coords" % k] = ref.conditioning.align_frames(rolled, data, return_type="coordinates")
    out["af_ref"] = data
    # center_of_mass_average
    imgs = np.zeros((3, 24, 24), np.complex64)
    for k, (dr, dc) in enumerate(((0, 0), (2, -3), (-4, 1))):
        imgs[k, 8 + dr:14 + dr, 9 + dc:15 + dc] = (1 + k) * (1 + 0.5j)
    out["com_in"] = imgs.copy()
    out["com_out"] = ref.phasing.center_of_mass_average(imgs.copy())
    np.savez_compressed(os.path.join(HERE, "helpers.npz"), **out)


def gaussian_ipsf(N, sigma):
    """Transform of a normalised Gaussian point spread (sigma in pixels,
    centred on pixel 0 with wrap-around): the ``ipsf`` that ``load`` takes."""
    q = np.fft.fftfreq(N) * N
    g = np.exp(-0.5 * (q[:, None] ** 2 + q[None, :] ** 2) / sigma ** 2)
    g /= g.sum()
    return np.fft.fft2(g).astype(np.complex64)


def coherence():
    """Partially coherent projections: one reference iteration of each
    algorithm with ``load(ipsf=...)``, and a short trajectory."""
    out = {}
    for N in (32, 64):
        psi, modulus, support = _inputs(N, 300 + N)
        ipsf = gaussian_ipsf(N, 1.5)
        out["N%d_psi" % N] = psi
        out["N%d_modulus" % N] = modulus
        out["N%d_support" % N] = support
        out["N%d_ipsf" % N] = ipsf
        for alg in ("hio", "er", "raar", "sf", "dm"):
            beta = 0.9 if alg != "raar" else 0.87
            r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
            _quiet(r.load, modulus=modulus, support=support, ipsf=ipsf, numtrials=1)
            r.psi_in = psi.copy()
            _quiet(r.iterate, 1, order=((alg, 1),), beta=beta)
            out["N%d_%s_psi_in" % (N, alg)] = np.asarray(r.psi_in)
            out["N%d_%s_beta" % (N, alg)] = np.float64(beta)
    N = 32
    psi, modulus, support = _inputs(N, 7)
    ipsf = gaussian_ipsf(N, 1.0)
    r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
    _quiet(r.load, modulus=modulus, support=support, ipsf=ipsf, numtrials=1)
    r.psi_in = psi.copy()
    _quiet(r.iterate, 8, order=(("hio", 3), ("dm", 2), ("er", 1)), beta=0.9)
    out["traj_psi0"], out["traj_modulus"], out["traj_support"] = psi, modulus, support
    out["traj_ipsf"] = ipsf
    out["traj_psi_in"] = np.asarray(r.psi_in)
    np.savez_compressed(os.path.join(HERE, "coherence.npz"), **out)


def quality():
    """rftf (phasing.py:1521-1608) and remove_hot_pixels
    (conditioning.py:207-313) of the reference's numpy path."""
    out = {}
    for N in (32, 64):
        rng = np.random.default_rng(500 + N)
        B = N // 4
        obj = np.zeros((N, N), np.complex128)
        obj[:B, :B] = rng.random((B, B)) * np.exp(1j * rng.uniform(-0.5, 0.5, (B, B)))
        goal = (np.abs(np.fft.fft2(obj)) + 0.05).astype(np.float32)
        est = (obj[:B, :B] + 0.05 * rng.standard_normal((B, B))).astype(np.complex64)
        ipsf = gaussian_ipsf(N, 1.5)
        out["N%d_goal" % N], out["N%d_est" % N], out["N%d_ipsf" % N] = goal, est, ipsf
        out["N%d_plain" % N] = ref.phasing.rftf(est, goal)
        out["N%d_centred" % N] = ref.phasing.rftf(est, np.fft.fftshift(goal))
        out["N%d_ipsf_out" % N] = ref.phasing.rftf(est, goal, ipsf=ipsf)
        out["N%d_scale" % N] = ref.phasing.rftf(est, goal, scale=True)
        out["N%d_hot" % N] = ref.phasing.rftf(est, goal, hot_pixels=True)
        # (rftfq=True cannot run under Python 3: N/2 is a float in wrapping.unwrap)
        frames = (rng.random((2, N, N)) * 3).astype(np.float32)
        frames[0, 5, 7] = 40.0
        frames[1, N - 1, 0] = 25.0
        out["N%d_hp_in" % N] = frames
        out["N%d_hp_out" % N] = ref.conditioning.remove_hot_pixels(frames.copy(), iterations=2)
    np.savez_compressed(os.path.join(HERE, "quality.npz"), **out)


def coherence_opt():
    """optimize_coherence (phasing.py:507-930), numpy branch: Richardson-Lucy
    on one frame (the branch fails on a second) and the Gaussian fit on two."""
    import warnings
    out = {}
    N, B = 32, 10
    rng = np.random.default_rng(9)
    obj = np.zeros((N, N), np.complex128)
    obj[11:11 + B, 11:11 + B] = rng.random((B, B)) * np.exp(1j * rng.uniform(-0.5, 0.5, (B, B)))
    blur = gaussian_ipsf(N, 1.2)
    M = np.sqrt(np.abs(np.fft.ifft2(np.fft.fft2(np.abs(np.fft.fft2(obj)) ** 2) * blur))).astype(np.float32)
    est1 = obj[8:24, 8:24].astype(np.complex64)[None]
    est2 = np.stack([obj[8:24, 8:24], obj[8:24, 8:24] * 0.9 + 0.01]).astype(np.complex64)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
        rl = _quiet(r.optimize_coherence, est1.copy(), modulus=M, force_cpu=True, load=False,
                    silent=True, iterations=6, method="richardson_lucy")
        r2 = _quiet(ref.phasing.phasing, force_cpu=True, force_np_fft=True)
        cl = _quiet(r2.optimize_coherence, est2.copy(), modulus=M, force_cpu=True, load=False,
                    silent=True, method="gaussian")
    out["modulus"], out["est1"], out["est2"] = M, est1, est2
    out["rl_iterations"] = np.int64(6)
    out["rl_ipsf"] = np.asarray(rl)
    out["gaussian_lengths"] = np.asarray(cl)
    np.savez_compressed(os.path.join(HERE, "coherence_opt.npz"), **out)


def unwraps():
    """The polar-unwrap outputs (``prtfq``, ``rftfq``): ``prtf(prtfq=True)``
    on seeded trial sets at N = 32 and 64, ``rftf(rftfq=True)`` on the
    quality fixture's inputs, and ``wrapping.unwrap`` of a smooth 512 x 512
    map (row means, a sample of the unwrapped pixels)."""
    out = {}
    for N, frames in ((32, 6), (64, 8)):
        est = inputs.prtf_estimates(N, frames, 40 + N)
        out["prtf%d_in" % N] = est
        arr, q = _quiet(ref.phasing.prtf, est, prtfq=True)
        out["prtf%d_array" % N], out["prtf%d_q" % N] = arr, q
    for N in (32, 64):
        rng = np.random.default_rng(500 + N)   # the inputs of quality()
        B = N // 4
        obj = np.zeros((N, N), np.complex128)
        obj[:B, :B] = rng.random((B, B)) * np.exp(1j * rng.uniform(-0.5, 0.5, (B, B)))
        goal = (np.abs(np.fft.fft2(obj)) + 0.05).astype(np.float32)
        est = (obj[:B, :B] + 0.05 * rng.standard_normal((B, B))).astype(np.complex64)
        for name, kw in (("plain", {}), ("scale", {"scale": True})):
            arr, q = ref.phasing.rftf(est, goal, rftfq=True, **kw)
            out["rftf%d_%s_q" % (N, name)] = q
    N = 512
    m = inputs.smooth_map(N, 77)
    out["map512_sums"] = np.array([np.sum(m.astype(np.float64)), np.sum(m.astype(np.float64) ** 2)])
    uw = ref.wrapping.unwrap(m, (0, N // 2, (N // 2, N // 2)))
    out["map512_mean"] = np.average(uw, axis=1)
    idx = np.random.default_rng(3).choice(uw.size, 4096, replace=False)
    out["map512_idx"] = idx.astype(np.int64)
    out["map512_samples"] = uw.ravel()[idx]
    out["map512_shape"] = np.array(uw.shape)
    np.savez_compressed(os.path.join(HERE, "unwrap.npz"), **out)


ALL = ("projections", "projections_large", "trajectories", "seeds", "helpers", "coherence",
       "quality", "coherence_opt", "unwraps")

if __name__ == "__main__":
    # make_golden.py <reference root> [fixture function ...] (default: all)
    for name in (sys.argv[2:] or ALL):
        globals()[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
