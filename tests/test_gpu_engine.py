"""GPU parity of the fused engine and the standalone FFT against the oracle
and the reference's golden vectors.

Tolerances: a single projection matches to 1e-5 relative L2 norm
(||a-b||/||b||); the 2-D FFT to 2e-6; short trajectories of the chaotic
iteration to 1e-4.
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


def dev(x, dt=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t.to(dt) if dt is not None else t


@pytest.fixture(scope="module")
def engine():
    from als_speckle_b200.engine import Engine
    e = Engine(use_graph=False)
    yield e
    e.close()


# ---------------------------------------------------------------- 2-D FFT
@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_fft2_matches_numpy(N):
    from als_speckle_b200.phasing import fft2
    rng = np.random.default_rng(N)
    batch = 2 if N <= 2048 else 1
    x = (rng.standard_normal((batch, N, N)) + 1j * rng.standard_normal((batch, N, N))).astype(np.complex64)
    f = fft2(dev(x)).cpu().numpy()
    assert rel(f, np.fft.fft2(x.astype(np.complex128))) < 2e-6
    b = fft2(dev(x), inverse=True).cpu().numpy()
    assert rel(b, np.fft.ifft2(x.astype(np.complex128))) < 2e-6


# ------------------------------------------------- one projection vs golden
def _spec(psi, M, S, iters, order, beta, **kw):
    from als_speckle_b200.engine import TrialSpec
    return TrialSpec(psi=psi, modulus=M, support=S, iterations=iters, order=order, beta=beta, **kw)


@pytest.mark.parametrize("N", [8, 32, 64])
@pytest.mark.parametrize("alg", ["hio", "er", "raar", "sf", "dm"])
def test_single_projection_vs_reference_golden(engine, N, alg):
    g = np.load(os.path.join(G, "projections.npz"))
    psi = dev(g["N%d_psi" % N])
    M = dev(g["N%d_modulus" % N])
    S = dev(g["N%d_support" % N])
    beta = float(g["N%d_%s_beta" % (N, alg)])
    engine.solve([_spec(psi, M, S, 1, ((alg, 1),), beta, quirks="cpu")])
    assert rel(psi.cpu().numpy(), g["N%d_%s_psi_in" % (N, alg)]) < 1e-5


@pytest.mark.parametrize("N", [256, 512])
@pytest.mark.parametrize("alg", ["hio", "er", "raar", "sf", "dm"])
def test_single_projection_vs_reference_golden_large(engine, N, alg):
    """One iteration at 256^2 and 512^2 against the reference's own numpy
    path: its output at 4096 fixed pixels (half inside the support) and its
    FP64 whole-plane sums, on inputs rebuilt from the fixture's seed."""
    import sys
    sys.path.insert(0, G)
    import golden_inputs as inputs
    g = np.load(os.path.join(G, "projections_large.npz"))
    psi0, M, S = inputs.projection_inputs(N, int(g["N%d_seed" % N]))
    np.testing.assert_allclose(inputs.input_sums(psi0, M, S), g["N%d_input_sums" % N], rtol=1e-12)
    psi = dev(psi0)
    beta = float(g["N%d_%s_beta" % (N, alg)])
    engine.solve([_spec(psi, dev(M), dev(S), 1, ((alg, 1),), beta, quirks="cpu")])
    got = psi.cpu().numpy()
    assert rel(got.ravel()[g["N%d_idx" % N]], g["N%d_%s_samples" % (N, alg)]) < 1e-5
    r = got.astype(np.complex128)
    sums = np.array([np.sum(np.abs(r) ** 2), np.sum(r).real, np.sum(r).imag])
    want = g["N%d_%s_sums" % (N, alg)]
    assert abs(sums[0] - want[0]) / want[0] < 1e-5
    scale = np.sqrt(want[0] * r.size)  # bound on |sum| by Cauchy-Schwarz
    assert np.all(np.abs(sums[1:] - want[1:]) / scale < 1e-5)


@pytest.mark.parametrize("E", [8, 16, 32])
@pytest.mark.parametrize("N", [128, 256, 512, 1024, 2048])
@pytest.mark.parametrize("alg", ["hio", "er", "raar", "sf", "dm"])
def test_single_projection_vs_fp64_oracle(N, alg, E):
    """One projection + update of every algorithm, for every values-per-thread
    choice E, against the FP64 oracle; the FP64 error sums too."""
    from als_speckle_b200 import synth
    from als_speckle_b200.engine import Engine
    obj, M, S = synth.pattern(N, n_ellipses=6, box=N // 4, peak=1e6, seed=N, support_edge=N // 4 + N // 16)
    rng = np.random.default_rng(1)
    psi0 = ((rng.random((N, N)) + 1j * rng.random((N, N))) * S).astype(np.complex64)
    beta = 0.87 if alg == "raar" else 0.9
    want, _ = O.iteration(psi0, M, S, alg, beta, quirks="gpu", mode="f64")
    psi = dev(psi0)
    err = torch.zeros((1, 2), dtype=torch.float64, device="cuda")
    engine = Engine(use_graph=False, e_per_n={N: E})
    engine.solve([_spec(psi, dev(M), dev(S), 1, ((alg, 1),), beta, errors=err)])
    assert rel(psi.cpu().numpy(), want) < 1e-5
    e, r = O.modulus_errors(psi0, M)
    m = M.astype(np.float64)
    got = err.cpu().numpy()[0]
    assert abs(got[0] / np.sum(m * m) - e) / e < 1e-5
    assert abs(got[1] / np.sum(m) - r) / r < 1e-5
    engine.close()


@pytest.mark.parametrize("N", [512])
def test_projection_e16_equals_e32(N):
    """Per-thread radix choices give the same result to FP32 rounding."""
    from als_speckle_b200.engine import Engine
    from als_speckle_b200 import synth
    _, M, S = synth.pattern(N, n_ellipses=6, box=128, peak=1e6, seed=3, support_edge=160)
    rng = np.random.default_rng(2)
    psi0 = ((rng.random((N, N)) + 1j * rng.random((N, N))) * S).astype(np.complex64)
    outs = []
    for E in (8, 16, 32):
        e = Engine(use_graph=False, e_per_n={N: E})
        psi = dev(psi0)
        e.solve([_spec(psi, dev(M), dev(S), 3, None, 0.9)])
        outs.append(psi.cpu().numpy())
        e.close()
    assert rel(outs[0], outs[2]) < 1e-5
    assert rel(outs[1], outs[2]) < 1e-5


def test_short_trajectories_vs_reference_golden(engine):
    t = np.load(os.path.join(G, "trajectories.npz"))
    for name, order in (("default", None), ("hio_er", (("hio", 8), ("er", 2))),
                        ("raar_dm", (("raar", 3), ("dm", 2)))):
        psi = dev(t["psi0"])
        engine.solve([_spec(psi, dev(t["modulus"]), dev(t["support"]), int(t[name + "_iters"]),
                            order, float(t[name + "_beta"]), quirks="cpu")])
        assert rel(psi.cpu().numpy(), t[name + "_final"]) < 1e-4, name


def test_random_phase_start_vs_oracle(engine):
    from als_speckle_b200 import synth
    N = 256
    _, M, S = synth.pattern(N, n_ellipses=8, box=64, peak=1e5, seed=5, support_edge=80)
    psi = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    engine.solve([_spec(psi, dev(M), dev(S), 0, None, 0.9, random_phase=True, seed=11, trial=3)])
    want = O.seed_random_phase(M, S, 11, 3)
    assert rel(psi.cpu().numpy(), want) < 1e-5


# ------------------------------------------------ batching is exact
def _batch_inputs(sizes, seed=0):
    from als_speckle_b200 import synth
    out = []
    for k, N in enumerate(sizes):
        _, M, S = synth.pattern(N, n_ellipses=5, box=N // 4, peak=1e6, seed=seed + k,
                                support_edge=N // 4 + 8)
        out.append((dev(M), dev(S)))
    return out


def test_batched_equals_alone_uneven_sizes_and_algorithms():
    """A mixed batch (sizes, algorithms, iteration counts) gives bit-identical
    psi to running each trial alone; L2 grouping and CUDA graphs too."""
    from als_speckle_b200.engine import Engine
    sizes = [64, 256, 512, 128, 256, 1024]
    orders = [(("hio", 4), ("er", 1)), (("raar", 3),), (("dm", 2), ("er", 1)), (("sf", 2), ("hio", 2)),
              (("dm", 1),), (("hio", 5),)]
    iters = [7, 5, 6, 4, 3, 5]
    inp = _batch_inputs(sizes)

    def specs(psis, saves):
        out = []
        for k, N in enumerate(sizes):
            M, S = inp[k]
            out.append(_spec(psis[k], M, S, iters[k], orders[k], 0.85, random_phase=True, seed=9,
                             trial=k, box=(N // 4, N // 8, N // 2, N // 3), save=saves[k]))
        return out

    def fresh():
        psis = [torch.zeros((N, N), dtype=torch.complex64, device="cuda") for N in sizes]
        saves = [torch.zeros((N // 2, N // 3), dtype=torch.complex64, device="cuda") for N in sizes]
        return psis, saves

    alone, alone_save = fresh()
    e = Engine(use_graph=False)
    for k, s in enumerate(specs(alone, alone_save)):
        e.solve([s])
    for l2, graph in ((0, False), (8 << 20, False), (0, True), (8 << 20, True)):
        psis, saves = fresh()
        eng = Engine(use_graph=graph, l2_group_bytes=l2)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            eng.solve(specs(psis, saves), stream=stream)
        stream.synchronize()
        for k in range(len(sizes)):
            assert torch.equal(psis[k], alone[k]), (l2, graph, k)
            assert torch.equal(saves[k], alone_save[k]), (l2, graph, k)
        eng.close()
    N = sizes[0]
    assert torch.equal(alone_save[0], alone[0][N // 4:N // 4 + N // 2, N // 8:N // 8 + N // 3])
    e.close()


# ------------------------------------------------ operator API (_kexec)
def test_kexec_operators_match_formulas():
    from als_speckle_b200.gpu import common
    rng = np.random.default_rng(0)
    n = 4096
    s = rng.random(n).astype(np.float32)
    pi = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    po = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    dm = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    m = rng.random(n).astype(np.float32)
    b, g = 0.9, -1 / 0.9
    c = common()
    out = torch.empty(n, dtype=torch.complex64, device="cuda")
    cases = {
        "hio": ((b, dev(s), dev(pi), dev(po), out), (1 - s) * (pi - b * po) + s * po),
        "er": ((dev(s), dev(po), out), s * po),
        "raar": ((b, dev(s), dev(pi), dev(po), out), (1 - s) * (b * pi + (1 - 2 * b) * po) + s * po),
        "sf": ((dev(s), dev(pi), dev(po), out), (1 - s) * (-po) + s * po),
        "dm1": ((1 / b, dev(s), dev(pi), out), -(1 / b) * (1 - s) * pi + s * pi),
        "dm2": ((b, g, dev(s), dev(pi), dev(po), dev(dm), out),
                s * (2 * po - b * dm + b * ((1 + g) * po - g * pi)) + (1 - s) * (pi - b * po)),
        "fourier": ((dev(pi), dev(np.abs(pi).astype(np.complex64)), dev(m), out), m * pi / np.abs(pi)),
        "abs_f2_f2": ((dev(pi), out), np.abs(pi).astype(np.complex64)),
    }
    for name, (args, want) in cases.items():
        c._kexec(name, *args)
        assert rel(out.cpu().numpy(), want) < 1e-6, name
    # copy_to_buffer_f2 (dst, src, c0, r0, n, N, shape=(cols, rows))
    N = 32
    src = dev((rng.standard_normal((N, N)) + 1j).astype(np.complex64))
    dst = torch.zeros((3, 10, 7), dtype=torch.complex64, device="cuda")
    c._kexec("copy_to_buffer_f2", dst, src, 4, 5, 1, N, shape=(7, 10))
    assert torch.equal(dst[1], src[5:15, 4:11])


# ------------------------------------------------ post-processing
def test_align_global_phase_vs_oracle():
    from als_speckle_b200.phasing import align_global_phase
    h = np.load(os.path.join(G, "helpers.npz"))
    got = align_global_phase(h["agp_in"])
    want = O.align_global_phase(h["agp_in"].astype(np.complex128))
    assert rel(got, want) < 2e-6
    for n in range(got.shape[0]):
        assert np.abs(got[n] - h["agp_out"][n]).max() < 5e-4 * np.abs(h["agp_in"][n]).max()


def test_prtf_vs_golden():
    from als_speckle_b200.phasing import prtf
    h = np.load(os.path.join(G, "helpers.npz"))
    # the golden (pinned in the CPU suite) is at N = 12, not a power of two;
    # the device PRTF is checked against the pinned oracle at N = 16 and 32
    for N in (16, 32):
        got = prtf(h["prtf_in"], N=N)
        assert np.allclose(got, O.prtf(h["prtf_in"], N=N), rtol=1e-5, atol=1e-6)
    with pytest.raises(ValueError):
        prtf(h["prtf_in"])


def test_refine_support_vs_golden():
    from als_speckle_b200.phasing import refine_support
    h = np.load(os.path.join(G, "helpers.npz"))
    for j in range(3):
        blur, lt, gt = h["rs%d_params" % j]
        refined, blurred = refine_support(h["rs%d_support" % j], h["rs%d_avg" % j], blur=float(blur),
                                          local_threshold=float(lt), global_threshold=float(gt))
        # the golden blur is an FFT convolution of |avg| computed in complex64
        assert np.allclose(blurred, h["rs%d_blurred" % j], rtol=1e-5, atol=1e-7)
        assert np.array_equal(refined, h["rs%d_refined" % j])


def test_center_of_mass_average_vs_golden():
    from als_speckle_b200.phasing import center_of_mass_average
    h = np.load(os.path.join(G, "helpers.npz"))
    assert np.allclose(center_of_mass_average(h["com_in"]), h["com_out"], atol=1e-6)


def test_align_frames_device_known_answers():
    """test/test_conditioning.py:34-52 semantics at a power-of-two size."""
    from als_speckle_b200.phasing import align_frames_device
    rng = np.random.default_rng(4)
    data = rng.random((64, 64)).astype(np.complex64)
    for ry, rx in ((3, 5), (0, 11), (30, 2)):
        rolled = np.roll(np.roll(data, rx, axis=1), ry, axis=0)
        out = align_frames_device(dev(rolled), dev(data)).cpu().numpy()
        assert np.array_equal(out, data)


# ------------------------------------------------ the phasing class
def test_phasing_class_matches_reference_trajectory():
    from als_speckle_b200.phasing import phasing
    t = np.load(os.path.join(G, "trajectories.npz"))
    r = phasing(quirks="cpu")
    r.load(modulus=t["modulus"], support=t["support"], numtrials=2)
    r.psi_in.copy_(dev(t["psi0"]))
    r.iterate(int(t["default_iters"]))
    assert rel(r.get(r.psi_in), t["default_final"]) < 1e-4
    sb = r.get(r.savebuffer)
    assert sb.shape[0] == 3 and np.array_equal(sb[0], r.get(r.psi_in)[r.r0:r.r0 + r.rows, r.c0:r.c0 + r.cols])
    assert r.numtrial == 1
    # chunked iteration (silent=int) walks the same cyclic order
    r2 = phasing(quirks="cpu")
    r2.load(modulus=t["modulus"], support=t["support"], numtrials=2)
    r2.psi_in.copy_(dev(t["psi0"]))
    r2.iterate(int(t["default_iters"]), silent=5)
    assert torch.equal(r2.psi_in, r.psi_in)


def test_phasing_seed_matches_reference():
    from als_speckle_b200.phasing import phasing
    s = np.load(os.path.join(G, "seed.npz"))
    r = phasing()
    N = s["psi"].shape[0]
    r.load(modulus=np.ones((N, N), np.float32), support=s["support"], numtrials=1)
    r.seed(int(s["val"]))
    assert np.array_equal(r.get(r.psi_in), s["psi"])


def test_plain_path_matches_engine():
    from als_speckle_b200 import _lib, synth
    from als_speckle_b200.engine import Engine, expand_runs
    import ctypes as C
    N = 256
    _, M, S = synth.pattern(N, n_ellipses=8, box=64, peak=1e5, seed=2, support_edge=80)
    rng = np.random.default_rng(0)
    psi0 = ((rng.random((N, N)) + 1j * rng.random((N, N))) * S).astype(np.complex64)
    order = (("hio", 3), ("er", 1), ("dm", 1))
    a = dev(psi0)
    Engine(use_graph=False).solve([_spec(a, dev(M), dev(S), 5, order, 0.9)])
    b = dev(psi0)
    Md, Sd = dev(M), dev(S)
    algs, counts = expand_runs(order)
    work = torch.empty((4, N, N), dtype=torch.complex64, device="cuda")
    alg_arr = (C.c_int32 * len(algs))(*algs)
    cnt_arr = (C.c_int32 * len(counts))(*counts)
    _lib.call("sp_plain_iterate", N, 5, len(algs), alg_arr, cnt_arr, C.c_float(0.9), _lib.ptr(b),
              _lib.ptr(Md), _lib.ptr(Sd), _lib.ptr(work), _lib.stream_ptr())
    torch.cuda.synchronize()
    assert rel(a.cpu().numpy(), b.cpu().numpy()) < 1e-4


def test_split_prtf_and_average_equal_one_shot():
    """Partial phasor/frame sums over two halves, added and finished, equal
    the PRTF and mean of all frames at once (the multi-GPU reduction path)."""
    from als_speckle_b200.distributed import local_sums, finish_prtf
    from als_speckle_b200.phasing import prtf, mean_frames
    rng = np.random.default_rng(9)
    fr = (rng.random((9, 20, 24)) * np.exp(1j * rng.normal(0, 0.4, (9, 20, 24)))).astype(np.complex64)
    t = dev(fr)
    f1, p1 = local_sums(t[:4], 32)
    f2, p2 = local_sums(t[4:], 32)
    got = finish_prtf(p1 + p2, 9).cpu().numpy()
    assert np.allclose(got, prtf(t, N=32).cpu().numpy(), rtol=1e-5, atol=1e-6)
    assert np.allclose(((f1 + f2) / 9).cpu().numpy(), mean_frames(t).cpu().numpy(), atol=1e-6)
