"""sp_engine_run_static, the engine entry point that allocates nothing.

It serves callers that cannot allocate device memory themselves (a host
framework that owns all allocations, a plugin without an allocator): its
scratch is a fixed 48 MiB array inside the library.  These tests call it
through the C ABI and check that two calls in a row give what
sp_engine_run gives with a caller-allocated workspace -- coherent trials of
several sizes and algorithms, and partially coherent ones (ipsf, energy
spectrum) -- to the engine's
single-projection tolerance (1e-5 relative L2 norm) -- in practice bit for bit.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _trials(seed=0):
    """A small mixed batch: sizes, algorithms and starts differ per trial;
    the last two project partially coherently (an ipsf, and an energy
    spectrum with an ipsf), which adds divisor planes and a job table to the
    scratch layout."""
    from als_speckle_b200 import synth
    from als_speckle_b200.workloads import gaussian_ipsf
    out = []
    for k, (N, order, iters, coh) in enumerate(((256, (("hio", 6), ("er", 2)), 8, None),
                                                (512, (("raar", 5),), 5, None),
                                                (128, (("dm", 3), ("er", 1)), 4, None),
                                                (128, (("hio", 3), ("dm", 2)), 5, "ipsf"),
                                                (64, (("raar", 4),), 4, "spectrum"))):
        _, M, S = synth.pattern(N, n_ellipses=5, box=N // 4, peak=1e6, seed=seed + k,
                                support_edge=N // 4 + 8)
        d = dict(N=N, order=order, iters=iters, M=torch.from_numpy(M).cuda(),
                 S=torch.from_numpy(S).cuda(), trial=k, ipsf=None, spectrum=None)
        if coh is not None:
            d["ipsf"] = torch.from_numpy(gaussian_ipsf(N, 1.5)).cuda()
        if coh == "spectrum":
            e = np.linspace(0.96, 1.04, 5)
            w = np.exp(-0.5 * np.linspace(-2, 2, 5) ** 2)
            d["spectrum"] = (torch.from_numpy((e / e[2]).astype(np.float32)).cuda(),
                             torch.from_numpy(w.astype(np.float32)).cuda())
        out.append(d)
    return out


def _specs(inp, psis, saves, errs):
    from als_speckle_b200.engine import TrialSpec
    return [TrialSpec(psi=psis[k], modulus=d["M"], support=d["S"], iterations=d["iters"],
                      order=d["order"], beta=0.9, random_phase=True, seed=5, trial=d["trial"],
                      box=(d["N"] // 4, d["N"] // 4, d["N"] // 2, d["N"] // 2), save=saves[k],
                      errors=errs[k], ipsf=d["ipsf"], spectrum=d["spectrum"])
            for k, d in enumerate(inp)]


def _buffers(inp):
    psis = [torch.zeros((d["N"], d["N"]), dtype=torch.complex64, device="cuda") for d in inp]
    saves = [torch.zeros((d["N"] // 2, d["N"] // 2), dtype=torch.complex64, device="cuda") for d in inp]
    errs = [torch.zeros((d["iters"], 2), dtype=torch.float64, device="cuda") for d in inp]
    return psis, saves, errs


def _rel(a, b):
    a = a.cpu().numpy().astype(np.complex128)
    b = b.cpu().numpy().astype(np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_static_entry_matches_workspace_entry_twice():
    from als_speckle_b200 import _lib
    from als_speckle_b200.engine import Engine, _to_struct
    inp = _trials()

    # reference result: the existing entry point with a torch-allocated workspace,
    # with the library's default E per size, as the static call below uses
    psis, saves, errs = _buffers(inp)
    eng = Engine(use_graph=False, e_per_n={})
    eng.solve(_specs(inp, psis, saves, errs))
    torch.cuda.synchronize()

    for call in range(2):
        p2, s2, e2 = _buffers(inp)
        specs = _specs(inp, p2, s2, e2)
        arr = (_lib.sp_trial * len(specs))(*[_to_struct(t) for t in specs])
        opts = _lib.sp_run_opts()
        status = _lib.lib.sp_engine_run_static(arr, len(specs), C.byref(opts), _lib.stream_ptr())
        assert status == 0, _lib.lib.sp_last_error()
        torch.cuda.synchronize()
        for k in range(len(inp)):
            assert _rel(p2[k], psis[k]) < 1e-5, (call, k)
            assert _rel(s2[k], saves[k]) < 1e-5, (call, k)
            assert torch.allclose(e2[k], errs[k], rtol=1e-9, atol=0), (call, k)
    eng.close()


def test_static_entry_rejects_oversize_request():
    from als_speckle_b200 import _lib
    from als_speckle_b200.engine import _to_struct, TrialSpec
    N = 2048
    M = torch.ones((N, N), dtype=torch.float32, device="cuda")
    S = torch.ones((N, N), dtype=torch.float32, device="cuda")
    psi = torch.zeros((N, N), dtype=torch.complex64, device="cuda")
    # 2 trials of 2048^2 with DM need 2 * 2 * 32 MiB of work planes
    specs = [TrialSpec(psi=psi, modulus=M, support=S, iterations=1, order=(("dm", 1),), beta=0.9)
             for _ in range(2)]
    arr = (_lib.sp_trial * 2)(*[_to_struct(t) for t in specs])
    status = _lib.lib.sp_engine_run_static(arr, 2, None, _lib.stream_ptr())
    assert status == 2
    assert b"static array" in _lib.lib.sp_last_error()
