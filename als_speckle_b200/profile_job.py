"""A small, fixed engine job for profiling (ncu launch lists and captures).

    python -m als_speckle_b200.profile_job --n 512 --trials 12 --iters 8 [--e 32]
        [--ipsf] [--spectrum]

Runs one warm-up solve and one profiled solve of ``trials`` random-phase HIO
trials of size N without CUDA graphs, so every pass is a separate launch that
ncu can select by name (``row_pass_kernel`` / ``col_pass_kernel``, and the
``pc_*`` kernels of partially coherent trials).  The working set is
2 * trials * N^2 * 8 bytes plus the modulus and support (and the divisor
planes of partially coherent trials).  ``--ipsf`` gives every trial a Gaussian
ipsf (sigma 2 px), ``--spectrum`` a 7-sample energy spectrum (+-5%, Gaussian
weights), as the ``coherence512`` workload does.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import synth
from .engine import Engine, TrialSpec
from .workloads import gaussian_ipsf


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--trials", type=int, default=12)
    ap.add_argument("--iters", type=int, default=8)
    ap.add_argument("--e", type=int, default=32)
    ap.add_argument("--alg", default="hio")
    ap.add_argument("--ipsf", action="store_true")
    ap.add_argument("--spectrum", action="store_true")
    a = ap.parse_args()
    N = a.n
    _, M, S = synth.pattern(N, n_ellipses=8, box=N // 4, peak=1e6, seed=0, support_edge=N // 4 + N // 16)
    Md = torch.from_numpy(M).cuda()
    Sd = torch.from_numpy(S).cuda()
    psis = torch.empty((a.trials, N, N), dtype=torch.complex64, device="cuda")
    errs = torch.zeros((a.trials, a.iters, 2), dtype=torch.float64, device="cuda")
    ipsf = torch.from_numpy(gaussian_ipsf(N, 2.0)).cuda() if a.ipsf else None
    spec = None
    if a.spectrum:
        e = np.linspace(0.95, 1.05, 7)
        w = np.exp(-0.5 * np.linspace(-2, 2, 7) ** 2)
        spec = (torch.from_numpy((e / e[3]).astype(np.float32)).cuda(),
                torch.from_numpy(w.astype(np.float32)).cuda())
    eng = Engine(use_graph=False, e_per_n={N: a.e})
    specs = [TrialSpec(psi=psis[k], modulus=Md, support=Sd, iterations=a.iters,
                       order=((a.alg, a.iters),), beta=0.9, random_phase=True, seed=1, trial=k,
                       errors=errs[k], ipsf=ipsf, spectrum=spec) for k in range(a.trials)]
    eng.solve(specs)
    torch.cuda.synchronize()
    eng.solve(specs)
    torch.cuda.synchronize()
    r = (errs[:, -1, 1] / Md.double().sum()).mean().item()
    print("N=%d trials=%d iters=%d E=%d final R=%.4f" % (N, a.trials, a.iters, a.e, r))
    eng.close()


if __name__ == "__main__":
    main()
