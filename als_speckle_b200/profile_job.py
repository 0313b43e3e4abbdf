"""A small, fixed engine job for profiling (ncu launch lists and captures).

    python -m als_speckle_b200.profile_job --n 512 --trials 12 --iters 8 [--e 32]

Runs one warm-up solve and one profiled solve of ``trials`` random-phase HIO
trials of size N without CUDA graphs, so every pass is a separate launch that
ncu can select by name (``row_pass_kernel`` / ``col_pass_kernel``).  The
working set is 2 * trials * N^2 * 8 bytes plus the modulus and support.
"""
from __future__ import annotations

import argparse

import torch

from . import synth
from .engine import Engine, TrialSpec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--trials", type=int, default=12)
    ap.add_argument("--iters", type=int, default=8)
    ap.add_argument("--e", type=int, default=32)
    ap.add_argument("--alg", default="hio")
    a = ap.parse_args()
    N = a.n
    _, M, S = synth.pattern(N, n_ellipses=8, box=N // 4, peak=1e6, seed=0, support_edge=N // 4 + N // 16)
    Md = torch.from_numpy(M).cuda()
    Sd = torch.from_numpy(S).cuda()
    psis = torch.empty((a.trials, N, N), dtype=torch.complex64, device="cuda")
    errs = torch.zeros((a.trials, a.iters, 2), dtype=torch.float64, device="cuda")
    eng = Engine(use_graph=False, e_per_n={N: a.e})
    specs = [TrialSpec(psi=psis[k], modulus=Md, support=Sd, iterations=a.iters,
                       order=((a.alg, a.iters),), beta=0.9, random_phase=True, seed=1, trial=k,
                       errors=errs[k]) for k in range(a.trials)]
    eng.solve(specs)
    torch.cuda.synchronize()
    eng.solve(specs)
    torch.cuda.synchronize()
    r = (errs[:, -1, 1] / Md.double().sum()).mean().item()
    print("N=%d trials=%d iters=%d E=%d final R=%.4f" % (N, a.trials, a.iters, a.e, r))
    eng.close()


if __name__ == "__main__":
    main()
