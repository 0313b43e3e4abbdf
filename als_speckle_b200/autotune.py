"""Autotuner for the engine's per-size launch parameters.

For a size N it times, on the current device, the fused iteration for every
values-per-thread choice E (8, 16 or 32: the radix of the in-register first
Stockham stage, the tile each CTA owns and, through registers, how many CTAs
share an SM) and for several L2 group sizes
(trials whose planes are kept L2-resident together), and keeps the fastest.
Results are cached in ``autotune.json`` next to this file, keyed by device
name and N.

    python -m als_speckle_b200.autotune 256 512 1024 2048
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "autotune.json")

DEFAULTS = {
    # values per thread and L2 group budget (bytes) when nothing was tuned
    "E": 32,
    "l2_group_bytes": 48 << 20,
}


def _device_key():
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "unknown"


def load(path=CACHE):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def tuned_e_per_n(path=CACHE, device_name=None):
    """{N: E} for every size tuned on this device (empty when none was)."""
    entries = load(path).get(device_name or _device_key(), {})
    out = {}
    for n, entry in entries.items():
        if isinstance(entry, dict) and "E" in entry:
            out[int(n)] = int(entry["E"])
    return out


def load_or_default(N, path=CACHE):
    entry = load(path).get(_device_key(), {}).get(str(N))
    out = dict(DEFAULTS)
    if entry:
        out.update({k: entry[k] for k in ("E", "l2_group_bytes") if k in entry})
    return out


def _time_config(N, E, l2, trials, iters, reps=3):
    import torch
    from . import synth
    from .engine import Engine, TrialSpec
    _, M, S = synth.pattern(N, n_ellipses=8, box=N // 4, peak=1e6, seed=0,
                            support_edge=N // 4 + N // 16)
    Md = torch.from_numpy(M).cuda()
    Sd = torch.from_numpy(S).cuda()
    psis = torch.empty((trials, N, N), dtype=torch.complex64, device="cuda")
    eng = Engine(use_graph=True, l2_group_bytes=l2, e_per_n={N: E})
    specs = [TrialSpec(psi=psis[k], modulus=Md, support=Sd, iterations=iters,
                       order=(("hio", iters),), beta=0.9, random_phase=True, seed=1, trial=k)
             for k in range(trials)]
    eng.solve(specs)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        eng.solve(specs)
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b) / 1e3)
    eng.close()
    return trials * iters / best


def tune(N, trials=None, iters=60, path=CACHE, verbose=True):
    """Time every (E, group) choice for size N and store the fastest."""
    plane = N * N * 8
    if trials is None:
        trials = max(1, min(128, (1 << 30) // (3 * plane)))
    groups = sorted({g for g in (8, 16, 32, trials) if g <= trials})
    results = []
    for E in (8, 16, 32):
        for g in groups:
            l2 = g * 2 * plane if g < trials else 0
            rate = _time_config(N, E, l2, trials, iters)
            results.append({"E": E, "group": g, "l2_group_bytes": l2, "rate": rate})
            if verbose:
                print("N=%d E=%d group=%d: %.0f trial-iter/s" % (N, E, g, rate), flush=True)
    best = max(results, key=lambda r: r["rate"])
    data = load(path)
    data.setdefault(_device_key(), {})[str(N)] = {
        "E": best["E"], "l2_group_bytes": best["l2_group_bytes"], "rate": best["rate"],
        "trials": trials, "iters": iters, "sweep": results}
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    return best


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("sizes", type=int, nargs="*", default=[512])
    ap.add_argument("--out", default=CACHE)
    ap.add_argument("--trials", type=int, default=None)
    ap.add_argument("--iters", type=int, default=60)
    a = ap.parse_args()
    for n in a.sizes:
        print(n, tune(n, trials=a.trials, iters=a.iters, path=a.out))
