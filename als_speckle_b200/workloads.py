"""The benchmark workloads other than the headline batched HIO job.

    python -m als_speckle_b200.workloads single256 | raar_dm1024 | uneven | serving | coherence512 | quality [--out f.json]

* ``single256``   one 256^2 trial, 200 HIO (beta 0.9) + 20 ER, random-phase start,
                   through ``phasing.iterate_trials``; final R-factor.
* ``raar_dm1024`` one 1024^2 trial, 1500 RAAR (beta 0.87) + 500 DM, shrinkwrap
                   every 20 iterations (sigma annealed 3 -> 0.7 px, local threshold
                   0.15); per-iteration modulus error.
* ``uneven``      64 x 256^2 + 32 x 512^2 + 8 x 1024^2 + 2 x 2048^2 trials,
                   HIO / RAAR / DM round robin, 1000 iterations each, in one
                   engine call versus one call per trial.
* ``serving``     Poisson request stream through the continuous-batching
                   service; p50 / p99 latency, throughput, sustainable rate.
* ``coherence512`` 32 x 512^2 trials, 200 HIO (beta 0.9), random-phase starts:
                   coherent, with an ipsf (Gaussian point spread, sigma 2 px),
                   with an energy spectrum (7 samples, +-5%), and with both;
                   trial-iterations/s of each.
* ``quality``     128 reconstructions (180^2 crops of one object plus noise):
                   gpu_rftf against a 512^2 goal, rftf of their average, and
                   covar_results over all 8256 pairs (256^2 transforms).

All inputs are seeded synthetic patterns (``synth``); results are printed as
one JSON object.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import synth
from .engine import Engine, TrialSpec
from .masking import bounding_box


def _timed(fn):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0


def single256(seed=0):
    from .phasing import phasing
    _, M, S = synth.config_pattern("plain_256", seed=seed)
    r = phasing()
    r.load(modulus=M, support=S, numtrials=1)
    order = (("hio", 200), ("er", 20))
    r.iterate_trials(220, 1, order=order, beta=0.9, seed=seed)  # warm-up
    r.numtrial = 0
    (psis, errs), dt = _timed(lambda: r.iterate_trials(220, 1, order=order, beta=0.9, seed=seed,
                                                       errors=True))
    m = M.astype(np.float64)
    e = errs[0].cpu().numpy()
    return {"workload": "single256", "iterations": 220, "seconds": dt, "iter_per_s": 220 / dt,
            "final_error": float(e[-1, 0] / np.sum(m * m)), "final_r_factor": float(e[-1, 1] / np.sum(m))}


def raar_dm1024(seed=0, rounds=None):
    """RAAR 1500 + DM 500 with shrinkwrap every 20 iterations on one 1024^2
    instance.  The support is refined on its crop (bounding box, pad 10) of
    |psi| and put back in place, so the running iterate stays aligned."""
    from .phasing import refine_support
    _, M, S = synth.config_pattern("raar_dm_1024", seed=seed)
    N = M.shape[0]
    dev = torch.device("cuda")
    # everything on a private stream, where the engine's launch sequence is
    # replayed as a CUDA graph (a lone 1024^2 trial gains ~20% from it)
    stream = torch.cuda.Stream(dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(stream):
        Md = torch.from_numpy(M).to(dev)
        sup = S.copy()
        psi = torch.zeros((N, N), dtype=torch.complex64, device=dev)
        eng = Engine(device=dev, use_graph=True)
        schedule = [("raar", 0.87)] * 75 + [("dm", 0.87)] * 25  # 100 blocks of 20 iterations
        if rounds is not None:
            schedule = schedule[:rounds]
        sigmas = np.linspace(3.0, 0.7, len(schedule))
        m = M.astype(np.float64)
        errs = []
        t_iter = t_sw = 0.0
        for b, (alg, beta) in enumerate(schedule):
            Sd = torch.from_numpy(sup).to(dev)
            err = torch.zeros((20, 2), dtype=torch.float64, device=dev)
            spec = TrialSpec(psi=psi, modulus=Md, support=Sd, iterations=20, order=((alg, 20),), beta=beta,
                             random_phase=(b == 0), seed=seed, trial=0, errors=err)
            _, dt = _timed(lambda: eng.solve([spec], stream=stream))
            t_iter += dt
            e = err.cpu().numpy()
            errs.extend((e[:, 0] / np.sum(m * m)).tolist())
            # shrinkwrap on the support's crop
            bb = bounding_box(sup, pad=10)
            r0, r1, c0, c1 = (int(v) for v in bb)
            t0 = time.perf_counter()
            crop = psi[r0:r1, c0:c1].contiguous()
            refined, _ = refine_support(sup[r0:r1, c0:c1], crop, blur=float(sigmas[b]),
                                        local_threshold=0.15, global_threshold=0.0)
            if refined.sum() > 0:
                sup = np.zeros_like(sup)
                sup[r0:r1, c0:c1] = refined
            t_sw += time.perf_counter() - t0
        eng.close()
    n_it = 20 * len(schedule)
    return {"workload": "raar_dm1024", "iterations": n_it, "iterate_seconds": t_iter,
            "iter_per_s": n_it / t_iter, "shrinkwrap_seconds": t_sw,
            "error_first": errs[:5], "error_every_100": errs[::100], "final_error": errs[-1],
            "support_pixels": int(sup.sum())}


def uneven(iters=1000, seed=0):
    """Uneven-size batch in one engine call versus one call per trial."""
    plan = [(256, 64), (512, 32), (1024, 8), (2048, 2)]
    algs = [("hio", 0.9), ("raar", 0.87), ("dm", 0.9)]
    dev = torch.device("cuda")
    trials = []
    k = 0
    for N, count in plan:
        _, M, S = synth.pattern(N, n_ellipses=40, box=N // 4, peak=1e6, seed=seed + N,
                                support_edge=int(round(1.25 * (N // 4))))
        Md, Sd = torch.from_numpy(M).to(dev), torch.from_numpy(S).to(dev)
        for _ in range(count):
            alg, beta = algs[k % 3]
            trials.append(dict(N=N, M=Md, S=Sd, alg=alg, beta=beta, k=k))
            k += 1

    def specs(psis):
        return [TrialSpec(psi=psis[i], modulus=t["M"], support=t["S"], iterations=iters,
                          order=((t["alg"], iters),), beta=t["beta"], random_phase=True, seed=seed,
                          trial=t["k"]) for i, t in enumerate(trials)]

    psis = [torch.zeros((t["N"], t["N"]), dtype=torch.complex64, device=dev) for t in trials]
    from . import autotune
    e_per_n = {N: autotune.load_or_default(N)["E"] for N, _ in plan}
    eng = Engine(device=dev, use_graph=True, e_per_n=e_per_n)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        eng.solve(specs(psis), stream=stream)  # warm-up (graph capture)
        stream.synchronize()
        _, t_batched = _timed(lambda: eng.solve(specs(psis), stream=stream))
        stream.synchronize()
        # serial: one engine call per trial on the same GPU
        sp = specs(psis)
        eng1 = Engine(device=dev, use_graph=True, e_per_n=e_per_n)
        for _ in range(2):  # the workspace settles at its largest size, graphs get cached
            for s in sp:
                eng1.solve([s], stream=stream)
        stream.synchronize()
        _, t_serial = _timed(lambda: [eng1.solve([s], stream=stream) for s in sp])
    px_it = sum(t["N"] ** 2 for t in trials) * iters
    eng.close()
    eng1.close()
    return {"workload": "uneven", "trials": len(trials), "iterations": iters,
            "batched_seconds": t_batched, "serial_seconds": t_serial,
            "speedup": t_serial / t_batched, "batched_gpx_it_per_s": px_it / t_batched / 1e9,
            "e_per_n": e_per_n}


def serving(rate=200.0, window=0.5, seed=0, budget_gb=120, chunk=64, sizes=(256, 512, 1024, 2048),
            probs=(0.4, 0.3, 0.2, 0.1)):
    from .serving import ServingEngine, poisson_workload
    reqs = poisson_workload(window=window, rate=rate, seed=seed, sizes=sizes, probs=probs)
    srv = ServingEngine(hbm_budget=int(budget_gb) << 30, chunk=chunk)
    for r in reqs:
        srv.submit(r)
    t0 = time.perf_counter()
    res = srv.run(realtime=True)
    wall = time.perf_counter() - t0
    lat = np.array([r.latency for r in res.values()])
    px_it = sum(r.n ** 2 * r.iterations * r.trials for r in reqs)
    work_per_req = px_it / max(1, len(reqs))
    capacity = px_it / wall  # pixel-iterations per second actually delivered
    return {"workload": "serving", "rate": rate, "window_s": window, "requests": len(reqs),
            "wall_s": wall, "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "rounds": srv.rounds,
            "trial_iterations_per_s": srv.trial_iterations / wall,
            "gpx_iterations_per_s": capacity / 1e9,
            "sustainable_rate_per_s": capacity / work_per_req}


def gaussian_ipsf(N, sigma):
    """Transform of a normalised Gaussian point spread of ``sigma`` pixels,
    corner-centred: the ``ipsf`` of ``phasing.load``."""
    q = np.fft.fftfreq(N) * N
    g = np.exp(-0.5 * (q[:, None] ** 2 + q[None, :] ** 2) / sigma ** 2)
    return np.fft.fft2(g / g.sum()).astype(np.complex64)


def coherence512(trials=32, iters=200, seed=0):
    """Partially coherent against coherent projections on the same job."""
    _, M, S = synth.config_pattern("hio_512x128", seed=seed)
    N = M.shape[0]
    dev = torch.device("cuda")
    Md, Sd = torch.from_numpy(M).to(dev), torch.from_numpy(S).to(dev)
    ipsf = torch.from_numpy(gaussian_ipsf(N, 2.0)).to(dev)
    psis = torch.zeros((trials, N, N), dtype=torch.complex64, device=dev)
    from . import autotune
    eng = Engine(device=dev, use_graph=True, e_per_n={N: autotune.load_or_default(N)["E"]})
    stream = torch.cuda.Stream()
    out = {"workload": "coherence512", "trials": trials, "iterations": iters}
    e = np.linspace(0.95, 1.05, 7)
    w = np.exp(-0.5 * np.linspace(-2, 2, 7) ** 2)
    spec = (torch.from_numpy((e / e[3]).astype(np.float32)).to(dev),
            torch.from_numpy(w.astype(np.float32)).to(dev))
    for name, ip, sp in (("coherent", None, None), ("partially_coherent", ipsf, None),
                         ("spectrum", None, spec), ("ipsf_and_spectrum", ipsf, spec)):
        specs = [TrialSpec(psi=psis[k], modulus=Md, support=Sd, iterations=iters,
                           order=(("hio", iters),), beta=0.9, random_phase=True, seed=seed,
                           trial=k, ipsf=ip, spectrum=sp) for k in range(trials)]
        with torch.cuda.stream(stream):
            eng.solve(specs, stream=stream)  # warm-up (graph capture)
            stream.synchronize()
            _, dt = _timed(lambda: eng.solve(specs, stream=stream))
        out[name + "_trial_iter_per_s"] = trials * iters / dt
    eng.close()
    out["ratio"] = out["partially_coherent_trial_iter_per_s"] / out["coherent_trial_iter_per_s"]
    return out


def quality(frames=128, seed=0):
    """Trial-quality measures on a batch of reconstructions."""
    from .phasing import gpu_rftf, rftf, covar_results
    rng = np.random.default_rng(seed)
    obj, M, _ = synth.config_pattern("hio_512x128", seed=seed)
    crop = obj[166:346, 166:346]
    recs = (crop[None] * np.exp(1j * rng.uniform(-np.pi, np.pi, (frames, 1, 1)))
            + 0.05 * (rng.standard_normal((frames, 180, 180)) + 1j * rng.standard_normal((frames, 180, 180))))
    recs = recs.astype(np.complex64)
    dev = torch.device("cuda")
    recs_d = torch.from_numpy(recs).to(dev)
    Md = torch.from_numpy(M).to(dev)
    gpu_rftf(None, recs_d[:2], Md)  # warm-up
    _, t_gr = _timed(lambda: gpu_rftf(None, recs_d, Md))
    avg = recs_d.mean(0)
    rftf(avg, Md)
    _, t_r = _timed(lambda: rftf(avg, Md))
    covar_results(None, recs[:4], threshold=0.9)
    (cc, cov, stats, _), t_c = _timed(lambda: covar_results(None, recs, threshold=0.9))
    pairs = frames * (frames + 1) // 2
    return {"workload": "quality", "frames": frames, "gpu_rftf_seconds": t_gr,
            "rftf_seconds": t_r, "covar_results_seconds": t_c, "covar_pairs": pairs,
            "covar_pairs_per_s": pairs / t_c, "covar_transform": 256,
            "mean_covariance": float(cov.mean())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=("single256", "raar_dm1024", "uneven", "serving", "coherence512",
                                         "quality"))
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--window", type=float, default=0.5)
    ap.add_argument("--rounds", type=int, default=None)
    ap.add_argument("--iters", type=int, default=1000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.workload == "single256":
        r = single256()
    elif a.workload == "raar_dm1024":
        r = raar_dm1024(rounds=a.rounds)
    elif a.workload == "uneven":
        r = uneven(iters=a.iters)
    elif a.workload == "coherence512":
        r = coherence512()
    elif a.workload == "quality":
        r = quality()
    else:
        r = serving(rate=a.rate, window=a.window)
    line = json.dumps(r)
    print(line)
    if a.out:
        with open(a.out, "a") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
