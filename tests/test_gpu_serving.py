"""The continuous-batching service on the GPU: a request's result is the same
alone and in a mix of other requests, for any round length, and equals a
plain engine solve of the same trials."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests():
    from als_speckle_b200 import synth
    from als_speckle_b200.serving import Request
    specs = [(64, (("hio", 4), ("er", 1)), 23, 3), (128, (("raar", 1),), 17, 2),
             (256, (("dm", 2), ("er", 1)), 11, 2), (128, (("er", 1),), 9, 1),
             (64, (("sf", 3), ("hio", 2)), 30, 2)]
    out = []
    for rid, (N, order, iters, trials) in enumerate(specs):
        _, M, S = synth.pattern(N, n_ellipses=5, box=N // 4, peak=1e6, seed=rid,
                                support_edge=N // 4 + 8)
        out.append(Request(rid=rid, modulus=M, support=S, iterations=iters, trials=trials,
                           order=order, beta=0.87 if "raar" in order[0] else 0.9, seed=100 + rid))
    return out


def _serve(reqs, chunk):
    from als_speckle_b200.serving import ServingEngine
    srv = ServingEngine(chunk=chunk)
    for r in reqs:
        srv.submit(r)
    return srv.run(realtime=False)


def test_same_alone_and_in_the_mix_for_any_chunk():
    reqs = _requests()
    mix = _serve(reqs, chunk=7)
    mix2 = _serve(reqs, chunk=1000)
    for r in reqs:
        alone = _serve([r], chunk=5)[r.rid]
        for other in (mix[r.rid], mix2[r.rid]):
            assert np.array_equal(other.save, alone.save), r.rid
            assert np.allclose(other.errors, alone.errors, rtol=1e-12, atol=0), r.rid


def test_service_equals_engine_solve():
    from als_speckle_b200.engine import Engine, TrialSpec
    r = _requests()[2]  # DM + ER at 256^2, two trials
    res = _serve([r], chunk=4)[r.rid]
    M = torch.from_numpy(r.modulus).cuda()
    sup = r.support / r.support.max()
    S = torch.from_numpy(sup.astype(np.float32)).cuda()
    r0, c0, rows, cols = res.box
    eng = Engine(use_graph=False)
    psis = torch.zeros((r.trials, r.n, r.n), dtype=torch.complex64, device="cuda")
    saves = torch.zeros((r.trials, rows, cols), dtype=torch.complex64, device="cuda")
    eng.solve([TrialSpec(psi=psis[k], modulus=M, support=S, iterations=r.iterations, order=r.order,
                         beta=r.beta, random_phase=True, seed=r.seed, trial=k, box=res.box,
                         save=saves[k]) for k in range(r.trials)])
    torch.cuda.synchronize()
    assert np.array_equal(saves.cpu().numpy(), res.save)
    eng.close()


def test_final_r_factor_vs_fp64_oracle():
    """Requests of the serving mix (sizes, algorithms, trial counts drawn as
    the service's Poisson workload draws them, shortened so the FP64 oracle
    finishes in seconds): every trial's R-factor, sum||F|-M| / sum M, beside
    the oracle's from the same random-phase start.  The first three
    iterations must agree to 1e-5 relative (same start, same algorithm, no
    chaos yet: this is where a wrong start, order or beta would show); the
    final R-factor, after 12-40 chaotic iterations, to 2% (measured up to
    0.8% for a 64^2 RAAR request)."""
    from als_speckle_b200.serving import poisson_workload
    from oracle import phasing_oracle as O
    reqs = poisson_workload(n_requests=6, window=10.0, rate=50.0, seed=3, sizes=(64, 128),
                            probs=(0.5, 0.5), iters=(12, 40), trials=(1, 3), patterns_per_size=1)
    assert len(reqs) == 6
    res = _serve(reqs, chunk=16)
    rows = []
    for r in reqs:
        out = res[r.rid]
        assert out.status == "done"
        M = r.modulus.astype(np.float32)
        S = (r.support / r.support.max()).astype(np.float32)
        for k in range(r.trials):
            psi = O.seed_random_phase(M, S, r.seed, k, mode="f64")
            _, errs = O.iterate(psi, M, S, r.iterations, order=r.order, beta=r.beta, mode="f64",
                                errors=True)
            rs = out.errors[k, :, 1] / float(np.sum(M.astype(np.float64)))
            early = np.abs(rs[:3] - errs[:3, 1]) / errs[:3, 1]
            want = errs[-1][1]
            got = rs[-1]
            rows.append((r.rid, r.n, r.order[0][0], r.iterations, k, got, want))
            assert early.max() < 1e-5, (rows[-1], early)
            assert abs(got - want) <= 2e-2 * want, rows[-1]
    for row in rows:
        print("request %d N=%d %s x%d trial %d: R gpu %.6f fp64 %.6f" % row)
