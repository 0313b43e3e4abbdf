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
