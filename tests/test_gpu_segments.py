"""Trials of different sizes run as concurrent launch chains (one per size,
forked onto auxiliary streams and joined back): the results equal each trial
run alone bit for bit, eager and as a CUDA graph, and each size's chain stops
at its own longest trial."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _specs(psis, inputs, trials=None):
    from als_speckle_b200.engine import TrialSpec
    trials = trials if trials is not None else range(len(psis))
    return [TrialSpec(psi=p, modulus=M, support=S, iterations=it, order=((alg, it),), beta=0.9,
                      random_phase=True, seed=3, trial=k)
            for k, p, (M, S, it, alg) in zip(trials, psis, inputs)]


def _inputs():
    from als_speckle_b200 import synth
    out = []
    for k, (N, it, alg) in enumerate(((64, 5, "hio"), (128, 9, "raar"), (256, 3, "dm"), (64, 7, "er"))):
        _, M, S = synth.pattern(N, n_ellipses=4, box=N // 4, peak=1e6, seed=k, support_edge=N // 4 + 6)
        out.append((torch.from_numpy(M).cuda(), torch.from_numpy(S).cuda(), it, alg))
    return out


def test_concurrent_size_chains_equal_alone_and_count_launches():
    from als_speckle_b200 import _lib
    from als_speckle_b200.engine import Engine
    inp = _inputs()
    alone = []
    for k, (M, S, it, alg) in enumerate(inp):
        p = torch.zeros(M.shape, dtype=torch.complex64, device="cuda")
        eng = Engine(use_graph=False, e_per_n={})
        eng.solve(_specs([p], [(M, S, it, alg)], trials=[k]))  # the same random start as in the batch
        torch.cuda.synchronize()
        alone.append(p.cpu().numpy())
        eng.close()
    stream = torch.cuda.Stream()
    for use_graph in (False, True):
        psis = [torch.zeros(M.shape, dtype=torch.complex64, device="cuda") for M, _, _, _ in inp]
        eng = Engine(use_graph=use_graph, e_per_n={})
        with torch.cuda.stream(stream):
            for _ in range(2):  # the second call replays the captured graph
                for p in psis:
                    p.zero_()
                eng.solve(_specs(psis, inp), stream=stream)
        stream.synchronize()
        for p, want in zip(psis, alone):
            assert np.array_equal(p.cpu().numpy(), want)
        # 4 distinct moduli transposed; per size: n_iter + 1 ticks of a column
        # and a row pass, the 64^2 chain sized by its longer (7-iteration) trial
        assert int(_lib.lib.sp_engine_last_launches()) == 4 + 2 * (8 + 10 + 4)
        eng.close()


def test_graph_cache_is_trimmed_and_results_hold():
    """An engine whose launch shapes keep changing (here: iteration counts)
    drops its device's cached graphs once it holds more than MAX_GRAPHS, and
    every solve still gives the eager result."""
    from als_speckle_b200 import _lib
    from als_speckle_b200.engine import Engine
    M, S, _, _ = _inputs()[1]
    stream = torch.cuda.Stream()
    eager = Engine(use_graph=False, e_per_n={})
    graphed = Engine(use_graph=True, e_per_n={})
    graphed.MAX_GRAPHS = 2
    for iters in (2, 3, 4, 5, 6):
        a = torch.zeros(M.shape, dtype=torch.complex64, device="cuda")
        b = torch.zeros(M.shape, dtype=torch.complex64, device="cuda")
        with torch.cuda.stream(stream):
            eager.solve(_specs([a], [(M, S, iters, "hio")]), stream=stream)
            graphed.solve(_specs([b], [(M, S, iters, "hio")]), stream=stream)
        stream.synchronize()
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
        assert int(_lib.lib.sp_engine_graph_count()) <= 3
    eager.close()
    graphed.close()


def test_chains_from_threads_that_exit():
    """Concurrent chains launched from short-lived host threads (each makes
    its own auxiliary streams, released when it exits) give the same bits as
    from the main thread."""
    import threading
    from als_speckle_b200.engine import Engine
    inp = _inputs()

    def run(out):
        psis = [torch.zeros(M.shape, dtype=torch.complex64, device="cuda") for M, _, _, _ in inp]
        stream = torch.cuda.Stream()
        eng = Engine(use_graph=False, e_per_n={})
        with torch.cuda.stream(stream):
            eng.solve(_specs(psis, inp), stream=stream)
        stream.synchronize()
        eng.close()
        out.extend(p.cpu().numpy() for p in psis)

    want = []
    run(want)
    for _ in range(3):
        got, errors = [], []

        def worker():
            try:
                run(got)
            except Exception as e:  # reported below, on the main thread
                errors.append(e)

        t = threading.Thread(target=worker)
        t.start()
        t.join()
        assert not errors, errors
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
