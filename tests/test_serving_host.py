"""Host logic of the continuous-batching service (no GPU: a fake engine)."""
import numpy as np
import torch

from oracle import phasing_oracle as O


class FakeEngine:
    """Records each round's trials instead of launching kernels."""

    def __init__(self):
        self.calls = []

    def solve(self, specs, stream=None):
        self.calls.append([(s.n, s.iterations, s.random_phase, s.save is not None) for s in specs])
        for s in specs:
            s.psi += 1  # one mark per round
            if s.save is not None:
                s.save.fill_(s.psi.real.max().item())


def _req(rid, N=16, iters=10, trials=2, arrival=0.0, order=(("hio", 3), ("er", 1))):
    from als_speckle_b200.serving import Request
    M = np.ones((N, N), np.float32)
    S = np.zeros((N, N), np.float32)
    S[4:12, 4:12] = 1
    return Request(rid=rid, modulus=M, support=S, iterations=iters, trials=trials, order=order,
                   arrival=arrival)


def test_rotated_order_walks_the_cyclic_list():
    from als_speckle_b200.serving import rotated_order
    from als_speckle_b200.engine import expand_runs
    order = (("hio", 5), ("er", 2), ("dm", 1))
    algs, counts = expand_runs(order)
    flat = [a for a, c in zip(algs, counts) for _ in range(c)]
    names = O.expand_order(order)
    for off in range(0, 17):
        rot = rotated_order(flat, off)
        got = [n for n, c in rot for _ in range(c)]
        assert got == [names[(off + i) % len(names)] for i in range(len(names))]


def test_rounds_chunks_and_first_chunk_random_start():
    from als_speckle_b200.serving import ServingEngine
    eng = FakeEngine()
    srv = ServingEngine(device="cpu", chunk=4, engine=eng)
    srv.submit(_req(0, iters=10))
    res = srv.run(realtime=False)
    # 10 iterations in chunks of 4: 4, 4, 2; random start only in the first chunk
    assert [c[0][1] for c in eng.calls] == [4, 4, 2]
    assert [c[0][2] for c in eng.calls] == [True, False, False]
    assert [c[0][3] for c in eng.calls] == [False, False, True]
    assert res[0].save.shape[0] == 2 and srv.rounds == 3
    assert srv.trial_iterations == 20


def test_budget_admission_is_first_come_first_served():
    from als_speckle_b200.serving import ServingEngine
    eng = FakeEngine()
    one = _req(0).bytes_needed()
    srv = ServingEngine(device="cpu", chunk=5, engine=eng, hbm_budget=int(one * 1.5))
    for rid in range(3):
        srv.submit(_req(rid, iters=10))
    srv.run(realtime=False)
    # only one request fits at a time: each round carries exactly one request's trials
    assert all(len(c) == 2 for c in eng.calls)
    assert len(eng.calls) == 6 and srv.in_use == 0


def test_requests_join_as_others_finish():
    from als_speckle_b200.serving import ServingEngine
    eng = FakeEngine()
    srv = ServingEngine(device="cpu", chunk=5, engine=eng)
    srv.submit(_req(0, iters=5, trials=1))
    srv.submit(_req(1, iters=15, trials=3))
    res = srv.run(realtime=False)
    assert [len(c) for c in eng.calls] == [4, 3, 3]
    assert set(res) == {0, 1}


def test_oversize_request_rejected():
    import pytest
    from als_speckle_b200.serving import ServingEngine
    srv = ServingEngine(device="cpu", engine=FakeEngine(), hbm_budget=1000)
    with pytest.raises(ValueError):
        srv.submit(_req(0))


def test_poisson_workload_is_seeded():
    from als_speckle_b200.serving import poisson_workload
    a = poisson_workload(window=0.05, rate=200, sizes=(16, 32), probs=(0.5, 0.5), iters=(5, 9),
                         trials=(1, 3), patterns_per_size=1)
    b = poisson_workload(window=0.05, rate=200, sizes=(16, 32), probs=(0.5, 0.5), iters=(5, 9),
                         trials=(1, 3), patterns_per_size=1)
    assert [(r.n, r.iterations, r.trials, r.order, r.arrival) for r in a] == \
        [(r.n, r.iterations, r.trials, r.order, r.arrival) for r in b]
    assert all(np.diff([r.arrival for r in a]) > 0)


def test_non_finite_and_empty_inputs_rejected():
    import pytest
    from als_speckle_b200.serving import ServingEngine
    srv = ServingEngine(device="cpu", engine=FakeEngine())
    bad = _req(0)
    bad.modulus = bad.modulus.copy()
    bad.modulus[3, 3] = np.nan
    with pytest.raises(ValueError):
        srv.submit(bad)
    empty = _req(1)
    empty.support = np.zeros_like(empty.support)
    with pytest.raises(ValueError):
        srv.submit(empty)


class PoisonEngine(FakeEngine):
    """Writes NaN error sums for one trial's request, as a diverging iterate would."""

    def __init__(self, poison_n):
        super().__init__()
        self.poison_n = poison_n

    def solve(self, specs, stream=None):
        super().solve(specs, stream)
        for s in specs:
            if s.n == self.poison_n and s.errors is not None:
                s.errors.fill_(float("nan"))


def test_diverged_request_is_stopped_and_freed():
    from als_speckle_b200.serving import ServingEngine
    eng = PoisonEngine(poison_n=32)
    srv = ServingEngine(device="cpu", chunk=4, engine=eng)
    srv.submit(_req(0, N=16, iters=12))
    srv.submit(_req(1, N=32, iters=12))
    res = srv.run(realtime=False)
    assert res[1].status == "diverged" and res[0].status == "done"
    # rounds are pipelined: round 2 was enqueued before round 1's divergence
    # was read back, so the diverged request rides along once more, then stops
    assert len(eng.calls) == 3 and [len(c) for c in eng.calls] == [4, 4, 2]
    assert srv.in_use == 0


def test_cancel_pending_and_active():
    from als_speckle_b200.serving import ServingEngine
    eng = FakeEngine()
    srv = ServingEngine(device="cpu", chunk=4, engine=eng)
    srv.submit(_req(0, iters=8))
    srv.submit(_req(1, iters=8, arrival=5.0))
    assert srv.cancel(1) and not srv.cancel(7)
    srv._admit(0.0)
    assert srv.cancel(0) and srv.in_use == 0 and not srv.active
    res = srv.run(realtime=False)
    assert res[0].status == "cancelled" and res[1].status == "cancelled"
    assert eng.calls == []


def test_next_round_is_enqueued_before_the_current_one_completes():
    """Pipelined rounds: when round k is collected, round k+1 is already on
    the stream (the GPU is never left without queued work while the host
    collects results and admits requests)."""
    from als_speckle_b200.serving import ServingEngine
    eng = FakeEngine()
    srv = ServingEngine(device="cpu", chunk=4, engine=eng)
    seen = []
    orig = srv._complete

    def spy(r, t, realtime):
        seen.append((r.index, len(eng.calls)))
        return orig(r, t, realtime)

    srv._complete = spy
    srv.submit(_req(0, iters=12))
    res = srv.run(realtime=False)
    assert res[0].status == "done" and srv.in_use == 0
    # rounds 0 and 1 are collected with one more round already enqueued
    assert seen == [(0, 2), (1, 3), (2, 3)]


def test_cancel_while_a_round_is_queued_defers_the_release():
    """Cancelling a request that the queued round still uses: its result is
    "cancelled" at once, its memory is released only after that round, and it
    takes part in no round after it."""
    from als_speckle_b200.serving import ServingEngine
    eng = FakeEngine()
    srv = ServingEngine(device="cpu", chunk=4, engine=eng)
    srv.submit(_req(0, N=16, iters=16))
    srv.submit(_req(1, N=32, iters=16))
    orig = srv._complete
    seen = []

    def spy(r, t, realtime):
        out = orig(r, t, realtime)
        if r.index == 0:
            before = srv.in_use
            assert srv.cancel(1)
            # round 1 (already queued) still holds request 1's buffers
            seen.append((before, srv.in_use))
        return out

    srv._complete = spy
    res = srv.run(realtime=False)
    assert res[1].status == "cancelled" and res[0].status == "done"
    assert seen[0][0] == seen[0][1]  # nothing released while round 1 is queued
    assert srv.in_use == 0
    # request 1 (N = 32) is in rounds 0 and 1 only
    assert [sum(1 for c in call if c[0] == 32) for call in eng.calls] == [2, 2, 0, 0]
