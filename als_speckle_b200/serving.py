"""Continuous-batching reconstruction service on one GPU.

Requests (a modulus, a support, an iteration order, a trial count) arrive
over time.  The service admits them against an HBM budget as earlier
requests finish, and advances every admitted trial in rounds: one engine call
per round moves each active trial forward by up to ``chunk`` iterations, so
requests of different sizes, algorithms and lengths share the same launches
and new requests join at the next round.  Rounds are pipelined: round k+1 is
built and enqueued before round k's results are collected, so the device
always has queued work while the host reads back one batch of per-request
finiteness flags, copies finished results out on a second stream and admits
new requests.  Between rounds a trial's state is
only its psi (the Fourier work plane is rebuilt from psi at the start of a
round, which is the same arithmetic the uninterrupted iteration performs), so
a request's result does not depend on what else is in flight.

This is an addition to the reference, which has no service: its trials run
serially inside ``phasing.iterate`` (``speckle/phasing.py:181-289``).
"""
from __future__ import annotations

import contextlib
import dataclasses
import heapq
import time
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .engine import Engine, TrialSpec, expand_runs
from .masking import bounding_box

_NAMES = {_lib.SP_HIO: "hio", _lib.SP_ER: "er", _lib.SP_RAAR: "raar", _lib.SP_SF: "sf",
          _lib.SP_DM: "dm", _lib.SP_ER_CPU: "er_cpu", _lib.SP_SF_CPU: "sf_cpu"}


def rotated_order(flat: Sequence[int], offset: int):
    """Run-length order that starts at iteration ``offset`` of the cyclic list."""
    k = len(flat)
    runs = []
    for i in range(k):
        a = flat[(offset + i) % k]
        if runs and runs[-1][0] == a:
            runs[-1][1] += 1
        else:
            runs.append([a, 1])
    return [(_NAMES[a], c) for a, c in runs]


@dataclasses.dataclass
class Request:
    """One reconstruction request: ``trials`` random-phase starts iterated
    ``iterations`` times with ``order``; results are the crops of every trial
    and the per-iteration FP64 error sums."""
    rid: int
    modulus: np.ndarray
    support: np.ndarray
    iterations: int
    trials: int = 1
    order: Optional[Sequence] = None
    beta: float = 0.9
    seed: int = 0
    arrival: float = 0.0  # seconds after the service clock starts

    @property
    def n(self):
        return int(self.modulus.shape[0])

    def bytes_needed(self):
        """Device bytes while in flight: per trial psi + work plane(s) +
        errors + crop, plus the shared modulus and support."""
        N = self.n
        dm = any(a == _lib.SP_DM for a in expand_runs(self.order)[0])
        per_trial = N * N * 8 * (3 if dm else 2) + self.iterations * 16 + N * N * 8
        return self.trials * per_trial + N * N * 8


@dataclasses.dataclass
class Result:
    rid: int
    save: np.ndarray          # (trials, rows, cols) complex64 crops
    errors: np.ndarray        # (trials, iterations, 2) FP64 sums
    box: tuple
    arrival: float
    admitted: float
    finished: float
    status: str = "done"      # "done", "diverged" (non-finite error sums) or "cancelled"

    @property
    def latency(self):
        return self.finished - self.arrival


class _Active:
    def __init__(self, req: Request, device, admitted):
        self.req = req
        N = req.n
        self.M = torch.from_numpy(np.ascontiguousarray(req.modulus, np.float32)).to(device)
        sup = np.ascontiguousarray(req.support, np.float32)
        sup = sup / sup.max()
        self.S = torch.from_numpy(sup).to(device)
        bb = bounding_box(sup, pad=10)
        self.box = (int(bb[0]), int(bb[2]), int(bb[1] - bb[0]), int(bb[3] - bb[2]))
        self.psi = torch.zeros((req.trials, N, N), dtype=torch.complex64, device=device)
        self.save = torch.zeros((req.trials, self.box[2], self.box[3]), dtype=torch.complex64,
                                device=device)
        self.errors = torch.zeros((req.trials, max(1, req.iterations), 2), dtype=torch.float64,
                                  device=device)
        algs, counts = expand_runs(req.order)
        self.flat = [a for a, c in zip(algs, counts) for _ in range(c)]
        self.done = 0        # iterations whose round has completed
        self.scheduled = 0   # iterations enqueued (one round may be in flight beyond done)
        self.last_round = -1  # the latest round that uses this request's buffers
        self.dead = False    # diverged or cancelled while a round held it
        self.admitted = admitted
        self.bytes = req.bytes_needed()

    def specs(self, chunk):
        """The next round's trials: up to ``chunk`` iterations from where the
        enqueued work ends."""
        start = self.scheduled
        n = min(chunk, self.req.iterations - start)
        last = start + n >= self.req.iterations
        order = rotated_order(self.flat, start)
        out = []
        for k in range(self.req.trials):
            out.append(TrialSpec(
                psi=self.psi[k], modulus=self.M, support=self.S, iterations=n, order=order,
                beta=self.req.beta, random_phase=(start == 0), seed=self.req.seed, trial=k,
                box=self.box if last else None, save=self.save[k] if last else None,
                errors=self.errors[k, start:start + n], quirks="gpu"))
        return n, out


class _Round:
    """One enqueued engine call: its requests with their iteration counts,
    the per-request finiteness flags (pinned host copy) and the event that
    marks the round's end on the service stream."""

    def __init__(self, index, members, flags_host, event):
        self.index = index
        self.members = members  # [(active, n)]
        self.flags_host = flags_host
        self.event = event

    def wait(self):
        if self.event is not None:
            self.event.synchronize()
        return [bool(v) for v in self.flags_host.tolist()]


class ServingEngine:
    """Admit requests against ``hbm_budget`` bytes and advance them in rounds
    of up to ``chunk`` iterations (continuous batching)."""

    # cached launch graphs kept before the service drops them (each active set
    # of requests has its own launch shape, hence its own graph)
    MAX_GRAPHS = 32

    def __init__(self, device=None, hbm_budget=120 << 30, chunk=64, engine: Engine = None,
                 max_active_trials=4096, use_graph=True):
        self.device = torch.device(device if device is not None else "cuda")
        self.budget = int(hbm_budget)
        self.chunk = int(chunk)
        # rounds whose active set did not change replay the previous round's
        # CUDA graph (one launch for the round's 2 x chunk kernels)
        self.engine = engine or Engine(device=self.device, use_graph=use_graph)
        self.max_active_trials = max_active_trials
        self.pending: List = []     # heap of (arrival, rid, request)
        self.active: List[_Active] = []
        self.results: Dict[int, Result] = {}
        self.in_use = 0
        self.rounds = 0
        self.trial_iterations = 0
        cuda = self.device.type == "cuda"
        self.stream = torch.cuda.Stream(self.device) if cuda else None
        self.copy_stream = torch.cuda.Stream(self.device) if cuda else None
        self._inflight: Optional[_Round] = None
        self._retiring: List[_Active] = []

    def _on_stream(self):
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def submit(self, req: Request):
        """Queue a request.  Rejected at once: a request larger than the
        whole budget, or one whose modulus or support is not finite."""
        if req.bytes_needed() > self.budget:
            raise ValueError("request %d needs %d bytes, more than the whole budget" % (req.rid, req.bytes_needed()))
        if not (np.all(np.isfinite(req.modulus)) and np.all(np.isfinite(req.support))):
            raise ValueError("request %d: modulus and support must be finite" % req.rid)
        if not np.any(req.support > 0):
            raise ValueError("request %d: empty support" % req.rid)
        heapq.heappush(self.pending, (req.arrival, req.rid, req))

    def cancel(self, rid: int):
        """Drop a request whether it is waiting or in flight; its result is
        recorded with status "cancelled" and its memory is released (once no
        enqueued round uses it any more)."""
        for i, (_, r, req) in enumerate(self.pending):
            if r == rid:
                self.pending.pop(i)
                heapq.heapify(self.pending)
                self.results[rid] = Result(rid, np.zeros((0, 0, 0), np.complex64),
                                           np.zeros((0, 0, 2)), (0, 0, 0, 0), req.arrival, -1.0, -1.0,
                                           "cancelled")
                return True
        for a in self.active:
            if a.req.rid == rid:
                self.active.remove(a)
                self.results[rid] = Result(rid, np.zeros((0, 0, 0), np.complex64),
                                           np.zeros((0, 0, 2)), a.box, a.req.arrival, a.admitted,
                                           -1.0, "cancelled")
                self._retire(a)
                return True
        return False

    def _retire(self, a):
        """Release a request's memory now, or after the last enqueued round
        that uses its buffers."""
        a.dead = True
        if self._inflight is not None and a.last_round >= self._inflight.index:
            self._retiring.append(a)
        else:
            self.in_use -= a.bytes

    def _admit(self, now):
        trials = sum(a.req.trials for a in self.active)
        while self.pending and self.pending[0][0] <= now:
            req = self.pending[0][2]
            if self.in_use + req.bytes_needed() > self.budget or \
                    trials + req.trials > self.max_active_trials:
                break  # first come, first served: wait until memory frees up
            heapq.heappop(self.pending)
            with self._on_stream():
                a = _Active(req, self.device, now)
            self.active.append(a)
            self.in_use += a.bytes
            trials += req.trials

    def _enqueue(self, members):
        """Enqueue one round: the engine call and the per-request finiteness
        flags of its last iteration (copied to pinned host memory behind it).
        Returns the round without waiting for it."""
        specs, used = [], []
        for a in members:
            n, sp = a.specs(self.chunk)
            a.scheduled += n
            a.last_round = self.rounds
            specs.extend(sp)
            used.append((a, n))
            self.trial_iterations += n * a.req.trials
        with self._on_stream():
            self.engine.solve(specs, stream=self.stream)
            flags = torch.stack([torch.isfinite(a.errors[:, a.scheduled - 1]).all()
                                 for a, n in used])
            event = None
            if self.stream is not None:
                host = torch.empty(flags.shape, dtype=torch.bool, pin_memory=True)
                host.copy_(flags, non_blocking=True)
                event = torch.cuda.Event()
                event.record(self.stream)
            else:
                host = flags
        r = _Round(self.rounds, used, host, event)
        self.rounds += 1
        return r

    def _host_copy(self, t, event):
        """Copy a result buffer to the host behind ``event`` on the copy stream,
        so the round enqueued after it keeps running."""
        if self.copy_stream is None:
            return t.numpy().copy()
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(event)
            out = t.to("cpu", non_blocking=True)
        self.copy_stream.synchronize()
        return out.numpy()

    def _complete(self, r: _Round, t, realtime):
        """Account for a finished round: requests whose last iteration was in
        it are done (their crops and error sums are copied out), requests whose
        error sums turned non-finite are stopped."""
        finite = r.wait()
        # trim the graph cache of launch shapes that have come and gone; the
        # queued round must finish first (one pipeline bubble per trim)
        if getattr(self.engine, "use_graph", False) and \
                _lib.lib.sp_engine_graph_count() > self.MAX_GRAPHS:
            torch.cuda.synchronize(self.device)
            with torch.cuda.device(self.device):
                _lib.call("sp_engine_release_device_graphs")
        for (a, n), ok in zip(r.members, finite):
            a.done += n
            if a.dead:
                continue
            status = None
            if not ok:
                status = "diverged"  # the iterate has become non-finite
            elif a.done >= a.req.iterations:
                status = "done"
            if status is None:
                continue
            self.results[a.req.rid] = Result(
                a.req.rid, self._host_copy(a.save, r.event), self._host_copy(a.errors, r.event),
                a.box, a.req.arrival if realtime else 0.0, a.admitted if realtime else 0.0, t,
                status)
            self.active.remove(a)
            self._retire(a)
        # memory of stopped requests whose last round has now finished
        keep = []
        for a in self._retiring:
            if a.last_round <= r.index:
                self.in_use -= a.bytes
            else:
                keep.append(a)
        self._retiring = keep

    def run(self, clock=None, realtime=True):
        """Serve until every submitted request is finished.  With
        ``realtime`` the arrival times are honoured against ``clock``
        (seconds); otherwise every request is available immediately.

        Rounds are pipelined: the next round is built and enqueued while the
        current one runs (which trials finish when is known in advance; only
        a divergence is learnt afterwards, and costs the diverged request at
        most one extra round), so the GPU is not left idle while the host
        collects results and admits requests.  Returns the results by request
        id."""
        clock = clock or time.perf_counter
        t0 = clock()
        now = lambda: (clock() - t0) if realtime else float("inf")
        while self.pending or self.active or self._inflight is not None:
            self._admit(now())
            ready = [a for a in self.active if not a.dead and a.scheduled < a.req.iterations]
            nxt = self._enqueue(ready) if ready else None
            if self._inflight is not None:
                done, self._inflight = self._inflight, nxt
                self._complete(done, clock() - t0, realtime)
            elif nxt is not None:
                self._inflight = nxt
            else:
                # idle until the next arrival
                wait = self.pending[0][0] - now() if self.pending else 0.0
                if wait > 0:
                    time.sleep(min(wait, 0.01))
        return self.results


def poisson_workload(n_requests=None, window=1.0, rate=200.0, seed=0, sizes=(256, 512, 1024, 2048),
                     probs=(0.4, 0.3, 0.2, 0.1), iters=(200, 2000), trials=(1, 16),
                     patterns_per_size=2):
    """Seeded request stream: Poisson arrivals at ``rate`` per second over
    ``window`` seconds; sizes, algorithm (uniform over HIO/ER/RAAR/DM),
    iteration count and trial count drawn as given.  Patterns follow the
    large-instance recipe (ellipses in an N/4 box, 1e7 photons, Poisson noise),
    a few per size reused across requests."""
    from . import synth
    rng = np.random.default_rng(seed)
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window or (n_requests is not None and len(arrivals) >= n_requests):
            break
        arrivals.append(t)
    pats = {}
    for N in sizes:
        for p in range(patterns_per_size):
            _, M, S = synth.pattern(N, n_ellipses=60, box=N // 4, peak=1e7, seed=1000 * N + p,
                                    support_edge=int(round(1.25 * (N // 4))))
            pats[(N, p)] = (M, S)
    algs = ("hio", "er", "raar", "dm")
    reqs = []
    for i, ta in enumerate(arrivals):
        N = int(rng.choice(sizes, p=probs))
        M, S = pats[(N, int(rng.integers(patterns_per_size)))]
        alg = algs[int(rng.integers(4))]
        beta = 0.87 if alg == "raar" else 0.9
        reqs.append(Request(rid=i, modulus=M, support=S,
                            iterations=int(rng.integers(iters[0], iters[1] + 1)),
                            trials=int(rng.integers(trials[0], trials[1] + 1)),
                            order=((alg, 1),), beta=beta, seed=int(rng.integers(1 << 31)),
                            arrival=ta))
    return reqs
