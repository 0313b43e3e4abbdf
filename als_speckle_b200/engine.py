"""Batched phase-retrieval engine: many trials per call through sp_engine_run.

``solve`` advances any number of independent trials (uneven sizes,
algorithms, iteration counts) with the fused CUDA engine.  Each trial is a
``TrialSpec``; device arrays are torch tensors.  This is the batched form of
``phasing.iterate`` (reference ``speckle/phasing.py:181-289``), which in the
reference runs one trial at a time.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional, Sequence

import torch

from . import _lib
from ._lib import ALG_CODES, CPU_QUIRK_CODES, SP_MAX_RUNS, call, ptr, stream_ptr


# explicit names of the CPU-branch forms (phasing.py:1257, :1284)
_RAW_CODES = {"er_cpu": _lib.SP_ER_CPU, "sf_cpu": _lib.SP_SF_CPU}


def expand_runs(order=None, quirks="gpu"):
    """(alg codes, counts) for an ``order`` as ``phasing.iterate`` takes it.

    Default ``(('hio',99),('er',1))`` (``phasing.py:244-257``).  Adjacent
    entries with the same algorithm are merged; at most 8 runs are kept.
    """
    if order is None:
        order = (("hio", 99), ("er", 1))
    algs, counts = [], []
    for entry in order:
        try:
            name = str(entry[0]).lower()
            count = int(entry[1])
        except (IndexError, TypeError, ValueError):
            raise ValueError("entry %r in iteration order is improperly formatted" % (entry,))
        if name in _RAW_CODES:
            code = _RAW_CODES[name]
        elif name not in ALG_CODES:
            raise ValueError("real space enforcement algorithm %s is unknown" % name)
        else:
            code = CPU_QUIRK_CODES.get(name, ALG_CODES[name]) if quirks == "cpu" else ALG_CODES[name]
        if count <= 0:
            continue
        if algs and algs[-1] == code:
            counts[-1] += count
        else:
            algs.append(code)
            counts.append(count)
    if not algs:
        raise ValueError("iteration order is empty")
    if len(algs) > SP_MAX_RUNS:
        raise ValueError("iteration order has %d runs; at most %d are supported" % (len(algs), SP_MAX_RUNS))
    return algs, counts


@dataclasses.dataclass
class TrialSpec:
    """One independent reconstruction on the device."""
    psi: torch.Tensor                      # complex64 (N, N), in/out psi_in
    modulus: torch.Tensor                  # float32 (N, N), corner-centred
    support: torch.Tensor                  # float32 (N, N) in [0, 1]
    iterations: int
    order: Optional[Sequence] = None
    beta: float = 0.8
    random_phase: bool = False             # start from S*IFFT(M exp(i phi)) instead of psi
    seed: int = 0
    trial: int = 0
    box: Optional[tuple] = None            # (r0, c0, rows, cols) savebuffer crop
    save: Optional[torch.Tensor] = None    # complex64 (rows, cols) destination
    errors: Optional[torch.Tensor] = None  # float64 (iterations, 2) per-iteration sums
    quirks: str = "gpu"
    ipsf: Optional[torch.Tensor] = None    # complex64 (N, N): partially coherent projection
    spectrum: Optional[tuple] = None       # (rescales, weights) float32 CUDA tensors (n,)

    @property
    def n(self):
        return int(self.modulus.shape[-1])


def _to_struct(t: TrialSpec) -> _lib.sp_trial:
    s = _lib.sp_trial()
    N = t.n
    for name, x, dt in (("psi", t.psi, torch.complex64), ("modulus", t.modulus, torch.float32),
                        ("support", t.support, torch.float32)):
        if x.dtype != dt or tuple(x.shape) != (N, N) or not x.is_cuda or not x.is_contiguous():
            raise ValueError("%s must be a contiguous CUDA %s tensor of shape (%d, %d)" % (name, dt, N, N))
    s.n = N
    s.n_iter = int(t.iterations)
    algs, counts = expand_runs(t.order, t.quirks)
    s.n_runs = len(algs)
    for i, (a, c) in enumerate(zip(algs, counts)):
        s.run_alg[i] = a
        s.run_count[i] = c
    s.beta = float(t.beta)
    s.init = _lib.SP_INIT_RANDOM_PHASE if t.random_phase else _lib.SP_INIT_GIVEN
    s.seed = int(t.seed) & 0xFFFFFFFF
    s.trial = int(t.trial) & 0xFFFFFFFF
    s.psi_dev = t.psi.data_ptr()
    s.modulus_dev = t.modulus.data_ptr()
    s.support_dev = t.support.data_ptr()
    if t.save is not None:
        r0, c0, rows, cols = t.box
        if t.save.dtype != torch.complex64 or tuple(t.save.shape) != (rows, cols) or not t.save.is_contiguous():
            raise ValueError("save must be a contiguous complex64 tensor of shape (rows, cols)")
        s.r0, s.c0, s.rows, s.cols = int(r0), int(c0), int(rows), int(cols)
        s.save_dev = t.save.data_ptr()
    if t.errors is not None:
        if t.errors.dtype != torch.float64 or t.errors.numel() < 2 * max(1, t.iterations) or not t.errors.is_contiguous():
            raise ValueError("errors must be a contiguous float64 tensor with 2*iterations entries")
        s.errors_dev = t.errors.data_ptr()
    if t.ipsf is not None:
        x = t.ipsf
        if x.dtype != torch.complex64 or tuple(x.shape) != (N, N) or not x.is_cuda or not x.is_contiguous():
            raise ValueError("ipsf must be a contiguous CUDA complex64 tensor of shape (%d, %d)" % (N, N))
        s.ipsf_dev = x.data_ptr()
    if t.spectrum is not None:
        r, w = t.spectrum
        for x in (r, w):
            if x.dtype != torch.float32 or not x.is_cuda or not x.is_contiguous() or x.dim() != 1:
                raise ValueError("spectrum must be two contiguous CUDA float32 vectors")
        if r.numel() != w.numel() or r.numel() == 0:
            raise ValueError("spectrum rescales and weights must have the same, non-zero length")
        s.spectrum_rescale_dev = r.data_ptr()
        s.spectrum_weight_dev = w.data_ptr()
        s.spectrum_n = r.numel()
    return s


class Engine:
    """Holds the workspace and options for repeated solves on one device.

    ``l2_group_bytes`` groups trials so each group's planes stay in L2 while it
    iterates; ``use_graph`` captures each group's launches in a CUDA graph
    (cached per workspace and shape); ``e_per_n`` maps N to the per-thread
    radix E (16 or 32).  Left as None it is the autotuner's table for this
    device (``autotune.json``), so every caller gets the tuned E per size;
    ``{}`` leaves every size to the library's default (E = 32).  The choice
    depends only on N, never on how many trials a call carries, so a trial's
    result is the same alone and batched with others.
    """

    def __init__(self, device=None, l2_group_bytes=0, use_graph=True, e_per_n=None,
                 ctas_per_sm=0):
        self.device = torch.device(device if device is not None else "cuda")
        self.l2_group_bytes = int(l2_group_bytes)
        self.use_graph = bool(use_graph)
        if e_per_n is None:
            e_per_n = {}
            if torch.cuda.is_available():
                from . import autotune
                with torch.cuda.device(self.device):
                    e_per_n = autotune.tuned_e_per_n()
        self.e_per_n = dict(e_per_n)
        self.ctas_per_sm = int(ctas_per_sm)
        self._ws = None

    def opts(self):
        o = _lib.sp_run_opts()
        o.l2_group_bytes = self.l2_group_bytes
        o.use_graph = 1 if self.use_graph else 0
        o.ctas_per_sm = self.ctas_per_sm
        for N, E in self.e_per_n.items():
            o.e_per_logn[int(N).bit_length() - 1] = int(E)
        return o

    def workspace(self, nbytes):
        if self._ws is None or self._ws.numel() < nbytes:
            if self._ws is not None:
                torch.cuda.synchronize(self.device)
                call("sp_engine_release_graphs")
            self._ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        return self._ws

    # cached CUDA graphs (one per workspace and launch shape, process-wide)
    # kept before solve drops them all
    MAX_GRAPHS = 64

    def solve(self, trials: Sequence[TrialSpec], stream=None):
        """Enqueue every trial's iterations on ``stream`` (asynchronous)."""
        if not trials:
            return
        if self.use_graph and _lib.lib.sp_engine_graph_count() > self.MAX_GRAPHS:
            # a long-lived caller whose launch shapes keep changing (different
            # iteration counts, trial mixes): drop this device's cached graphs
            # once nothing runs on it
            torch.cuda.synchronize(self.device)
            with torch.cuda.device(self.device):
                call("sp_engine_release_device_graphs")
        arr = (_lib.sp_trial * len(trials))(*[_to_struct(t) for t in trials])
        need = C.c_size_t(0)
        call("sp_engine_workspace_size", arr, len(trials), C.byref(need))
        ws = self.workspace(need.value)
        opts = self.opts()
        with torch.cuda.device(self.device):
            call("sp_engine_run", arr, len(trials), ptr(ws), ws.numel(), C.byref(opts),
                 stream_ptr(stream))

    def close(self):
        if self._ws is not None:
            torch.cuda.synchronize(self.device)
            call("sp_engine_release_graphs")
            self._ws = None


def solve(trials: Sequence[TrialSpec], engine: Optional[Engine] = None, stream=None):
    """One-shot batched solve with a temporary Engine (graphs off)."""
    eng = engine or Engine(device=trials[0].psi.device if trials else None, use_graph=False)
    eng.solve(trials, stream)
    return eng
