"""Benchmark: batched HIO phase retrieval, 512^2 x 128 trials (500 HIO + 50 ER).

One step = one full reconstruction job: 128 seeded uniform-random-phase
starts iterated 500 HIO (beta 0.9) + 50 ER through the fused engine, the crop
saved per trial, then global-phase alignment, the average and the PRTF, all
on the device.  The metric is trial-iterations per second over the job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own 128-trial job (weak scaling, no
collective on the data path); the printed value is the sum over ranks
divided by the slowest rank's time.  ``--mode strong`` instead splits one
128-trial job over the ranks (distributed.solve_sharded: one broadcast and
two all-reduces after the iterations).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 512
TRIALS = 128
ORDER = (("hio", 500), ("er", 50))
ITERS = 550
BETA = 0.9
UPSAMPLE = 64  # subpixel registration to 1/64 pixel
BYTES_PER_PX = 24  # algorithmic bytes per trial-iteration per pixel: psi r+w 16, modulus 4, support 4
METRIC = "HIO trial-iterations/s, 512^2 x 128 trials (500 HIO + 50 ER), batched"
UNIT = "trial-iter/s"
WORKLOAD = "hio_512x128: N=512, 40 ellipses in a 128^2 box, 1e6 photons Poisson, support 160^2"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
        except Exception:
            rows = []
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


# ------------------------------------------------------------- CPU side
REF_ROOT = os.path.join(ROOT, "baseline", "_ref")


def reference_available():
    """The reference install (pip --target baseline/_ref) is present."""
    return os.path.exists(os.path.join(REF_ROOT, "speckle", "phasing.py"))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


_W = {}


def _cpu_init(kind):
    """Pool initialiser: the pattern and, for kind "reference", the
    reference's own phasing object (speckle/phasing.py loaded unmodified from
    baseline/_ref through the Python-3 loader, numpy branch); for kind "port"
    the oracle's bit-exact restatement of that numpy arithmetic."""
    import contextlib
    import io
    from als_speckle_b200 import synth
    from oracle import phasing_oracle as O
    obj, M, S = synth.config_pattern("hio_512x128", seed=0)
    _W.update(kind=kind, M=M, S=S, O=O)
    if kind == "reference":
        os.environ["SPECKLE_REF_ROOT"] = REF_ROOT
        from oracle import refshim
        ref = refshim.load_reference()
        with contextlib.redirect_stdout(io.StringIO()):
            r = ref.phasing.phasing(force_cpu=True, force_np_fft=True)
            r.load(modulus=M, support=S, numtrials=1)
        _W["r"] = r


def _cpu_task(args):
    """One trial x ``iters`` HIO iterations from a random-phase start; only
    the iteration itself is timed."""
    import contextlib
    import io
    trial, iters = args
    O, M, S = _W["O"], _W["M"], _W["S"]
    psi = O.seed_random_phase(M, S, 1234, trial, mode="ref64")
    if _W["kind"] == "reference":
        r = _W["r"]
        r.psi_in = psi
        r.numtrial = 0
        with contextlib.redirect_stdout(io.StringIO()):
            t0 = time.perf_counter()
            r.iterate(iters, order=(("hio", iters),), beta=BETA)
            dt = time.perf_counter() - t0
    else:
        t0 = time.perf_counter()
        O.iterate(psi, M, S, iters, order=(("hio", iters),), beta=BETA, quirks="cpu", mode="ref64")
        dt = time.perf_counter() - t0
    return dt


class CpuPool:
    """A persistent pool of one process per host core, each holding its
    inputs (and the reference's phasing object), so a timed step is only the
    iterations: each of ``procs`` tasks runs one trial concurrently."""

    def __init__(self, procs=None):
        import multiprocessing as mp
        self.kind = "reference" if reference_available() else "port"
        self.procs = procs or max(1, min(cpu_cores(), 64))
        self.pool = mp.get_context("spawn").Pool(self.procs, initializer=_cpu_init,
                                                 initargs=(self.kind,))
        self.pool.map(_cpu_task, [(k, 1) for k in range(self.procs)], chunksize=1)  # warm

    def run(self, iters):
        """(trial-iterations/s over the step, step wall seconds, task times)"""
        t0 = time.perf_counter()
        times = self.pool.map(_cpu_task, [(k, iters) for k in range(self.procs)], chunksize=1)
        wall = time.perf_counter() - t0
        return self.procs * iters / wall, wall, times

    def close(self):
        self.pool.close()
        self.pool.join()

    def describe(self, iters):
        what = ("the reference's own numpy iteration (speckle/phasing.py, phasing(force_cpu=True, "
                "force_np_fft=True).iterate, loaded from baseline/_ref)" if self.kind == "reference"
                else "the oracle's bit-exact restatement of the reference's numpy complex64 "
                     "iteration (the reference install is absent)")
        return ("%d processes x 1 trial x %d HIO iterations at 512^2 per step, %s, on %s"
                % (self.procs, iters, what, cpu_model()))


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline(iters=24):
    """The host-core baseline: one trial per core at once (the line's value),
    and one process alone (numpy's FFT is single-threaded)."""
    pool = CpuPool()
    try:
        value, wall, _ = pool.run(iters)
        alone = pool.pool.apply(_cpu_task, ((0, iters),))
    finally:
        pool.close()
    return {"value": value, "unit": UNIT, "cores": pool.procs, "kind": pool.kind,
            "sample": pool.describe(iters) + ", %.1f s wall" % wall,
            "single_process": {"value": iters / alone, "unit": UNIT, "cores": 1,
                               "sample": "1 trial x %d HIO iterations at 512^2, alone" % iters}}


def _precision_worker(args):
    """One trial of the benchmark job (the same random-phase start) iterated
    by the oracle in FP64 (mode "f64") or in numpy complex64 (mode "ref64",
    the reference's CPU arithmetic), cropped: the checkers of the FP32
    average."""
    seed, trial, box, mode = args
    from als_speckle_b200 import synth
    from oracle import phasing_oracle as O
    obj, M, S = synth.config_pattern("hio_512x128", seed=0)
    psi = O.seed_random_phase(M, S, seed, trial, mode=mode)
    psi = O.iterate(psi, M, S, ITERS, order=ORDER, beta=BETA, quirks="gpu", mode=mode)
    r0, c0, rows, cols = box
    return np.asarray(psi[r0:r0 + rows, c0:c0 + cols], np.complex128)


def _truth_error(avg, truth, reg_n):
    """Relative error of a reconstruction against the true object after
    registration (subpixel shift), a complex least-squares scale (the
    global phase and the photon scaling) and the twin ambiguity (the
    conjugate point-inverted image is an equally valid solution)."""
    from oracle import phasing_oracle as O
    best = np.inf
    for cand in (avg, np.conj(avg[::-1, ::-1])):
        _, al = O.register_subpixel(cand[None], truth, N=reg_n, upsample=UPSAMPLE)
        a = al[0]
        c = np.vdot(truth, a) / np.vdot(truth, truth)
        best = min(best, float(np.linalg.norm(a - c * truth) / np.linalg.norm(c * truth)))
    return best


def precision_check(job, trials=4):
    """The averaged reconstruction in FP32 against FP64, on the job's first
    ``trials`` trials from the same starts (part of the CPU-baseline leg; the
    oracle runs them in spawned processes).

    * value: ||avg_gpu - avg_fp64|| / ||avg_fp64||, both aligned to trial 0
      (global phase + subpixel shift) and averaged;
    * numpy_c64_vs_fp64: the same for the reference's complex64 numpy
      arithmetic -- HIO iterations are chaotic, so FP32 and FP64 runs from one
      start drift apart (their R-factor curves differ by ~1e-4 after 50
      iterations and ~1e-2 after a few hundred) and end at different,
      equally valid solutions; this figure is that drift for the reference's
      own precision, the yardstick for the first;
    * err_vs_truth: each average against the true (synthetic) object after
      registration, a complex scale and the twin choice -- the precision-
      independent quality of the result."""
    import multiprocessing as mp
    from als_speckle_b200 import synth
    from oracle import phasing_oracle as O
    t0 = time.perf_counter()
    args = [(job.seed, k, job.box, mode) for mode in ("f64", "ref64") for k in range(trials)]
    with mp.get_context("spawn").Pool(len(args)) as pool:
        frames = pool.map(_precision_worker, args)
    f64, c64 = np.stack(frames[:trials]), np.stack(frames[trials:])

    def average(fr):
        fr = O.align_global_phase(fr)
        _, fr = O.register_subpixel(fr, fr[0], N=job.reg_n, upsample=UPSAMPLE)
        return fr.mean(axis=0)

    avg64, avgc64 = average(f64), average(c64)
    save = job.save.cpu().numpy().astype(np.complex128)  # aligned to trial 0 already
    avg32 = save[:trials].mean(axis=0)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    obj, _, _ = synth.config_pattern("hio_512x128", seed=0)
    r0, c0, rows, cols = job.box
    truth = np.asarray(obj[r0:r0 + rows, c0:c0 + cols], np.complex128)
    return {"value": rel(avg32, avg64), "trials": trials,
            "numpy_c64_vs_fp64": rel(avgc64, avg64),
            "err_vs_truth": {"gpu_fp32_all_%d" % TRIALS: _truth_error(save.mean(axis=0), truth, job.reg_n),
                             "gpu_fp32": _truth_error(avg32, truth, job.reg_n),
                             "fp64": _truth_error(avg64, truth, job.reg_n),
                             "numpy_c64": _truth_error(avgc64, truth, job.reg_n)},
            "seconds": round(time.perf_counter() - t0, 1),
            "what": "average of the first %d trials (500 HIO + 50 ER from the same starts, aligned "
                    "to trial 0): GPU FP32 vs the oracle's FP64 (value) and numpy complex64 vs FP64; "
                    "errors against the true object after registration, complex scale and twin "
                    "choice" % trials}


# ------------------------------------------------------------ GPU side
def build_inputs(torch, device):
    from als_speckle_b200 import synth
    from als_speckle_b200.masking import bounding_box
    obj, M, S = synth.config_pattern("hio_512x128", seed=0)
    bb = bounding_box(S, pad=10)
    box = (int(bb[0]), int(bb[2]), int(bb[1] - bb[0]), int(bb[3] - bb[2]))
    return M, S, box


class Job:
    """Device-resident job: buffers allocated once, one step = full solve."""

    def __init__(self, torch, device, M, S, box, engine, seed):
        from als_speckle_b200.engine import TrialSpec
        self.torch = torch
        self.device = device
        self.M = torch.from_numpy(M).to(device)
        self.S = torch.from_numpy(S).to(device)
        self.box = box
        r0, c0, rows, cols = box
        self.psis = torch.empty((TRIALS, N, N), dtype=torch.complex64, device=device)
        self.save = torch.empty((TRIALS, rows, cols), dtype=torch.complex64, device=device)
        self.errs = torch.zeros((TRIALS, ITERS, 2), dtype=torch.float64, device=device)
        self.engine = engine
        self.seed = seed
        self.specs = [TrialSpec(psi=self.psis[k], modulus=self.M, support=self.S, iterations=ITERS,
                                order=ORDER, beta=BETA, random_phase=True, seed=seed, trial=k,
                                box=box, save=self.save[k], errors=self.errs[k])
                      for k in range(TRIALS)]
        self.prtf_work = torch.empty((TRIALS, N, N), dtype=torch.complex64, device=device)
        self.prtf = torch.empty((N, N), dtype=torch.float32, device=device)
        self.avg = torch.empty((rows, cols), dtype=torch.complex64, device=device)
        self.sums = torch.empty(5 * TRIALS, dtype=torch.float64, device=device)
        self.angles = torch.empty(TRIALS, dtype=torch.float64, device=device)
        # subpixel registration to trial 0: crops in the next power-of-two transform
        from als_speckle_b200._lib import call
        import ctypes
        self.reg_n = 1 << (max(rows, cols) - 1).bit_length()
        nb = ctypes.c_size_t(0)
        call("sp_register_workspace_size", TRIALS, self.reg_n, UPSAMPLE, ctypes.byref(nb))
        self.reg_bytes = nb.value
        self.reg_work = torch.empty(nb.value, dtype=torch.uint8, device=device)
        self.shifts = torch.empty((TRIALS, 3), dtype=torch.float64, device=device)
        self.launches = 0

    def step(self):
        from als_speckle_b200._lib import call, ptr, stream_ptr, lib
        self.engine.solve(self.specs)
        eng = int(lib.sp_engine_last_launches())
        r0, c0, rows, cols = self.box
        s = stream_ptr()
        call("sp_align_global_phase", ptr(self.save), TRIALS, rows * cols, ptr(self.angles),
             ptr(self.sums), s)
        # subpixel shift and global phase of every trial onto trial 0, in place
        call("sp_register_subpixel", ptr(self.save), TRIALS, rows, cols, ptr(self.save[0]),
             self.reg_n, UPSAMPLE, ptr(self.reg_work), self.reg_bytes, ptr(self.shifts),
             ptr(self.save), s)
        call("sp_mean_frames", ptr(self.save), TRIALS, rows * cols, ptr(self.avg), s)
        call("sp_prtf", ptr(self.save), TRIALS, rows, cols, N, ptr(self.prtf_work), ptr(self.prtf), s)
        # align: 2 kernels; register: 2 embeds, 3 two-pass FFTs, cross, argmax,
        # table, 2 upsampled DFTs, finish, shift, crop; mean: 1; prtf: embed +
        # 2 FFT passes + accumulate
        self.launches = eng + 2 + 16 + 1 + 4

    def r_factor(self):
        m = self.M.double()
        return (self.errs[:, -1, 1] / m.sum()).cpu().numpy()


class ShardedJob:
    """The same 128-trial job split across the ranks (strong scaling):
    ``distributed.solve_sharded`` -- each rank iterates its share, trial 0's
    owner broadcasts its phase-aligned crop, every rank registers to it, and
    the frame and PRTF-phasor sums are all-reduced before the average and
    the PRTF are finished."""

    def __init__(self, torch, device, M, S, box, engine, seed):
        from als_speckle_b200.distributed import DeviceOps
        self.M = torch.from_numpy(M).to(device)
        self.S = torch.from_numpy(S).to(device)
        self.box = box
        self.seed = seed
        self.ops = DeviceOps(engine=engine)
        self.launches = 0
        self.mine = []

    def step(self):
        from als_speckle_b200._lib import lib
        from als_speckle_b200.distributed import solve_sharded
        self.avg, self.prtf, count, self.mine = solve_sharded(
            self.M, self.S, TRIALS, ITERS, order=ORDER, beta=BETA, seed=self.seed, box=self.box,
            N_prtf=N, upsample=UPSAMPLE, ops=self.ops)
        self.launches = int(lib.sp_engine_last_launches()) + 2 + 16 + 1 + 5

    def r_factor(self):
        return None  # the sharded solve keeps no per-iteration error sums


def flush_l2(torch, buf):
    buf.fill_(1)


def kernel_pass_times(torch, engine, job, reps=20):
    """Average device time of one column-pass and one row-pass launch over
    one L2 group, measured with CUDA events on the launching stream."""
    from als_speckle_b200.engine import Engine
    from als_speckle_b200 import _lib
    group = max(1, int(engine.l2_group_bytes // (2 * N * N * 8))) if engine.l2_group_bytes else TRIALS
    group = min(group, TRIALS)
    eng = Engine(device=job.device, use_graph=False, l2_group_bytes=0, e_per_n=engine.e_per_n)
    specs = job.specs[:group]
    # one solve of 2 iterations gives launches C0 R0 C1 R1 C2 R2; time solves
    # of 1 and 1+reps iterations and difference them to isolate steady ticks
    import copy
    def timed(iters):
        sp = [copy.copy(s) for s in specs]
        for s in sp:
            s.iterations = iters
            s.order = (("hio", iters),)
            s.errors = None
            s.save = None
        eng.solve(sp)  # warm
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        eng.solve(sp)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3
    t1 = timed(1)
    tn = timed(1 + reps)
    eng.close()
    per_tick = (tn - t1) / reps
    return per_tick, group


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    # a dedicated stream: CUDA graphs cannot be captured on the legacy default stream
    torch.cuda.set_stream(torch.cuda.Stream(device))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)
    from als_speckle_b200.engine import Engine
    from als_speckle_b200 import autotune
    tune = autotune.load_or_default(N)
    engine = Engine(device=device, use_graph=True, l2_group_bytes=tune["l2_group_bytes"],
                    e_per_n={N: tune["E"]})
    M, S, box = build_inputs(torch, device)
    strong = args.mode == "strong"
    job = ShardedJob(torch, device, M, S, box, engine, seed=1000) if strong else \
        Job(torch, device, M, S, box, engine, seed=1000 + rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)  # 256 MiB > L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        job.step()
    barrier()
    stream = torch.cuda.current_stream()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_all0 = torch.cuda.Event(enable_timing=True)
    t_all1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        t_all0.record(stream)
        for k in range(args.steps):
            flush_l2(torch, flush)
            starts[k].record(stream)
            job.step()
            ends[k].record(stream)
        t_all1.record(stream)
        barrier()
    total_s = t_all0.elapsed_time(t_all1) / 1e3
    step_s = [s.elapsed_time(e) / 1e3 for s, e in zip(starts, ends)]
    t = torch.tensor([total_s], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_s = float(t.item())
    # replicas: every rank runs a whole job; strong: the ranks share one job
    work = TRIALS * ITERS * (1 if strong else world) * args.steps
    value = work / total_s
    launches = job.launches * args.steps
    rfac = job.r_factor()

    # e2e through the public API with host inputs and host outputs: every rank
    # runs the job; the whole-job figure is all ranks' work over the slowest time
    e2e = run_e2e(torch, device, M, S, args, engine, sync=barrier)
    et = torch.tensor([e2e.pop("seconds")], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e["value"] = TRIALS * ITERS * args.steps * world / float(et.item())
    # kernel-level roofline: one steady iteration tick of one L2 group
    per_tick, group = kernel_pass_times(
        torch, engine, Job(torch, device, M, S, box, engine, seed=1000) if strong else job)
    peak, peak_kind = _peaks()
    achieved = BYTES_PER_PX * N * N * group / per_tick / 1e9
    plain = run_plain(torch, device, M, S)
    single = run_single_trial(torch, device, M, S, engine)
    cufft = run_cufft_pair(torch, device, per_tick, group)
    serving = run_serving() if world == 1 and args.serving else None

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "strong" if strong else "weak",
        "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (seeded ellipse objects, Poisson noise; reference example data unavailable)",
        "config": {"workload": WORKLOAD, "trials": TRIALS, "iterations": "500 hio + 50 er",
                   "beta": BETA, "l2": "inputs larger than L2 (512 MiB psi+G per job) and a "
                   "256 MiB L2 flush before every step", "parallelism": ("trial-sharded x%d (one job)" % world) if strong
                   else "replicas x%d" % world,
                   "E": tune["E"], "l2_group_bytes": tune["l2_group_bytes"]},
        "latency_ms": {"p50": 1e3 * float(np.percentile(step_s, 50)),
                       "p99": 1e3 * float(np.percentile(step_s, 99))},
        "final_r_factor": None if rfac is None else
        {"mean": float(np.mean(rfac)), "median": float(np.median(rfac))},
        "e2e": e2e,
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "kernel": "%s + sp::row_pass_kernel<512,%d> (one iteration tick of %d trials, "
                               "24 B/px)" % ("sp::col_pass_sb_kernel<512,32>" if tune["E"] >= 32 else
                                             "sp::col_pass_kernel<512,%d>" % tune["E"], min(tune["E"], 32),
                                             group),
                     "traffic": traffic_per_tick(group)},
        # 10 N^2 log2(N^2) flop per forward + inverse 2-D FFT pair, one pair per
        # trial-iteration, over the same tick
        "fft_tflops": 10.0 * N * N * math.log2(N * N) * group / per_tick / 1e12,
        "plain_gpu": plain,
        "single_trial_engine": single,
        "cufft_transforms_only": cufft,
        "batched_over_plain": value / world / plain["value"],
        "batched_over_single_trial_engine": value / world / single["value"],
        "clocks": clk.summary(),
    }
    if serving is not None:
        line["serving"] = serving
    if args.cpu_baseline and world == 1:  # the host-core baseline: rank 0 at N = 1 only
        line["cpu_baseline"] = cpu_baseline()
        if not strong:
            line["avg_err_vs_fp64"] = precision_check(job)
    print(json.dumps(line))


def traffic_per_tick(group):
    """DRAM bytes per tick from the committed ncu capture, scaled by trials."""
    path = os.path.join(ROOT, "profiles", "traffic_hio_512.json")
    try:
        with open(path) as f:
            t = json.load(f)
        return float(t["dram_bytes_per_trial_tick"]) * group
    except Exception:
        return None


def run_e2e(torch, device, M, S, args, engine, sync=None):
    """Same job through the phasing API with host buffers every step.  Under
    torchrun every rank runs its own job; ``sync`` (a barrier) lines the ranks
    up before the timed loop and the caller takes the slowest rank's time."""
    from als_speckle_b200.phasing import (phasing, align_global_phase, align_frames_subpixel, prtf,
                                          mean_frames)
    Mh = torch.from_numpy(M).pin_memory()
    Sh = torch.from_numpy(S).pin_memory()
    r = phasing(device=device, engine=engine)

    def one():
        r.numtrial = 0
        r.load(modulus=Mh.numpy(), support=Sh.numpy(), numtrials=TRIALS)
        psis, errs = r.iterate_trials(ITERS, TRIALS, order=ORDER, beta=BETA, seed=7, errors=True)
        sb = r.savebuffer[:TRIALS]
        al = align_frames_subpixel(align_global_phase(sb), upsample=UPSAMPLE)
        avg = mean_frames(al).cpu()
        p = prtf(al, N=N).cpu()
        rf = errs[:, -1, 1].cpu()
        return avg.numel() * 8 + p.numel() * 4 + rf.numel() * 8

    for _ in range(max(1, args.warmup)):
        one()
    torch.cuda.synchronize()
    if sync is not None:
        sync()
    t0 = time.perf_counter()
    d2h = 0
    for _ in range(args.steps):
        d2h = one()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"value": TRIALS * ITERS * args.steps / dt, "unit": UNIT,
            "h2d_bytes_per_step": int(M.nbytes + S.nbytes), "d2h_bytes_per_step": int(d2h),
            "api": "phasing.load + iterate_trials + align_global_phase + align_frames_subpixel + "
                   "mean_frames + prtf",
            "seconds": dt}


def run_plain(torch, device, M, S, iters=40):
    """The plain single-instance path: one trial, cuFFT + one kernel per step
    with a synchronisation after each (the reference's GPU dataflow)."""
    from als_speckle_b200 import _lib
    from als_speckle_b200.engine import expand_runs
    Md = torch.from_numpy(M).to(device)
    Sd = torch.from_numpy(S).to(device)
    psi = torch.zeros((N, N), dtype=torch.complex64, device=device)
    psi.real.copy_(Sd)
    work = torch.empty((4, N, N), dtype=torch.complex64, device=device)
    algs, counts = expand_runs((("hio", iters),))
    a = (C.c_int32 * 1)(*algs)
    c = (C.c_int32 * 1)(*counts)

    def go(n):
        _lib.call("sp_plain_iterate", N, n, 1, a, c, C.c_float(BETA), _lib.ptr(psi), _lib.ptr(Md),
                  _lib.ptr(Sd), _lib.ptr(work), _lib.stream_ptr())
    go(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    go(iters)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"value": iters / dt, "unit": "iter/s", "what": "1 trial, cuFFT + elementwise kernels, "
            "sync after every launch (reference GPU dataflow)"}


def run_cufft_pair(torch, device, per_tick, group, reps=20):
    """cuFFT (through torch.fft) on the same planes: a forward and an inverse
    2-D transform of ``group`` 512^2 complex64 planes, beside one engine tick
    (the whole iteration: both transforms, the projection and the update)."""
    x = torch.randn(group, N, N, dtype=torch.complex64, device=device)
    for _ in range(3):
        y = torch.fft.ifft2(torch.fft.fft2(x))
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        y = torch.fft.ifft2(torch.fft.fft2(x))
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    del x, y
    return {"fft2_ifft2_ms": ms, "engine_tick_ms": 1e3 * per_tick,
            "what": "torch.fft.fft2 then ifft2 of %d planes of %d^2 (cuFFT), against one engine "
                    "iteration tick of the same trials" % (group, N)}


def run_single_trial(torch, device, M, S, engine, iters=200):
    """The fused engine on a single trial (no batching)."""
    from als_speckle_b200.engine import Engine, TrialSpec
    Md = torch.from_numpy(M).to(device)
    Sd = torch.from_numpy(S).to(device)
    psi = torch.zeros((N, N), dtype=torch.complex64, device=device)
    eng = Engine(device=device, use_graph=True, e_per_n=engine.e_per_n)
    spec = TrialSpec(psi=psi, modulus=Md, support=Sd, iterations=iters, order=(("hio", iters),),
                     beta=BETA, random_phase=True, seed=1)
    eng.solve([spec])
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    eng.solve([spec])
    b.record()
    torch.cuda.synchronize()
    eng.close()
    return {"value": iters / (a.elapsed_time(b) / 1e3), "unit": "iter/s",
            "what": "1 trial through the fused engine (CUDA graph)"}


def run_serving(rate=4.0, window=5.0):
    """The continuous-batching service on the mixed request stream (sizes
    256^2..2048^2 at .4/.3/.2/.1, HIO/ER/RAAR/DM, 200-2000 iterations, 1-16
    trials) offered at a rate it sustains: p50/p99 request latency (arrival to
    result on the host) and delivered pixel-iterations per second."""
    from als_speckle_b200 import workloads
    r = workloads.serving(rate=rate, window=window, seed=0)
    keep = ("rate", "window_s", "requests", "wall_s", "p50_latency_s", "p99_latency_s",
            "gpx_iterations_per_s", "trial_iterations_per_s", "rounds")
    out = {k: r[k] for k in keep}
    out["what"] = ("Poisson arrivals, sizes 256^2-2048^2 (.4/.3/.2/.1), HIO/ER/RAAR/DM, 200-2000 "
                   "iterations, 1-16 trials, 120 GB budget, rounds of 64 iterations")
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    iters = 12
    pool = CpuPool()
    try:
        for _ in range(args.warmup):
            pool.run(iters)
        vals, walls = [], []
        for _ in range(args.steps):
            v, w, _ = pool.run(iters)
            vals.append(v)
            walls.append(w)
    finally:
        pool.close()
    value = float(np.sum([pool.procs * iters for _ in walls]) / np.sum(walls))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(walls)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (seeded ellipse objects, Poisson noise)",
        "config": {"workload": WORKLOAD, "trials": TRIALS, "iterations": "500 hio + 50 er",
                   "beta": BETA},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": pool.procs, "kind": pool.kind,
                         "sample": pool.describe(iters)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-serving", dest="serving", action="store_false")
    ap.add_argument("--mode", choices=("replicas", "strong"), default="replicas",
                    help="replicas: one whole job per rank (weak scaling); strong: one job "
                         "sharded over the ranks")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
