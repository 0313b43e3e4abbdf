"""Drop-in for ``speckle.phasing`` (dhparks/als_speckle, ``speckle/phasing.py``).

Same class and function names, keyword arguments, defaults and state
machine as the reference; the arithmetic runs in libspeckle_b200 on the GPU.
Iterations are fused (one column pass and one row pass per iteration, see
``csrc/sp_engine_kernels.cuh``); trials can also be run many at a time with
``phasing.iterate_trials`` (an addition: the reference runs trials serially).

Differences from the reference, all deliberate:
* No CPU branch: ``force_cpu=True`` raises.  ER/SF follow the OpenCL kernels
  (``phasing_er.cl``, ``phasing_sf.cl``); ``quirks="cpu"`` selects the
  reference's CPU-branch forms instead (``phasing.py:1257``, ``:1284``).
* Where ``|FFT(psi)| == 0`` the reference divides by zero
  (``phasing_fourier.cl:14``); here the modulus is kept with zero phase.
* ``debug_on`` FITS dumps cover the coherent projection (they raise with an
  ipsf or a spectrum loaded).  ``ipsf`` (transverse coherence) and
  ``spectrum`` (longitudinal coherence, the reference's GPU-only
  ``radial_rescale``) are supported; where the blurred divisor is 0 the
  modulus is kept with zero phase, like the coherent case.
* ``reconstruct`` runs what the reference's version describes (that one
  cannot run as written), all trials of a round in one engine call.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib, masking
from ._lib import call, ptr, stream_ptr
from .engine import Engine, TrialSpec, expand_runs
from .gpu import common


class phasing(common):
    """A reconstruction: modulus, support, trials and a savebuffer
    (``phasing.py:33-1353``)."""

    def __init__(self, force_cpu=False, force_np_fft=False, gpu_info=None, device=None,
                 quirks="gpu", engine=None):
        if force_cpu:
            raise ValueError("als_speckle_b200 has no CPU path; use the reference for force_cpu=True")
        if not torch.cuda.is_available():
            raise RuntimeError("als_speckle_b200 needs a CUDA device")
        if quirks not in ("gpu", "cpu"):
            raise ValueError("quirks must be 'gpu' or 'cpu'")
        self.device = torch.device(device if device is not None else "cuda")
        self.use_gpu = True
        self.compute_device = "gpu"
        self.quirks = quirks
        # the engine runs on a private stream ordered after (and before) the
        # caller's current stream, so its launch sequence can be replayed as a
        # CUDA graph (graphs cannot be captured on the legacy default stream)
        self.engine = engine or Engine(device=self.device, use_graph=True)
        with torch.cuda.device(self.device):
            call("sp_device_init")
            self._engine_stream = torch.cuda.Stream(self.device)
        self.modulus_state = 0
        self.support_state = 0
        self.ipsf_state = 0
        self.ipsf = None
        self.buffer_state = 0
        self.spectrum_state = 0
        self.can_iterate = False
        self.numtrial = 0
        self.N = self.shape = self.size = None
        self.modulus = self.support = self.psi_in = self.psi_out = None
        self.numtrials = None
        self.r0 = self.c0 = self.rows = self.cols = None
        self.savebuffer = None
        self.errors = None  # (iterations, 2) FP64 sums of the last iterate()
        self.reconstruction = None

    # ------------------------------------------------------------------ load
    def load(self, modulus=None, support=None, ipsf=None, spectrum=None, numtrials=None):
        """Load data (keyword arguments only), ``phasing.py:291-505``."""
        for name, x in (("modulus", modulus), ("support", support), ("ipsf", ipsf)):
            if x is not None and not isinstance(x, np.ndarray):
                raise TypeError("%s must be ndarray if supplied" % name)
        # spectrum: (2, n) array of (energies, weights); rescale factors are
        # energies / the energy of the largest weight (phasing.py:426-450)
        if spectrum is not None:
            if not isinstance(spectrum, np.ndarray) or spectrum.ndim != 2 or spectrum.shape[0] != 2:
                raise ValueError("spectrum must be an ndarray of shape (2, n)")
            energies, weights = spectrum[0], spectrum[1]
            rescales = energies / energies[weights.argmax()]
            self.rescales = torch.from_numpy(rescales.astype(np.float32)).to(self.device)
            self.sweights = torch.from_numpy(weights.astype(np.float32)).to(self.device)
            self.N_spctrm = int(energies.shape[0])
            self.spectrum_state = 2
        if modulus is not None:
            if modulus.ndim != 2:
                raise ValueError("modulus must be 2d")
            modulus = modulus.astype(np.float32)
            if self.modulus_state == 2:
                if modulus.shape != self.shape:
                    raise ValueError("modulus shape %s differs from %s" % (modulus.shape, self.shape))
            else:
                if modulus.shape[0] != modulus.shape[1]:
                    raise ValueError("modulus must be square")
                N = modulus.shape[0]
                if N & (N - 1) or not 8 <= N <= 4096:
                    raise ValueError("N=%d must be a power of two in [8, 4096]" % N)
                self.N, self.shape, self.size = N, modulus.shape, modulus.size
                self.modulus = self._allocate(self.shape, np.float32, "modulus")
                self.psi_in = self._allocate(self.shape, np.complex64, "psi_in")
                self.psi_out = self._allocate(self.shape, np.complex64, "psi_out")
            self.modulus = self._set(modulus, self.modulus)
            self.modulus_state = 2
        if support is not None:
            if support.ndim != 2:
                raise ValueError("support is %s-dim" % support.ndim)
            if support.shape[0] != support.shape[1]:
                raise ValueError("support shape is %s %s, must be square" % support.shape)
            support = support.astype(np.float32)
            support *= 1.0 / support.max()
            if self.support_state == 2:
                self.numtrial = 0
            self._support_host = support
            bounds = masking.bounding_box(support, pad=10)
            self.r0, self.rows = int(bounds[0]), int(bounds[1] - bounds[0])
            self.c0, self.cols = int(bounds[2]), int(bounds[3] - bounds[2])
            self.support_state = 1
        if numtrials is not None:
            self.numtrials = int(numtrials)
            if self.buffer_state == 0:
                self.buffer_state = 1
        # ipsf: transform of the coherence point spread, same shape as the
        # modulus (phasing.py:413-424, dependency check :455-459)
        if ipsf is not None:
            if ipsf.ndim != 2 or ipsf.shape[0] != ipsf.shape[1]:
                raise ValueError("ipsf must be a square 2d array")
            ipsf = ipsf.astype(np.complex64)
            if self.ipsf_state == 2 and ipsf.shape != tuple(self.ipsf.shape):
                raise ValueError("ipsf shape %s differs from %s" % (ipsf.shape, tuple(self.ipsf.shape)))
            self.ipsf = self._set(ipsf, self._allocate(ipsf.shape, np.complex64, "ipsf"))
            self.ipsf_state = 1
        if self.modulus_state == 2 and self.ipsf_state > 0:
            if tuple(self.ipsf.shape) != self.shape:
                raise ValueError("ipsf shape %s differs from the modulus %s" % (tuple(self.ipsf.shape), self.shape))
            self.ipsf_state = 2
        if self.modulus_state == 2 and self.support_state > 0:
            sup = self._support_host
            if sup.shape != self.shape:
                if self.rows > self.shape[0] or self.cols > self.shape[1]:
                    raise ValueError("support crop larger than the modulus")
                crop = sup[self.r0:self.r0 + self.rows, self.c0:self.c0 + self.cols]
                new = np.zeros(self.shape, np.float32)
                new[:self.rows, :self.cols] = crop
                bounds = masking.bounding_box(new, force_to_square=True, pad=4)
                self.r0, self.rows = int(bounds[0]), int(bounds[1] - bounds[0])
                self.c0, self.cols = int(bounds[2]), int(bounds[3] - bounds[2])
                sup = new
                self._support_host = sup
            self.support = self._allocate(self.shape, np.float32, "support")
            self.support = self._set(sup, self.support)
            self.support_state = 2
            if self.buffer_state > 0:
                shape = (self.numtrials + 1, self.rows, self.cols)
                if self.buffer_state == 1 or tuple(self.savebuffer.shape) != shape:
                    self.savebuffer = self._allocate(shape, np.complex64, "savebuffer")
                    self.buffer_state = 2
        self.can_iterate = self.modulus_state == 2 and self.support_state == 2 and self.buffer_state == 2

    def _ipsf(self):
        """The loaded ipsf when the projection is partially coherent, else None."""
        return self.ipsf if self.ipsf_state == 2 else None

    def _spectrum(self):
        """(rescales, weights) on the device when a spectrum is loaded, else None."""
        return (self.rescales, self.sweights) if self.spectrum_state == 2 else None

    # ------------------------------------------------------- coherence estimate
    def optimize_coherence(self, best_estimate, modulus=None, force_cpu=False, load=True,
                           silent=False, iterations=500, method="richardson_lucy",
                           is_fourier=False):
        """Estimate the coherence function from reconstructions
        (``phasing.py:507-930``).

        ``richardson_lucy``: for every frame at once, Richardson-Lucy
        deconvolution of the measured intensity M^2 by the frame's intensity
        (``iterations`` steps from a Gaussian of width N/4); the result is the
        last frame's transform divided by its value at (0,0), as in the
        reference (its sum over frames is unused), loaded as the ipsf if
        ``load`` and returned fftshifted.  ``gaussian``: per frame, the
        coherence lengths minimising the misfit between the modulus and the
        speckle of the damped autocorrelation (``scipy.optimize.fmin`` on the
        host, each evaluation on the device); their mean loads a Gaussian
        ipsf if ``load``; returns the (2, frames) lengths.  ``force_cpu``
        raises (no CPU branch)."""
        if force_cpu:
            raise NotImplementedError("als_speckle_b200 has no CPU branch")
        if method not in ("richardson_lucy", "gaussian"):
            raise ValueError("unknown coherence method %s" % method)
        if modulus is None:
            if self.modulus is None:
                raise RuntimeError("no modulus: load one or pass modulus=")
            modulus = self.modulus.cpu().numpy()
        modulus = np.asarray(modulus)
        if modulus.ndim != 2 or modulus.shape[0] != modulus.shape[1]:
            raise ValueError("modulus must be square 2d")
        N = modulus.shape[0]
        est = best_estimate.cpu().numpy() if isinstance(best_estimate, torch.Tensor) else np.asarray(best_estimate)
        if est.ndim == 2:
            est = est[None]
        if est.ndim != 3 or est.shape[1] > N or est.shape[2] > N:
            raise ValueError("best_estimate must be 2d or 3d and no larger than the modulus")
        F = est.shape[0]
        dev = self.device
        st = stream_ptr()
        active = torch.zeros((F, N, N), dtype=torch.complex64, device=dev)
        active[:, :est.shape[1], :est.shape[2]] = torch.from_numpy(est.astype(np.complex64)).to(dev)
        if method == "richardson_lucy":
            # p = |FFT(estimate)|^2 / sum (the estimate is already a modulus if
            # is_fourier), P = FFT(p), PH = P flipped; d = M^2 / sum
            p = active.clone()
            if not is_fourier:
                call("sp_fft2", ptr(p), ptr(p), N, F, 0, st)
                call("sp_abs_f2_f2", ptr(p), ptr(p), p.numel(), st)
            call("sp_multiply_f2_f2", ptr(p), ptr(p), ptr(p), p.numel(), st)
            sums = p.real.sum(dim=(1, 2), dtype=torch.float64)
            p.mul_((1.0 / sums).to(torch.float32).view(F, 1, 1))
            call("sp_fft2", ptr(p), ptr(p), N, F, 0, st)
            ph = torch.empty_like(p)
            call("sp_flip_f2", ptr(p), ptr(ph), N, F, st)
            m2 = modulus.astype(np.float64) ** 2
            d = torch.from_numpy((m2 / m2.sum()).astype(np.complex64)).to(dev)
            u = torch.empty((F, N, N), dtype=torch.complex64, device=dev)
            call("sp_gaussian", ptr(u[0]), N, C.c_float(N / 4.0), C.c_float(N / 4.0), 1, st)
            u[1:] = u[0]
            work = torch.empty_like(u)
            call("sp_richardson_lucy", ptr(u), ptr(p), ptr(ph), ptr(d), ptr(work), N, F,
                 int(iterations), st)
            last = u[F - 1].contiguous()
            call("sp_fft2", ptr(last), ptr(last), N, 1, 0, st)
            ipsf = last.cpu().numpy()
            ipsf = (ipsf * (1.0 / abs(ipsf[0, 0]))).astype(np.complex64)
            if load:
                self.load(ipsf=ipsf)
            return np.fft.fftshift(ipsf)
        # gaussian: autocorrelation IFFT(|FFT(estimate)|^2) per frame, then fmin
        from scipy.optimize import fmin
        call("sp_fft2", ptr(active), ptr(active), N, F, 0, st)
        call("sp_abs2_f2_f2", ptr(active), ptr(active), active.numel(), st)
        call("sp_fft2", ptr(active), ptr(active), N, F, 1, st)
        m = torch.from_numpy(np.ascontiguousarray(modulus, np.float32)).to(dev)
        work = torch.empty((N, N), dtype=torch.complex64, device=dev)
        acc = torch.empty(1, dtype=torch.float64, device=dev)
        optcls = np.zeros((2, F), np.float32)
        for n in range(F):
            ac = active[n]

            def misfit(cl):
                call("sp_coherence_misfit", ptr(ac), ptr(m), C.c_float(cl[0]), C.c_float(cl[1]), N,
                     ptr(work), ptr(acc), st)
                return float(acc.item())
            optcls[:, n] = fmin(misfit, (N / 2, N / 2), disp=False, ftol=.1, xtol=0.1)
        ave = np.average(optcls, axis=1)
        if load:
            rows, cols = np.indices((N, N)) - N / 2.
            rows, cols = np.fft.fftshift(rows), np.fft.fftshift(cols)
            self.load(ipsf=np.exp(-rows ** 2 / (2 * ave[0] ** 2)) * np.exp(-cols ** 2 / (2 * ave[1] ** 2)))
        return optcls

    # ------------------------------------------------------------------ seed
    def seed(self, val=None, supplied=None):
        """psi_in = (U[0,1) + i U[0,1)) * support from numpy's global RNG, or a
        supplied guess rolled onto the support (``phasing.py:990-1031``)."""
        if self.N is None:
            raise RuntimeError("cannot seed without N being set. load data first.")
        if val is not None:
            np.random.seed(val)
        if supplied is None:
            s = (np.random.rand(self.N, self.N) + 1j * np.random.rand(self.N, self.N)).astype(np.complex64)
            s = s * self._support_host
            self._set(s.astype(np.complex64), self.psi_in)
            return
        s = np.asarray(supplied)
        if s.ndim != 2 or s.shape[0] > self.N or s.shape[1] > self.N:
            raise ValueError("supplied guess must be 2d and no larger than N")
        if s.shape != (self.N, self.N):
            s2 = np.zeros(self.shape, np.complex64)
            s2[:s.shape[0], :s.shape[1]] = s.astype(np.complex64)
            s = s2
        dev = torch.from_numpy(s.astype(np.complex64)).to(self.device)
        ref = self.support.to(torch.complex64)
        rolled = align_frames_device(dev, ref, use_mag_only=True)
        rolled = rolled * self.support
        self.psi_in.copy_(rolled)

    # --------------------------------------------------------------- iterate
    def _check_ready(self):
        if not self.can_iterate:
            raise RuntimeError("cant iterate before loading support, modulus and numtrials "
                               "(states %d %d %d)" % (self.modulus_state, self.support_state,
                                                      self.buffer_state))

    def iterate(self, iterations, order=None, silent=True, beta=0.8, debug_on=None):
        """Run ``iterations`` of the cyclic ``order`` on psi_in, then copy the
        crop into ``savebuffer[numtrial]`` (``phasing.py:181-289``).

        The per-iteration FP64 modulus error sums of FFT(psi_in) are kept in
        ``self.errors`` (see ``modulus_error``).  Iterations listed in
        ``debug_on`` run one operator at a time and write the reference's
        debugging FITS files to the working directory (``_debug_iteration``);
        the others run fused."""
        self._check_ready()
        iterations = int(iterations)
        debug = set(int(i) for i in (debug_on or ()))
        if debug and (self._ipsf() is not None or self._spectrum() is not None):
            raise NotImplementedError("debug_on dumps cover the coherent projection only")
        if self.numtrial >= self.savebuffer.shape[0]:
            raise IndexError("savebuffer is full (%d slots); load(numtrials=...) to enlarge"
                             % self.savebuffer.shape[0])
        algs, counts = expand_runs(order, self.quirks)
        flat = [a for a, c in zip(algs, counts) for _ in range(c)]
        chunk = iterations
        if silent is not True:
            chunk = 1 if isinstance(silent, bool) else max(1, int(silent))
        self.errors = torch.zeros((iterations, 2), dtype=torch.float64, device=self.device)
        done = 0
        while done < iterations:
            if done in debug:
                self._debug_iteration(flat[done % len(flat)], done, beta)
                n = 1
            else:
                n = min(chunk, iterations - done)
                nxt = [i for i in debug if i > done]
                if nxt:
                    n = min(n, min(nxt) - done)
                rot = [flat[(done + i) % len(flat)] for i in range(len(flat))]
                last = done + n >= iterations
                spec = TrialSpec(psi=self.psi_in, modulus=self.modulus, support=self.support,
                                 iterations=n, order=_runs_from_flat(rot), beta=beta,
                                 box=(self.r0, self.c0, self.rows, self.cols) if last else None,
                                 save=self.savebuffer[self.numtrial] if last else None,
                                 errors=self.errors[done:done + n], quirks="gpu",
                                 ipsf=self._ipsf(), spectrum=self._spectrum())
                self._solve([spec])
            done += n
            if silent is not True and (isinstance(silent, bool) or done % chunk == 0):
                print("  iteration %s" % done)
        if iterations == 0 or (iterations - 1) in debug:
            self._kexec("copy_to_buffer_f2", self.savebuffer, self.psi_in, self.c0, self.r0,
                        self.numtrial, self.N, shape=(self.cols, self.rows))
        self.numtrial += 1

    def _debug_iteration(self, alg, iteration, beta):
        """One iteration through the operator API, as the reference's GPU
        branch runs it (``phasing.py:1187-1353``: FFT, divisor |FFT|, the
        ``fourier`` kernel, inverse FFT, then the update kernel; DM repeats the
        projection on ``dm1(psi_in)``), saving what the reference's debug mode
        saves (``phasing.py:1193-1227``, ``:1244-1246``) under the same names:
        ``gpu i<it> psi_fourier_1`` / ``fourier_div`` / ``psi_fourier_2``
        (fftshifted, magnitude and phase), ``gpu i<it> out`` (real and
        imaginary) and, for HIO, ``gpu i<it> hio update``.  The iteration's
        FP64 error sums go to ``self.errors[iteration]`` as the fused path's do."""
        from . import io
        shift = np.fft.fftshift
        tag = "%s i%s " % (self.compute_device, iteration)
        N = self.N
        st = stream_ptr()
        m = self.modulus

        def dump(name, array, components):
            # DM projects twice per iteration under the same names: keep the last
            io.save(tag + name + ".fits", array, components=components, overwrite=True)

        def constraint(data):
            pf = torch.empty_like(data)
            call("sp_fft2", ptr(data), ptr(pf), N, 1, 0, st)
            dump("psi_fourier_1", shift(self.get(pf)), "polar")
            div = torch.empty_like(pf)
            self._cl_abs(pf, div)
            dump("fourier_div", shift(self.get(div)), "polar")
            self._kexec("fourier", pf, div, m, pf)
            dump("psi_fourier_2", shift(self.get(pf)), "polar")
            out = torch.empty_like(pf)
            call("sp_fft2", ptr(pf), ptr(out), N, 1, 1, st)
            dump("out", self.get(out), "cartesian")
            return out, div

        psi, sup = self.psi_in, self.support
        out, div = constraint(psi)
        d = div.real.double() - m.double()
        self.errors[iteration, 0] = (d * d).sum()
        self.errors[iteration, 1] = d.abs().sum()
        name = _CODE_NAMES[alg]
        if name == "hio":
            self._kexec("hio", beta, sup, psi, out, psi)
            dump("hio update", self.get(psi), "cartesian")
        elif name == "er":
            self._kexec("er", sup, out, psi)
        elif name == "raar":
            self._kexec("raar", beta, sup, psi, out, psi)
        elif name == "sf":
            self._kexec("sf", sup, psi, out, psi)
        elif name == "er_cpu":  # phasing.py:1257
            psi.mul_(sup)
        elif name == "sf_cpu":  # phasing.py:1284
            psi.copy_((1 - sup) * (-psi) + sup * out)
        else:  # dm: gamma_m = 1/beta, gamma_s = -gamma_m (phasing.py:1294-1295)
            tmp = torch.empty_like(psi)
            self._kexec("dm1", 1.0 / beta, sup, psi, tmp)
            tmp, _ = constraint(tmp)
            self._kexec("dm2", beta, -1.0 / beta, sup, psi, out, tmp, psi)

    def iterate_trials(self, iterations, trials, order=None, beta=0.8, seed=0,
                       random_phase=True, errors=False):
        """Batched extension: run ``trials`` independent starts at once and
        fill ``savebuffer[numtrial:numtrial+trials]``.

        Starts are S*IFFT(M exp(i phi)) with phi from (seed, trial index) when
        ``random_phase``; otherwise every trial starts from the current psi_in.
        Returns the final psi of every trial (trials, N, N) and, with
        ``errors=True``, the FP64 error sums (trials, iterations, 2)."""
        self._check_ready()
        if self.numtrial + trials > self.savebuffer.shape[0]:
            raise IndexError("savebuffer has %d free slots, %d trials requested"
                             % (self.savebuffer.shape[0] - self.numtrial, trials))
        psis = torch.empty((trials, self.N, self.N), dtype=torch.complex64, device=self.device)
        if not random_phase:
            psis.copy_(self.psi_in.expand(trials, self.N, self.N))
        errs = (torch.zeros((trials, max(iterations, 1), 2), dtype=torch.float64, device=self.device)
                if errors else None)
        specs = []
        for k in range(trials):
            specs.append(TrialSpec(psi=psis[k], modulus=self.modulus, support=self.support,
                                   iterations=int(iterations), order=order, beta=beta,
                                   random_phase=random_phase, seed=seed, trial=self.numtrial + k,
                                   box=(self.r0, self.c0, self.rows, self.cols),
                                   save=self.savebuffer[self.numtrial + k],
                                   errors=errs[k] if errors else None, quirks=self.quirks,
                                   ipsf=self._ipsf(), spectrum=self._spectrum()))
        self._solve(specs)
        self.numtrial += trials
        return (psis, errs) if errors else psis

    def reconstruct(self, iterations=100, rounds=1, order=None, refine_support=True,
                    refinement_parameters=None):
        """Seed and iterate every trial, average them, refine the support;
        ``rounds`` times (``phasing.py:932-988``).

        The reference's method cannot run as written (it loops over the
        integer ``rounds`` and reads an undefined ``self.trials``); this runs
        what it describes.  Per round, each of the ``numtrials`` trials is
        seeded as ``seed()`` seeds (numpy's global RNG, in trial order) and
        iterated ``iterations`` times with ``order`` (default
        ``(('hio', 99), ('er', 1))``) at beta 0.8 into the next savebuffer
        slot, all trials in one engine call (the same arithmetic as one
        ``iterate`` per trial); ``psi_in`` is left holding the last trial's
        iterate.  A copy of the savebuffer is aligned by each frame's global
        phase and its last slot is replaced by the mean over all slots, that
        slot included, as the reference's ``np.mean(save_buffer, axis=0)``
        is; the mean is ``self.reconstruction`` (numpy).  With
        ``refine_support`` the support's crop is refined from the mean
        (``refine_support`` with ``local_threshold`` 0.08, ``blur_sigma`` 3,
        ``global_threshold`` 0.0 unless ``refinement_parameters`` overrides
        them; ``kill_weakest`` is accepted and, as in the reference, not
        used), placed at the corner of an N x N plane and loaded, which
        restarts the trial count.  A refinement that leaves no pixel raises
        ValueError (the reference would load a support of NaNs)."""
        if refinement_parameters is not None and not isinstance(refinement_parameters, dict):
            raise TypeError("refinement_parameters must be a dict or None")
        rp = {"local_threshold": 0.08, "blur_sigma": 3, "global_threshold": 0.0,
              "kill_weakest": False}
        if refinement_parameters is not None:
            rp.update(refinement_parameters)
        beta = 0.8
        for _ in range(int(rounds)):
            self._check_ready()
            T = int(self.numtrials)
            if self.numtrial + T > self.savebuffer.shape[0]:
                raise IndexError("savebuffer has %d free slots, %d trials requested"
                                 % (self.savebuffer.shape[0] - self.numtrial, T))
            starts = np.empty((T, self.N, self.N), np.complex64)
            for k in range(T):
                s = (np.random.rand(self.N, self.N) + 1j * np.random.rand(self.N, self.N))
                starts[k] = s.astype(np.complex64) * self._support_host
            psis = torch.from_numpy(starts).to(self.device)
            algs, counts = expand_runs(order, self.quirks)
            runs = _runs_from_flat([a for a, c in zip(algs, counts) for _ in range(c)])
            specs = [TrialSpec(psi=psis[k], modulus=self.modulus, support=self.support,
                               iterations=int(iterations), order=runs, beta=beta,
                               box=(self.r0, self.c0, self.rows, self.cols),
                               save=self.savebuffer[self.numtrial + k], quirks="gpu",
                               ipsf=self._ipsf(), spectrum=self._spectrum()) for k in range(T)]
            self._solve(specs)
            self.psi_in.copy_(psis[T - 1])
            self.numtrial += T
            frames = align_global_phase(self.savebuffer)
            frames[-1] = mean_frames(frames)
            self.reconstruction = frames[-1].cpu().numpy()
            if refine_support:
                crop = self._support_host[self.r0:self.r0 + self.rows, self.c0:self.c0 + self.cols]
                refined = _shrinkwrap(
                    crop, self.reconstruction, blur=rp["blur_sigma"],
                    local_threshold=rp["local_threshold"],
                    global_threshold=rp["global_threshold"])[0]
                if not np.any(refined > 0):
                    raise ValueError("the refined support is empty")
                new_support = np.zeros(self.shape, np.float32)
                new_support[:refined.shape[0], :refined.shape[1]] = refined
                self.load(support=new_support)

    def _solve(self, specs):
        """Run the engine on the private stream, ordered after everything the
        caller's current stream has queued and before anything it queues
        next."""
        cur = torch.cuda.current_stream(self.device)
        self._engine_stream.wait_stream(cur)
        with torch.cuda.stream(self._engine_stream):
            self.engine.solve(specs, stream=self._engine_stream)
        cur.wait_stream(self._engine_stream)

    def modulus_error(self):
        """Per-iteration (E, R) of the last ``iterate``: E = sum(|F|-M)^2/sum M^2,
        R = sum||F|-M|/sum M, F = FFT(psi_in) before each projection."""
        m = self.modulus.double()
        s2, s1 = float((m * m).sum()), float(m.sum())
        e = self.errors.cpu().numpy()
        return np.stack([e[:, 0] / s2, e[:, 1] / s1], axis=1)

    def status(self):
        ro = {2: "complete", 1: "incomplete", 0: "nothing"}
        print("states:")
        print("  modulus %s %s" % (ro[self.modulus_state], self.shape))
        print("  support %s" % ro[self.support_state])
        print("  ipsf    %s" % ro[self.ipsf_state])
        print("  buffer  %s" % ro[self.buffer_state])
        print("  spectrm %s" % ro[self.spectrum_state])
        print("  device  %s" % self.compute_device)


def _runs_from_flat(flat):
    """Order list -> run-length ('alg', count) order with raw codes."""
    runs = []
    for a in flat:
        if runs and runs[-1][0] == a:
            runs[-1][1] += 1
        else:
            runs.append([a, 1])
    return [(_CODE_NAMES[a], c) for a, c in runs]


_CODE_NAMES = {_lib.SP_HIO: "hio", _lib.SP_ER: "er", _lib.SP_RAAR: "raar", _lib.SP_SF: "sf",
               _lib.SP_DM: "dm", _lib.SP_ER_CPU: "er_cpu", _lib.SP_SF_CPU: "sf_cpu"}


# ---------------------------------------------------------------------------
# module functions
# ---------------------------------------------------------------------------
def _device_frames(data):
    """(tensor on cuda complex64 (F, r, c), was_numpy, was_2d)."""
    was_np = isinstance(data, np.ndarray)
    t = torch.from_numpy(np.ascontiguousarray(data)).cuda() if was_np else data
    if not torch.is_complex(t):
        raise TypeError("data must be complex")
    was2d = t.dim() == 2
    if t.dim() not in (2, 3):
        raise ValueError("data must be 2d or 3d")
    t = t.to(torch.complex64)
    if was2d:
        t = t.unsqueeze(0)
    return t.contiguous(), was_np, was2d


def align_global_phase(data_in):
    """Remove each frame's global phase: the minimiser of
    sum|Re sin p + Im cos p|^2 from FP64 sums, then the sign rule
    (``phasing.py:1355-1404``; closed form instead of ``fminbound``)."""
    t, was_np, was2d = _device_frames(data_in)
    t = t.clone()
    F = t.shape[0]
    sums = torch.empty(5 * F, dtype=torch.float64, device=t.device)
    angles = torch.empty(F, dtype=torch.float64, device=t.device)
    call("sp_align_global_phase", ptr(t), F, t[0].numel(), ptr(angles), ptr(sums), stream_ptr())
    out = t[0] if was2d else t
    return out.cpu().numpy() if was_np else out


def prtf(estimates, N=None, silent=True, prtfq=False):
    """|mean_n F_n/|F_n||, fftshifted, estimates embedded at the corner of
    N x N (``phasing.py:1406-1461``, ``gpu_prtf`` ``:1463-1519``)."""
    t, was_np, _ = _device_frames(estimates)
    F, r, c = t.shape
    if N is None:
        N = max(r, c)
    Np = 1 << (int(N) - 1).bit_length()
    if Np != N:
        raise ValueError("N=%d must be a power of two" % N)
    work = torch.empty((F, N, N), dtype=torch.complex64, device=t.device)
    out = torch.empty((N, N), dtype=torch.float32, device=t.device)
    call("sp_prtf", ptr(t), F, r, c, N, ptr(work), ptr(out), stream_ptr())
    res = out.cpu().numpy() if was_np else out
    if prtfq:
        return res, unwrap_average(out, as_numpy=was_np)
    return res


def gpu_prtf(gpuinfo, estimates, N=None, prtfq=False):
    """``phasing.gpu_prtf`` signature; ``gpuinfo`` is ignored."""
    return prtf(estimates, N=N, prtfq=prtfq)


def unwrap_average(arr, as_numpy=True):
    """Azimuthal average of an N x N float map about (N/2, N/2) at radii
    0 .. N/2 - 1: ``np.average(wrapping.unwrap(arr, (0, N/2, (N/2, N/2))),
    axis=1)`` (``phasing.py:1454-1458``; ``wrapping.py:8-67``, ``:131-176``),
    the polar samples taken by cubic B-spline interpolation on the device
    (``sp_unwrap``).  Returns float32 (numpy if ``as_numpy``)."""
    a = torch.from_numpy(np.ascontiguousarray(arr, np.float32)).cuda() \
        if isinstance(arr, np.ndarray) else arr.to(torch.float32).contiguous()
    if a.dim() != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("unwrap_average needs a square 2d map")
    N = int(a.shape[0])
    work = torch.empty((N, N), dtype=torch.float64, device=a.device)
    mean = torch.empty(N // 2, dtype=torch.float32, device=a.device)
    call("sp_unwrap", ptr(a), N, 0, N // 2, float(N // 2), float(N // 2), 0, ptr(work), None,
         ptr(mean), stream_ptr())
    return mean.cpu().numpy() if as_numpy else mean


def _gaussian_1d_kernel(n, sigma):
    """fftshift of exp(-(x-n//2)^2/(2 sigma^2)), normalised: one factor of the
    separable kernel of ``refine_support`` (``phasing.py:1787-1789`` with
    ``shape.gaussian`` ``shape.py:494-508``)."""
    x = np.arange(n).astype(float)
    g = np.exp(-(x - n // 2) ** 2 / (2 * float(sigma) ** 2))
    g = np.fft.fftshift(g)
    return g / g.sum()


def refine_support(support, average_mag, blur=3, local_threshold=.2, global_threshold=0,
                   kill_weakest=False):
    """Shrinkwrap (``phasing.py:1747-1815``): blur |avg| with a circular
    Gaussian, keep the pixels above ``global_threshold`` of the maximum and,
    within each connected part of ``support``, above ``local_threshold`` of
    the part's maximum.  Returns (refined, blurred) as numpy arrays."""
    support = np.asarray(support)
    if support.ndim != 2:
        raise ValueError("support must be 2d")
    avg = average_mag
    if isinstance(avg, np.ndarray):
        if avg.ndim != 2:
            raise ValueError("average_mag must be 2d")
        avg_t = torch.from_numpy(np.ascontiguousarray(avg.astype(np.complex64))).cuda()
    else:
        avg_t = avg.to(torch.complex64).contiguous()
    for name, v in (("blur", blur), ("global_threshold", global_threshold),
                    ("local_threshold", local_threshold)):
        if not isinstance(v, (float, int, np.floating, np.integer)):
            raise TypeError("%s must be a number (is %s)" % (name, type(v)))
    rows, cols = support.shape
    if tuple(avg_t.shape) != (rows, cols):
        raise ValueError("support and average_mag must have the same shape")
    dev = avg_t.device
    kr = torch.from_numpy(_gaussian_1d_kernel(rows, blur)).to(dev)
    kc = torch.from_numpy(_gaussian_1d_kernel(cols, blur)).to(dev)
    labels, n = masking.label_parts(support)
    lab = torch.from_numpy(labels.astype(np.int32)).to(dev)
    work = torch.empty(rows * cols + n + 1, dtype=torch.float64, device=dev)
    blurred = torch.empty((rows, cols), dtype=torch.float64, device=dev)
    refined = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    sums = torch.empty(n + 1, dtype=torch.float64, device=dev)
    call("sp_shrinkwrap", ptr(avg_t), rows, cols, ptr(kr), ptr(kc), ptr(lab), n,
         float(local_threshold), float(global_threshold), 1 if kill_weakest else 0,
         ptr(work), ptr(blurred), ptr(refined), ptr(sums), stream_ptr())
    ref = refined.cpu().numpy().astype(support.dtype if support.dtype.kind == "f" else np.int64)
    return ref, blurred.cpu().numpy()


# the module function under a second name, for methods whose keyword
# argument ``refine_support`` (a flag, as in the reference) hides it
_shrinkwrap = refine_support


def align_frames_device(frames, align_to, use_mag_only=False):
    """Integer-roll alignment of N x N device frames to ``align_to``
    (``conditioning.align_frames`` :316-430, ``crosscorr.alignment_coordinates``
    :526-568).  Returns the rolled frames."""
    single = frames.dim() == 2
    fr = frames.unsqueeze(0) if single else frames
    N = fr.shape[-1]
    if fr.shape[-2] != N:
        raise ValueError("frames must be square N x N")
    ref = align_to.to(torch.complex64).contiguous()
    work = torch.empty((2, N, N), dtype=torch.complex64, device=fr.device)
    best = torch.empty(1, dtype=torch.int64, device=fr.device)
    out = torch.empty_like(fr)
    for k in range(fr.shape[0]):
        f = fr[k].contiguous()
        call("sp_xcorr_peak", ptr(f), ptr(ref), N, 1 if use_mag_only else 0, ptr(work), ptr(best),
             stream_ptr())
        key = int(best.item()) & 0xFFFFFFFFFFFFFFFF
        sidx = 0xFFFFFFFF - (key & 0xFFFFFFFF)
        mr, mc = divmod(sidx, N)
        mr -= N // 2
        mc -= N // 2
        if mr > N // 2:
            mr -= N
        if mc > N // 2:
            mc -= N
        call("sp_roll", ptr(f), ptr(out[k]), N, N, -mr, -mc, stream_ptr())
    return out[0] if single else out


def align_frames_subpixel(data, align_to=None, upsample=64, return_type="data"):
    """Align frames to ``align_to`` (default: the first frame) by subpixel
    shifts and a global phase: the cross-correlation convention and
    whole-pixel answers of ``conditioning.align_frames``
    (``conditioning.py:316-430``, ``crosscorr.py:526-568``), refined to
    1/``upsample`` pixel by the upsampled DFT of Guizar-Sicairos et al. (2008)
    and applied as a Fourier shift (``sp_register_subpixel``).  The reference
    aligns by whole pixels only; this is the batched workload's "align to
    trial 0".  ``return_type``: ``"data"`` (aligned frames, same shape and
    kind as ``data``), ``"coordinates"`` ((F, 3) array of dy, dx, theta) or
    ``"both"``."""
    t, was_np, was2d = _device_frames(data)
    F, rows, cols = t.shape
    if align_to is None:
        ref = t[0].contiguous()
    else:
        r, _, r2d = _device_frames(align_to)
        if not r2d or tuple(r.shape[1:]) != (rows, cols):
            raise ValueError("align_to must be one frame of the data's shape")
        ref = r[0].contiguous()
    N = 1 << (max(rows, cols) - 1).bit_length()
    N = max(N, 8)
    nbytes = C.c_size_t(0)
    call("sp_register_workspace_size", F, N, int(upsample), C.byref(nbytes))
    work = torch.empty(nbytes.value, dtype=torch.uint8, device=t.device)
    shifts = torch.empty((F, 3), dtype=torch.float64, device=t.device)
    out = torch.empty_like(t) if return_type != "coordinates" else None
    call("sp_register_subpixel", ptr(t), F, rows, cols, ptr(ref), N, int(upsample), ptr(work),
         nbytes.value, ptr(shifts), ptr(out), stream_ptr())
    coords = shifts.cpu().numpy() if was_np else shifts
    if return_type == "coordinates":
        return coords[0] if was2d else coords
    o = out[0] if was2d else out
    o = o.cpu().numpy() if was_np else o
    if return_type == "both":
        return o, (coords[0] if was2d else coords)
    return o


def center_of_mass_average(imgs):
    """Sum of frames rolled so their |img| centres of mass coincide with the
    first frame's (``phasing.py:1710-1745``)."""
    t, was_np, _ = _device_frames(imgs)
    F, r, c = t.shape
    sums = torch.empty(3 * F, dtype=torch.float64, device=t.device)
    call("sp_com_sums", ptr(t), F, r, c, ptr(sums), stream_ptr())
    s = sums.cpu().numpy().reshape(F, 3)
    coms = [(int(s[k, 1] / s[k, 0]), int(s[k, 2] / s[k, 0])) for k in range(F)]
    shifts = np.array([(coms[k][0] - coms[0][0], coms[k][1] - coms[0][1]) for k in range(F)],
                      np.int32)
    sh = torch.from_numpy(shifts).to(t.device)
    out = torch.empty((r, c), dtype=torch.complex64, device=t.device)
    call("sp_roll_accumulate", ptr(t), F, r, c, ptr(sh), ptr(out), stream_ptr())
    return out.cpu().numpy() if was_np else out


def mean_frames(frames):
    """Mean over the frame axis of device frames (complex64)."""
    t, was_np, _ = _device_frames(frames)
    out = torch.empty(t.shape[1:], dtype=torch.complex64, device=t.device)
    call("sp_mean_frames", ptr(t), t.shape[0], t[0].numel(), ptr(out), stream_ptr())
    return out.cpu().numpy() if was_np else out


def fft2(x, inverse=False):
    """Batched N x N complex FFT on the device (numpy conventions)."""
    t = x.to(torch.complex64).contiguous()
    N = t.shape[-1]
    out = torch.empty_like(t)
    call("sp_fft2", ptr(t), ptr(out), N, t.numel() // (N * N), 1 if inverse else 0, stream_ptr())
    return out


def _pow2_size(N, who):
    if N & (N - 1) or not 8 <= N <= 4096:
        raise ValueError("%s: N=%d must be a power of two in [8, 4096]" % (who, N))


def _embed(frames, N):
    """Frames (F, r, c) placed at the corner of zeroed (F, N, N) planes."""
    F, r, c = frames.shape
    if r > N or c > N:
        raise ValueError("estimate must be smaller than goal_modulus")
    out = torch.zeros((F, N, N), dtype=torch.complex64, device=frames.device)
    out[:, :r, :c] = frames
    return out


def _hot_pixels(x, threshold, iterations=1):
    """remove_hot_pixels on a device float32 array (2d or 3d), in place."""
    rows, cols = x.shape[-2], x.shape[-1]
    frames = x.numel() // (rows * cols)
    work = torch.empty((rows, cols), dtype=torch.float32, device=x.device)
    call("sp_remove_hot_pixels", ptr(x), ptr(work), frames, rows, cols, iterations,
         C.c_float(threshold), stream_ptr())
    return x


def remove_hot_pixels(data_in, iterations=1, threshold=2, gpu_info=None):
    """``conditioning.remove_hot_pixels`` (``conditioning.py:207-313``): pixels
    above ``threshold`` times the local 3 x 3 median (+0.1) are replaced by
    it, ``iterations`` times; ``gpu_info`` is ignored."""
    was_np = isinstance(data_in, np.ndarray)
    x = torch.from_numpy(np.ascontiguousarray(data_in, np.float32)).cuda() if was_np else \
        data_in.to(torch.float32).contiguous().clone()
    if x.dim() not in (2, 3):
        raise ValueError("data must be 2d or 3d")
    _hot_pixels(x, threshold, iterations)
    return x.cpu().numpy() if was_np else x


def rftf(estimate, goal_modulus, hot_pixels=False, ipsf=None, rftfq=False, scale=False):
    """RFTF of one estimate against the goal modulus (``phasing.py:1521-1608``):
    the speckle modulus of the estimate embedded at the corner (blurred by
    ``ipsf`` if given: the modulus is convolved, as the reference's numpy
    function does), lined up with the goal (centred at (0,0) or (N/2,N/2),
    whichever fits better), ``sqrt(1/(1+(F-g)^2/g^2))`` in the centred layout,
    optionally rescaled to [0, 1] and cleaned of hot pixels.  N must be a
    power of two here.  ``rftfq`` adds the polar-unwrapped azimuthal average
    (``unwrap_average``, ``phasing.py:1603-1605``)."""
    est, was_np, _ = _device_frames(estimate)
    g = torch.from_numpy(np.ascontiguousarray(goal_modulus, np.float32)).cuda() \
        if isinstance(goal_modulus, np.ndarray) else goal_modulus.to(torch.float32).contiguous()
    N = int(g.shape[0])
    _pow2_size(N, "rftf")
    if g.shape != (N, N):
        raise ValueError("goal_modulus must be square")
    st = stream_ptr()
    f = _embed(est[:1], N)
    call("sp_fft2", ptr(f), ptr(f), N, 1, 0, st)
    call("sp_abs_f2_f2", ptr(f), ptr(f), N * N, st)
    if ipsf is not None:
        ip = torch.from_numpy(np.ascontiguousarray(ipsf, np.complex64)).cuda() \
            if isinstance(ipsf, np.ndarray) else ipsf.to(torch.complex64).contiguous()
        if tuple(ip.shape) != (N, N):
            raise ValueError("ipsf must have the goal modulus' shape")
        call("sp_fft2", ptr(f), ptr(f), N, 1, 0, st)
        call("sp_multiply_f2_f2", ptr(f), ptr(ip), ptr(f), N * N, st)
        call("sp_fft2", ptr(f), ptr(f), N, 1, 1, st)
        call("sp_sqrt_abs_f2", ptr(f), ptr(f), N * N, st)
    sums = torch.empty(2, dtype=torch.float64, device=g.device)
    err = torch.empty((N, N), dtype=torch.float32, device=g.device)
    out = torch.empty((N, N), dtype=torch.float32, device=g.device)
    call("sp_rftf_map", ptr(f), ptr(g), N, 1 if scale else 0, ptr(sums), ptr(err), ptr(out), st)
    if hot_pixels:
        _hot_pixels(err, 2.0)
        call("sp_rftf_from_error", ptr(err), ptr(out), N * N, 1 if scale else 0, st)
        _hot_pixels(out, 1.1)
    res = out.cpu().numpy() if was_np else out
    if rftfq:
        return res, unwrap_average(out, as_numpy=was_np)
    return res


def gpu_rftf(gpuinfo, estimates, goal_modulus, ipsf=None, rftfq=False):
    """``phasing.gpu_rftf`` (``phasing.py:1611-1708``) over many estimates:
    each estimate's transform F (with ``ipsf``: the intensity |F|^2 blurred
    by the real part of ipsf, then the principal square root), then the mean
    over estimates of ``1/sqrt(1 + (g - Re F)^2/g^2)``, fftshifted.
    ``gpuinfo`` is ignored."""
    est, was_np, _ = _device_frames(estimates)
    g = torch.from_numpy(np.ascontiguousarray(goal_modulus, np.float32)).cuda() \
        if isinstance(goal_modulus, np.ndarray) else goal_modulus.to(torch.float32).contiguous()
    N = int(g.shape[0])
    _pow2_size(N, "gpu_rftf")
    L = est.shape[0]
    st = stream_ptr()
    f = _embed(est, N)
    call("sp_fft2", ptr(f), ptr(f), N, L, 0, st)
    if ipsf is not None:
        ip = np.real(np.asarray(ipsf)).astype(np.float32) if not isinstance(ipsf, torch.Tensor) \
            else ipsf.real.cpu().numpy().astype(np.float32)
        ipd = torch.from_numpy(np.ascontiguousarray(ip)).cuda()
        call("sp_abs2_f2_f2", ptr(f), ptr(f), f.numel(), st)
        call("sp_fft2", ptr(f), ptr(f), N, L, 0, st)
        call("sp_multiply_axis_f_f2", L, ptr(ipd), ptr(f), ptr(f), N * N, st)
        call("sp_fft2", ptr(f), ptr(f), N, L, 1, st)
        call("sp_sqrt_f2", ptr(f), ptr(f), f.numel(), st)
    else:
        call("sp_abs_f2_f2", ptr(f), ptr(f), f.numel(), st)
    acc = torch.empty((N, N), dtype=torch.float32, device=g.device)
    call("sp_rftf_accumulate", L, ptr(g), ptr(acc), ptr(f), N, 1, st)
    res = acc.cpu().numpy() if was_np else acc
    if rftfq:
        return res, unwrap_average(acc, as_numpy=was_np)
    return res


def covar_results(gpuinfo, data, threshold=0.85, mask=None):
    """Pair-wise similarity of reconstructions for configuration sorting
    (``phasing.py:1817-1982``): frames zero-padded to N x N (the larger edge
    if a power of two, else 2**(round(log2 edge) + 1), as ``_reshape_data``
    computes it), their transforms D, cc[n, m] = max |IFFT2(conj(D_n) D_m)|
    for the pairs the mask selects, covars = cc/sqrt(cc_nn cc_mm) (NaN -> 0),
    and per-row stats (row, mean covariance, count above ``threshold``).
    ``mask``: an array, or a float p drawing a random pair mask with numpy's
    global RNG as the reference does (default 1.0: every pair).  Returns
    (cc, covars, stats, transforms).  The reference's own version cannot run
    (it reads an undefined ``self``); ``gpuinfo`` is ignored."""
    data = np.asarray(data)
    if data.ndim != 3:
        raise ValueError("data must be 3d")
    frames, rows, cols = data.shape
    e = max(rows, cols)
    N = e if e & (e - 1) == 0 else 2 ** (int(round(np.log2(e))) + 1)
    _pow2_size(N, "covar_results")
    if mask is None:
        mask = 1.0
    if not isinstance(mask, np.ndarray):
        mask = np.where(np.random.rand(frames, frames) < mask, 1, 0)
    d = torch.zeros((frames, N, N), dtype=torch.complex64, device="cuda")
    d[:, :rows, :cols] = torch.from_numpy(np.ascontiguousarray(data.astype(np.complex64))).cuda()
    st = stream_ptr()
    call("sp_fft2", ptr(d), ptr(d), N, frames, 0, st)
    pairs = [(n, m) for n in range(frames) for m in (np.nonzero(mask[n, n:])[0] + n)]
    cc = np.zeros((frames, frames))
    if pairs:
        pr = torch.tensor(pairs, dtype=torch.int32, device="cuda").contiguous()
        planes = max(1, min(len(pairs), (512 << 20) // (N * N * 8)))
        work = torch.empty((planes, N, N), dtype=torch.complex64, device="cuda")
        vals = torch.empty(len(pairs), dtype=torch.float32, device="cuda")
        call("sp_covar_pairs", ptr(d), N, ptr(pr), len(pairs), ptr(work), planes, ptr(vals), st)
        for (n, m), v in zip(pairs, vals.cpu().numpy().astype(np.float64)):
            cc[n, m] = cc[m, n] = v
    covars = np.zeros((frames, frames))
    with np.errstate(divide="ignore", invalid="ignore"):
        for n, m in pairs:
            covars[n, m] = covars[m, n] = cc[n, m] / np.sqrt(cc[n, n] * cc[m, m])
    covars = np.nan_to_num(covars)
    stats = None
    if threshold > 0:
        stats = np.zeros((frames, 3))
        for row in range(frames):
            stats[row] = row, np.average(covars[row]), np.sum(covars[row] > threshold)
    return cc, covars, stats, d.cpu().numpy()
