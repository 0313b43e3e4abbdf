"""Device dispatch, the counterpart of ``speckle/gpu.py``'s ``common`` class.

The reference looks kernels up by name (``common._kexec``, ``gpu.py:295-372``:
``<project>_<name>.cl`` then ``common_<name>.cl``) and passes buffers and
scalars positionally.  Here the same names map to entry points of
libspeckle_b200 with the same argument order; there is no CPU branch.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream_ptr


def _numel(args):
    sizes = [a.numel() for a in args if isinstance(a, torch.Tensor)]
    if not sizes:
        raise ValueError("_kexec needs at least one device buffer")
    return max(sizes)


def _f(x):
    return float(np.float32(x))


# name -> (entry point, positional layout).  'b','g' are float scalars, 'i' ints,
# 'B' a device buffer; the element count is appended like the reference's
# global size (max buffer size, gpu.py:311-320).
_OPS = {
    "hio": ("sp_hio", "fBBBB"),            # (b, support, psi_in, psi_out, output)
    "er": ("sp_er", "BBB"),                # (support, psi_out, output)
    "raar": ("sp_raar", "fBBBB"),          # (b, support, psi_in, psi_out, output)
    "sf": ("sp_sf", "BBBB"),               # (support, psi_in, psi_out, output)
    "dm1": ("sp_dm1", "fBBB"),             # (g, support, psi_in, output)
    "dm2": ("sp_dm2", "ffBBBBB"),          # (b, g, support, psi_in, psi_out, dm_tmp, output)
    "fourier": ("sp_fourier", "BBBB"),     # (psi, div, mod, out)
    "abs_f2_f2": ("sp_abs_f2_f2", "BB"),   # (in, out)
}


class common:
    """Mixin with the reference's device helpers (``gpu.py:17-421``)."""

    use_gpu = True
    device = None

    def _stream(self):
        return stream_ptr()

    def _kexec(self, name, *args, **kwargs):
        """Run the operator ``name`` with the reference's positional arguments."""
        if name == "copy_to_buffer_f2":
            # (dst, src, c0, r0, n, N, shape=(cols, rows)), phasing_copy_to_buffer_f2.cl
            dst, src, c0, r0, n, N = args
            cols, rows = kwargs["shape"]
            call("sp_copy_to_buffer_f2", ptr(dst), ptr(src), int(c0), int(r0), int(n), int(N),
                 int(cols), int(rows), self._stream())
            return
        if name == "prtf_accumulate2":
            # (frames, fft, prtf, shape=(N, N)), phasing_prtf_accumulate2.cl
            frames, fft, prtf = args
            N = kwargs["shape"][0]
            call("sp_prtf_accumulate", int(frames), ptr(fft), ptr(prtf), int(N), self._stream())
            return
        if name not in _OPS:
            raise _lib.SpeckleError(6, "no operator named %r" % name)
        entry, layout = _OPS[name]
        if len(args) != len(layout):
            raise TypeError("%s takes %d arguments (%d given)" % (name, len(layout), len(args)))
        conv = []
        for kind, a in zip(layout, args):
            if kind == "f":
                conv.append(_f(a))
            else:
                if not isinstance(a, torch.Tensor) or not a.is_cuda:
                    raise TypeError("%s: buffers must be CUDA tensors" % name)
                conv.append(ptr(a))
        n = kwargs.get("n", _numel(args))
        call(entry, *conv, int(n), self._stream())

    def _cl_abs(self, in1, out):
        self._kexec("abs_f2_f2", in1, out)

    def _allocate(self, size, dtype, name=None):
        dt = {np.float32: torch.float32, np.complex64: torch.complex64}.get(np.dtype(dtype).type)
        if dt is None:
            raise TypeError("unsupported dtype %s" % dtype)
        return torch.zeros(size, dtype=dt, device=self.device)

    def _set(self, what, where):
        """Copy host ``what`` into device ``where`` (gpu.py:374-387)."""
        what = np.ascontiguousarray(what)
        if tuple(what.shape) != tuple(where.shape):
            raise ValueError("incompatible shapes %s %s" % (what.shape, tuple(where.shape)))
        where.copy_(torch.from_numpy(what).to(where.dtype))
        return where

    def get(self, something):
        """Device tensor -> numpy (gpu.py:389-397); other objects pass through."""
        if isinstance(something, torch.Tensor):
            return something.detach().cpu().numpy()
        return something
