"""ctypes bindings of libspeckle_b200.so (the C ABI in include/speckle_b200.h).

The library is required: importing this module raises if it is missing,
so no operation silently runs elsewhere.  Device memory is owned by torch;
the bindings pass raw pointers and sizes only.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspeckle_b200.so")

SP_OK = 0
SP_HIO, SP_ER, SP_RAAR, SP_SF, SP_DM, SP_ER_CPU, SP_SF_CPU = range(7)
SP_INIT_GIVEN, SP_INIT_RANDOM_PHASE = 0, 1
SP_MAX_RUNS = 8

ALG_CODES = {"hio": SP_HIO, "er": SP_ER, "raar": SP_RAAR, "sf": SP_SF, "dm": SP_DM}
CPU_QUIRK_CODES = {"er": SP_ER_CPU, "sf": SP_SF_CPU}


class SpeckleError(RuntimeError):
    """A libspeckle_b200 call returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__("%s (status %d): %s" % (STATUS_NAMES.get(status, "error"), status, message))
        self.status = status


STATUS_NAMES = {1: "invalid argument", 2: "unsupported size", 3: "CUDA error",
                4: "workspace too small", 5: "unsupported", 6: "not found"}


class sp_trial(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("n_iter", C.c_int32), ("n_runs", C.c_int32),
        ("run_alg", C.c_int32 * SP_MAX_RUNS), ("run_count", C.c_int32 * SP_MAX_RUNS),
        ("beta", C.c_float), ("init", C.c_int32), ("seed", C.c_uint32), ("trial", C.c_uint32),
        ("r0", C.c_int32), ("c0", C.c_int32), ("rows", C.c_int32), ("cols", C.c_int32),
        ("psi_dev", C.c_void_p), ("modulus_dev", C.c_void_p), ("support_dev", C.c_void_p),
        ("save_dev", C.c_void_p), ("errors_dev", C.c_void_p), ("ipsf_dev", C.c_void_p),
        ("spectrum_rescale_dev", C.c_void_p), ("spectrum_weight_dev", C.c_void_p),
        ("spectrum_n", C.c_int32),
    ]


class sp_run_opts(C.Structure):
    _fields_ = [("l2_group_bytes", C.c_int64), ("use_graph", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("e_per_logn", C.c_int32 * 13)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libspeckle_b200.so is not built (expected at %s); run "
            "`python -m als_speckle_b200.build` with the CUDA toolkit" % LIB_PATH)
    return C.CDLL(LIB_PATH)


lib = _load()

_i, _p, _f, _d, _i64, _sz = C.c_int, C.c_void_p, C.c_float, C.c_double, C.c_int64, C.c_size_t
_SIGS = {
    "sp_version": ([], _i),
    "sp_status_string": ([_i], C.c_char_p),
    "sp_last_error": ([], C.c_char_p),
    "sp_device_init": ([], _i),
    "sp_engine_workspace_size": ([C.POINTER(sp_trial), _i, C.POINTER(_sz)], _i),
    "sp_engine_run": ([C.POINTER(sp_trial), _i, _p, _sz, C.POINTER(sp_run_opts), _p], _i),
    "sp_engine_release_graphs": ([], _i),
    "sp_engine_last_launches": ([], C.c_int64),
    "sp_engine_graph_count": ([], C.c_int64),
    "sp_engine_release_device_graphs": ([], _i),
    "sp_engine_run_static": ([C.POINTER(sp_trial), _i, C.POINTER(sp_run_opts), _p], _i),
    "sp_hio": ([_f, _p, _p, _p, _p, _i64, _p], _i),
    "sp_er": ([_p, _p, _p, _i64, _p], _i),
    "sp_raar": ([_f, _p, _p, _p, _p, _i64, _p], _i),
    "sp_sf": ([_p, _p, _p, _p, _i64, _p], _i),
    "sp_dm1": ([_f, _p, _p, _p, _i64, _p], _i),
    "sp_dm2": ([_f, _f, _p, _p, _p, _p, _p, _i64, _p], _i),
    "sp_fourier": ([_p, _p, _p, _p, _i64, _p], _i),
    "sp_abs_f2_f2": ([_p, _p, _i64, _p], _i),
    "sp_copy_to_buffer_f2": ([_p, _p, _i, _i, _i, _i, _i, _i, _p], _i),
    "sp_prtf_accumulate": ([_i, _p, _p, _i, _p], _i),
    "sp_fft2": ([_p, _p, _i, _i, _i, _p], _i),
    "sp_align_global_phase": ([_p, _i, _i64, _p, _p, _p], _i),
    "sp_prtf": ([_p, _i, _i, _i, _i, _p, _p, _p], _i),
    "sp_shrinkwrap": ([_p, _i, _i, _p, _p, _p, _i, _d, _d, _i, _p, _p, _p, _p, _p], _i),
    "sp_mean_frames": ([_p, _i, _i64, _p, _p], _i),
    "sp_prtf_phasors": ([_p, _i, _i, _i, _i, _p, _p, _p], _i),
    "sp_prtf_finish": ([_p, _i, _i, _p, _p], _i),
    "sp_xcorr_peak": ([_p, _p, _i, _i, _p, _p, _p], _i),
    "sp_roll": ([_p, _p, _i, _i, _i, _i, _p], _i),
    "sp_com_sums": ([_p, _i, _i, _i, _p, _p], _i),
    "sp_roll_accumulate": ([_p, _i, _i, _i, _p, _p, _p], _i),
    "sp_plain_iterate": ([_i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _p], _i),
    "sp_unwrap": ([_p, _i, _i, _i, _d, _d, _i, _p, _p, _p, _p], _i),
    "sp_register_workspace_size": ([_i, _i, _i, C.POINTER(_sz)], _i),
    "sp_register_subpixel": ([_p, _i, _i, _i, _p, _i, _i, _p, _sz, _p, _p, _p], _i),
    "sp_abs2_f2_f2": ([_p, _p, _i64, _p], _i),
    "sp_sqrt_f2": ([_p, _p, _i64, _p], _i),
    "sp_sqrt_abs_f2": ([_p, _p, _i64, _p], _i),
    "sp_multiply_axis_f_f2": ([_i, _p, _p, _p, _i64, _p], _i),
    "sp_multiply_f2_f2": ([_p, _p, _p, _i64, _p], _i),
    "sp_rftf_accumulate": ([_i, _p, _p, _p, _i, _i, _p], _i),
    "sp_rftf_map": ([_p, _p, _i, _i, _p, _p, _p, _p], _i),
    "sp_rftf_from_error": ([_p, _p, _i64, _i, _p], _i),
    "sp_remove_hot_pixels": ([_p, _p, _i, _i, _i, _i, _f, _p], _i),
    "sp_covar_pairs": ([_p, _i, _p, _i, _p, _i, _p, _p], _i),
    "sp_divide_f2_f2": ([_p, _p, _p, _i64, _p], _i),
    "sp_flip_f2": ([_p, _p, _i, _i, _p], _i),
    "sp_gaussian": ([_p, _i, _f, _f, _i, _p], _i),
    "sp_richardson_lucy": ([_p, _p, _p, _p, _p, _i, _i, _i, _p], _i),
    "sp_coherence_misfit": ([_p, _p, _f, _f, _i, _p, _p, _p], _i),
}
for _name, (_args, _res) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res


def check(status):
    if status != SP_OK:
        msg = lib.sp_last_error()
        raise SpeckleError(status, msg.decode() if msg else "")
    return status


def call(name, *args):
    """Call ``sp_<name>`` and raise SpeckleError on a non-zero status."""
    return check(getattr(lib, name)(*args))


def ptr(t):
    """Device (or host) address of a tensor, or None for None."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def symbols():
    """Names of the C entry points bound here."""
    return sorted(_SIGS)
