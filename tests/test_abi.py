"""The C-ABI library loads, exports every declared symbol, and its struct
layouts agree with the Python bindings.  No GPU needed."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "speckle_b200.h")
LIB = os.path.join(ROOT, "als_speckle_b200", "libspeckle_b200.so")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|int64_t|const char\*)\s+(sp_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from als_speckle_b200 import build
        build.build()
    return C.CDLL(LIB)


def test_every_declared_symbol_is_exported(lib):
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n


def test_bindings_cover_header():
    from als_speckle_b200 import _lib
    assert set(declared()) <= set(_lib.symbols())


def test_struct_layout_matches_c(tmp_path):
    """Compile a host C program against the header and compare sizes/offsets."""
    from als_speckle_b200 import _lib
    src = tmp_path / "layout.c"
    src.write_text('''
#include <stdio.h>
#include <stddef.h>
#include "speckle_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(sp_trial), offsetof(sp_trial, beta),
         offsetof(sp_trial, psi_dev), offsetof(sp_trial, errors_dev), sizeof(sp_run_opts),
         offsetof(sp_run_opts, e_per_logn), offsetof(sp_trial, r0), offsetof(sp_trial, ipsf_dev),
         offsetof(sp_trial, spectrum_n));
  return 0;
}''')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)])
    vals = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    T, O = _lib.sp_trial, _lib.sp_run_opts
    assert vals == [C.sizeof(T), T.beta.offset, T.psi_dev.offset, T.errors_dev.offset,
                    C.sizeof(O), O.e_per_logn.offset, T.r0.offset, T.ipsf_dev.offset,
                    T.spectrum_n.offset]


def test_host_side_errors_without_gpu(lib):
    """Argument checks run before any CUDA call and return status codes."""
    from als_speckle_b200 import _lib
    t = (_lib.sp_trial * 1)()
    t[0].n = 100  # not a power of two
    need = C.c_size_t(0)
    assert _lib.lib.sp_engine_workspace_size(t, 1, C.byref(need)) == 2
    assert b"power of two" in _lib.lib.sp_last_error()
    assert _lib.lib.sp_fft2(None, None, 512, 1, 0, None) == 1
    assert _lib.lib.sp_fft2(C.c_void_p(16), C.c_void_p(16), 48, 1, 0, None) == 2
    assert _lib.lib.sp_status_string(4) == b"workspace too small"
    t[0].n = 64
    t[0].n_runs = 0
    assert _lib.lib.sp_engine_run(t, 1, None, 0, None, None) == 1
    with pytest.raises(_lib.SpeckleError):
        _lib.call("sp_fft2", None, None, 512, 1, 0, None)


def test_registration_and_unwrap_argument_checks_without_gpu(lib):
    """The subpixel registration and the polar unwrap reject bad arguments
    before any CUDA call; the registration workspace size is host
    arithmetic and grows with the frame count."""
    from als_speckle_b200 import _lib
    L = _lib.lib
    b = C.c_size_t(0)
    assert L.sp_register_workspace_size(4, 256, 64, C.byref(b)) == 0 and b.value > 0
    b4 = b.value
    assert L.sp_register_workspace_size(8, 256, 64, C.byref(b)) == 0 and b.value > b4
    assert L.sp_register_workspace_size(4, 100, 64, C.byref(b)) == 2   # N not a power of two
    assert L.sp_register_workspace_size(4, 256, 0, C.byref(b)) == 1    # upsample below 1
    assert L.sp_register_workspace_size(4, 256, 171, C.byref(b)) == 1  # upsample above 170
    assert L.sp_register_workspace_size(0, 256, 64, C.byref(b)) == 1   # no frames
    p = C.c_void_p(256)
    d = C.cast(p, C.POINTER(C.c_double))
    # frames larger than N, then a missing reference
    assert L.sp_register_subpixel(p, 2, 300, 300, p, 256, 64, p, b4, d, p, None) == 1
    assert L.sp_register_subpixel(p, 2, 100, 100, None, 256, 64, p, b4, d, p, None) == 1
    f = C.cast(p, C.POINTER(C.c_float))
    w = C.cast(p, C.POINTER(C.c_double))
    # no input, no output, empty radius range, grid outside the map
    assert L.sp_unwrap(None, 64, 0, 32, 32.0, 32.0, 0, w, f, f, None) == 1
    assert L.sp_unwrap(f, 64, 0, 32, 32.0, 32.0, 0, w, None, None, None) == 1
    assert L.sp_unwrap(f, 64, 10, 10, 32.0, 32.0, 0, w, f, f, None) == 1
    assert L.sp_unwrap(f, 64, 0, 40, 32.0, 32.0, 0, w, f, f, None) == 1
