"""``phasing.iterate(debug_on=...)``: the listed iterations run one operator
at a time (the reference's GPU dataflow) and write the reference's debugging
FITS files (``phasing.py:1193-1227``, ``:1244-1246``); the run's result equals
the fused run's to the engine's trajectory tolerance (1e-4 relative: the
operator path transforms with the standalone FFT, whose rounding differs)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(tmp_path, debug_on):
    import torch
    from als_speckle_b200 import synth
    from als_speckle_b200.phasing import phasing
    _, M, S = synth.pattern(64, n_ellipses=4, box=16, peak=1e5, seed=2, support_edge=20)
    r = phasing()
    r.load(modulus=M, support=S, numtrials=2)
    r.seed(7)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        r.iterate(5, order=(("hio", 2), ("dm", 1), ("er", 1), ("raar", 1)), beta=0.9,
                  debug_on=debug_on)
    finally:
        os.chdir(cwd)
    torch.cuda.synchronize()
    return r


def test_debug_dumps_and_result(tmp_path):
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    a = _run(tmp_path / "a", None)
    b = _run(tmp_path / "b", (0, 2, 4))
    names = sorted(os.listdir(tmp_path / "b"))
    for it in (0, 2, 4):
        for stem, comps in (("psi_fourier_1", ("mag", "phase")), ("fourier_div", ("mag", "phase")),
                            ("psi_fourier_2", ("mag", "phase")), ("out", ("real", "imag"))):
            for c in comps:
                assert "gpu i%d %s_%s.fits" % (it, stem, c) in names, names
    assert "gpu i0 hio update_real.fits" in names and "gpu i0 hio update_imag.fits" in names
    assert not os.listdir(tmp_path / "a")
    pa, pb = a.psi_in.cpu().numpy(), b.psi_in.cpu().numpy()
    assert np.linalg.norm(pa - pb) / np.linalg.norm(pa) < 1e-4
    sa, sb = a.savebuffer[0].cpu().numpy(), b.savebuffer[0].cpu().numpy()
    assert np.linalg.norm(sa - sb) / np.linalg.norm(sa) < 1e-4
    ea, eb = a.modulus_error(), b.modulus_error()
    assert np.allclose(ea, eb, rtol=1e-4)
    # the dumped modulus of the first transform is |FFT(psi_0)|, fftshifted
    from als_speckle_b200 import io
    mag = io.openfits(str(tmp_path / "b" / "gpu i0 psi_fourier_1_mag.fits"))
    assert mag.shape == (64, 64)
