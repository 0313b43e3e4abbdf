"""FITS input/output (the reference's speckle.io FITS functions, written here
from the FITS standard since pyfits is not available): round trips, a
hand-built known-answer file, IMAGE extensions with the LabView
orientation, scaling keywords, header items and the complex helpers."""
import os
import struct

import numpy as np
import pytest

from als_speckle_b200 import io as sio


def card(text):
    return text.ljust(80).encode("ascii")


def block(b, fill=b" "):
    return b + fill * ((-len(b)) % 2880)


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.int32, np.int64, np.float32, np.float64,
                                   np.uint16, np.uint32])
@pytest.mark.parametrize("shape", [(5, 7), (3, 4, 9), (64, 64)])
def test_round_trip(tmp_path, dtype, shape):
    rng = np.random.default_rng(1)
    if np.dtype(dtype).kind == "f":
        a = rng.standard_normal(shape).astype(dtype)
    else:
        info = np.iinfo(dtype)
        a = rng.integers(max(info.min, -10 ** 6), min(info.max, 10 ** 6), shape).astype(dtype)
        a.flat[0] = info.max if dtype in (np.uint16, np.uint32, np.uint8) else a.flat[0]
    f = str(tmp_path / "a.fits")
    sio.writefits(f, a)
    assert os.path.getsize(f) % 2880 == 0
    b = sio.openfits(f)
    assert b.dtype == a.dtype and b.shape == a.shape and np.array_equal(a, b)


def test_known_answer_file(tmp_path):
    """A file built by hand from the standard: BITPIX -32, NAXIS1 = 3 (the
    fast axis), NAXIS2 = 2, big-endian floats."""
    head = b"".join(card(c) for c in ["SIMPLE  =                    T", "BITPIX  =                  -32",
                                       "NAXIS   =                    2", "NAXIS1  =                    3",
                                       "NAXIS2  =                    2", "OBJECT  = 'speckle '", "END"])
    vals = [1.5, -2.0, 3.25, 0.0, 1e-3, 7.0]
    data = struct.pack(">6f", *vals)
    f = tmp_path / "k.fits"
    f.write_bytes(block(head) + block(data, b"\0"))
    a = sio.openfits(str(f))
    assert a.shape == (2, 3)
    assert np.array_equal(a, np.array(vals, np.float32).reshape(2, 3))
    assert sio.openheader(str(f))["OBJECT"] == "speckle"


def test_written_header_layout(tmp_path):
    f = str(tmp_path / "w.fits")
    sio.writefits(f, np.zeros((2, 3), np.float64), header_items={"EXPOSURE": 0.5, "LONGKEYWORD": 3})
    raw = open(f, "rb").read()
    cards = [raw[i:i + 80].decode() for i in range(0, 2880, 80)]
    assert cards[0] == "SIMPLE  =                    T".ljust(80)
    assert cards[1].startswith("BITPIX  =                  -64")
    assert cards[3].startswith("NAXIS1  =                    3")
    assert cards[4].startswith("NAXIS2  =                    2")
    h = sio.openheader(f)
    assert h["EXPOSURE"] == 0.5 and h["LONGKEYWORD"] == 3
    assert raw[2880:2880 + 48] == b"\0" * 48


def test_image_extension_and_labview_orientation(tmp_path):
    img = np.arange(12, dtype=">i2").reshape(3, 4)
    prim = b"".join(card(c) for c in ["SIMPLE  =                    T", "BITPIX  =                    8",
                                       "NAXIS   =                    0", "EXTEND  =                    T", "END"])
    ext = b"".join(card(c) for c in ["XTENSION= 'IMAGE   '", "BITPIX  =                   16",
                                      "NAXIS   =                    2", "NAXIS1  =                    4",
                                      "NAXIS2  =                    3", "PCOUNT  =                    0",
                                      "GCOUNT  =                    1", "END"])
    f = tmp_path / "lv.fits"
    f.write_bytes(block(prim) + block(ext) + block(img.tobytes(), b"\0"))
    raw = sio.openfits(str(f), orientImageHDU=False)
    assert np.array_equal(raw, img.astype(np.int16))
    assert np.array_equal(sio.openfits(str(f)), np.rot90(np.fliplr(img.astype(np.int16))))


def test_bzero_bscale(tmp_path):
    head = b"".join(card(c) for c in ["SIMPLE  =                    T", "BITPIX  =                   16",
                                       "NAXIS   =                    1", "NAXIS1  =                    3",
                                       "BZERO   =                 10.0", "BSCALE  =                  0.5", "END"])
    f = tmp_path / "s.fits"
    f.write_bytes(block(head) + block(struct.pack(">3h", -4, 0, 6), b"\0"))
    assert np.allclose(sio.openfits(str(f)), [8.0, 10.0, 13.0])


def test_overwrite(tmp_path):
    f = str(tmp_path / "o.fits")
    sio.writefits(f, np.ones((2, 2), np.float32))
    with pytest.raises(IOError):
        sio.writefits(f, np.zeros((2, 2), np.float32))
    sio.writefits(f, np.zeros((2, 2), np.float32), overwrite=True)
    assert np.all(sio.openfits(f) == 0)


def test_complex_helpers(tmp_path):
    rng = np.random.default_rng(2)
    z = (rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8))).astype(np.complex64)
    base = str(tmp_path / "z")
    sio.write_complex_fits(base, z)
    assert np.allclose(sio.open_complex_fits(base), z)
    base2 = str(tmp_path / "p")
    sio.write_mag_phase_fits(base2, z)
    assert np.allclose(sio.open_complex_fits(base2), z, atol=1e-6)  # falls back to mag/phase
    sio.save(str(tmp_path / "s.fits"), z, components=["polar"])
    assert os.path.exists(str(tmp_path / "s_mag.fits")) and os.path.exists(str(tmp_path / "s_phase.fits"))
    with pytest.raises(NotImplementedError):
        sio.open(str(tmp_path / "x.png"))
