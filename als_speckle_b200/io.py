"""FITS input and output for moduli, supports and reconstructions, replacing
the pyfits-based functions of ``speckle.io`` (``io.py:35-94`` ``open`` /
``save``, ``:384-443`` ``openfits``, ``:502-624`` the writers and complex
helpers, ``:626-645`` ``_labview_to_andor``, ``:714-748`` ``save_fits``).

pyfits is not available, so files are read and written here directly from
the FITS standard (version 4.0): a file is a sequence of header-data units;
a header is 80-character ASCII cards in 2880-byte blocks ending with END; the
data that follows is big-endian, ``BITPIX`` 8/16/32/64 (integers) or
-32/-64 (IEEE floats), ``NAXISn`` with the fastest axis first, physical
value = ``BZERO + BSCALE * stored``, padded with zeros to a 2880-byte block.
Primary HDUs and IMAGE extensions are supported; other extensions are
skipped.  Same function names, arguments and behaviour as the reference;
other formats of ``io.open`` / ``io.save`` (images, text, pickles, DS9
masks) are outside this library.
"""
from __future__ import annotations

import builtins
import os

import numpy as np

BLOCK = 2880
CARD = 80

overwrite_default = False


def set_overwrite(val):
    """Default overwrite behaviour of the FITS writers (``io.py:20-32``)."""
    global overwrite_default
    if isinstance(val, bool):
        overwrite_default = val


# --------------------------------------------------------------------------
# header cards
# --------------------------------------------------------------------------
def _parse_value(text):
    """Value of a card's value field (after '= '), comment stripped."""
    t = text.strip()
    if t.startswith("'"):
        # string: '' is an escaped quote; trailing blanks are not significant
        out, i = [], 1
        while i < len(t):
            if t[i] == "'":
                if i + 1 < len(t) and t[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(t[i])
            i += 1
        return "".join(out).rstrip()
    if "/" in t:
        t = t[:t.index("/")].strip()
    if t == "T":
        return True
    if t == "F":
        return False
    if t == "":
        return None
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(t.replace("D", "E"))
    except ValueError:
        return t


def _format_value(v):
    if isinstance(v, (bool, np.bool_)):
        return "%20s" % ("T" if v else "F")
    if isinstance(v, (int, np.integer)):
        return "%20d" % int(v)
    if isinstance(v, (float, np.floating)):
        s = repr(float(v)).upper()
        if "E" not in s and "." not in s and "N" not in s:
            s += ".0"
        return "%20s" % s
    s = str(v).replace("'", "''")
    return "'%-8s'" % s


def _card(key, value=None, comment=None):
    key = key.upper()
    if len(key) > 8 or " " in key:
        # long or spaced keywords use the HIERARCH convention, as io.py:534
        body = "HIERARCH %s = %s" % (key, _format_value(value).strip())
    elif value is None and key in ("END", "COMMENT", "HISTORY", ""):
        body = "%-8s%s" % (key, comment or "")
    else:
        body = "%-8s= %s" % (key, _format_value(value))
        if comment:
            body += " / " + comment
    if len(body) > CARD:
        raise ValueError("header card too long: %s" % body)
    return body.ljust(CARD)


def _read_header(f):
    """Cards of one header as an ordered dict, or None at end of file."""
    cards = {}
    while True:
        block = f.read(BLOCK)
        if not block:
            return None
        if len(block) < BLOCK:
            raise ValueError("truncated FITS header")
        text = block.decode("ascii", errors="replace")
        for k in range(0, BLOCK, CARD):
            c = text[k:k + CARD]
            key = c[:8].strip()
            if key == "END":
                return cards
            if key == "HIERARCH" and "=" in c:
                name, val = c[9:].split("=", 1)
                cards[name.strip()] = _parse_value(val)
            elif c[8:10] == "= ":
                cards[key] = _parse_value(c[10:])
            elif key in ("COMMENT", "HISTORY"):
                cards.setdefault(key, []).append(c[8:].rstrip())


_DTYPES = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


def _data_bytes(h):
    """Bytes of the data unit (|BITPIX|/8 * GCOUNT * (PCOUNT + NAXIS1*...*NAXISn))
    and the axis lengths."""
    naxis = int(h.get("NAXIS", 0))
    if naxis == 0:
        return 0, ()
    dims = tuple(int(h["NAXIS%d" % i]) for i in range(1, naxis + 1))
    n = abs(int(h["BITPIX"])) // 8 * int(h.get("GCOUNT", 1)) * (int(h.get("PCOUNT", 0)) + int(np.prod(dims)))
    return n, dims


def _read_data(f, h):
    n, dims = _data_bytes(h)
    if n == 0:
        return None, 0
    raw = f.read(n)
    if len(raw) < n:
        raise ValueError("truncated FITS data")
    pad = (-n) % BLOCK
    if pad:
        f.read(pad)
    bitpix = int(h["BITPIX"])
    a = np.frombuffer(raw[:abs(bitpix) // 8 * int(np.prod(dims))], dtype=_DTYPES[bitpix])
    a = a.reshape(dims[::-1])  # NAXIS1 is the fastest axis
    bzero, bscale = h.get("BZERO", 0), h.get("BSCALE", 1)
    if bitpix == 16 and bzero == 32768 and bscale == 1:
        return (a.astype(np.int32) + 32768).astype(np.uint16), n
    if bitpix == 32 and bzero == 2147483648 and bscale == 1:
        return (a.astype(np.int64) + 2147483648).astype(np.uint32), n
    if bzero != 0 or bscale != 1:
        return bzero + bscale * a.astype(np.float64 if bitpix in (32, 64, -64) else np.float32), n
    return a.astype(a.dtype.newbyteorder("=")), n


def read_hdus(filename):
    """Every header-data unit of a FITS file: a list of (header dict, data)."""
    out = []
    with builtins.open(filename, "rb") as f:
        while True:
            h = _read_header(f)
            if h is None:
                break
            data, _ = _read_data(f, h)
            out.append((h, data))
    if not out:
        raise ValueError("%s is not a FITS file" % filename)
    return out


# --------------------------------------------------------------------------
# the reference's functions
# --------------------------------------------------------------------------
def _labview_to_andor(img):
    """LabView rotates and flips its images; undo it (``io.py:626-645``):
    rotate 90 degrees counter-clockwise after a left-right flip, per frame."""
    if img.ndim not in (2, 3):
        raise ValueError("_labview_to_andor: Image is neither 2D nor 3D.")
    if img.ndim == 3:
        img = np.array(img)
        for f in range(img.shape[0]):
            img[f] = np.rot90(np.fliplr(img[f]))
        return img
    return np.rot90(np.fliplr(img))


def openfits(filename, quiet=True, orientImageHDU=True):
    """Open a FITS file (``io.py:384-443``): the data of the first IMAGE
    extension if there is one (written by LabView; reoriented if
    ``orientImageHDU``), else the primary HDU's."""
    if not os.path.exists(filename):
        raise AssertionError("unknown file %s" % filename)
    hdus = read_hdus(filename)
    for h, data in hdus[1:]:
        if h.get("XTENSION") == "IMAGE":
            if not quiet:
                print("openfits: %s data located in ImageHDU" % filename)
            return _labview_to_andor(data) if orientImageHDU else data
    if not quiet:
        print("openfits: %s data located in PrimaryHDU" % filename)
    return hdus[0][1]


def openframe(filename, frame=0, quiet=True):
    """One frame of a 3d FITS image (``io.py:445-466``)."""
    data = openfits(filename, quiet=quiet)
    if data.ndim == 3:
        return data[frame]
    return data


def openheader(filename, card=0):
    """The header of HDU ``card`` as a dict (``io.py:468-478``)."""
    return read_hdus(filename)[card][0]


open_fits_header = openheader


def _bitpix_of(img):
    kinds = {np.dtype(np.uint8): (8, None), np.dtype(np.int16): (16, None),
             np.dtype(np.int32): (32, None), np.dtype(np.int64): (64, None),
             np.dtype(np.float32): (-32, None), np.dtype(np.float64): (-64, None),
             np.dtype(np.uint16): (16, 32768), np.dtype(np.uint32): (32, 2147483648),
             np.dtype(np.bool_): (8, None), np.dtype(np.int8): (16, None)}
    dt = np.dtype(img.dtype).newbyteorder("=")
    if dt not in kinds:
        raise TypeError("cannot write data of type %s to FITS" % img.dtype)
    return kinds[dt]


def writefits(filename, img, header_items=None, overwrite=None):
    """Write ``img`` as the primary HDU of a FITS file (``io.py:502-552``),
    with ``header_items`` added to the header (keys longer than eight
    characters as HIERARCH cards).  An existing file is replaced only with
    ``overwrite`` (default: ``set_overwrite``'s value)."""
    if header_items is None:
        header_items = {}
    if not isinstance(header_items, dict):
        raise AssertionError("header_items must be a dictionary")
    if overwrite is None:
        overwrite = overwrite_default
    if not isinstance(img, np.ndarray):
        raise AssertionError("array to save must be an array")
    if os.path.exists(filename) and not overwrite:
        raise IOError("File %s already exists. Try overwrite=True keyword with "
                      "speckle.io.writefits()" % filename)
    bitpix, bzero = _bitpix_of(img)
    cards = [_card("SIMPLE", True), _card("BITPIX", bitpix), _card("NAXIS", img.ndim)]
    for i, n in enumerate(img.shape[::-1]):
        cards.append(_card("NAXIS%d" % (i + 1), int(n)))
    cards.append(_card("EXTEND", True))
    if bzero is not None:
        cards.append(_card("BZERO", bzero))
        cards.append(_card("BSCALE", 1))
    for k, v in header_items.items():
        cards.append(_card(k, v))
    cards.append(_card("END"))
    head = "".join(cards).encode("ascii")
    head += b" " * ((-len(head)) % BLOCK)
    if bzero is not None:
        stored = (img.astype(np.int64) - bzero).astype(_DTYPES[bitpix])
    elif img.dtype == np.bool_:
        stored = img.astype(">u1")
    elif img.dtype == np.int8:
        stored = img.astype(">i2")
    else:
        stored = img.astype(_DTYPES[bitpix])
    data = np.ascontiguousarray(stored).tobytes()
    data += b"\0" * ((-len(data)) % BLOCK)
    with builtins.open(filename, "wb") as f:
        f.write(head)
        f.write(data)


def write_complex_fits(base, fits, header_items=None, overwrite=None):
    """``base_imag.fits`` and ``base_real.fits`` (``io.py:554-568``)."""
    writefits(base + "_imag.fits", np.imag(fits), header_items or {}, overwrite)
    writefits(base + "_real.fits", np.real(fits), header_items or {}, overwrite)


def write_mag_phase_fits(base, fits, header=None, header_items=None, overwrite=None):
    """``base_mag.fits`` and ``base_phase.fits`` (``io.py:570-590``)."""
    writefits(base + "_mag.fits", np.abs(fits), header_items or {}, overwrite)
    writefits(base + "_phase.fits", np.angle(fits), header_items or {}, overwrite)


def open_mag_phase_fits(base):
    """mag * exp(i phase) from ``write_mag_phase_fits`` files (``io.py:592-606``)."""
    return openfits(base + "_mag.fits") * np.exp(1j * openfits(base + "_phase.fits"))


def open_complex_fits(base):
    """real + i imag from ``write_complex_fits`` files, else the mag/phase
    pair (``io.py:608-624``)."""
    try:
        return openfits(base + "_real.fits") + 1j * openfits(base + "_imag.fits")
    except AssertionError:
        return open_mag_phase_fits(base)


_COMPONENTS = {"mag": np.abs, "phase": np.angle, "real": np.real, "imag": np.imag}


def save_fits(filename, img, header=None, components=None, overwrite=None, append_component=True):
    """Save components of ``img`` (``io.py:714-748``): ``components`` from
    'mag', 'phase', 'real', 'imag', 'polar' (= mag, phase) and 'cartesian'
    (= real, imag), default ['mag'] for complex data and the data itself
    otherwise; with several components (or ``append_component``) each goes
    to ``name_<component>.fits``."""
    if components is None:
        components = ["mag"] if np.iscomplexobj(img) else ["raw"]
    if isinstance(components, str):
        components = [components]
    comps = []
    for c in components:
        comps += {"polar": ["mag", "phase"], "cartesian": ["real", "imag"]}.get(c, [c])
    base = filename[:-5] if filename.endswith(".fits") else filename
    for c in comps:
        if c == "raw":
            writefits(base + ".fits", np.asarray(img), {}, overwrite)
            continue
        if c not in _COMPONENTS:
            raise ValueError("unknown component %s" % c)
        name = base + "_" + c + ".fits" if (append_component or len(comps) > 1) else base + ".fits"
        writefits(name, _COMPONENTS[c](img).astype(np.float32 if np.asarray(img).dtype in
                                                   (np.complex64, np.float32) else np.float64),
                  {}, overwrite)


def open(filename, quiet=True, orientImageHDU=True, **kwargs):
    """``io.open`` (``io.py:35-92``) for FITS files (.fits, .fit)."""
    ext = filename.rsplit(".", 1)[-1].lower() if "." in filename else ""
    if ext not in ("fits", "fit"):
        raise NotImplementedError("only FITS files are handled here (got .%s)" % ext)
    return openfits(filename, quiet=quiet, orientImageHDU=orientImageHDU)


def save(filename, data, header=None, components=None, overwrite=None, append_component=True,
         **kwargs):
    """``io.save`` (``io.py:94-222``) for FITS files."""
    ext = filename.rsplit(".", 1)[-1].lower() if "." in filename else ""
    if ext not in ("fits", "fit"):
        raise NotImplementedError("only FITS files are handled here (got .%s)" % ext)
    return save_fits(filename, data, header=header, components=components, overwrite=overwrite,
                     append_component=append_component)
