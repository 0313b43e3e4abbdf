"""Load the reference's numpy phasing path under Python 3, read-only.

TEST AND BASELINE INFRASTRUCTURE ONLY.  The reference (dhparks/als_speckle)
is Python-2 source.  This loader reads the needed modules' text from a
reference checkout or install (``SPECKLE_REF_ROOT``), applies mechanical
source-level fixes in memory (print statements, backslash continuations,
implicit relative imports, Python-2 integer division where the path needs
it) and executes them as modules.  Nothing on disk is modified.  Users:
``tests/golden/make_golden.py`` (the golden fixtures) and ``bench.py``'s
reference arm and CPU baseline, which time the reference's own numpy
iteration from the install in ``baseline/_ref``.  The product never imports
it.
"""
import os
import re
import sys
import types

def _pkg_dir():
    """The reference's ``speckle`` package folder, from ``SPECKLE_REF_ROOT``
    (the root of a dhparks/als_speckle checkout or install)."""
    root = os.environ.get("SPECKLE_REF_ROOT")
    if not root:
        raise RuntimeError("set SPECKLE_REF_ROOT to the reference checkout (or pass it to "
                           "make_golden.py)")
    return os.path.join(root, "speckle")

_PRINT_RE = re.compile(r"^(\s*)print\s+(?!\()(.*)$")
_EXCEPT_RE = re.compile(r"^(\s*)except\s+([\w.]+)\s*,\s*(\w+)\s*:")
_RAISE_RE = re.compile(r"^(\s*)raise\s+([\w.]+)\s*,\s*(.+)$")


def _py3_text(src):
    # join backslash continuations so print rewriting sees whole statements
    src = re.sub(r"\\\n", " ", src)
    out = []
    for line in src.split("\n"):
        m = _PRINT_RE.match(line)
        if m:
            body = m.group(2).rstrip()
            if body.endswith(","):
                body = body[:-1]
            line = "%sprint(%s)" % (m.group(1), body)
        elif re.match(r"^\s*print\s*$", line):
            line = re.sub(r"print", "print()", line)
        line = _EXCEPT_RE.sub(r"\1except \2 as \3:", line)
        line = _RAISE_RE.sub(r"\1raise \2(\3)", line)
        out.append(line)
    return "\n".join(out)


def _package():
    pkg = sys.modules.get("speckle")
    if pkg is None or not getattr(pkg, "__refshim__", False):
        pkg = types.ModuleType("speckle")
        pkg.__path__ = [_pkg_dir()]
        pkg.__refshim__ = True
        sys.modules["speckle"] = pkg
        # speckle.io needs pyfits (absent); the phasing path only uses it for
        # debug dumps, so an empty stand-in module is registered instead.
        stub = types.ModuleType("speckle.io")
        stub.__refshim__ = True
        sys.modules["speckle.io"] = stub
        pkg.io = stub
    return pkg


def _load(name, fixups=()):
    pkg = _package()
    full = "speckle." + name
    if full in sys.modules and getattr(sys.modules[full], "__refshim__", False):
        return sys.modules[full]
    path = os.path.join(_pkg_dir(), name + ".py")
    with open(path) as f:
        src = _py3_text(f.read())
    for a, b in fixups:
        assert a in src, (name, a)
        src = src.replace(a, b)
    mod = types.ModuleType(full)
    mod.__file__ = path
    mod.__package__ = "speckle"
    mod.__refshim__ = True
    sys.modules[full] = mod
    sys.modules[name] = mod      # implicit relative imports (Python 2 style)
    setattr(pkg, name, mod)
    exec(compile(src, path, "exec"), mod.__dict__)
    return mod


def load_reference():
    """Return a namespace with the reference modules used on the phasing path."""
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", SyntaxWarning)
        shape = _load("shape")
        masking = _load("masking")
        # wrapping.py:161 shapes the unwrapped rows with len/(R-r), a float
        # that Python 2's numpy truncated and Python 3's rejects
        wrapping = _load("wrapping", fixups=[
            ("uw.shape = (R-r, len(plan[0])/(R-r))",
             "uw.shape = (int(R-r), int(len(plan[0])/(R-r)))")])
        _load("averaging")
        gpu = _load("gpu")
        # crosscorr.py:557-566 relies on Python-2 integer division
        crosscorr = _load("crosscorr", fixups=[
            ("max_row, max_col = cc_max/cols, cc_max%cols",
             "max_row, max_col = cc_max//cols, cc_max%cols"),
            ("max_row += -rows/2", "max_row += -rows//2"),
            ("max_col += -cols/2", "max_col += -cols//2"),
            ("if max_row > rows/2:", "if max_row > rows//2:"),
            ("if max_col > cols/2:", "if max_col > cols//2:")])
        # conditioning.py compares arrays with None (old numpy returned a scalar)
        conditioning = _load("conditioning", fixups=[
            ("if region != None:", "if region is not None:"),
            ("if align_to == None:", "if align_to is None:")])
        # phasing.py:1456, :1514, :1604, :1703 pass (0, N/2, (N/2, N/2)) with
        # Python-2 integer division
        phasing = _load("phasing", fixups=[("import wrapping, masking, gpu, sys, time, io",
                                            "import wrapping, masking, gpu, sys, time"),
                                           ("(0, N/2, (N/2, N/2))", "(0, N//2, (N//2, N//2))")])
    return types.SimpleNamespace(shape=shape, masking=masking, wrapping=wrapping,
                                 gpu=gpu, crosscorr=crosscorr,
                                 conditioning=conditioning, phasing=phasing)
