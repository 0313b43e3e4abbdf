"""Seeded synthetic diffraction patterns for the phasing workloads.

The reference's own example data is an external download; these patterns
stand in for it.  An object is the union of K anti-aliased ellipses
(``shape.ellipse`` semantics, ``speckle/shape.py:330-408``: rotated, stretched
coordinates and edge ``1 - clip(r - radius, 0, 1)``) with semi-axes U[3, 15]
px, random angle and centres chosen so each ellipse lies inside a centred
B x B box; amplitude 1 and one phase U[-pi/4, pi/4] per ellipse (where
ellipses overlap, the larger edge weight wins).  The pattern is |FFT(obj)|^2
scaled to ``peak`` photons with Poisson noise; the modulus is its square
root with q = 0 at the corner.  The support is a centred square.
"""
from __future__ import annotations

import numpy as np


def _ellipse_patch(cy, cx, ay, ax, angle_deg, y0, x0, h, w):
    rows, cols = np.indices((h, w)).astype(float)
    rows += y0 - cy
    cols += x0 - cx
    a = np.deg2rad(angle_deg)
    r = rows * np.cos(a) + cols * np.sin(a)
    c = cols * np.cos(a) - rows * np.sin(a)
    ratio = ax / ay
    if ratio >= 1:
        r = r * ratio
        radius = ax
    else:
        c = c / ratio
        radius = ay
    return 1 - np.clip(np.hypot(r, c) - radius, 0, 1)


def make_object(N, n_ellipses, box, seed, axes=(3.0, 15.0)):
    """Complex object (N, N) complex128 and the per-ellipse parameters."""
    rng = np.random.default_rng(seed)
    amp = np.zeros((N, N))
    phase = np.zeros((N, N))
    c = N / 2.0
    amax = axes[1] + 1.0
    lo, hi = c - box / 2.0 + amax, c + box / 2.0 - amax
    if hi <= lo:
        lo = hi = c
    params = []
    for _ in range(n_ellipses):
        ay, ax = rng.uniform(axes[0], axes[1], 2)
        cy, cx = rng.uniform(lo, hi, 2)
        ang = rng.uniform(0, 180)
        ph = rng.uniform(-np.pi / 4, np.pi / 4)
        params.append((cy, cx, ay, ax, ang, ph))
        y0, x0 = int(np.floor(cy - amax)) - 1, int(np.floor(cx - amax)) - 1
        h = w = int(2 * amax) + 4
        y0, x0 = max(0, y0), max(0, x0)
        h, w = min(h, N - y0), min(w, N - x0)
        e = _ellipse_patch(cy, cx, ay, ax, ang, y0, x0, h, w)
        a = amp[y0:y0 + h, x0:x0 + w]
        p = phase[y0:y0 + h, x0:x0 + w]
        take = e > a
        a[take] = e[take]
        p[take] = ph
    return amp * np.exp(1j * phase), params


def centred_square(N, edge):
    s = np.zeros((N, N), np.float32)
    a = (N - edge) // 2
    s[a:a + edge, a:a + edge] = 1
    return s


def pattern(N, n_ellipses, box, peak, seed, support_edge=None, noise=True):
    """(object, modulus float32, support float32) for one seeded pattern."""
    obj, _ = make_object(N, n_ellipses, box, seed)
    I = np.abs(np.fft.fft2(obj)) ** 2
    I *= peak / I.max()
    if noise:
        rng = np.random.default_rng(seed + 0x5EED)
        I = rng.poisson(I).astype(np.float64)
    modulus = np.sqrt(I).astype(np.float32)
    if support_edge is None:
        support_edge = int(round(1.25 * box))
    return obj, modulus, centred_square(N, support_edge)


# The workloads (sizes, counts, photons) of the benchmark configurations
CONFIGS = {
    "plain_256": dict(N=256, n_ellipses=20, box=64, peak=1e5, support_edge=80),
    "raar_dm_1024": dict(N=1024, n_ellipses=60, box=256, peak=1e7, support_edge=320),
    "hio_512x128": dict(N=512, n_ellipses=40, box=128, peak=1e6, support_edge=160),
}


def config_pattern(name, seed=0, noise=True):
    c = dict(CONFIGS[name])
    return pattern(c.pop("N"), seed=seed, noise=noise, **c)
