"""Host-side helpers of the phasing path: crop boxes and support parts.

Both work on small host arrays that the caller already holds (the support
mask); nothing here touches pixel data of the iterates.
"""
from __future__ import annotations

import numpy as np


def bounding_box(data, threshold=1e-10, force_to_square=False, pad=0):
    """(rmin, rmax, cmin, cmax) of ``data > threshold``.

    Same rules as ``masking.bounding_box`` (``speckle/masking.py:7-159``):
    padding clipped at the edges, optional squaring with Python-2 integer
    halving, and negative minima moved back to zero.  ``power_of_2`` is not
    used on the phasing path and is not provided.
    """
    data = np.asarray(data)
    if data.ndim != 2:
        raise ValueError("data must be a 2d ndarray")
    if not isinstance(pad, (int, np.integer)):
        raise TypeError("pad must be an integer")
    rows, cols = data.shape
    aw = np.argwhere(data > threshold)
    if aw.size == 0:
        raise ValueError("bounding_box: nothing above threshold")
    rmin, cmin = (int(v) for v in aw.min(0))
    rmax, cmax = (int(v) + 1 for v in aw.max(0))
    rmin = 0 if rmin < pad else rmin - pad
    rmax = rows if rmax + pad > rows else rmax + pad
    cmin = 0 if cmin < pad else cmin - pad
    cmax = cols if cmax + pad > cols else cmax + pad
    if force_to_square:
        dr, dc = rmax - rmin, cmax - cmin
        if dr % 2 == 1:
            dr += 1
            if rmax < rows:
                rmax += 1
            else:
                rmin -= 1
        if dc % 2 == 1:
            dc += 1
            if cmax < cols:
                cmax += 1
            else:
                cmin -= 1
        if dr > dc:
            mid = (cmax + cmin) // 2
            cmin, cmax = mid - dr // 2, mid + dr // 2
        elif dc > dr:
            mid = (rmax + rmin) // 2
            rmin, rmax = mid - dc // 2, mid + dc // 2
    if rmin < 0:
        rmin, rmax = 0, rmax - rmin
    if cmin < 0:
        cmin, cmax = 0, cmax - cmin
    return np.array([rmin, rmax, cmin, cmax]).astype(int)


def label_parts(data, detect_val=(0.95, 1.05)):
    """Connected parts of a (nearly binary) support, numbered 1..n.

    Connectivity is 8-neighbour with periodic wrap and parts are numbered in
    raster order of their first pixel, which is the order in which
    ``masking.find_all_objects`` (``speckle/masking.py:379-435``, flood fill
    ``trace_object`` ``:271-377``) returns them.  Returns (labels int32, n);
    n counts empty parts (isolated pixels), whose label has no pixels.
    """
    from scipy import ndimage
    data = np.asarray(data)
    mask = (data >= detect_val[0]) & (data <= detect_val[1])
    R, C = mask.shape
    lab, n = ndimage.label(mask, structure=np.ones((3, 3), bool))
    if n == 0:
        return np.zeros((R, C), np.int32), 0
    # merge parts that touch across the periodic edges (rows 0/R-1, cols 0/C-1)
    parent = np.arange(n + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    edges = []
    top, bot = lab[0], lab[R - 1]
    for dc in (-1, 0, 1):
        edges.append((top, np.roll(bot, dc)))
    left, right = lab[:, 0], lab[:, C - 1]
    for dr in (-1, 0, 1):
        edges.append((left, np.roll(right, dr)))
    for a, b in edges:
        both = (a > 0) & (b > 0)
        for x, y in zip(a[both], b[both]):
            rx, ry = find(int(x)), find(int(y))
            if rx != ry:
                parent[max(rx, ry)] = min(rx, ry)
    roots = np.array([find(i) for i in range(n + 1)])
    merged = roots[lab]
    flat = merged.ravel()
    # number parts by the raster position of their first pixel
    ids, first = np.unique(flat, return_index=True)
    keep = ids > 0
    ids, first = ids[keep], first[keep]
    order = ids[np.argsort(first)]
    remap = np.zeros(n + 1, np.int32)
    remap[order] = np.arange(1, len(order) + 1, dtype=np.int32)
    out = remap[merged]
    # the flood fill never marks its start pixel itself, so a pixel with no
    # neighbour in the mask is returned as an empty part (masking.py:357-372)
    sizes = np.bincount(out.ravel(), minlength=len(order) + 1)
    single = sizes == 1
    single[0] = False
    out[single[out]] = 0
    return out.astype(np.int32), len(order)
