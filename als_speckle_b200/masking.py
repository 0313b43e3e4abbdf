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
    data = np.asarray(data)
    mask = (data >= detect_val[0]) & (data <= detect_val[1])
    R, Cc = mask.shape
    parent = np.arange(R * Cc, dtype=np.int64)

    def find(a):
        root = a
        while parent[root] != root:
            root = parent[root]
        while parent[a] != root:
            parent[a], a = root, parent[a]
        return root

    idx = np.flatnonzero(mask.ravel())
    for k in idx:
        r, c = divmod(int(k), Cc)
        for dr, dc in ((0, 1), (1, -1), (1, 0), (1, 1)):
            rr, cc = (r + dr) % R, (c + dc) % Cc
            if mask[rr, cc]:
                a, b = find(int(k)), find(rr * Cc + cc)
                if a != b:
                    parent[max(a, b)] = min(a, b)
    labels = np.zeros(R * Cc, np.int32)
    order = {}
    size = {}
    for k in idx:
        root = find(int(k))
        size[root] = size.get(root, 0) + 1
    for k in idx:
        root = find(int(k))
        if root not in order:
            order[root] = len(order) + 1
        # the flood fill never marks its start pixel itself, so a pixel with no
        # neighbour in the mask is returned as an empty part (masking.py:357-372)
        if size[root] > 1:
            labels[k] = order[root]
    return labels.reshape(R, Cc), len(order)
