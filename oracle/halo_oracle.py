"""Halo exchange oracle: test infrastructure only, never the product path.

Restates, in numpy, what the path's rpn_comm_xch_halo calls do on a
non-periodic 2-D tile decomposition (src/gemdyn/src/base/dynstep.F90:52-53,
adz_interp_hlt.F90:87-88, adz_traject.F90:121-122).  rpn_comm is the rpncomm
submodule (src/rpn-si/rpncomm, branch main), which is not vendored and has no
pinned commit in the reference's tree.  Its published behaviour is: every
halo cell of width (hx, hy) whose global position lies inside the domain takes
the value of the tile that owns that position; halos on the domain edges keep
their values.

Parity pin: no golden vectors exist for rpn_comm.  The exchange is pinned by
a property instead: a step on a decomposed domain, with halos exchanged,
equals the step on the undivided domain, which is pinned to the adz oracle.

Arrays are numpy views of Fortran arrays (minx:maxx, miny:maxy, planes),
i.e. C arrays of shape (planes, ny, nx).  Buffer layout (pack / unpack, for
bit-level checks of the library's buffers): segments by neighbour slot
q = 3*(dy+1) + (dx+1), slot 4 unused; in a segment array, plane, j, i
(i fastest).
"""
from __future__ import annotations

import numpy as np


def strip(d: int, n: int, hw: int, send: bool):
    """First index and length of a strip along one axis (Fortran indices)."""
    if d == 0:
        return 1, n
    if d < 0:
        return (1 if send else 1 - hw), hw
    return (n - hw + 1 if send else n + 1), hw


def layout(ni, nj, hx, hy, nplanes, narrays, nbr):
    """Element offsets of the 9 segments and the total (10 numbers)."""
    off, o = [], 0
    for q in range(9):
        off.append(o)
        if q == 4 or not nbr[q]:
            continue
        _, w = strip(q % 3 - 1, ni, hx, True)
        _, h = strip(q // 3 - 1, nj, hy, True)
        o += w * h * nplanes * narrays
    off.append(o)
    return off


def _region(a, bounds, q, ni, nj, hx, hy, send):
    minx, _, miny, _ = bounds
    x0, w = strip(q % 3 - 1, ni, hx, send)
    y0, h = strip(q // 3 - 1, nj, hy, send)
    return a[:, y0 - miny:y0 - miny + h, x0 - minx:x0 - minx + w]


def pack(arrays, bounds, ni, nj, hx, hy, nbr):
    """Send buffer of a tile: segment q = its interior strip facing slot q."""
    nplanes = arrays[0].shape[0]
    off = layout(ni, nj, hx, hy, nplanes, len(arrays), nbr)
    buf = np.empty(off[9], dtype=arrays[0].dtype)
    for q in range(9):
        if q == 4 or not nbr[q]:
            continue
        parts = [_region(a, bounds, q, ni, nj, hx, hy, True).ravel() for a in arrays]
        buf[off[q]:off[q + 1]] = np.concatenate(parts)
    return buf


def unpack(arrays, buf, bounds, ni, nj, hx, hy, nbr):
    """Write received segment q into the halo strip on the side of slot q."""
    nplanes = arrays[0].shape[0]
    off = layout(ni, nj, hx, hy, nplanes, len(arrays), nbr)
    for q in range(9):
        if q == 4 or not nbr[q]:
            continue
        seg = buf[off[q]:off[q + 1]]
        n = seg.size // len(arrays)
        for k, a in enumerate(arrays):
            r = _region(a, bounds, q, ni, nj, hx, hy, False)
            r[...] = seg[k * n:(k + 1) * n].reshape(r.shape)


def expected(tiles, bounds_of, gni, gnj, hx, hy):
    """What the exchange leaves in every tile's array.

    tiles: list of (i0g, j0g, ni, nj, array); bounds_of(ni, nj) gives the
    array bounds.  Halo cells within (hx, hy) of the interior whose global
    position is inside the domain take the owner's interior value; every
    other cell keeps its value."""
    nplanes = tiles[0][4].shape[0]
    glob = np.full((nplanes, gnj, gni), np.nan, dtype=tiles[0][4].dtype)
    for i0, j0, ni, nj, a in tiles:
        minx, _, miny, _ = bounds_of(ni, nj)
        glob[:, j0 - 1:j0 - 1 + nj, i0 - 1:i0 - 1 + ni] = a[:, 1 - miny:1 - miny + nj, 1 - minx:1 - minx + ni]
    out = []
    for i0, j0, ni, nj, a in tiles:
        minx, _, miny, _ = bounds_of(ni, nj)
        b = a.copy()
        for j in range(1 - hy, nj + hy + 1):
            for i in range(1 - hx, ni + hx + 1):
                if 1 <= i <= ni and 1 <= j <= nj:
                    continue
                gi, gj = i0 - 1 + i, j0 - 1 + j
                if 1 <= gi <= gni and 1 <= gj <= gnj:
                    b[:, j - miny, i - minx] = glob[:, gj - 1, gi - 1]
        out.append(b)
    return out
