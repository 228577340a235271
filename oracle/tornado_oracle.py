"""Oracle (test infrastructure only) for the tornado-candidate search of the sub-grid tornado scheme.

CPU restatement of tornadoCandidates (app.js:1453-1466) on the readback maps: map0 = (composite dBZ, 1-km dBZ, low-level
theta', 1-km vertical vorticity), map1 = (max updraft, 2-5 km updraft helicity, ...), each (ny, nx, 4) float32. On the
stride-2 lattice from 6 to n-7, a point is a candidate when its vorticity z1 is at least zeta_min (0.003 * 1500/dx,
app.js:1451-1452), its theta' is not below -4.5 K, no other point of its stride-2 5 x 5 window has a larger vorticity,
and the window's maxima of helicity and updraft (both started at 0) exceed 60 m2/s2 and 12 m/s.

Two forms: `candidates_loop` follows the reference's loops literally (small grids), `candidates` is the vectorised
numpy form used at full size; tests check that they agree. The reference is browser JavaScript with no test of this
function and no JavaScript runtime is installed here, so the restatement is not pinned to outputs of the reference
itself (parity unpinned for this row); the comparisons are in float64 of the float32 map values against float64
thresholds, as in JavaScript.
"""
from __future__ import annotations

import numpy as np


def zeta_min(dx):
    """app.js:1451-1452."""
    return 0.003 * (1500.0 / dx)


def candidates_loop(m0, m1, dx, zmin=None):
    """Literal restatement: list of (i, j, x, y, z1, uh, w) in the reference's order (j outer, i inner)."""
    ny, nx = m0.shape[:2]
    zmin = zeta_min(dx) if zmin is None else zmin
    out = []
    for j in range(6, ny - 6, 2):
        for i in range(6, nx - 6, 2):
            z1 = float(m0[j, i, 3])
            if z1 < zmin or float(m0[j, i, 2]) < -4.5:
                continue
            is_max, uh, w = True, 0.0, 0.0
            for dj in range(-4, 5, 2):
                for di in range(-4, 5, 2):
                    if (di or dj) and float(m0[j + dj, i + di, 3]) > z1:
                        is_max = False
                    uh = max(uh, float(m1[j + dj, i + di, 1]))
                    w = max(w, float(m1[j + dj, i + di, 0]))
            if is_max and uh > 60 and w > 12:
                out.append((i, j, (i + 0.5) * dx, (j + 0.5) * dx, z1, uh, w))
    return out


def candidates(m0, m1, dx, zmin=None):
    """Vectorised form of candidates_loop, same output and order."""
    ny, nx = m0.shape[:2]
    zmin = zeta_min(dx) if zmin is None else zmin
    js = np.arange(6, ny - 6, 2)
    is_ = np.arange(6, nx - 6, 2)
    if js.size == 0 or is_.size == 0:
        return []
    J, I = np.meshgrid(js, is_, indexing="ij")
    z1 = m0[J, I, 3].astype(np.float64)
    ok = (z1 >= zmin) & (m0[J, I, 2].astype(np.float64) >= -4.5)
    is_max = np.ones_like(ok)
    uh = np.zeros(J.shape)
    w = np.zeros(J.shape)
    for dj in range(-4, 5, 2):
        for di in range(-4, 5, 2):
            if di or dj:
                is_max &= ~(m0[J + dj, I + di, 3].astype(np.float64) > z1)
            uh = np.maximum(uh, m1[J + dj, I + di, 1].astype(np.float64))
            w = np.maximum(w, m1[J + dj, I + di, 0].astype(np.float64))
    sel = ok & is_max & (uh > 60) & (w > 12)
    return [(int(I[a, b]), int(J[a, b]), (int(I[a, b]) + 0.5) * dx, (int(J[a, b]) + 0.5) * dx, float(z1[a, b]),
             float(uh[a, b]), float(w[a, b])) for a, b in zip(*np.nonzero(sel))]
