"""Dose comparison helpers for the tests: the per-voxel tolerance and the
gamma index used as parity criteria.

* ``dose_diff``: max |a - b| over voxels with b above ``thresh`` x max(b),
  as a fraction of max(b) (the criterion |dD| <= 0.5 % Dmax above 10 % Dmax);
  optionally over a voxel subset.
* ``gamma_pass_rate``: global gamma (dose difference ``dd`` of max(ref),
  distance to agreement ``dta_mm``), evaluated at voxels where ref is above
  ``thresh`` x max(ref); the search is over whole-voxel shifts within
  1.5 x DTA (no sub-voxel interpolation, which can only lower gamma).
"""
from __future__ import annotations

import numpy as np


WET_MAX_CM = 0.1        # no voxel further apart than 1 mm of water
WET_CLOSE_CM = 1e-3     # ... and 99.5 % of voxels within 0.01 mm
WET_CLOSE_FRAC = 0.995


def wet_close(a, b):
    """WET (cm) agreement between two implementations of the reference's
    sampling: the 1 mm march plus the smoothing, whose radius test
    (r < 10 * WET) and nearest-voxel picks are knife edges, so a 1e-4 cm
    difference can flip a few voxels' neighbour sets."""
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return bool(d.max() <= WET_MAX_CM and np.mean(d <= WET_CLOSE_CM) >= WET_CLOSE_FRAC)


def dose_diff(a, b, thresh=0.10, where=None, dmax=None):
    """With ``where`` (boolean volume) only those voxels count, and ``dmax``
    (default: max of b over them) normalises."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    sel = np.ones(b.shape, bool) if where is None else np.asarray(where, bool)
    m = float(np.abs(b[sel]).max()) if dmax is None else float(dmax)
    if m == 0.0:
        return float(np.abs(a[sel]).max())
    mask = (b > thresh * m) & sel
    return float(np.abs(a - b)[mask].max() / m) if mask.any() else 0.0


def gamma_pass_rate(test, ref, spacing_mm, dd=0.02, dta_mm=2.0, thresh=0.10, where=None, dmax=None):
    """With ``where`` only those reference voxels are evaluated, and ``dmax``
    (default: max of ref over them) is the dose criterion's normalisation."""
    test = np.asarray(test, np.float64)
    ref = np.asarray(ref, np.float64)
    sel = np.ones(ref.shape, bool) if where is None else np.asarray(where, bool)
    dmax = float(ref[sel].max()) if dmax is None else float(dmax)
    sp = np.broadcast_to(np.asarray(spacing_mm, np.float64), (3,))[::-1]  # (z, y, x)
    reach = [int(np.ceil(1.5 * dta_mm / s)) for s in sp]
    best = np.full(ref.shape, np.inf)
    pad = [(r, r) for r in reach]
    tp = np.pad(test, pad, mode="edge")
    nz, ny, nx = ref.shape
    for dz in range(-reach[0], reach[0] + 1):
        for dy in range(-reach[1], reach[1] + 1):
            for dx in range(-reach[2], reach[2] + 1):
                r2 = (dz * sp[0]) ** 2 + (dy * sp[1]) ** 2 + (dx * sp[2]) ** 2
                if r2 > (1.5 * dta_mm) ** 2:
                    continue
                sh = tp[reach[0] + dz:reach[0] + dz + nz, reach[1] + dy:reach[1] + dy + ny,
                        reach[2] + dx:reach[2] + dx + nx]
                g2 = ((sh - ref) / (dd * dmax)) ** 2 + r2 / dta_mm ** 2
                np.minimum(best, g2, out=best)
    mask = (ref > thresh * dmax) & sel
    return float((best[mask] <= 1.0).mean()) if mask.any() else 1.0
