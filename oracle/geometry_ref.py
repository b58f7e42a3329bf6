"""Literal numpy restatement of toolbox/+orf/epsFromBoxes.m:16-30 (open source
in the reference).  TEST COMPARATOR ONLY: checks the product's vectorised
geometry helpers (opticrcwafdtd_b200.geometry)."""
from __future__ import annotations

import numpy as np


def epsFromBoxes_ref(x, z, nBackground, boxes, nSub=4):
    x = np.asarray(x, dtype=float).ravel()
    z = np.asarray(z, dtype=float).ravel()
    boxes = np.asarray(boxes, dtype=float).reshape(-1, 5)
    dx = x[1] - x[0]
    dz = z[1] - z[0]
    off = (np.arange(1, nSub + 1) - (nSub + 1) / 2) / nSub       # epsFromBoxes.m:17
    eps = np.zeros((x.size, z.size))
    for ox in off:                                              # :19-29
        for oz in off:
            X, Z = np.meshgrid(x + ox * dx, z + oz * dz, indexing="ij")
            e = nBackground ** 2 * np.ones(X.shape)
            for b in boxes:
                e[(X >= b[0]) & (X < b[1]) & (Z >= b[2]) & (Z < b[3])] = b[4] ** 2
            eps = eps + e
    return eps / nSub ** 2                                      # :30
