"""Subpixel-averaged permittivity on the Yee grid (host-side preparation).

Mirrors the reference's geometry front end of the FDTD:
  - epsFromBoxes     toolbox/+orf/epsFromBoxes.m:1-31 (open code)
  - epsCellMean      toolbox/+orf/epsCellMean.m:1-9 (documented behaviour)
  - epsComponents2D  toolbox/+orf/epsComponents2D.m:1-10 (documented behaviour)
  - epsComponents3D  toolbox/+orf/epsComponents3D.m:1-27 (documented behaviour)

Boxes are painted in order, later rows over earlier (epsFromBoxes.m:4-5), a
sample at (X, Z) being inside a box when x1 <= X < x2 and z1 <= Z < z2
(epsFromBoxes.m:25).  Each painter visits only the sample columns/rows a box
covers (found by binary search), so cost scales with box area, not grid area.
"""
from __future__ import annotations

from typing import Any, Sequence

import numpy as np


def _offsets(nsub: int) -> np.ndarray:
    # epsFromBoxes.m:17
    return (np.arange(1, nsub + 1) - (nsub + 1) / 2.0) / nsub


def _ranges(coords: np.ndarray, lo: float, hi: float) -> tuple[int, int]:
    """Index range [a, b) of sorted coords with lo <= c < hi."""
    a = int(np.searchsorted(coords, lo, side="left"))
    b = int(np.searchsorted(coords, hi, side="left"))
    return a, b


def _paint2d(xs: np.ndarray, zs: np.ndarray, nbg: float, boxes: np.ndarray,
             wrap_z: tuple[float, float] | None = None) -> np.ndarray:
    """eps of axis-aligned boxes at sample points xs (sorted) x zs."""
    e = np.full((xs.size, zs.size), float(nbg) ** 2)
    if wrap_z is not None:
        z0, L = wrap_z
        zf = z0 + np.mod(zs - z0, L)
        order = np.argsort(zf, kind="stable")
        zsorted = zf[order]
    for b in boxes:
        i0, i1 = _ranges(xs, b[0], b[1])
        if i1 <= i0:
            continue
        val = b[4] ** 2
        if wrap_z is None:
            k0, k1 = _ranges(zs, b[2], b[3])
            if k1 > k0:
                e[i0:i1, k0:k1] = val
        else:
            # the structure repeats with period L: fold the box into [z0, z0+L)
            lo, hi = b[2], b[3]
            if hi - lo >= L:
                spans = [(z0, z0 + L)]
            else:
                a = z0 + np.mod(lo - z0, L)
                end = a + (hi - lo)
                spans = [(a, min(end, z0 + L))]
                if end > z0 + L:
                    spans.append((z0, end - L))
            for s0, s1 in spans:
                k0, k1 = _ranges(zsorted, s0, s1)
                if k1 > k0:
                    e[i0:i1, order[k0:k1]] = val
    return e


def _as_boxes(boxes) -> np.ndarray:
    b = np.asarray(boxes, dtype=float)
    if b.size == 0:
        return np.zeros((0, 5))
    return b.reshape(-1, 5)


def epsCellMean(xc, yc, dx: float, dy: float, boxes, nBg: float, harmonicDir: str = "none",
                NSub: int = 4, WrapY: Sequence[float] | None = None) -> np.ndarray:
    """Cell-averaged eps of boxes [x1 x2 y1 y2 n] at points (xc, yc), ndgrid layout.

    harmonicDir "none": arithmetic mean of NSub x NSub samples; "x" / "y":
    harmonic mean along that direction, then arithmetic along the other
    (epsCellMean.m:6-8).  WrapY = [y0 Ly] folds sample y into [y0, y0+Ly).
    """
    xc = np.asarray(xc, dtype=float).ravel()
    yc = np.asarray(yc, dtype=float).ravel()
    boxes = _as_boxes(boxes)
    off = _offsets(NSub)
    wrap = None if WrapY is None else (float(WrapY[0]), float(WrapY[1]))
    if harmonicDir not in ("none", "x", "y"):
        raise ValueError('harmonicDir must be "none", "x" or "y"')
    if wrap is None and NSub > 1 and xc.size * yc.size > 4096:
        return _cell_mean_banded(xc, yc, dx, dy, boxes, nBg, harmonicDir, NSub, off)
    return _cell_mean_full(xc, yc, dx, dy, boxes, nBg, harmonicDir, NSub, off, wrap)


def _straddled(c: np.ndarray, lo: float, hi: float, edges) -> np.ndarray:
    """Indices q whose sample span [c_q + lo, c_q + hi] puts samples on both
    sides of an edge (some sample < e <= another sample), for sorted c."""
    out = []
    for e in edges:
        if not np.isfinite(e):
            continue
        # c + lo < e <= c + hi  <=>  e - hi <= c < e - lo (up to rounding: widen by one)
        a = max(0, int(np.searchsorted(c, e - hi, side="left")) - 1)
        b = min(c.size, int(np.searchsorted(c, e - lo, side="left")) + 1)
        q = np.arange(a, b)
        if q.size:
            out.append(q[(c[q] + lo < e) & (e <= c[q] + hi)])
    return np.unique(np.concatenate(out)) if out else np.zeros(0, dtype=np.int64)


def _label2d(xs: np.ndarray, zs: np.ndarray, boxes: np.ndarray) -> np.ndarray:
    """Index (1-based, 0 = background) of the last box covering each sample
    point xs (sorted) x zs, in Fortran order: the label form of _paint2d."""
    lab = np.zeros((xs.size, zs.size), dtype=np.int32, order="F")
    for q, b in enumerate(boxes):
        i0, i1 = _ranges(xs, b[0], b[1])
        if i1 <= i0:
            continue
        k0, k1 = _ranges(zs, b[2], b[3])
        if k1 > k0:
            lab[i0:i1, k0:k1] = q + 1
    return lab


def _cell_mean_banded(xc, yc, dx, dy, boxes, nBg, harmonicDir, NSub, off):
    """epsCellMean without wrap, sub-sampling only where a box edge passes
    between a cell's samples.  A cell whose samples all lie inside or all
    outside every box has NSub^2 equal samples: its mean depends only on that
    material and is formed by the same sequence of operations as the full
    sub-sampled mean (one evaluation per material), and the cells an edge
    crosses (whole columns and rows) are computed by the full mean, so the
    result is bitwise the full computation's."""
    lo_x, hi_x = off[0] * dx, off[-1] * dx
    lo_y, hi_y = off[0] * dy, off[-1] * dy
    bx = [e for b in boxes if b[1] > b[0] and b[3] > b[2] for e in (b[0], b[1])]
    by = [e for b in boxes if b[1] > b[0] and b[3] > b[2] for e in (b[2], b[3])]
    cols = _straddled(xc, lo_x, hi_x, bx)
    rows = _straddled(yc, lo_y, hi_y, by)
    # uniform cells: the material at the cells' own samples (any one of them)
    lab = _label2d(xc + off[0] * dx, yc + off[0] * dy, boxes)
    vals = np.concatenate([[float(nBg) ** 2], boxes[:, 4] ** 2]) if boxes.size else np.array([float(nBg) ** 2])
    table = np.empty_like(vals)
    for m, v in enumerate(vals):
        v = np.float64(v)
        if harmonicDir == "none":
            acc = np.float64(0.0)
            for _ in range(NSub * NSub):
                acc = acc + v
            table[m] = acc / NSub ** 2
        else:
            inv = np.float64(0.0)
            for _ in range(NSub):
                inv = inv + 1.0 / v
            acc = np.float64(0.0)
            for _ in range(NSub):
                acc = acc + NSub / inv
            table[m] = acc / NSub
    out = table[lab]
    if cols.size:
        out[cols, :] = _cell_mean_full(xc[cols], yc, dx, dy, boxes, nBg, harmonicDir, NSub, off, None)
    if rows.size:
        out[:, rows] = _cell_mean_full(xc, yc[rows], dx, dy, boxes, nBg, harmonicDir, NSub, off, None)
    return out


def _cell_mean_full(xc, yc, dx, dy, boxes, nBg, harmonicDir, NSub, off, wrap):
    """epsCellMean with every cell sub-sampled NSub x NSub times."""
    if harmonicDir == "none":
        acc = np.zeros((xc.size, yc.size))
        for ox in off:
            xs = xc + ox * dx
            for oy in off:
                acc += _paint2d(xs, yc + oy * dy, nBg, boxes, wrap)
        return acc / NSub ** 2
    if harmonicDir == "x":
        acc = np.zeros((xc.size, yc.size))
        for oy in off:
            inv = np.zeros((xc.size, yc.size))
            for ox in off:
                inv += 1.0 / _paint2d(xc + ox * dx, yc + oy * dy, nBg, boxes, wrap)
            acc += NSub / inv
        return acc / NSub
    if harmonicDir == "y":
        acc = np.zeros((xc.size, yc.size))
        for ox in off:
            inv = np.zeros((xc.size, yc.size))
            for oy in off:
                inv += 1.0 / _paint2d(xc + ox * dx, yc + oy * dy, nBg, boxes, wrap)
            acc += NSub / inv
        return acc / NSub
    raise ValueError('harmonicDir must be "none", "x" or "y"')


def epsFromBoxes(x, z, nBackground: float, boxes, nSub: int = 4) -> np.ndarray:
    """Arithmetic cell mean at the grid points (epsFromBoxes.m:1-31)."""
    x = np.asarray(x, dtype=float).ravel()
    z = np.asarray(z, dtype=float).ravel()
    return epsCellMean(x, z, x[1] - x[0], z[1] - z[0], boxes, nBackground, "none", nSub)


def epsComponents2D(x, z, nBg: float, boxes, NSub: int = 4, PeriodicZ: bool = False) -> dict:
    """eps at the 2D Yee locations (epsComponents2D.m:2-10).

    e["y"] at (x_i, z_k): arithmetic mean (numel(x) x numel(z));
    e["x"] at (x_i, z_k+1/2): harmonic along x, arithmetic along z
           (numel(x) x numel(z)-1, or numel(z) when PeriodicZ);
    e["z"] at (x_i+1/2, z_k): harmonic along z, arithmetic along x
           ((numel(x)-1) x numel(z)).
    Column-major arrays (MATLAB's layout): the engine takes them without a copy.
    """
    x = np.asarray(x, dtype=float).ravel()
    z = np.asarray(z, dtype=float).ravel()
    dx, dz = x[1] - x[0], z[1] - z[0]
    wrap = (z[0] - dz / 2, z.size * dz) if PeriodicZ else None
    zh = z + dz / 2 if PeriodicZ else z[:-1] + dz / 2
    xh = x[:-1] + dx / 2
    return {
        "y": np.asfortranarray(epsCellMean(x, z, dx, dz, boxes, nBg, "none", NSub, wrap)),
        "x": np.asfortranarray(epsCellMean(x, zh, dx, dz, boxes, nBg, "x", NSub, wrap)),
        "z": np.asfortranarray(epsCellMean(xh, z, dx, dz, boxes, nBg, "y", NSub, wrap)),
    }


# --------------------------------------------------------------------- 3D --
def _shape_list(shapes) -> list[tuple[str, Any]]:
    out = []
    for s in shapes or []:
        kind, par = s[0], s[1]
        out.append((str(kind).lower(), par))
    return out


def _get(p, name, default=None):
    if isinstance(p, dict):
        return p.get(name, default)
    return getattr(p, name, default)


class _Shape:
    """Inside test and interface band of one epsComponents3D shape."""

    def __init__(self, kind: str, par: Any):
        self.kind = kind
        if kind == "box":
            b = np.asarray(par, dtype=float).ravel()
            self.lo = b[[0, 2, 4]]
            self.hi = b[[1, 3, 5]]
            self.n = b[6]
        elif kind in ("cyl", "cone"):
            b = np.asarray(par, dtype=float).ravel()
            if kind == "cyl":
                cx, cy, r, z1, z2, n = b
                r1 = r2 = r
            else:
                cx, cy, r1, r2, z1, z2, n = b
            self.c = (cx, cy)
            self.r1, self.r2, self.z1, self.z2, self.n = r1, r2, z1, z2, n
            rmax = max(r1, r2)
            self.lo = np.array([cx - rmax, cy - rmax, z1])
            self.hi = np.array([cx + rmax, cy + rmax, z2])
        elif kind == "polygon":
            self.xy = np.asarray(_get(par, "xy"), dtype=float).reshape(-1, 2)
            self.z1, self.z2 = float(_get(par, "z1")), float(_get(par, "z2"))
            self.n = float(_get(par, "n"))
            self.lo = np.array([self.xy[:, 0].min(), self.xy[:, 1].min(), self.z1])
            self.hi = np.array([self.xy[:, 0].max(), self.xy[:, 1].max(), self.z2])
        elif kind == "lattice":
            self.x0, self.y0 = float(_get(par, "x0")), float(_get(par, "y0"))
            self.P = float(_get(par, "period"))
            self.R = np.atleast_2d(np.asarray(_get(par, "R"), dtype=float))
            self.z1, self.z2 = float(_get(par, "z1")), float(_get(par, "z2"))
            self.n = float(_get(par, "n"))
            self.dRdz = float(_get(par, "dRdz", 0.0) or 0.0)
            rmax = float(self.R.max()) + abs(self.dRdz) * (self.z2 - self.z1)
            self.rmax = rmax
            self.lo = np.array([self.x0 - rmax, self.y0 - rmax, self.z1])
            self.hi = np.array([self.x0 + (self.R.shape[0] - 1) * self.P + rmax,
                                self.y0 + (self.R.shape[1] - 1) * self.P + rmax, self.z2])
        else:
            raise ValueError(f"unknown shape kind {kind!r}")

    def inside(self, X, Y, Z):
        k = self.kind
        if k == "box":
            return ((X >= self.lo[0]) & (X < self.hi[0]) & (Y >= self.lo[1]) & (Y < self.hi[1])
                    & (Z >= self.lo[2]) & (Z < self.hi[2]))
        if k in ("cyl", "cone"):
            zin = (Z >= self.z1) & (Z < self.z2)
            t = np.clip((Z - self.z1) / max(self.z2 - self.z1, 1e-300), 0.0, 1.0)
            r = self.r1 + (self.r2 - self.r1) * t
            return zin & ((X - self.c[0]) ** 2 + (Y - self.c[1]) ** 2 < r * r)
        if k == "polygon":
            zin = (Z >= self.z1) & (Z < self.z2)
            xs, ys = self.xy[:, 0], self.xy[:, 1]
            inside = np.zeros(np.broadcast(X, Y).shape, dtype=bool)
            Xb, Yb = np.broadcast_arrays(X, Y)
            for a in range(xs.size):
                b = (a + 1) % xs.size
                cond = (ys[a] > Yb) != (ys[b] > Yb)
                xcross = (xs[b] - xs[a]) * (Yb - ys[a]) / np.where(ys[b] != ys[a], ys[b] - ys[a], 1.0) + xs[a]
                inside ^= cond & (Xb < xcross)
            return zin & inside
        if k == "lattice":
            ix = np.rint((X - self.x0) / self.P).astype(np.int64)
            iy = np.rint((Y - self.y0) / self.P).astype(np.int64)
            ok = (ix >= 0) & (ix < self.R.shape[0]) & (iy >= 0) & (iy < self.R.shape[1])
            ixc = np.clip(ix, 0, self.R.shape[0] - 1)
            iyc = np.clip(iy, 0, self.R.shape[1] - 1)
            r = self.R[ixc, iyc] + self.dRdz * (Z - self.z1)
            cx = self.x0 + ixc * self.P
            cy = self.y0 + iyc * self.P
            zin = (Z >= self.z1) & (Z < self.z2)
            return ok & zin & (r > 0) & ((X - cx) ** 2 + (Y - cy) ** 2 < r * r)
        raise AssertionError

    def z_extruded(self) -> bool:
        """True when the cross-section does not change with z inside [z1, z2)."""
        if self.kind in ("cyl", "cone"):
            return self.r1 == self.r2
        if self.kind == "lattice":
            return self.dRdz == 0.0
        return True

    def band(self, X, Y, Z, h):
        """Cells (centres X, Y, Z, half-size h) that the shape boundary may cross."""
        near = ((X >= self.lo[0] - h) & (X <= self.hi[0] + h) & (Y >= self.lo[1] - h)
                & (Y <= self.hi[1] + h) & (Z >= self.lo[2] - h) & (Z <= self.hi[2] + h))
        k = self.kind
        if k == "box":
            full = ((X - h >= self.lo[0]) & (X + h < self.hi[0]) & (Y - h >= self.lo[1])
                    & (Y + h < self.hi[1]) & (Z - h >= self.lo[2]) & (Z + h < self.hi[2]))
            return near & ~full
        if k in ("cyl", "cone", "lattice", "polygon"):
            zface = (np.abs(Z - self.z1) <= h) | (np.abs(Z - self.z2) <= h)
            hd = h * np.sqrt(2.0) * 1.0000001
            if k in ("cyl", "cone"):
                rho = np.sqrt((X - self.c[0]) ** 2 + (Y - self.c[1]) ** 2)
                rlo = min(self.r1, self.r2)
                rhi = max(self.r1, self.r2)
                side = (rho >= rlo - hd) & (rho <= rhi + hd)
                return near & (zface | side)
            if k == "lattice":
                # a pillar whose rim passes through the cell has its centre at
                # one of the 3 x 3 lattice sites around the cell's nearest site
                # (radii stay below P/2)
                dz = abs(self.dRdz) * h
                ix0 = np.rint((X - self.x0) / self.P).astype(np.int64)
                iy0 = np.rint((Y - self.y0) / self.P).astype(np.int64)
                side = np.zeros(np.broadcast(X, Y, Z if self.dRdz else 0.0).shape, dtype=bool)
                for di in (-1, 0, 1):
                    for dj in (-1, 0, 1):
                        ix, iy = ix0 + di, iy0 + dj
                        ok = (ix >= 0) & (ix < self.R.shape[0]) & (iy >= 0) & (iy < self.R.shape[1])
                        ixc = np.clip(ix, 0, self.R.shape[0] - 1)
                        iyc = np.clip(iy, 0, self.R.shape[1] - 1)
                        r = self.R[ixc, iyc] + (self.dRdz * (Z - self.z1) if self.dRdz else 0.0)
                        rho = np.sqrt((X - (self.x0 + ixc * self.P)) ** 2 + (Y - (self.y0 + iyc * self.P)) ** 2)
                        side |= ok & (np.abs(rho - r) <= hd + dz)
                return near & (zface | side)
            # polygon: distance to any edge
            xs, ys = self.xy[:, 0], self.xy[:, 1]
            dmin = np.full(np.broadcast(X, Y).shape, np.inf)
            for a in range(xs.size):
                b = (a + 1) % xs.size
                ex, ey = xs[b] - xs[a], ys[b] - ys[a]
                L2 = max(ex * ex + ey * ey, 1e-300)
                t = np.clip(((X - xs[a]) * ex + (Y - ys[a]) * ey) / L2, 0, 1)
                u, v = X - xs[a] - t * ex, Y - ys[a] - t * ey
                dmin = np.minimum(dmin, np.sqrt(u * u + v * v))
            return near & (zface | (dmin <= hd))
        raise AssertionError


def _fold(v, L):
    if L is None or not np.isfinite(L):
        return v
    return np.mod(v + L / 2, L) - L / 2


def epsComponents3D(x, y, z, nBg: float, shapes, NSub: int = 4, Period=None,
                    Method: str = "directional", device=None) -> dict:
    """eps at the 3D Yee E locations (epsComponents3D.m:1-27).

    e["x"] at (x+d/2, y, z), e["y"] at (x, y+d/2, z), e["z"] at (x, y, z+d/2),
    each numel(x) x numel(y) x numel(z), column-major (MATLAB's layout, which
    the engine takes without a copy).  Shapes paint in order (box, cyl,
    cone, polygon, lattice).  "directional": harmonic mean along the
    component's own axis, arithmetic over the other two; "kottke":
    1/eps_cc = n_c^2 <1/eps> + (1 - n_c^2)/<eps> with n from the first moment
    of eps.  Only cells an interface crosses are sub-sampled; Period = [Lx Ly]
    folds x, y into [-L/2, L/2).

    device: a Context (or True for the current device's default context)
    computes either form on the GPU (orf_eps3d), bitwise the same values, in
    milliseconds per component instead of seconds.
    """
    x = np.asarray(x, dtype=float).ravel()
    y = np.asarray(y, dtype=float).ravel()
    z = np.asarray(z, dtype=float).ravel()
    d = x[1] - x[0]
    h = d / 2
    sh = [_Shape(k, p) for k, p in _shape_list(shapes)]
    Lx = Ly = None
    if Period is not None:
        Lx, Ly = (float(Period[0]), float(Period[1]))
    if device is not None and device is not False:
        if Method not in ("directional", "kottke"):
            raise ValueError('Method must be "directional" or "kottke"')
        return _eps3d_device(x, y, z, nBg, sh, NSub, Period, device, Method)
    off = _offsets(NSub)
    out = {}
    for c, name in enumerate(("x", "y", "z")):
        shift = [0.0, 0.0, 0.0]
        shift[c] = h
        X = (x + shift[0])[:, None, None]
        Y = (y + shift[1])[None, :, None]
        Zall = z + shift[2]
        # planes whose cells no shape face crosses and that lie inside the
        # same z-ranges of z-extruded shapes carry the same x-y map: compute
        # one representative of each such class, and every other plane alone
        rep, inv = _z_classes(Zall, sh, h)
        e = _component(c, X, Y, Zall[rep][None, None, :], sh, nBg, h, d, off, NSub, Lx, Ly, Method)
        if rep.size < Zall.size:
            # column-major (the layout the engine takes without a copy): each
            # plane is one contiguous block, copied from its representative
            full = np.empty(e.shape[:2] + (Zall.size,), order="F")
            for k in range(Zall.size):
                full[:, :, k] = e[:, :, inv[k]]
            e = full
        out[name] = e
    return out


def _eps3d_device(x, y, z, nBg, sh, NSub, Period, device, Method="directional") -> dict:
    """epsComponents3D on the GPU through orf_eps3d (csrc/eps3d.cu)."""
    import ctypes as C
    from . import _abi, _lib
    lib = _lib.load()
    kinds = {"box": 0, "cyl": 1, "cone": 1, "polygon": 2, "lattice": 3}
    arr = (_abi.OrfEpsShape * max(1, len(sh)))()
    keep = []
    for q, s in enumerate(sh):
        o = arr[q]
        o.kind = kinds[s.kind]
        o.n = float(s.n)
        for t in range(3):
            o.lo[t], o.hi[t] = float(s.lo[t]), float(s.hi[t])
        p = []
        if s.kind in ("cyl", "cone"):
            p = [s.c[0], s.c[1], s.r1, s.r2, s.z1, s.z2]
        elif s.kind == "polygon":
            p = [s.z1, s.z2]
            tab = np.ascontiguousarray(s.xy, dtype=float)
            o.n0 = tab.shape[0]
        elif s.kind == "lattice":
            p = [s.x0, s.y0, s.P, s.z1, s.z2, s.dRdz]
            tab = np.ascontiguousarray(s.R, dtype=float)
            o.n0, o.n1 = tab.shape
        for t, v in enumerate(p):
            o.p[t] = float(v)
        if s.kind in ("polygon", "lattice"):
            keep.append(tab)
            o.data = _abi._ptr(tab)
    shape = (x.size, y.size, z.size)
    out = {k: np.empty(shape, order="F") for k in ("x", "y", "z")}
    per = None if Period is None else np.array([float(Period[0]), float(Period[1])])
    ctx = getattr(device, "handle", None)
    st = lib.orf_eps3d(ctx, _abi._ptr(x), _abi._ptr(y), _abi._ptr(z), x.size, y.size, z.size, float(nBg),
                       int(NSub), 1 if Method == "kottke" else 0, _abi._ptr(per), len(sh),
                       C.cast(arr, C.c_void_p),
                       _abi._ptr(out["x"]), _abi._ptr(out["y"]), _abi._ptr(out["z"]))
    _lib.check(st, "epsComponents3D")
    return out


def _z_classes(Z: np.ndarray, sh: list, h: float):
    """(representative plane indices, plane -> representative map)."""
    n = Z.size
    everything = (np.arange(n), np.arange(n))
    zb = []
    for s in sh:
        if not s.z_extruded():
            return everything
        for v in (s.lo[2], s.hi[2]):
            if np.isfinite(v):
                zb.append(float(v))
    zb = np.array(sorted(set(zb)))
    if zb.size == 0:
        face = np.zeros(n, dtype=bool)
        keys = np.zeros((n, 0), dtype=bool)
    else:
        # planes within 2h of a z boundary are computed one by one: farther
        # out, every band, inside and sub-sample test of a plane depends only
        # on which side of each boundary it lies (its key), with no rounding
        # at a threshold, so the planes of one class carry the same map
        face = (np.abs(Z[:, None] - zb[None, :]) <= 2 * h).any(axis=1)
        keys = Z[:, None] >= zb[None, :]
    rep, inv, seen = [], np.empty(n, dtype=np.int64), {}
    for k in range(n):
        key = None if face[k] else keys[k].tobytes()
        if key is not None and key in seen:
            inv[k] = seen[key]
            continue
        inv[k] = len(rep)
        if key is not None:
            seen[key] = len(rep)
        rep.append(k)
    return np.array(rep, dtype=np.int64), inv


def _component(c, X, Y, Z, sh, nBg, h, d, off, NSub, Lx, Ly, Method):
    """One eps component at cell centres X (nx,1,1), Y (1,ny,1), Z (1,1,nz)."""
    Xf, Yf = _fold(X, Lx), _fold(Y, Ly)
    shape3 = (X.shape[0], Y.shape[1], Z.shape[2])
    # material at the cell centres (column-major, as the engine takes it)
    e = np.full(shape3, float(nBg) ** 2, order="F")
    band = np.zeros(shape3, dtype=bool, order="F")
    for s in sh:
        e[np.broadcast_to(s.inside(Xf, Yf, Z), shape3)] = s.n ** 2
        band |= np.broadcast_to(s.band(Xf, Yf, Z, h), shape3)
    if NSub > 1 and band.any():
        ii, jj, kk = np.nonzero(band)
        cx, cy, cz = X.ravel()[ii], Y.ravel()[jj], Z.ravel()[kk]
        m = ii.size
        val = np.empty(m)
        # sub-sample in bounded chunks of band cells (memory: chunk x NSub^3)
        step = max(1, (1 << 22) // (NSub ** 3))
        for q0 in range(0, m, step):
            q1 = min(m, q0 + step)
            # samples s[m, a, b, c] with a along x, b along y, c along z
            sx = cx[q0:q1, None] + off[None, :] * d
            sy = cy[q0:q1, None] + off[None, :] * d
            sz = cz[q0:q1, None] + off[None, :] * d
            SX = _fold(sx[:, :, None, None], Lx)
            SY = _fold(sy[:, None, :, None], Ly)
            SZ = sz[:, None, None, :]
            SXb, SYb, SZb = np.broadcast_arrays(SX, SY, SZ)
            es = np.full(SXb.shape, float(nBg) ** 2)
            for s in sh:
                es[np.broadcast_to(s.inside(SXb, SYb, SZb), es.shape)] = s.n ** 2
            mq = q1 - q0
            if Method == "directional":
                # harmonic mean along c, then arithmetic over the other two
                # axes, each sum sequential in index order (the GPU generator,
                # csrc/eps3d.cu, adds in the same order: same bits)
                # (np.cumsum accumulates left to right, one addition at a time)
                inv = np.moveaxis(1.0 / es, 1 + c, 1)                   # (m, along, r1, r2)
                acc = np.cumsum(inv, axis=1)[:, -1]
                r = (1.0 / (acc / NSub)).reshape(mq, NSub * NSub)
                tot = np.cumsum(r, axis=1)[:, -1]
                val[q0:q1] = tot / (NSub * NSub)
            elif Method == "kottke":
                # sums sequential over the samples in row-major (x, y, z)
                # order, as the GPU generator adds them
                flat = es.reshape(mq, -1)
                inv = 1.0 / flat
                n3 = NSub ** 3
                q3 = np.arange(n3)
                w = [off[q3 // (NSub * NSub)], off[(q3 // NSub) % NSub], off[q3 % NSub]]
                se = np.cumsum(flat, axis=1)[:, -1]
                si = np.cumsum(inv, axis=1)[:, -1]
                grads = [np.cumsum(flat * w[ax][None, :], axis=1)[:, -1] for ax in range(3)]
                mean_e, mean_inv = se / n3, si / n3
                gn = np.sqrt(sum(g * g for g in grads))
                nc2 = np.where(gn > 0, (grads[c] / np.where(gn > 0, gn, 1.0)) ** 2, 0.0)
                val[q0:q1] = 1.0 / (nc2 * mean_inv + (1.0 - nc2) / mean_e)
            else:
                raise ValueError('Method must be "directional" or "kottke"')
        e[ii, jj, kk] = val
    return e
