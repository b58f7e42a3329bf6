"""Host-side geometry and mode helpers (product code) against the reference's
open algorithms and known answers."""
import numpy as np

import oracle
from opticrcwafdtd_b200 import epsComponents2D, epsComponents3D, epsFromBoxes, slabModes


def test_eps_from_boxes_matches_literal_restatement():
    # toolbox/+orf/epsFromBoxes.m:16-30 restated literally in oracle/geometry_ref.py
    rng = np.random.default_rng(3)
    x = np.arange(60) * 0.03 - 0.2
    z = np.arange(45) * 0.03 + 0.1
    boxes = []
    for _ in range(8):
        a, b = sorted(rng.uniform(-0.3, 1.9, 2))
        c, d = sorted(rng.uniform(0.0, 1.5, 2))
        boxes.append([a, b, c, d, rng.uniform(1, 3.5)])
    boxes.append([0.4, np.inf, -np.inf, 0.5, 2.2])
    for nsub in (1, 3, 4):
        assert np.array_equal(epsFromBoxes(x, z, 1.3, boxes, nsub),
                              oracle.epsFromBoxes_ref(x, z, 1.3, boxes, nsub)) or \
            np.max(np.abs(epsFromBoxes(x, z, 1.3, boxes, nsub) - oracle.epsFromBoxes_ref(x, z, 1.3, boxes, nsub))) < 1e-13


def test_directional_eps_averaging_known_answers():
    # tests/TestFDTD2D.m:86-97
    x = np.round(np.arange(0, 2.0001, 0.1), 12)
    z = np.round(np.arange(0, 1.0001, 0.1), 12)
    e = epsComponents2D(x, z, 1, [1.0, np.inf, -np.inf, np.inf, 2])
    i = int(np.nonzero(np.abs(x - 1.0) < 1e-12)[0][0])
    assert abs(e["y"][i, 4] - 2.5) < 1e-12
    assert abs(e["x"][i, 4] - 1.6) < 1e-12
    assert abs(e["z"][i, 4] - 4) < 1e-12
    assert abs(e["z"][i - 1, 4] - 1) < 1e-12


def test_eps_components_shapes_and_periodic():
    x = np.arange(20) * 0.05
    z = (np.arange(16) + 0.5) * 0.05 - 0.4
    e = epsComponents2D(x, z, 1, [0.3, 0.7, -0.1, 0.1, 2], PeriodicZ=True)
    assert e["y"].shape == (20, 16) and e["x"].shape == (20, 16) and e["z"].shape == (19, 16)
    e2 = epsComponents2D(x, z, 1, [0.3, 0.7, -0.1, 0.1, 2])
    assert e2["x"].shape == (20, 15)
    # a box straddling the periodic seam paints both ends
    e3 = epsComponents2D(x, z, 1, [0.3, 0.7, 0.35, 0.45, 2], PeriodicZ=True)
    assert e3["y"][8, 0] > 1 and e3["y"][8, -1] > 1


def test_eps_components_3d_box_directional():
    d = 0.1
    x = np.arange(12) * d
    e = epsComponents3D(x, x, x, 1, [["box", [0.5, np.inf, -np.inf, np.inf, -np.inf, np.inf, 2]]])
    # the face x = 0.5 cuts the Ex cell at x_i+1/2 = 0.45 + ... check the known 1D means
    i = 4   # Ey cell centred at x = 0.4 spans [0.35, 0.45): outside
    assert abs(e["y"][i, 3, 3] - 1) < 1e-12
    i = 5   # Ey cell at x = 0.5 spans [0.45, 0.55): half inside -> arithmetic 2.5
    assert abs(e["y"][i, 3, 3] - 2.5) < 1e-12
    i = 4   # Ex cell at x = 0.45 spans [0.4, 0.5): outside
    assert abs(e["x"][i, 3, 3] - 1) < 1e-12
    # Ex at x = 0.5 + 0.05 -> inside
    assert abs(e["x"][5, 3, 3] - 4) < 1e-12


def test_slab_modes_te_tm():
    dx = 0.02
    z = np.arange(-1.5, 1.5 + dx / 2, dx) + dx / 2
    epsw = epsFromBoxes(np.arange(3) * dx, z, 1.444, [-np.inf, np.inf, -0.11, 0.11, 3.476])
    m = slabModes(z, np.sqrt(epsw[0, :]), 1.55, "TE", 2)
    assert m["field"].shape == (z.size, 2)
    assert 2.8 < m["neff"][0] < 2.9 and m["neff"][0] > m["neff"][1]
    assert abs(np.max(np.abs(m["field"][:, 0])) - 1) < 1e-12 and np.max(m["field"][:, 0]) == 1.0
    # compare with a dense eig of the same matrix (slabModes.m:29-30, 44-47)
    N = z.size
    k0 = 2 * np.pi / 1.55
    A = (np.diag(np.full(N - 1, 1 / dx ** 2), -1) + np.diag(np.full(N - 1, 1 / dx ** 2), 1)
         + np.diag(-2 / dx ** 2 + k0 ** 2 * epsw[0, :]))
    w = np.sort(np.linalg.eigvals(A).real)[::-1]
    assert abs(np.sqrt(w[0]) / k0 - m["neff"][0]) < 1e-12
    mt = slabModes(z, np.sqrt(epsw[0, :]), 1.55, "TM")
    assert 2.0 < mt["neff"][0] < m["neff"][0]


def _eps3d_every_cell_sampled(x, y, z, nBg, shapes, c, NSub=4):
    """Directional average with every cell sub-sampled (no interface band)."""
    from opticrcwafdtd_b200.geometry import _Shape, _offsets, _shape_list
    sh = [_Shape(k, p) for k, p in _shape_list(shapes)]
    d = x[1] - x[0]
    off = _offsets(NSub) * d
    shift = np.zeros(3)
    shift[c] = d / 2
    X = (x + shift[0])[:, None] + off[None, :]
    Y = (y + shift[1])[:, None] + off[None, :]
    Z = (z + shift[2])[:, None] + off[None, :]
    SX = X[:, None, None, :, None, None]
    SY = Y[None, :, None, None, :, None]
    SZ = Z[None, None, :, None, None, :]
    SX, SY, SZ = np.broadcast_arrays(SX, SY, SZ)
    es = np.full(SX.shape, float(nBg) ** 2)
    for s in sh:
        es[s.inside(SX, SY, SZ)] = s.n ** 2
    inv_along = (1.0 / es).mean(axis=3 + c)
    return (1.0 / inv_along).reshape(x.size, y.size, z.size, -1).mean(axis=3)


def test_eps_components_3d_band_covers_every_interface():
    """Cells outside the interface band are homogeneous: the band-limited
    average equals sub-sampling every cell (pillar lattice, cylinder, cone,
    boxes), and extruded planes shared between z classes stay exact."""
    rng = np.random.default_rng(7)
    d = 0.02
    x = (np.arange(26) + 0.5) * d
    y = (np.arange(24) + 0.5) * d
    z = np.arange(30) * d
    shapes = [["box", [-np.inf, np.inf, -np.inf, np.inf, -np.inf, 0.17, 1.46]],
              ["lattice", dict(x0=0.1, y0=0.1, period=0.2, R=rng.uniform(0.03, 0.09, (3, 3)), z1=0.17, z2=0.43,
                               n=2.4)],
              ["cyl", [0.25, 0.2, 0.07, 0.45, 0.55, 3.0]],
              ["cone", [0.3, 0.25, 0.03, 0.1, 0.05, 0.3, 1.8]]]
    e = epsComponents3D(x, y, z, 1.0, shapes)
    for c, k in enumerate("xyz"):
        ref = _eps3d_every_cell_sampled(x, y, z, 1.0, shapes, c)
        np.testing.assert_allclose(e[k], ref, rtol=1e-13, atol=0)


def test_3d_plane_classes_change_no_bit(monkeypatch):
    """epsComponents3D computes one plane per class of z-extruded planes and
    copies it; the copies must equal planes computed one by one, also where a
    shape's top lies on a grid plane (the component shifted by h then sits a
    rounding away from the band test's threshold)."""
    from opticrcwafdtd_b200 import geometry
    d = 0.02
    x = (np.arange(40) + 0.5) * d
    y = x.copy()
    z = np.arange(120) * d
    R = np.random.default_rng(3).uniform(0.06, 0.18, (2, 2))
    shapes = [["box", [-np.inf, np.inf, -np.inf, np.inf, -np.inf, 0.9, 1.46]],
              ["lattice", dict(x0=0.2, y0=0.2, period=0.4, R=R, z1=0.9, z2=1.5, n=2.4)],
              ["cyl", [0.4, 0.4, 0.1, 1.71, 2.0, 3.0]]]
    a = geometry.epsComponents3D(x, y, z, 1.0, shapes)
    monkeypatch.setattr(geometry, "_z_classes", lambda Z, sh, h: (np.arange(Z.size), np.arange(Z.size)))
    b = geometry.epsComponents3D(x, y, z, 1.0, shapes)
    for k in "xyz":
        assert np.array_equal(a[k], b[k]), k


def test_3d_kottke_reduces_to_directional_on_planar_faces():
    """Method "kottke" (epsComponents3D.m:19-24: 1/eps_cc = n_c^2 <1/eps> +
    (1 - n_c^2)/<eps>, n from the first moment of eps): on the faces of a z
    slab the normal is z, so eps_zz is the harmonic mean of the samples and
    eps_xx, eps_yy the arithmetic one -- the directional form's values."""
    from opticrcwafdtd_b200 import geometry
    d = 0.02
    x = (np.arange(6) + 0.5) * d
    y = x.copy()
    z = np.arange(40) * d
    slab = [["box", [-np.inf, np.inf, -np.inf, np.inf, 0.213, 0.517, 2.2]]]
    k = geometry.epsComponents3D(x, y, z, 1.3, slab, Method="kottke")
    dr = geometry.epsComponents3D(x, y, z, 1.3, slab)
    for c in "xyz":
        assert np.allclose(k[c], dr[c], rtol=1e-12, atol=0), c
    # the interface planes are sub-sampled: their values lie between the materials
    mid = k["z"][0, 0, :]
    assert np.any((mid > 1.3 ** 2 + 1e-9) & (mid < 2.2 ** 2 - 1e-9))


def test_3d_shape_cross_sections():
    """Each 3D shape covers its documented cross-section: on a plane inside
    its z range the z component (harmonic along z over one material, then
    arithmetic over the in-plane sub-samples) is the in-plane fill fraction,
    whose sum is the area -- pi r^2 for a cylinder, the cone's radius at that
    height, a triangle's area, sum pi R^2 for a lattice (missing site R = 0)."""
    from opticrcwafdtd_b200 import geometry
    d = 0.01
    x = (np.arange(-60, 60) + 0.5) * d
    y = x.copy()
    z = np.arange(40) * d
    bg, n = 1.0, 2.0

    def area(shape, k):
        e = geometry.epsComponents3D(x, y, z, bg, [shape])["z"][:, :, k]
        return float(np.sum((e - bg ** 2) / (n ** 2 - bg ** 2))) * d * d

    k = 20   # the plane at z = 0.2 + h, inside every shape below
    zc = z[k] + d / 2
    assert abs(area(["cyl", [0.03, -0.05, 0.31, 0.05, 0.35, n]], k) / (np.pi * 0.31 ** 2) - 1) < 5e-3
    # a gentle cone: on a steep wall the radius changes within a cell's
    # height and the harmonic mean along z no longer measures the fill
    r = 0.2 + (0.26 - 0.2) * (zc - 0.05) / (0.35 - 0.05)
    assert abs(area(["cone", [0.0, 0.0, 0.2, 0.26, 0.05, 0.35, n]], k) / (np.pi * r * r) - 1) < 5e-3
    tri = dict(xy=[[-0.4, -0.3], [0.45, -0.2], [0.05, 0.5]], z1=0.05, z2=0.35, n=n)
    tri_area = 0.5 * abs((0.45 + 0.4) * (0.5 + 0.3) - (0.05 + 0.4) * (-0.2 + 0.3))
    assert abs(area(["polygon", tri], k) / tri_area - 1) < 5e-3
    R = np.array([[0.1, 0.12], [0.0, 0.09]])
    lat = dict(x0=-0.25, y0=-0.25, period=0.5, R=R, z1=0.05, z2=0.35, n=n)
    assert abs(area(["lattice", lat], k) / (np.pi * np.sum(R ** 2)) - 1) < 1e-2
