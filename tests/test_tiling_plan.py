"""CPU checks of the 2D tile plan (orf_plan2d, no device needed), over seeded
random grids, CPML widths, periodicity, precisions, fused depths T and
interior variants.  They stand in for a device-side bounds checker:

  - every cell of the grid is output by exactly one tile;
  - a tile's output lies in its loaded window, and every cell within T of an
    output cell (its T-step dependency cone) is in the loaded window or, for a
    frame tile, outside the grid (where the masks keep every field zero);
  - interior tiles (no CPML code, no masks) keep the cone of their outputs
    clear of the CPML slabs and the grid edge;
  - loaded windows start on 4-cell boundaries (the 4-byte material-index
    copies; 16 bytes of FP32 field rows);
  - a frame tile whose loaded window (with a cell of margin) reaches an x or z
    CPML slab carries that axis's flag (the kernel skips the psi arithmetic of
    an axis otherwise), the TF/SF flag marks windows holding the source
    column or the one left of it, and the monitor flags mark outputs holding a
    monitor line."""
import numpy as np
import pytest

from opticrcwafdtd_b200.fdtd import plan2d


def _sim(nx, nz, npx, npz, per, pol, precision, sx, mons, monz):
    x = np.arange(nx) * 0.02
    z = np.arange(nz) * 0.02
    sim = dict(pol=pol, x=x, z=z, npml=[npx, npz], periodicZ=per, lambdas=[1.55], monitors=mons,
               monitorsZ=monz, maxTime=1.0, shutoff=0.0, precision=precision)
    if pol == "TE":
        sim["eps"] = np.ones((nx, nz))
    else:
        sim["epsX"] = np.ones((nx, nz if per else nz - 1))
        sim["epsZ"] = np.ones((nx - 1, nz))
    sim["source"] = dict(ix=sx, profile=np.ones(nz), neff=1.5, lambda0=1.55, bw=0.2)
    return sim


def _check(sim, tsteps, variant):
    p = plan2d(sim, tsteps=tsteps, variant=variant)
    T = p["tsteps"]
    t = p["tiles"]
    nx, nz = sim["x"].size, sim["z"].size
    per = bool(sim["periodicZ"])
    npx, npz = sim["npml"][0], 0 if per else sim["npml"][1]
    sx = sim["source"]["ix"] - 1
    assert 1 <= T <= 16
    assert np.all(t["kind"][:p["n_interior"]] == 0) and np.all(t["kind"][p["n_interior"]:] == 1)
    cover = np.zeros((nx, nz), dtype=np.int32)
    for q in range(t["kind"].size):
        kind, li0, lk0, lx, lz = (int(t[k][q]) for k in ("kind", "li0", "lk0", "lx", "lz"))
        oi0, ok0, ow, oh, fl = (int(t[k][q]) for k in ("oi0", "ok0", "ow", "oh", "flags"))
        assert ow >= 1 and oh >= 1, q
        assert li0 % 4 == 0, (q, li0)
        assert 0 <= oi0 and oi0 + ow <= nx and 0 <= ok0 and ok0 + oh <= nz, q
        cover[oi0:oi0 + ow, ok0:ok0 + oh] += 1
        # the dependency cone of the outputs: [oi0 - T, oi0 + ow + T) x [ok0 - T, ok0 + oh + T)
        c_lo_x, c_hi_x = oi0 - T, oi0 + ow + T
        c_lo_z, c_hi_z = ok0 - T, ok0 + oh + T
        inside_x = (max(c_lo_x, 0) >= li0) and (min(c_hi_x, nx) <= li0 + lx)
        if per:
            inside_z = c_lo_z >= lk0 and c_hi_z <= lk0 + lz
        else:
            inside_z = (max(c_lo_z, 0) >= lk0) and (min(c_hi_z, nz) <= lk0 + lz)
        assert inside_x and inside_z, ("cone leaves the loaded window", q, T)
        if kind == 0:
            # interior: the cone is plain cells (no slab, no edge, no mask)
            assert c_lo_x >= npx and c_hi_x <= nx - npx, ("interior cone meets an x slab or edge", q)
            if not per:
                assert c_lo_z >= npz and c_hi_z <= nz - npz, ("interior cone meets a z slab or edge", q)
        else:
            # frame: axis flags for the slabs the loaded window reaches (one cell of margin)
            wx = np.arange(max(li0 - 1, 0), min(li0 + lx + 1, nx))
            if npx > 0 and np.any((wx < npx) | (wx >= nx - 1 - npx)):
                assert fl & 8, ("x CPML flag missing", q)
            if npz > 0:
                wz = np.arange(lk0 - 1, lk0 + lz + 1)
                wz = wz[(wz >= 0) & (wz < nz)]
                if np.any((wz < npz) | (wz >= nz - 1 - npz)):
                    assert fl & 16, ("z CPML flag missing", q)
        if (li0 <= sx - 1 < li0 + lx) or (li0 <= sx < li0 + lx):
            assert fl & 1, ("TF/SF flag missing", q)
        if any(oi0 <= m - 1 < oi0 + ow for m in sim["monitors"]):
            assert fl & 2, q
        if any(ok0 <= m - 1 < ok0 + oh for m in sim["monitorsZ"]):
            assert fl & 4, q
    assert np.all(cover == 1), ("cells output by", np.unique(cover))
    return p


def _random_case(rng):
    nx = int(rng.integers(12, 1300))
    nz = int(rng.integers(6, 600))
    npx = int(rng.integers(0, min(26, (nx - 2) // 2)))
    per = bool(rng.random() < 0.25)
    npz = 0 if per else int(rng.integers(0, min(26, (nz - 2) // 2)))
    pol = "TE" if rng.random() < 0.5 else "TM"
    prec = "single" if rng.random() < 0.5 else "double"
    sx = int(rng.integers(npx + 1, nx - npx + 1))
    mons = sorted(set(int(v) for v in rng.integers(1, nx + 1, 3)))
    monz = sorted(set(int(v) for v in rng.integers(1, nz + 1, 2)))
    tsteps = int(rng.choice([0, 1, 2, 3, 4, 5, 6, 8, 10]))
    variant = int(rng.choice([0, 1, 2]))
    return _sim(nx, nz, npx, npz, per, pol, prec, sx, mons, monz), tsteps, variant


@pytest.mark.parametrize("seed", range(8))
def test_random_plans_cover_once_and_keep_cones(seed):
    rng = np.random.default_rng(1000 + seed)
    for _ in range(25):
        sim, tsteps, variant = _random_case(rng)
        _check(sim, tsteps, variant)


@pytest.mark.parametrize("shape", [(4000, 1500, "TM"), (800, 300, "TE"), (600, 250, "TE"), (1200, 350, "TE")])
@pytest.mark.parametrize("precision", ["single", "double"])
def test_benchmark_grids(shape, precision):
    nx, nz, pol = shape
    sim = _sim(nx, nz, 20, 20, False, pol, precision, 101, [51, 301, nx - 30], [nz // 2], )
    for tsteps in (0, 4, 6, 8, 10):
        for variant in (1, 2):
            _check(sim, tsteps, variant)


def test_one_frame_tile_row_covers_the_cpml_strip():
    """With T = 8 and 64 x 40 frame tiles, a tile at the grid edge outputs 32
    rows (no margin on the edge side), enough for the 20 CPML rows plus the
    T rows the interior keeps clear: the bottom and top strips take one tile
    row each on the 800 x 300 coupler grid."""
    sim = _sim(800, 300, 20, 20, False, "TE", "single", 51, [26, 61, 770], [150])
    p = _check(sim, 8, 1)
    t = p["tiles"]
    fr, it = t["kind"] == 1, t["kind"] == 0
    # the interior spans rows [32, 268): the strips below and above are one tile row
    assert np.min(t["ok0"][it]) == 32 and np.max(t["ok0"][it] + t["oh"][it]) == 268
    bottom = fr & (t["ok0"] < 32)
    assert np.all(t["ok0"][bottom] == 0) and np.all(t["lk0"][bottom] == 0) and np.all(t["oh"][bottom] == 32)
    top = fr & (t["ok0"] + t["oh"] > 268)
    assert np.all(t["ok0"][top] == 268) and np.all(t["lk0"][top] + 40 == 300)


# --------------------------------------------------------------------- 3D ---
def _sim3d(n, npml, per):
    d = 0.04
    x, y, z = (np.arange(m) * d for m in n)
    src = dict(axis=3, index=max(2, npml[2] + 2) if not per[2] else 3, Ea=1.0, Hb=1.0, lambda0=0.6)
    return dict(x=x, y=y, z=z, eps={c: np.ones(n) for c in "xyz"}, npml=list(npml), periodic=list(per),
                source=src, lambdas=[0.6], monitors=[], maxTime=1.0, shutoff=0.0)


def _check3d(sim):
    from opticrcwafdtd_b200.fdtd import plan3d
    p = plan3d(sim)
    t = p["tiles"]
    n = (sim["x"].size, sim["y"].size, sim["z"].size)
    per = [bool(v) for v in sim["periodic"]]
    npml = [0 if per[q] else int(sim["npml"][q]) for q in range(3)]
    cover = np.zeros(n, dtype=np.int32)
    for q in range(t["kind"].size):
        kind, i0, j0, tw, th, k0, k1, tma, tx, tix = (int(t[k][q]) for k in
                                                      ("kind", "i0", "j0", "tw", "th", "k0", "k1", "tma", "tma_x",
                                                       "tma_index_x"))
        assert i0 % 32 == 0 and j0 % 8 == 0 and 1 <= tw <= 32 and 1 <= th <= 8, q
        assert 1 <= k1 - k0 <= 60, ("segment longer than the kernel's 64-bit plane mask allows", q)
        cover[i0:i0 + tw, j0:j0 + th, k0:k1] += 1
        if tma:
            # a TMA tile's halo (one cell each side in x and y) must not wrap ...
            if per[0]:
                assert i0 - 1 >= 0 and i0 + 32 < n[0], q
            if per[1]:
                assert j0 - 1 >= 0 and j0 + 8 < n[1], q
            # ... and every box must start on a 16-byte boundary in x
            for esz in (4, 8):
                assert (tx * esz) % 16 == 0, (q, tx, esz)
            for isz in (1, 2, 4):
                assert (tix * isz) % 16 == 0, (q, tix, isz)
        else:
            assert (per[0] and (i0 == 0 or i0 + 32 >= n[0])) or (per[1] and (j0 == 0 or j0 + 8 >= n[1])), q
        if kind == 0:
            # interior: every cell it updates or recomputes (halo of one cell,
            # the plane below the segment) keeps a cell of distance from the
            # slabs of E (u < np, u >= n - np) and H (u >= n - 1 - np)
            region = [(i0 - 1, i0 + tw + 1), (j0 - 1, j0 + th + 1), (k0 - 1, k1 + 1)]
            for ax, (lo, hi) in enumerate(region):
                if npml[ax] > 0:
                    assert lo - 1 >= npml[ax] and hi + 1 <= n[ax] - 1 - npml[ax], ("interior tile near a slab", q, ax)
    assert np.all(cover == 1)
    return p


@pytest.mark.parametrize("seed", range(4))
def test_random_3d_plans(seed):
    rng = np.random.default_rng(2000 + seed)
    for _ in range(12):
        n = tuple(int(v) for v in rng.integers(10, 170, 3))
        per = tuple(bool(v) for v in rng.random(3) < 0.4)
        npml = tuple(int(rng.integers(0, max(1, min(12, (m - 4) // 2)))) for m in n)
        _check3d(_sim3d(n, npml, per))


def test_pillar_lattice_3d_plan():
    p = _check3d(_sim3d((600, 600, 300), (0, 0, 20), (True, True, False)))
    assert p["n_interior"] > 0 and p["n_cpml"] > 0
