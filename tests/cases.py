"""Simulation setups shared by the tests, written after the reference's own
FDTD tests (tests/TestFDTD2D.m, TestFDTD3D.m, TestGUISupport.m, TestCPO.m)."""
from __future__ import annotations

import numpy as np

from opticrcwafdtd_b200 import epsComponents2D, epsFromBoxes, slabModes


def slab_sim(dx=0.01, extra=None):
    """TestFDTD2D.slabRun (tests/TestFDTD2D.m:11-32): plane wave, periodic z,
    0.5 um n = 2 slab; returns (sim, eps_empty, eps_slab)."""
    x = np.round(np.arange(0, 6 + dx / 2, dx), 12)
    z = np.arange(4) * dx
    lam = np.linspace(1.2, 1.8, 7)
    ixOf = lambda xx: int(round(xx / dx)) + 1
    s = dict(x=x, z=z, npml=[round(0.2 / dx), 0], periodicZ=True, lambdas=lam,
             monitors=[ixOf(0.6), ixOf(5)])
    s["source"] = dict(ix=ixOf(1), profile=np.ones(4), neff=1, lambda0=1.5, bw=0.3)
    if extra:
        s.update(extra)
    e0 = np.ones((x.size, z.size))
    e1 = epsFromBoxes(x, z, 1, [3.0, 3.5, -np.inf, np.inf, 2.0])
    return s, e0, e1


def slab_rt(run, dx=0.01, extra=None):
    s, e0, e1 = slab_sim(dx, extra)
    s["eps"] = e0
    o0 = run(s)
    s["eps"] = e1
    o1 = run(s)
    R = -o1["flux"][0] / o0["flux"][1]
    T = o1["flux"][1] / o0["flux"][1]
    Rempty = np.abs(o0["flux"][0] / o0["flux"][1])
    return R, T, Rempty


def waveguide_sim(lambdas=None):
    """TestFDTD2D.waveguideRun (tests/TestFDTD2D.m:38-48): Si slab in SiO2, TE0 source."""
    dx = 0.02
    x = np.round(np.arange(0, 8 + dx / 2, dx), 12)
    z = np.arange(-1.5, 1.5 + dx / 2, dx) + dx / 2
    epsw = epsFromBoxes(x, z, 1.444, [-np.inf, np.inf, -0.11, 0.11, 3.476])
    m = slabModes(z, np.sqrt(epsw[0, :]), 1.55, "TE")
    sim = dict(x=x, z=z, eps=epsw, npml=[15, 15],
               lambdas=np.linspace(1.5, 1.6, 5) if lambdas is None else lambdas, monitors=[51, 151, 301])
    sim["source"] = dict(ix=101, profile=m["field"][:, 0], neff=m["neff"][0], lambda0=1.55, bw=0.1)
    return sim, m


def waveguide_tm_sim():
    """TestFDTD2D.tmGuidedModeMatchesDiscreteDispersion (tests/TestFDTD2D.m:115-124)."""
    dx = 0.02
    x = np.round(np.arange(0, 8 + dx / 2, dx), 12)
    z = np.arange(-1.5, 1.5 + dx / 2, dx) + dx / 2
    e = epsComponents2D(x, z, 1.444, [-np.inf, np.inf, -0.11, 0.11, 3.476])
    m = slabModes(z, np.sqrt(e["z"][0, :]), 1.55, "TM", EpsHalf=e["x"][0, :])
    sim = dict(pol="TM", x=x, z=z, epsX=e["x"], epsZ=e["z"], npml=[15, 15], lambdas=[1.55],
               monitors=[51, 151, 301])
    sim["source"] = dict(ix=101, profile=m["field"][:, 0], neff=m["neff"][0], lambda0=1.55, bw=0.1)
    return sim, m, e


def progress_sim():
    """TestGUISupport.fdtdReportsProgressAndCanBeCancelled (tests/TestGUISupport.m:27-33)."""
    dx = 0.02
    x = np.round(np.arange(0, 4 + dx / 2, dx), 12)
    z = np.arange(4) * dx
    s = dict(x=x, z=z, npml=[15, 0], periodicZ=True, lambdas=[1.5], monitors=[30, 170],
             eps=np.ones((x.size, 4)))
    s["source"] = dict(ix=40, profile=np.ones(4), neff=1, lambda0=1.5, bw=0.3)
    return s


def mixed_te_sim(nx=150, nz=90, steps=400, precision="double", seed=0, pol="TE", periodic=False):
    """Small random-structure run touching every code path: CPML on all sides
    (or periodic z), TF/SF mode-like source, x and z monitors, many materials."""
    rng = np.random.default_rng(seed)
    dx = 0.02
    x = np.arange(nx) * dx
    z = np.arange(nz) * dx
    boxes = []
    for _ in range(12):
        x1 = rng.uniform(1.0, nx * dx - 0.6)
        z1 = rng.uniform(0.1, nz * dx - 0.3)
        boxes.append([x1, x1 + rng.uniform(0.05, 0.5), z1, z1 + rng.uniform(0.05, 0.4), rng.uniform(1.3, 3.5)])
    e = epsComponents2D(x, z, 1.444, boxes, PeriodicZ=periodic)
    prof = np.exp(-((z - z.mean()) / (0.2 * nz * dx)) ** 2)
    sim = dict(pol=pol, x=x, z=z, npml=[12, 0 if periodic else 10], periodicZ=periodic,
               lambdas=np.linspace(1.45, 1.65, 7), monitors=[20, nx - 25, nx // 2],
               monitorsZ=[15, nz - 14] if not periodic else [5], shutoff=0, maxTime=steps * 0.99 / np.sqrt(2) * dx,
               precision=precision)
    if pol == "TE":
        sim["eps"] = e["y"]
    else:
        sim["epsX"], sim["epsZ"] = e["x"], e["z"]
    sim["source"] = dict(ix=30, profile=prof, neff=1.8, lambda0=1.55, bw=0.25)
    return sim


def box3d_sim(n=(28, 24, 36), axis=3, per=(False, False, False), steps=150, precision="double", seed=0,
              npml=(6, 5, 7), mons=None):
    """Small 3D run touching every code path: CPML or wrap per axis, a few
    random boxes, a TF/SF plane normal to `axis` with a smooth profile, and a
    monitor plane normal to each axis."""
    from opticrcwafdtd_b200 import epsComponents3D
    rng = np.random.default_rng(seed)
    d = 0.04
    x, y, z = (np.arange(m) * d for m in n)
    shapes = []
    for _ in range(4):
        lo = [rng.uniform(0.2, m * d - 0.5) for m in n]
        hi = [a + rng.uniform(0.1, 0.4) for a in lo]
        shapes.append(["box", [lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], rng.uniform(1.3, 2.6)]])
    e = epsComponents3D(x, y, z, 1.0, shapes)
    ax = axis - 1
    a, b = (ax + 1) % 3, (ax + 2) % 3
    ca = np.arange(n[a]) * d
    cb = np.arange(n[b]) * d
    prof = np.exp(-((ca[:, None] - ca.mean()) / (0.3 * n[a] * d)) ** 2 - ((cb[None, :] - cb.mean()) / (0.3 * n[b] * d)) ** 2)
    np_ = [0 if per[q] else npml[q] for q in range(3)]
    src = dict(axis=axis, index=np_[ax] + 3, Ea=prof, Eb=0.3 * prof, Ha=-0.2 * prof, Hb=1.2 * prof, neff=1.2,
               lambda0=0.6, bw=0.3)
    if mons is None:
        mons = [dict(axis=q + 1, index=np_[q] + 5 + (2 if q == ax else 0)) for q in range(3)]
        mons.append(dict(axis=axis, index=n[ax] - np_[ax] - 3))
    S = 0.99 / np.sqrt(3) * d
    return dict(x=x, y=y, z=z, eps=e, npml=list(np_), periodic=list(per), source=src, monitors=mons,
                lambdas=[0.55, 0.6, 0.65], maxTime=steps * S, shutoff=0.0, precision=precision)


def plane_wave_3d(x, y, z, d, lam, lambda0, bw, zSrc, zR, zT):
    """TestFDTD3D.planeWaveSim (tests/TestFDTD3D.m:179-189)."""
    izOf = lambda zz: int(round((zz - z[0]) / d)) + 1
    Na, Nb = x.size, y.size
    src = dict(axis=3, index=izOf(zSrc), Ea=np.ones((Na, Nb)), Eb=np.zeros((Na, Nb)), Ha=np.zeros((Na, Nb)),
               Hb=np.ones((Na, Nb)), neff=1, lambda0=lambda0, bw=bw)
    return dict(x=x, y=y, z=z, npml=[0, 0, round(0.3 / d)], periodic=[True, True, False], source=src,
                lambdas=lam, monitors=[dict(axis=3, index=izOf(zR)), dict(axis=3, index=izOf(zT))])


def strip3d_sim(precision="double"):
    """tests/TestFDTD3D.m:36-58 (stripRun): a 500 x 220 nm SOI strip along x
    (d = 40 nm) fed by its TE0 mode, solved by wgModes2D on the 3D grid's own
    (y, z) permittivity plane.  Returns (sim, prof, ms_eps)."""
    from opticrcwafdtd_b200 import epsComponents3D, wgModes2D
    d = 0.04
    x = np.arange(0, 2.6 + 1e-9, d)
    y = (np.arange(-30, 30) + 0.5) * d
    z = (np.arange(-25, 25) + 0.5) * d
    e = epsComponents3D(x, y, z, 1.444, [["box", [-np.inf, np.inf, -0.25, 0.25, -0.11, 0.11, 3.476]]])
    # mode-solver plane (a, b) = (y, z): its E_x, E_y, E_z are the 3D E_y, E_z, E_x
    ms_eps = {"x": e["y"][0], "y": e["z"][0], "z": e["x"][0]}
    m = wgModes2D(y, z, 1.444, np.zeros((0, 5)), 1.55, 2, Eps=ms_eps)
    ite = int(np.argmax(m["teFraction"]))
    prof = {k: np.real(m[f][:, :, ite]) for k, f in (("Ea", "Ex"), ("Eb", "Ey"), ("Ha", "Hx"), ("Hb", "Hy"))}
    ix = lambda xx: int(round(xx / d)) + 1
    src = dict(axis=1, index=ix(0.6), neff=float(m["neff"][ite]), lambda0=1.55, bw=0.1, **prof)
    sim = dict(x=x, y=y, z=z, eps=e, npml=[8, 8, 8], source=src, lambdas=[1.55],
               monitors=[dict(axis=1, index=ix(0.4)), dict(axis=1, index=ix(0.9)), dict(axis=1, index=ix(2.0))],
               precision=precision)
    return sim, prof, ms_eps


def check_strip3d(o, sim, prof, ms_eps):
    """tests/TestFDTD3D.m:100-117: unidirectional (< 1e-4 back), lossless
    guide (1e-3), and the phase advance between monitors 2 and 3 matching
    the mode index at the numerical wavenumber through the exact Yee
    dispersion along x (1e-4)."""
    from opticrcwafdtd_b200 import wgModes2D
    flux = o["flux"][:, 0]
    assert -flux[0] / flux[1] < 1e-4
    assert abs(flux[2] / flux[1] - 1.0) <= 1e-3
    d = sim["x"][1] - sim["x"][0]
    S = 0.99 / np.sqrt(3) * d
    k0 = 2 * np.pi / 1.55
    k0n = 2 / S * np.sin(k0 * S / 2)
    mt = wgModes2D(sim["y"], sim["z"], 1.444, np.zeros((0, 5)), 2 * np.pi / k0n, 2, Eps=ms_eps)
    it = int(np.argmax(mt["teFraction"]))
    n_pred = 2 / d * np.arcsin(mt["neff"][it] * k0n * d / 2) / k0
    ov = lambda q: (np.sum(prof["Ea"] * o["mon"][q]["Ea"][:, :, 0]) +
                    np.sum(prof["Eb"] * o["mon"][q]["Eb"][:, :, 0]))
    L = (sim["monitors"][2]["index"] - sim["monitors"][1]["index"]) * d
    ph = np.angle(ov(2)) - np.angle(ov(1))
    q = round((n_pred * k0 * L - ph) / (2 * np.pi))
    assert abs((ph + 2 * np.pi * q) / (k0 * L) - n_pred) <= 1e-4
