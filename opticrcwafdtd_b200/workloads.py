"""Seeded synthetic inputs with the shapes of the benchmark workloads.

No dataset is involved: every structure is generated from a seed, with the
sizes, materials and value distributions the workloads name.

  coupler_sim          2D TE SOI grating coupler, 800 x 300 at 20 nm, FP64, 8000 steps
  pixel_region_sim     2D TM Si/SiO2 pixel design region, 4000 x 1500 at 10 nm, 30000 steps
  pillar_lattice_sim   3D TiO2 pillar lattice on SiO2, 600 x 600 x 300 at 20 nm, 6000 steps
  coupler_batch_sims   256 2D TE grating couplers of uneven size, 10000 steps each (batch)
  serve_stream         Poisson stream of mixed 2D / 3D jobs (serving)

The 100 nm source bandwidth of the workloads is read as a 1/e spectral
half-width of 50 nm, i.e. bw = 0.05 / 1.55 in the reference's relative units
(fdtd2DTE.m:14-15).
"""
from __future__ import annotations

import math

import numpy as np

from .geometry import epsComponents2D, epsComponents3D
from .modes import slabModes

N_SI, N_SIO2, N_TIO2 = 3.476, 1.444, 2.4
BW_100NM = 0.05 / 1.55


def _closing(mask: np.ndarray, width: int) -> np.ndarray:
    """Binary dilation then erosion with a width x width square (min feature)."""
    from scipy.ndimage import binary_dilation, binary_erosion
    pad = width
    m = np.pad(mask, pad, mode="edge")
    st = np.ones((width, width), dtype=bool)
    m = binary_erosion(binary_dilation(m, st), st)
    return m[pad:-pad, pad:-pad]


def _runs_to_boxes(mask: np.ndarray, x0: float, z0: float, px: float, pz: float, n: float) -> list:
    """Merge the True pixels of each row into [x1 x2 z1 z2 n] boxes."""
    boxes = []
    for r in range(mask.shape[1]):
        row = mask[:, r]
        i = 0
        while i < row.size:
            if row[i]:
                j = i
                while j < row.size and row[j]:
                    j += 1
                boxes.append([x0 + i * px, x0 + j * px, z0 + r * pz, z0 + (r + 1) * pz, n])
                i = j
            else:
                i += 1
    return boxes


def pixel_region_sim(seed: int = 0, steps: int = 30000, precision: str = "single", nx: int = 4000, nz: int = 1500,
                n_lambda: int = 101) -> dict:
    """2D TM, dx = 10 nm, 20-cell CPML: SOI waveguide (220 nm Si in SiO2) whose
    middle 10 um x 0.22 um is a Bernoulli(0.5) Si/SiO2 pixel map (20 nm pixels,
    5-pixel closing = 100 nm minimum feature).  TM0 mode source, 101-wavelength
    DFT monitors over 1.5-1.6 um (reflection, incident, transmission lines and
    up / down planes)."""
    dx = 0.01
    x = np.arange(nx) * dx
    z = np.arange(nz) * dx
    zc = round(nz * dx / 2 / dx) * dx
    z1, z2 = zc - 0.115, zc + 0.105          # 22 cells, edges on cell boundaries
    xd1 = round(0.375 * nx) * dx - dx / 2     # design region starts on a cell edge
    xd2 = xd1 + 10.0
    rng = np.random.default_rng(seed)
    pix = rng.random((500, 11)) < 0.5
    pix = _closing(pix, 5)
    boxes = [[-np.inf, xd1, z1, z2, N_SI], [xd2, np.inf, z1, z2, N_SI]]
    boxes += _runs_to_boxes(pix, xd1, z1, 0.02, 0.02, N_SI)
    e = epsComponents2D(x, z, N_SIO2, boxes)
    ix = 101
    m = slabModes(z, np.sqrt(e["z"][ix - 1, :]), 1.55, "TM", EpsHalf=e["x"][ix - 1, :])
    S = 0.99 / math.sqrt(2) * dx
    sim = dict(pol="TM", x=x, z=z, epsX=e["x"], epsZ=e["z"], npml=[20, 20],
               lambdas=np.linspace(1.5, 1.6, n_lambda), monitors=[51, 301, round(0.75 * nx) + 1],
               monitorsZ=[round(0.5 * nz) + 250, round(0.5 * nz) - 250],
               maxTime=steps * S, shutoff=0.0, precision=precision)
    sim["source"] = dict(ix=ix, profile=m["field"][:, 0], neff=float(m["neff"][0]), lambda0=1.55, bw=BW_100NM)
    return sim


def grating_coupler_geometry(period=0.63, ff=0.5, etch=0.07, n_per=20, box=2.0, t_si=0.22, x_start=1.5,
                             n_clad=N_SIO2):
    """Boxes [x1 x2 z1 z2 n] of a uniform SOI grating coupler (gratingCouplerTE.m:1-27
    geometry): Si core z in [0, tSi], BOX below on a Si substrate, cladding above,
    grooves of depth etch at the top of the core.  ff is the unetched fraction."""
    boxes = [[-np.inf, np.inf, -np.inf, -box, N_SI],          # substrate
             [-np.inf, np.inf, -box, 0.0, N_SIO2],            # BOX
             [-np.inf, np.inf, 0.0, t_si, N_SI]]              # core
    for p in range(n_per):
        g0 = x_start + p * period + ff * period
        boxes.append([g0, x_start + (p + 1) * period, t_si - etch, t_si, n_clad])
    return boxes


def core_mode(z, n, lambda0, pol="TE", core=(0.0, 0.22), n_modes=8, eps_half=None, substrate_top=None):
    """The guided mode of the Si core (not a substrate mode): the slab mode
    with the largest share of |field|^2 inside the core.  With substrate_top
    given, the Si substrate below it is replaced by oxide for the mode solve,
    so a thick substrate's many guided modes cannot crowd the core mode out."""
    n = np.asarray(n, dtype=float)
    if substrate_top is not None:
        n = np.where(np.asarray(z) < substrate_top, N_SIO2, n)
    m = slabModes(z, n, lambda0, pol, n_modes, EpsHalf=eps_half)
    inside = (z >= core[0]) & (z <= core[1])
    frac = [np.sum(m["field"][inside, q] ** 2) / np.sum(m["field"][:, q] ** 2) for q in range(n_modes)]
    q = int(np.argmax(frac))
    return float(np.real(m["neff"][q])), m["field"][:, q]


def coupler_sim(precision: str = "double", steps: int = 8000, n_lambda: int = 51, period=0.63, ff=0.5, etch=0.07,
                nx: int = 800, nz: int = 300) -> dict:
    """2D TE SOI grating coupler, 800 x 300 at 20 nm with 20-cell CPML.  The
    grating starts 1.5 um after the source (the reference's x = 4 um start does
    not fit a 16 um domain); TE0 mode source; up monitor 1 um above the grating."""
    dx = 0.02
    x = np.arange(nx) * dx
    z = np.arange(nz) * dx - 3.0 + dx / 2             # substrate at the bottom, cladding on top
    src_x = 1.0
    boxes = grating_coupler_geometry(period, ff, etch, x_start=src_x + 1.5, n_clad=1.444)
    e = epsComponents2D(x, z, N_SIO2, boxes)
    ix = int(round(src_x / dx)) + 1
    neff, prof = core_mode(z, np.sqrt(e["y"][ix - 1, :]), 1.55)
    S = 0.99 / math.sqrt(2) * dx
    kup = int(np.argmin(np.abs(z - (0.22 + 1.0)))) + 1
    kdn = int(np.argmin(np.abs(z - (-1.0)))) + 1
    sim = dict(pol="TE", x=x, z=z, eps=e["y"], npml=[20, 20], lambdas=np.linspace(1.5, 1.6, n_lambda),
               monitors=[ix - 25, ix + 10, nx - 30], monitorsZ=[kup, kdn], maxTime=steps * S, shutoff=0.0,
               precision=precision)
    sim["source"] = dict(ix=ix, profile=prof, neff=neff, lambda0=1.55, bw=BW_100NM)
    return sim


def coupler_batch_sims(n: int = 256, seed: int = 4, steps: int = 10000, precision: str = "single", n_lambda: int = 51):
    """n uneven grating couplers: period U[0.56, 0.70], fill U[0.3, 0.7], etch
    U[0.05, 0.12] um, domain width U[12, 24] um (600-1200 cells), height
    250-350 cells, dx = 20 nm."""
    rng = np.random.default_rng(seed)
    sims = []
    for _ in range(n):
        width = rng.uniform(12, 24)
        nx = int(round(width / 0.02))
        nz = int(rng.integers(250, 351))
        period, ff, etch = rng.uniform(0.56, 0.70), rng.uniform(0.3, 0.7), rng.uniform(0.05, 0.12)
        n_per = max(4, int((width - 4.0) / period))
        dx = 0.02
        x = np.arange(nx) * dx
        z = np.arange(nz) * dx - 0.4 * nz * dx + dx / 2
        boxes = grating_coupler_geometry(period, ff, etch, n_per=n_per, x_start=2.5, n_clad=1.444,
                                         box=min(2.0, 0.35 * nz * dx))
        e = epsComponents2D(x, z, N_SIO2, boxes)
        ix = 51
        neff, prof = core_mode(z, np.sqrt(e["y"][ix - 1, :]), 1.55)
        S = 0.99 / math.sqrt(2) * dx
        kup = int(np.argmin(np.abs(z - 1.22))) + 1
        sim = dict(pol="TE", x=x, z=z, eps=e["y"], npml=[20, 20], lambdas=np.linspace(1.5, 1.6, n_lambda),
                   monitors=[ix - 25, ix + 10, nx - 30], monitorsZ=[kup], maxTime=steps * S, shutoff=0.0,
                   precision=precision)
        sim["source"] = dict(ix=ix, profile=prof, neff=neff, lambda0=1.55, bw=BW_100NM)
        sims.append(sim)
    return sims


def pillar_lattice_sim(nx: int = 600, ny: int = 600, nz: int = 300, d: float = 0.02, seed: int = 3,
                       steps: int = 6000, precision: str = "single", n_lambda: int = 1, npml_z: int = 20,
                       device=None):
    """3D periodic TiO2 pillar array (n = 2.4, 600 nm tall, lattice 400 nm,
    radius U[60, 180] nm) on SiO2 (n = 1.46), periodic x/y, CPML in z, 532 nm
    x-polarised plane wave toward +z, 3 planar DFT monitors."""
    x = (np.arange(nx) + 0.5) * d
    y = (np.arange(ny) + 0.5) * d
    z = np.arange(nz) * d
    rng = np.random.default_rng(seed)
    P = 0.4
    npx, npy = int(round(nx * d / P)), int(round(ny * d / P))
    R = rng.uniform(0.06, 0.18, (npx, npy))
    zsub = 0.3 * nz * d
    shapes = [["box", [-np.inf, np.inf, -np.inf, np.inf, -np.inf, zsub, 1.46]],
              ["lattice", dict(x0=P / 2, y0=P / 2, period=P, R=R, z1=zsub, z2=zsub + 0.6, n=N_TIO2)]]
    e = epsComponents3D(x, y, z, 1.0, shapes, device=device)   # device: the GPU generator, same bits
    iz_src = int(zsub / d) - 15
    S = 0.99 / math.sqrt(3) * d
    src = dict(axis=3, index=iz_src, Ea=1.0, Eb=0.0, Ha=0.0, Hb=1.46, neff=1.46, lambda0=0.532, bw=0.1)
    mons = [dict(axis=3, index=iz_src - 10), dict(axis=3, index=int((zsub + 0.6) / d) + 10),
            dict(axis=3, index=nz - npml_z - 5)]
    sim = dict(x=x, y=y, z=z, eps=e, npml=[0, 0, npml_z], periodic=[True, True, False], source=src,
               monitors=mons, lambdas=np.linspace(0.52, 0.545, n_lambda) if n_lambda > 1 else [0.532],
               maxTime=steps * S, shutoff=0.0, precision=precision)
    return sim


def _coupler_instance(nx: int, nz: int, period: float, ff: float, etch: float, steps: int, precision: str,
                      n_lambda: int) -> dict:
    """One uniform SOI grating coupler on an nx x nz grid at 20 nm (the
    coupler_batch_sims layout)."""
    dx = 0.02
    width = nx * dx
    n_per = max(4, int((width - 4.0) / period))
    x = np.arange(nx) * dx
    z = np.arange(nz) * dx - 0.4 * nz * dx + dx / 2
    boxes = grating_coupler_geometry(period, ff, etch, n_per=n_per, x_start=2.5, n_clad=1.444,
                                     box=min(2.0, 0.35 * nz * dx))
    e = epsComponents2D(x, z, N_SIO2, boxes)
    ix = 51
    neff, prof = core_mode(z, np.sqrt(e["y"][ix - 1, :]), 1.55, substrate_top=-min(2.0, 0.35 * nz * dx))
    S = 0.99 / math.sqrt(2) * dx
    kup = int(np.argmin(np.abs(z - 1.22))) + 1
    sim = dict(pol="TE", x=x, z=z, eps=e["y"], npml=[20, 20], lambdas=np.linspace(1.5, 1.6, n_lambda),
               monitors=[ix - 25, ix + 10, nx - 30], monitorsZ=[kup], maxTime=steps * S, shutoff=0.0,
               precision=precision)
    sim["source"] = dict(ix=ix, profile=prof, neff=neff, lambda0=1.55, bw=BW_100NM)
    return sim


def coupler_instance_eta(out: dict, sim: dict, theta_deg=None, x_step: float = 0.5, w0: float = 5.2) -> np.ndarray:
    """Fiber coupling efficiency of one coupler_batch_sims / serve_stream 2D
    coupler from its DFT lines: Pinc = flux after the source + R with
    R = -flux behind it, Pup = up-line flux / Pinc, and eta = overlap of the
    up-line Ey with a tilted Gaussian fiber mode times Pup (the formula of
    fiberCoupling.m:16-31), on a theta (default 5..15 deg) x fiber centre x
    lambda grid.  The mode's phase exp(i k sin(theta) (x - x0)) is evaluated
    as exp(i k sin(theta) x) exp(-i k sin(theta) x0), so each wavelength and
    tilt is one real matrix-vector product over the fiber centres."""
    pinc = out["flux"][1] - out["flux"][0]
    pup = np.atleast_1d(out["fluxZ"][0] / pinc)
    x = np.asarray(sim["x"], dtype=float).ravel()
    lam = np.atleast_1d(np.asarray(sim["lambdas"], dtype=float))
    E = np.asarray(out["PZ"][:, :, 0]).reshape(x.size, -1)
    th = np.deg2rad(np.arange(5.0, 15.01, 1.0) if theta_deg is None else np.asarray(theta_deg, dtype=float))
    x0 = np.arange(3.0, x[-1] - 3.0, x_step)
    eta = np.zeros((th.size, x0.size, lam.size))
    EE = np.real(np.sum(np.conj(E) * E, axis=0))
    u = x[None, :] - x0[:, None]
    for i, t in enumerate(th):
        G = np.exp(-(u * np.cos(t) / w0) ** 2)            # |E_f|, real, (x0, x)
        GG = np.sum(G * G, axis=1)
        for l in range(lam.size):
            ks = 2 * np.pi * N_SIO2 / lam[l] * np.sin(t)
            v = G @ (np.exp(-1j * ks * x) * E[:, l])     # sum_x conj(E_f) E, up to the x0 phase
            eta[i, :, l] = np.abs(v) ** 2 / (EE[l] * GG) * pup[l]
    return eta


def serve_stream(n_jobs: int = 32, seed: int = 5, rate: float = 1.0, cells=(2e5, 5e7), steps=(2000, 20000),
                 frac3d: float = 0.2, precision: str = "single", n_lambda: int = 21, device=None) -> list[dict]:
    """A served stream: Poisson arrivals (rate jobs/s) of mixed jobs, frac3d
    of them 3D pillar lattices and the rest 2D grating couplers, cell counts
    log-uniform in [cells], step budgets uniform in [steps] (shutoff off, so
    every job runs its budget).  Returns [{"t", "dims", "cells", "steps",
    "sim"}] in arrival order.  device: as in pillar_lattice_sim (the 3D
    permittivity from the GPU generator, the same values as the host's)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for _ in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        is3d = rng.random() < frac3d
        nc = math.exp(rng.uniform(math.log(cells[0]), math.log(cells[1])))
        st = int(rng.integers(steps[0], steps[1] + 1))
        if is3d:
            # nx = ny = 2 nz, lattice-commensurate (20 cells per 400 nm period), nz >= 120
            nz = max(120, int(round((nc / 4) ** (1 / 3))))
            nxy = max(20, int(round(math.sqrt(nc / nz) / 20)) * 20)
            sim = pillar_lattice_sim(nx=nxy, ny=nxy, nz=nz, seed=int(rng.integers(1 << 30)), steps=st,
                                     precision=precision, n_lambda=3, device=device)
            jobs.append(dict(t=t, dims=3, cells=nxy * nxy * nz, steps=st, sim=sim))
        else:
            nz = max(150, int(round(math.sqrt(nc / 3))))
            nx = max(400, int(round(nc / nz)))
            period, ff, etch = rng.uniform(0.56, 0.70), rng.uniform(0.3, 0.7), rng.uniform(0.05, 0.12)
            sim = _coupler_instance(nx, nz, period, ff, etch, st, precision, n_lambda)
            jobs.append(dict(t=t, dims=2, cells=nx * nz, steps=st, sim=sim))
    return jobs


def fdfd_straight_guide(d: float = 0.02, lam: float = 1.55):
    """The FDFD straight-guide problem of tests/TestInverseDesign.m:12-24: an
    SOI slab (Si substrate below z = -2, 2 um BOX n = 1.444, 220 nm Si
    n = 3.476, air above) on x in [0, 10], z in [-2.6, 1.8] um (cell
    centres), fed at x = 2 um by its TE0 mode, solved over the window
    -1.5 < z < z_end - 30 d.  Returns (x, z, epsr, lam, J, mode, win)."""
    from .geometry import epsFromBoxes
    x = np.round(np.arange(0, 10 + d / 2, d), 12)
    z = np.arange(-2.6, 1.8 + d / 2, d) + d / 2
    epsr = epsFromBoxes(x, z, 1.0, np.array([[-np.inf, np.inf, -np.inf, -2, 3.476],
                                             [-np.inf, np.inf, -2, 0, 1.444],
                                             [-np.inf, np.inf, 0, 0.22, 3.476]]))
    win = (z > -1.5) & (z < z[-1] - 30 * d)
    i0 = int(round(2 / d))
    m = slabModes(z[win], np.sqrt(epsr[i0, win]), lam, "TE")
    J = np.zeros((x.size, z.size))
    J[i0, win] = np.real(m["field"][:, 0])
    return x, z, epsr, lam, J, m, win
