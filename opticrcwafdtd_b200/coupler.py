"""orf.gratingCouplerTE, orf.fiberCoupling, orf.bestFiberCoupling and
orf.apodizedGrating on the B200 engine.

gratingCouplerTE (toolbox/+orf/gratingCouplerTE.m:1-27, documented interface;
the implementation is closed) builds the SOI grating cross-section, launches
the TE0 slab mode toward +x with the one-sided TF/SF source, runs one 2D TE
FDTD job on the GPU and reduces the DFT lines of a closed monitor box to the
power budget.  fiberCoupling follows toolbox/+orf/fiberCoupling.m:16-31 (open
code) line for line.  gratingCouplerTE_batch runs many parameter sets as one
orf_batch2d_run submission (the sweeps of examples/cpo_box_scan.m:23-31).

Choices the documentation leaves open, stated here:
  - domain: CPML of 20 cells on every side; x from 0 to the grating end
    (x = 4 + length) plus 2.5 um; z from 1 um below the BOX to 1 um above the
    up monitor (Si substrate below the BOX when p.substrate);
  - source plane at x = 1.5 um; a reflection line at x = 1.0 um (scattered
    field only, left of the one-sided source); the input line at 2.5 um; the
    transmission line 1 um after the grating; up / down lines zUp above the
    Si top and zDown below the Si bottom;
  - the box faces are the segments between those lines; each flux is the
    Riemann sum 1/2 Re sum E_y H^* dx over its segment (fdtd2DTE.m:27-31);
  - Pinc = net flux through the input line + R (the documented definition);
    R, Pup, Pdown, Ptrans are fractions of Pinc, balance = 1 - their sum;
  - TE0 source: the fundamental slab mode of the source column with the Si
    substrate replaced by BOX oxide (a substrate mode is never picked);
  - pulse: centred at lambda0 with relative half-width bw (p.bw, default
    0.2, the fdtd2D source default); shutoff 1e-10 of the peak energy.
"""
from __future__ import annotations

import math
from typing import Any

import numpy as np

from .geometry import epsComponents2D
from .modes import slabModes

DEFAULTS = dict(lambda0=1.55, lambdas=None, dx=0.02, tSi=0.22, etch=0.07, period=0.62, ff=0.5, nPer=20, box=2.0,
                nSi=3.476, nBox=1.444, nClad=1.0, substrate=True, useGPU=True, precision="double", zUp=1.0,
                zDown=1.0, progress=None, sidewall=90.0, layout=None, bw=0.2, npml=20, maxTime=1e4,
                shutoff=1e-10, courant=None)

X_GRATING = 4.0          # the grating starts at x = 4 um (gratingCouplerTE.m:26)
X_REFL, X_SRC, X_IN = 1.0, 1.5, 2.5


def _params(p: Any) -> dict:
    q = dict(DEFAULTS)
    if p is None:
        p = {}
    items = p.items() if isinstance(p, dict) else vars(p).items()
    for k, v in items:
        if k not in q:
            raise ValueError(f"gratingCouplerTE:unknownField: unknown parameter {k!r}")
        q[k] = v
    if q["lambdas"] is None:
        q["lambdas"] = np.linspace(1.5, 1.6, 11)
    q["lambdas"] = np.atleast_1d(np.asarray(q["lambdas"], dtype=float))
    return q


def _grating_boxes(q: dict) -> tuple[list, float]:
    """Boxes [x1 x2 z1 z2 n] painted over the SOI stack, and the grating length."""
    n_per = int(q["nPer"])
    if q["layout"] is not None:
        lay = q["layout"]
        boxes = np.atleast_2d(np.asarray(lay["boxes"] if isinstance(lay, dict) else lay.boxes, dtype=float))
        length = float(lay["length"] if isinstance(lay, dict) else lay.length)
        return [list(b) for b in boxes], length
    period = np.broadcast_to(np.asarray(q["period"], dtype=float), (n_per,))
    ff = np.broadcast_to(np.asarray(q["ff"], dtype=float), (n_per,))
    t_si, etch, n_clad = float(q["tSi"]), float(q["etch"]), float(q["nClad"])
    dx = float(q["dx"])
    theta = math.radians(float(q["sidewall"]))
    boxes = []
    x = X_GRATING
    for k in range(n_per):
        g0, g1 = x + ff[k] * period[k], x + period[k]      # groove at the top surface (the mask)
        if theta >= math.pi / 2 - 1e-12:
            boxes.append([g0, g1, t_si - etch, t_si, n_clad])
        else:
            # walls lean inward with depth: quarter-cell steps in z
            step = dx / 4
            nsteps = max(1, int(math.ceil(etch / step - 1e-9)))
            for s in range(nsteps):
                z1 = t_si - min(etch, (s + 1) * step)
                z2 = t_si - s * step
                depth = 0.5 * (z1 + z2) - t_si                  # negative, at the step centre
                shrink = -depth / math.tan(theta)
                a, b = g0 + shrink, g1 - shrink
                if b > a:
                    boxes.append([a, b, z1, z2, n_clad])
        x += period[k]
    return boxes, x - X_GRATING


def _te0_mode(z, eps_col, q: dict):
    """Fundamental TE slab mode of the source column, substrate replaced by BOX."""
    n = np.sqrt(np.asarray(eps_col, dtype=float))
    if q["substrate"]:
        n = np.where(z < -float(q["box"]), float(q["nBox"]), n)
    m = slabModes(z, n, float(q["lambda0"]), "TE", 1)
    return float(np.real(m["neff"][0])), m["field"][:, 0]


def gratingCouplerTE_sim(p: Any = None) -> tuple[dict, dict]:
    """The fdtd2D sim of gratingCouplerTE(p) and the monitor-box description."""
    q = _params(p)
    dx = float(q["dx"])
    npml = int(q["npml"])
    boxes_g, length = _grating_boxes(q)
    x_end = X_GRATING + length
    x_tr = x_end + 1.0
    nx = int(math.ceil((x_end + 2.5) / dx)) + 1
    t_si, box = float(q["tSi"]), float(q["box"])
    z_up, z_dn = t_si + float(q["zUp"]), -float(q["zDown"])
    z_lo = -box - 1.0
    z_hi = z_up + 1.0
    nz = int(math.ceil((z_hi - z_lo) / dx)) + 1
    x = np.arange(nx) * dx
    z = z_lo + dx / 2 + np.arange(nz) * dx
    stack = []
    if q["substrate"]:
        stack.append([-np.inf, np.inf, -np.inf, -box, float(q["nSi"])])
    stack.append([-np.inf, np.inf, -box if q["substrate"] else -np.inf, 0.0, float(q["nBox"])])
    stack.append([-np.inf, np.inf, 0.0, t_si, float(q["nSi"])])
    e = epsComponents2D(x, z, float(q["nClad"]), stack + boxes_g)
    eps = e["y"]
    col = lambda xx: int(round(xx / dx))             # 0-based P column
    row = lambda zz: int(np.argmin(np.abs(z - zz)))   # 0-based P row
    ix_src = col(X_SRC)
    neff, prof = _te0_mode(z, eps[ix_src, :], q)
    mons = [col(X_REFL), col(X_IN), col(x_tr)]
    monz = [row(z_up), row(z_dn)]
    sim = dict(pol="TE", x=x, z=z, eps=eps, npml=[npml, npml], lambdas=q["lambdas"],
               monitors=[m + 1 for m in mons], monitorsZ=[k + 1 for k in monz], maxTime=float(q["maxTime"]),
               shutoff=float(q["shutoff"]), precision=q["precision"], progress=q["progress"])
    if q["courant"] is not None:
        sim["courant"] = float(q["courant"])
    sim["source"] = dict(ix=ix_src + 1, profile=prof, neff=neff, lambda0=float(q["lambda0"]), bw=float(q["bw"]))
    boxdesc = dict(q=q, dx=dx, x=x, z=z, eps=eps, neff=neff, mons=mons, monz=monz, grating=(X_GRATING, x_end),
                   k_lo=monz[1], k_hi=monz[0], i_lo=mons[1], i_hi=mons[2])
    return sim, boxdesc


def _segment_flux(E, H, lo, hi, d):
    """1/2 Re sum_{k=lo..hi} E H^* d for each wavelength (E, H: n x nL)."""
    return 0.5 * np.real(np.sum(E[lo:hi + 1, :] * np.conj(H[lo:hi + 1, :]), axis=0)) * d


def coupler_budget(out: dict, bd: dict) -> dict:
    """Power budget of the closed monitor box from the DFT lines of one run."""
    q, dx = bd["q"], bd["dx"]
    P, B = out["P"], out["B"]            # x-lines: Ey, Hz     (nz x nL x nMon)
    PZ, AZ = out["PZ"], out["AZ"]        # z-lines: Ey, Hx     (nx x nL x nMonZ)
    k_lo, k_hi, i_lo, i_hi = bd["k_lo"], bd["k_hi"], bd["i_lo"], bd["i_hi"]
    # x-directed flux 1/2 Re Ey Hz^* over z in the box; z-directed -1/2 Re Ey Hx^*
    f_refl = _segment_flux(P[:, :, 0], B[:, :, 0], k_lo, k_hi, dx)
    f_in = _segment_flux(P[:, :, 1], B[:, :, 1], k_lo, k_hi, dx)
    f_tr = _segment_flux(P[:, :, 2], B[:, :, 2], k_lo, k_hi, dx)
    f_up = -_segment_flux(PZ[:, :, 0], AZ[:, :, 0], i_lo, i_hi, dx)
    f_dn = -_segment_flux(PZ[:, :, 1], AZ[:, :, 1], i_lo, i_hi, dx)
    R = -f_refl
    Pinc = f_in + R
    res = dict(Pinc=Pinc, R=R / Pinc, Pup=f_up / Pinc, Pdown=-f_dn / Pinc, Ptrans=f_tr / Pinc)
    res["balance"] = 1.0 - (res["R"] + res["Pup"] + res["Pdown"] + res["Ptrans"])
    res["xUp"] = bd["x"].copy()
    res["EyUp"] = np.array(PZ[:, :, 0])
    res["lambdas"] = np.array(q["lambdas"])
    res["nClad"] = float(q["nClad"])
    res["neffIn"] = bd["neff"]
    res["steps"] = out["steps"]
    res["converged"] = out["converged"]
    res["geometry"] = dict(x=bd["x"], z=bd["z"], eps=bd["eps"])
    res["params"] = q
    res["grating"] = bd["grating"]
    return res


def gratingCouplerTE(p: Any = None, ctx=None) -> dict:
    """res = gratingCouplerTE(p): power budget of a uniform (or apodized)
    SOI grating coupler, one 2D TE FDTD run on the GPU."""
    from .fdtd import fdtd2D
    sim, bd = gratingCouplerTE_sim(p)
    out = fdtd2D(sim, ctx)
    return coupler_budget(out, bd)


def gratingCouplerTE_batch(ps, ctx=None, progress=None) -> list[dict]:
    """gratingCouplerTE for many parameter sets, advanced together by one
    orf_batch2d_run submission (all sets must share the precision).  Under an
    initialised torch.distributed process group (one process per GPU) the
    sets are sharded across ranks by grid size and every rank returns all
    results."""
    from .fdtd import fdtd2D_batch
    from .replicas import sharded_map
    built = [gratingCouplerTE_sim(p) for p in ps]
    sims = []
    for s, _ in built:
        s = dict(s)
        s.pop("progress", None)
        sims.append(s)
    costs = [s["x"].size * s["z"].size for s in sims]
    outs = sharded_map(lambda part: fdtd2D_batch(part, ctx, progress), sims, costs)
    return [coupler_budget(o, bd) for o, (_, bd) in zip(outs, built)]


def fiberCoupling(res: dict, theta, x0, w0: float):
    """[eta, overlap] = fiberCoupling(res, theta, x0, w0) (fiberCoupling.m:16-31).

    Gaussian fiber mode E_f(x) = exp(-((x - x0) cos(theta) / w0)^2)
    exp(i k nc sin(theta) (x - x0)); overlap = |sum E_up E_f^*|^2 /
    (sum |E_up|^2 sum |E_f|^2); eta = overlap * Pup.  Outputs are
    numel(theta) x numel(x0) x nL."""
    if not (w0 > 0):
        raise ValueError("fiberCoupling: w0 must be positive")
    x = np.asarray(res["xUp"], dtype=float).ravel()
    lambdas = np.atleast_1d(np.asarray(res["lambdas"], dtype=float))
    theta = np.atleast_1d(np.asarray(theta, dtype=float)).ravel()
    x0 = np.atleast_1d(np.asarray(x0, dtype=float)).ravel()
    EyUp = np.asarray(res["EyUp"]).reshape(x.size, -1)
    pup = np.atleast_1d(np.asarray(res["Pup"], dtype=float))
    nL = lambdas.size
    eta = np.zeros((theta.size, x0.size, nL))
    overlap = np.zeros_like(eta)
    for l in range(nL):
        E = EyUp[:, l]
        k = 2 * np.pi * float(res["nClad"]) / lambdas[l]
        EE = np.real(np.vdot(E, E))
        for i, th in enumerate(theta):
            for j, xc in enumerate(x0):
                u = x - xc
                Ef = np.exp(-(u * np.cos(th) / w0) ** 2) * np.exp(1j * k * np.sin(th) * u)
                overlap[i, j, l] = abs(np.vdot(Ef, E)) ** 2 / (EE * np.real(np.vdot(Ef, Ef)))
        eta[:, :, l] = overlap[:, :, l] * pup[l]
    return eta, overlap


def bestFiberCoupling(res: dict, thetaDeg=None, w0: float = 5.2) -> dict:
    """b = bestFiberCoupling(res, thetaDeg, w0) (bestFiberCoupling.m:1-8,
    documented interface): scans the fiber tilt over thetaDeg (default
    5:0.5:15) and its centre over the grating in 0.1 um steps, maximising the
    coupling at the design wavelength res.params.lambda0.
      b.eta, b.dB : coupling at lambda0;  b.theta [deg], b.x0 [um]
      b.spectrum  : coupling vs res.lambdas at that fiber position
      b.band1dB   : [min max] sampled wavelengths within 1 dB of the peak
      b.Pup       : upward power fraction at lambda0"""
    theta = np.arange(5.0, 15.0 + 1e-9, 0.5) if thetaDeg is None else np.atleast_1d(np.asarray(thetaDeg, float))
    lam = np.atleast_1d(np.asarray(res["lambdas"], dtype=float))
    lam0 = float(res.get("params", {}).get("lambda0", 1.55)) if isinstance(res.get("params"), dict) else 1.55
    g0, g1 = res.get("grating", (float(np.min(res["xUp"])), float(np.max(res["xUp"]))))
    x0 = np.arange(g0, g1 + 1e-9, 0.1)
    eta, _ = fiberCoupling(res, np.deg2rad(theta), x0, w0)
    il = int(np.argmin(np.abs(lam - lam0)))
    i, j = np.unravel_index(int(np.argmax(eta[:, :, il])), eta[:, :, il].shape)
    best = float(eta[i, j, il])
    spec = eta[i, j, :].copy()
    inband = lam[spec >= best / 10 ** 0.1]
    pup = np.atleast_1d(np.asarray(res["Pup"], dtype=float))
    return dict(eta=best, dB=10 * np.log10(best) if best > 0 else -np.inf, theta=float(theta[i]), x0=float(x0[j]),
                spectrum=spec, band1dB=np.array([inband.min(), inband.max()]) if inband.size else np.array([]),
                Pup=float(pup[il] if pup.size > 1 else pup[0]), lambdas=lam.copy())


def _slab_te0(n_core_top: float, q: dict) -> float:
    """TE0 effective index of the SOI slab whose Si is n_core_top thick (BOX
    below, cladding above), on a 5 nm grid."""
    dz = 0.005
    z = np.arange(-2.0, n_core_top + 2.0, dz) + dz / 2
    n = np.where(z < 0, float(q["nBox"]), np.where(z < n_core_top, float(q["nSi"]), float(q["nClad"])))
    m = slabModes(z, n, float(q["lambda0"]), "TE", 1)
    return float(np.real(m["neff"][0]))


def apodizedGrating(ffStart: float, ffEnd: float, thetaDeg: float, nPer: int, scale: float = 1.0, p: Any = None):
    """[period, ff] = apodizedGrating(ffStart, ffEnd, thetaDeg, nPer, scale, p)
    (apodizedGrating.m:1-9, documented interface): the unetched fraction
    ramps linearly from ffStart to ffEnd over nPer periods, and each period
    meets the local Bragg condition
        period_k = scale * lambda0 / (neff_k - nClad sin(theta)),
        neff_k = ff_k n_full + (1 - ff_k) n_etched,
    with n_full, n_etched the TE0 slab indices of the unetched (tSi) and
    etched (tSi - etch) cross-sections of the gratingCouplerTE stack p."""
    q = _params(p)
    ff = np.linspace(float(ffStart), float(ffEnd), int(nPer))
    n_full = _slab_te0(float(q["tSi"]), q)
    n_etch = _slab_te0(float(q["tSi"]) - float(q["etch"]), q)
    neff = ff * n_full + (1.0 - ff) * n_etch
    period = float(scale) * float(q["lambda0"]) / (neff - float(q["nClad"]) * np.sin(np.deg2rad(float(thetaDeg))))
    return period, ff
