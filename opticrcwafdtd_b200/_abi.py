"""ctypes mirror of include/orf_fdtd.h and marshalling of MATLAB-style sim structs.

The reference takes a MATLAB struct ``sim`` (toolbox/+orf/fdtd2D.m:9-23,
fdtd2DTE.m:7-25, fdtd3D.m:11-24) with 1-based indices and column-major arrays
indexed ``eps(i, k)``.  Here ``sim`` is a dict (or any object with those
attributes); arrays are numpy arrays indexed the same way, ``eps[i, k]`` with
shape ``(numel(x), numel(z))``.  Indices stay 1-based at this level, as in the
reference; marshalling converts them to the 0-based C ABI.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)

ORF_TE, ORF_TM = 0, 1
ORF_DOUBLE, ORF_SINGLE = 0, 1
ORF_EBUSY, ORF_ETOOLARGE = 7, 8

STATUS_NAMES = {
    0: "ORF_OK", 1: "ORF_EINVAL", 2: "ORF_ENOMEM_DEVICE", 3: "ORF_ECANCELLED",
    4: "ORF_ETIMEOUT_DEVICE", 5: "ORF_ECUDA", 6: "ORF_ENODEV", 7: "ORF_EBUSY",
    8: "ORF_ETOOLARGE",
}
# status -> MATLAB-style error identifier (what the MEX gateway raises)
STATUS_IDS = {
    1: "orf:invalidInput", 2: "orf:outOfDeviceMemory", 3: "orf:cancelled",
    4: "orf:deviceTimeout", 5: "orf:cuda", 6: "orf:noDevice", 7: "orf:busy",
    8: "orf:tooLarge",
}

PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_double, C.c_char_p, C.c_void_p)


class OrfSim2D(C.Structure):
    _fields_ = [
        ("pol", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32),
        ("x0", C.c_double), ("z0", C.c_double), ("dx", C.c_double),
        ("eps", c_double_p), ("eps_x", c_double_p), ("eps_z", c_double_p),
        ("npml_x", C.c_int32), ("npml_z", C.c_int32), ("periodic_z", C.c_int32),
        ("src_ix", C.c_int32), ("src_profile", c_double_p),
        ("src_neff", C.c_double), ("src_lambda0", C.c_double), ("src_bw", C.c_double),
        ("n_mon", C.c_int32), ("monitors", c_int32_p),
        ("n_monz", C.c_int32), ("monitors_z", c_int32_p),
        ("n_lambda", C.c_int32), ("lambdas", c_double_p),
        ("max_time", C.c_double), ("shutoff", C.c_double), ("courant", C.c_double),
        ("precision", C.c_int32), ("flags", C.c_int32),
    ]


class OrfOut2D(C.Structure):
    _fields_ = [
        ("flux", c_double_p), ("flux_z", c_double_p),
        ("P", c_double_p), ("B", c_double_p), ("PZ", c_double_p), ("AZ", c_double_p),
        ("converged", C.c_int32), ("_pad", C.c_int32), ("steps", C.c_int64),
        ("time", C.c_double), ("wall_time", C.c_double),
    ]


class OrfSim3D(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("_pad0", C.c_int32),
        ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("d", C.c_double),
        ("eps_x", c_double_p), ("eps_y", c_double_p), ("eps_z", c_double_p),
        ("npml", C.c_int32 * 3), ("periodic", C.c_int32 * 3),
        ("src_axis", C.c_int32), ("src_index", C.c_int32),
        ("src_Ea", c_double_p), ("src_Eb", c_double_p), ("src_Ha", c_double_p), ("src_Hb", c_double_p),
        ("src_neff", C.c_double), ("src_lambda0", C.c_double), ("src_bw", C.c_double),
        ("n_mon", C.c_int32), ("_pad1", C.c_int32),
        ("mon_axis", c_int32_p), ("mon_index", c_int32_p),
        ("n_lambda", C.c_int32), ("_pad2", C.c_int32), ("lambdas", c_double_p),
        ("max_time", C.c_double), ("shutoff", C.c_double), ("courant", C.c_double),
        ("precision", C.c_int32), ("flags", C.c_int32),
    ]


class OrfOut3D(C.Structure):
    _fields_ = [
        ("flux", c_double_p),
        ("mon_Ea", C.POINTER(c_double_p)), ("mon_Eb", C.POINTER(c_double_p)),
        ("mon_Ha", C.POINTER(c_double_p)), ("mon_Hb", C.POINTER(c_double_p)),
        ("converged", C.c_int32), ("_pad", C.c_int32), ("steps", C.c_int64),
        ("time", C.c_double), ("wall_time", C.c_double),
    ]


class OrfTuning(C.Structure):
    _fields_ = [("tsteps", C.c_int32), ("variant", C.c_int32),
                ("use_graph", C.c_int32), ("_pad", C.c_int32)]


class OrfTile2D(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("kind", "li0", "lk0", "lx", "lz", "oi0", "ok0", "ow", "oh", "flags")]


class OrfTile3D(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("kind", "i0", "j0", "tw", "th", "k0", "k1", "tma", "tma_x", "tma_index_x")]


class OrfKernelStats(C.Structure):
    _fields_ = [("interior_ms", C.c_double), ("interior_launches", C.c_int64),
                ("interior_cell_updates", C.c_int64),
                ("frame_ms", C.c_double), ("frame_launches", C.c_int64), ("frame_cell_updates", C.c_int64),
                ("flush_ms", C.c_double), ("flush_launches", C.c_int64),
                ("cell_updates", C.c_int64), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
                ("setup_ms", C.c_double), ("loop_ms", C.c_double), ("finish_ms", C.c_double)]


class OrfEpsShape(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n0", C.c_int32), ("n1", C.c_int32), ("reserved", C.c_int32),
                ("n", C.c_double), ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("p", C.c_double * 8),
                ("data", c_double_p)]


class OrfServeCfg(C.Structure):
    _fields_ = [("max_device_bytes", C.c_int64), ("max_jobs", C.c_int32),
                ("macro_steps", C.c_int32)]


class OrfServeJobInfo(C.Structure):
    _fields_ = [("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("steps", C.c_int64), ("cells", C.c_int64), ("status", C.c_int32),
                ("dims", C.c_int32), ("device_bytes", C.c_int64), ("preemptions", C.c_int32),
                ("reserved", C.c_int32)]


class OrfFdfd2D(C.Structure):
    _fields_ = [("nx", C.c_int32), ("nz", C.c_int32), ("dx", C.c_double), ("eps", c_double_p),
                ("lambda0", C.c_double), ("npml_x", C.c_int32), ("npml_z", C.c_int32),
                ("pml_reflection", C.c_double)]


class OrfError(RuntimeError):
    """Error raised for a non-zero orf_status; ``identifier`` mirrors MATLAB's
    error identifiers (e.g. ``'orf:cancelled'``, tests/TestGUISupport.m:39-43)."""

    def __init__(self, identifier: str, message: str, status: int = 1):
        super().__init__(f"{identifier}: {message}")
        self.identifier = identifier
        self.status = status


class NotConvergedWarning(UserWarning):
    """Issued when a run stops at maxTime (warning id fdtd2D:notConverged /
    fdtd3D:notConverged, fdtd2D.m:28, estimateResources.m:105)."""


def _get(sim: Any, name: str, default: Any = None) -> Any:
    if isinstance(sim, dict):
        return sim.get(name, default)
    return getattr(sim, name, default)


def _ptr(a: np.ndarray | None, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _fortran(a, shape: tuple[int, ...], name: str) -> np.ndarray:
    arr = np.asarray(a, dtype=np.float64)
    if arr.size == 1 and int(np.prod(shape)) == 1:
        arr = arr.reshape(shape)
    if arr.shape != shape:
        # MATLAB would accept a vector for a single-column profile
        if arr.size == int(np.prod(shape)) and arr.ndim == 1:
            arr = arr.reshape(shape, order="F")
        else:
            raise OrfError("orf:invalidInput", f"{name} must be {shape}, got {arr.shape}")
    if np.iscomplexobj(a):
        raise OrfError("orf:invalidInput", f"{name} must be real")
    return np.asfortranarray(arr)


def _grid(v, name: str) -> tuple[int, float, float]:
    v = np.asarray(v, dtype=np.float64).ravel()
    if v.size < 2:
        raise OrfError("orf:invalidInput", f"sim.{name} needs at least two points")
    d = float(v[1] - v[0])
    if not (d > 0) or np.max(np.abs(np.diff(v) - d)) > 1e-9 * max(1.0, abs(d)) * v.size:
        raise OrfError("orf:invalidInput", f"sim.{name} must be uniform and increasing")
    return v.size, float(v[0]), d


@dataclass
class Marshalled:
    struct: Any
    keep: list = field(default_factory=list)
    meta: dict = field(default_factory=dict)


def marshal_sim2d(sim: Any) -> Marshalled:
    """Build an OrfSim2D from a MATLAB-style sim (fdtd2D.m:9-23 defaults)."""
    keep: list = []
    pol = str(_get(sim, "pol", "TE")).upper()
    if pol not in ("TE", "TM"):
        raise OrfError("orf:invalidInput", 'sim.pol must be "TE" or "TM"')
    nx, x0, dx = _grid(_get(sim, "x"), "x")
    nz, z0, dz = _grid(_get(sim, "z"), "z")
    if abs(dz - dx) > 1e-9 * dx:
        raise OrfError("orf:invalidInput", "sim.x and sim.z must share one spacing")
    periodic = bool(_get(sim, "periodicZ", False))
    s = OrfSim2D()
    s.pol = ORF_TE if pol == "TE" else ORF_TM
    s.nx, s.nz, s.x0, s.z0, s.dx = nx, nz, x0, z0, dx
    if pol == "TE":
        eps = _get(sim, "eps")
        if eps is None:
            raise OrfError("orf:invalidInput", "sim.eps is required for TE")
        e = _fortran(eps, (nx, nz), "sim.eps")
        keep.append(e)
        s.eps = _ptr(e)
    else:
        ex, ez = _get(sim, "epsX"), _get(sim, "epsZ")
        if ex is None or ez is None:
            raise OrfError("orf:invalidInput", "sim.epsX and sim.epsZ are required for TM")
        nzA = nz if periodic else nz - 1
        ex = _fortran(ex, (nx, nzA), "sim.epsX")
        ez = _fortran(ez, (nx - 1, nz), "sim.epsZ")
        keep += [ex, ez]
        s.eps_x, s.eps_z = _ptr(ex), _ptr(ez)
    npml = np.atleast_1d(np.asarray(_get(sim, "npml", [0, 0]), dtype=np.int64)).ravel()
    if npml.size == 1:
        npml = np.array([npml[0], npml[0]])
    s.npml_x, s.npml_z = int(npml[0]), int(npml[1])
    s.periodic_z = 1 if periodic else 0
    src = _get(sim, "source")
    if src is None:
        raise OrfError("orf:invalidInput", "sim.source is required")
    s.src_ix = int(_get(src, "ix")) - 1
    prof = _fortran(np.asarray(_get(src, "profile"), dtype=np.float64).ravel(), (nz,), "sim.source.profile")
    keep.append(prof)
    s.src_profile = _ptr(prof)
    s.src_neff = float(np.real(_get(src, "neff", 1.0)))
    s.src_lambda0 = float(_get(src, "lambda0"))
    s.src_bw = float(_get(src, "bw", 0.2))
    mons = np.ascontiguousarray(np.atleast_1d(np.asarray(_get(sim, "monitors", []), dtype=np.int64)).ravel() - 1,
                                dtype=np.int32)
    monz = np.ascontiguousarray(np.atleast_1d(np.asarray(_get(sim, "monitorsZ", []), dtype=np.int64)).ravel() - 1,
                                dtype=np.int32)
    keep += [mons, monz]
    s.n_mon, s.monitors = mons.size, _ptr(mons, C.c_int32)
    s.n_monz, s.monitors_z = monz.size, _ptr(monz, C.c_int32)
    lam = np.ascontiguousarray(np.atleast_1d(np.asarray(_get(sim, "lambdas"), dtype=np.float64)).ravel())
    keep.append(lam)
    s.n_lambda, s.lambdas = lam.size, _ptr(lam)
    s.max_time = float(_get(sim, "maxTime", 1e4))
    s.shutoff = float(_get(sim, "shutoff", 1e-10))
    s.courant = float(_get(sim, "courant", 0.99 / math.sqrt(2.0)))
    prec = str(_get(sim, "precision", "double")).lower()
    if prec not in ("double", "single"):
        raise OrfError("orf:invalidInput", 'sim.precision must be "double" or "single"')
    s.precision = ORF_DOUBLE if prec == "double" else ORF_SINGLE
    s.flags = 0
    return Marshalled(s, keep, {"pol": pol, "nx": nx, "nz": nz, "nL": lam.size,
                                "nM": mons.size, "nMZ": monz.size, "lambdas": lam})


def _out2d_shapes(m: Marshalled) -> dict:
    nx, nz, nL, nM, nMZ = (m.meta[k] for k in ("nx", "nz", "nL", "nM", "nMZ"))
    return {"P": (nz, nL, nM), "B": (nz, nL, nM), "PZ": (nx, nL, nMZ), "AZ": (nx, nL, nMZ)}


def alloc_out2d(m: Marshalled, slab: np.ndarray | None = None) -> tuple[OrfOut2D, dict]:
    """Output buffers of one 2D run.  The DFT lines are written in full by
    the run's results (no zero fill); slab (a flat complex128 array, see
    alloc_out2d_many) holds them when given."""
    nL, nM, nMZ = (m.meta[k] for k in ("nL", "nM", "nMZ"))
    bufs = {"flux": np.zeros((nM, nL), order="F"), "fluxZ": np.zeros((nMZ, nL), order="F")}
    off = 0
    for k, shp in _out2d_shapes(m).items():
        n = int(np.prod(shp))
        if slab is None:
            bufs[k] = np.empty(shp, dtype=np.complex128, order="F")
        else:
            bufs[k] = slab[off:off + n].reshape(shp, order="F")
            off += n
    o = OrfOut2D()
    o.flux = _ptr(bufs["flux"]) if bufs["flux"].size else None
    o.flux_z = _ptr(bufs["fluxZ"]) if bufs["fluxZ"].size else None
    for k in ("P", "B", "PZ", "AZ"):
        setattr(o, k, _ptr(bufs[k]) if bufs[k].size else None)
    return o, bufs


def alloc_out2d_many(ms: list) -> list:
    """Output buffers of a batch: the DFT lines of every instance carved from
    one allocation (a batch of couplers returns most of a gigabyte; its
    pages are first written by the host threads finishing the batch, in
    parallel)."""
    sizes = [sum(int(np.prod(s)) for s in _out2d_shapes(m).values()) for m in ms]
    slab = np.empty(sum(sizes), dtype=np.complex128)
    outs, off = [], 0
    for m, n in zip(ms, sizes):
        outs.append(alloc_out2d(m, slab[off:off + n]))
        off += n
    return outs


def finish_out2d(m: Marshalled, o: OrfOut2D, bufs: dict) -> dict:
    """out struct of fdtd2D.m:25-29 with the TE/TM aliases (physical signs)."""
    out = dict(bufs)
    out["converged"] = bool(o.converged)
    out["steps"] = int(o.steps)
    out["time"] = float(o.time)
    out["wallTime"] = float(o.wall_time)
    out["lambdas"] = m.meta["lambdas"].copy()
    if m.meta["pol"] == "TE":
        out.update(Ey=bufs["P"], Hz=bufs["B"], EyZ=bufs["PZ"], HxZ=bufs["AZ"])
    else:
        out.update(Hy=bufs["P"], Ez=-bufs["B"], HyZ=bufs["PZ"], ExZ=-bufs["AZ"])
    return out


def _axis_sizes(n: tuple[int, int, int], axis: int) -> tuple[int, int]:
    return n[(axis + 1) % 3], n[(axis + 2) % 3]


def marshal_sim3d(sim: Any) -> Marshalled:
    """Build an OrfSim3D from a MATLAB-style sim (fdtd3D.m:11-24)."""
    keep: list = []
    nx, x0, dx = _grid(_get(sim, "x"), "x")
    ny, y0, dy = _grid(_get(sim, "y"), "y")
    nz, z0, dz = _grid(_get(sim, "z"), "z")
    if max(abs(dy - dx), abs(dz - dx)) > 1e-9 * dx:
        raise OrfError("orf:invalidInput", "sim.x, sim.y and sim.z must share one spacing")
    n = (nx, ny, nz)
    s = OrfSim3D()
    s.nx, s.ny, s.nz, s.x0, s.y0, s.z0, s.d = nx, ny, nz, x0, y0, z0, dx
    eps = _get(sim, "eps")
    if eps is None:
        raise OrfError("orf:invalidInput", "sim.eps (struct .x .y .z) is required")
    comps = []
    for c in ("x", "y", "z"):
        e = _fortran(_get(eps, c), n, f"sim.eps.{c}")
        keep.append(e)
        comps.append(_ptr(e))
    s.eps_x, s.eps_y, s.eps_z = comps
    npml = np.atleast_1d(np.asarray(_get(sim, "npml", [0, 0, 0]), dtype=np.int64)).ravel()
    if npml.size == 1:
        npml = np.repeat(npml, 3)
    per = np.atleast_1d(np.asarray(_get(sim, "periodic", [False, False, False]), dtype=bool)).ravel()
    if per.size == 1:
        per = np.repeat(per, 3)
    for q in range(3):
        s.npml[q] = 0 if per[q] else int(npml[q])
        s.periodic[q] = int(per[q])
    src = _get(sim, "source")
    if src is None:
        raise OrfError("orf:invalidInput", "sim.source is required")
    ax = int(_get(src, "axis")) - 1
    if ax not in (0, 1, 2):
        raise OrfError("orf:invalidInput", "sim.source.axis must be 1, 2 or 3")
    s.src_axis = ax
    s.src_index = int(_get(src, "index")) - 1
    na, nb = _axis_sizes(n, ax)
    profs = []
    for name in ("Ea", "Eb", "Ha", "Hb"):
        v = _get(src, name)
        arr = np.zeros((na, nb)) if v is None else np.asarray(v, dtype=np.float64)
        if arr.size == 1:
            arr = np.full((na, nb), float(arr.ravel()[0]))
        arr = _fortran(arr, (na, nb), f"sim.source.{name}")
        keep.append(arr)
        profs.append(_ptr(arr))
    s.src_Ea, s.src_Eb, s.src_Ha, s.src_Hb = profs
    s.src_neff = float(np.real(_get(src, "neff", 1.0)))
    s.src_lambda0 = float(_get(src, "lambda0"))
    s.src_bw = float(_get(src, "bw", 0.2))
    mons = _get(sim, "monitors", [])
    if isinstance(mons, dict):
        mons = [mons]
    axes = np.ascontiguousarray([int(_get(mq, "axis")) - 1 for mq in mons], dtype=np.int32)
    idxs = np.ascontiguousarray([int(_get(mq, "index")) - 1 for mq in mons], dtype=np.int32)
    keep += [axes, idxs]
    s.n_mon = axes.size
    s.mon_axis, s.mon_index = _ptr(axes, C.c_int32), _ptr(idxs, C.c_int32)
    lam = np.ascontiguousarray(np.atleast_1d(np.asarray(_get(sim, "lambdas"), dtype=np.float64)).ravel())
    keep.append(lam)
    s.n_lambda, s.lambdas = lam.size, _ptr(lam)
    s.max_time = float(_get(sim, "maxTime", 1e4))
    s.shutoff = float(_get(sim, "shutoff", 1e-10))
    s.courant = float(_get(sim, "courant", 0.99 / math.sqrt(3.0)))
    prec = str(_get(sim, "precision", "double")).lower()
    if prec not in ("double", "single"):
        raise OrfError("orf:invalidInput", 'sim.precision must be "double" or "single"')
    s.precision = ORF_DOUBLE if prec == "double" else ORF_SINGLE
    s.flags = 0
    planes = [_axis_sizes(n, int(a)) for a in axes]
    return Marshalled(s, keep, {"n": n, "nL": lam.size, "nM": axes.size, "planes": planes,
                                "lambdas": lam})


def alloc_out3d(m: Marshalled) -> tuple[OrfOut3D, dict]:
    nL = m.meta["nL"]
    bufs: dict = {"flux": np.zeros((m.meta["nM"], nL), order="F"), "mon": []}
    ptrs = {k: (c_double_p * max(1, m.meta["nM"]))() for k in ("Ea", "Eb", "Ha", "Hb")}
    for q, (na, nb) in enumerate(m.meta["planes"]):
        mon = {}
        for k in ("Ea", "Eb", "Ha", "Hb"):
            a = np.zeros((na, nb, nL), dtype=np.complex128, order="F")
            mon[k] = a
            ptrs[k][q] = _ptr(a)
        bufs["mon"].append(mon)
    o = OrfOut3D()
    o.flux = _ptr(bufs["flux"]) if bufs["flux"].size else None
    o.mon_Ea, o.mon_Eb, o.mon_Ha, o.mon_Hb = (ptrs[k] for k in ("Ea", "Eb", "Ha", "Hb"))
    bufs["_ptrs"] = ptrs
    return o, bufs


def finish_out3d(m: Marshalled, o: OrfOut3D, bufs: dict) -> dict:
    return {"flux": bufs["flux"], "mon": bufs["mon"], "converged": bool(o.converged),
            "steps": int(o.steps), "time": float(o.time), "wallTime": float(o.wall_time),
            "lambdas": m.meta["lambdas"].copy()}


def make_progress(cb):
    """Wrap a MATLAB-style progress(frac, msg) callback.  An exception raised in
    the callback cancels the run and is re-raised unchanged after the call
    returns (fdtd2D.m:18-20: 'throw an error in it (e.g. orf:cancelled)')."""
    if cb is None:
        return None, None
    box: dict = {}

    def _tramp(frac, msg, _user):
        try:
            cb(float(frac), msg.decode() if msg else "")
            return 0
        except BaseException as e:  # noqa: BLE001 - any error cancels, as in MATLAB
            box["exc"] = e
            return 1

    return PROGRESS_FN(_tramp), box
