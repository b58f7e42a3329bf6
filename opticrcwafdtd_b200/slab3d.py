"""One 3D run (orf.fdtd3D, fdtd3D.m:1-29) split into z slabs.

A grid too large for one GPU is cut along z into contiguous slabs, one per
GPU (one process per GPU under torch.distributed, NCCL point-to-point over
NVLink), or several on one GPU (a single process, device copies).  Each slab
is a device-resident 3D job over its own planes plus one ghost plane at
every end that borders another slab (orf_job3d_create_slab).  The job's CPML
profile in z is the whole grid's at its planes, so an inner end absorbs
nothing and every own cell updates exactly as in the whole grid, provided
the ghost planes hold the neighbours' values at the start of every step.
After each step (orf_job3d_step) the slabs therefore swap, per inner
boundary:

  - the slab below sends Ex, Ey, Ez of its last own plane into the ghost
    plane under the slab above (whose H update of that ghost plane then
    needs no other input from below: H of a plane depends on E of that
    plane and the one above, and on its own previous H);
  - the slab above sends Ex, Ey of its first own plane into the ghost plane
    over the slab below (the H update of the plane under it reads those).

The ghost planes' own updates are wrong (their outer neighbours are not in
the job) and are overwritten by the swap.  DFT monitors normal to z belong to
the slab that owns their plane; x- and y-normal monitor planes are cut along
z and put together from the slabs' own rows, with the flux summed over the
whole plane on the host.  Runs have a fixed step count (shutoff 0): the
energy of one slab says nothing about the run's.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi, _lib
from .fdtd import Context

# fields of a 3D job buffer (orf_job3d_plane)
EX, EY, EZ, HX, HY, HZ = range(6)
SEND_UP = (EX, EY, EZ)     # last own plane -> ghost plane under the slab above
SEND_DOWN = (EX, EY)       # first own plane -> ghost plane over the slab below


@dataclass(frozen=True)
class Slab:
    """Planes of one slab in global z indices: own planes [z0, z1), job
    planes [lo, hi) (own planes plus the ghost planes at inner ends)."""
    rank: int
    z0: int
    z1: int
    lo: int
    hi: int

    @property
    def n(self) -> int:
        return self.hi - self.lo

    @property
    def has_below(self) -> bool:
        return self.lo < self.z0

    @property
    def has_above(self) -> bool:
        return self.hi > self.z1


def split_z(nz: int, nslabs: int, npml: int) -> list[Slab]:
    """Cut nz planes into nslabs contiguous slabs of near-equal size.  An
    inner boundary b (first own plane of the slab above) must keep both
    neighbouring jobs' inner ends clear of the grid's CPML: npml + 1 <= b <=
    nz - npml - 2; and each job needs more than 2 npml + 1 planes."""
    if nslabs < 1:
        raise _abi.OrfError("orf:invalidInput", "nslabs must be at least 1")
    cuts = [round(nz * q / nslabs) for q in range(nslabs + 1)]
    slabs = []
    for r in range(nslabs):
        z0, z1 = cuts[r], cuts[r + 1]
        lo = z0 - 1 if r > 0 else z0
        hi = z1 + 1 if r < nslabs - 1 else z1
        slabs.append(Slab(r, z0, z1, lo, hi))
    for s in slabs[1:]:
        b = s.z0
        if not (npml + 1 <= b <= nz - npml - 2):
            raise _abi.OrfError("orf:invalidInput",
                                f"{nslabs} slabs of {nz} planes: the cut at z = {b} lies in or next to the "
                                f"{npml}-plane CPML")
    for s in slabs:
        if s.n < 2 * npml + 2:
            raise _abi.OrfError("orf:invalidInput",
                                f"{nslabs} slabs of {nz} planes: slab {s.rank} holds {s.n} planes, fewer than "
                                f"the {2 * npml + 2} its CPML layout needs")
    return slabs


def _npml_z(sim) -> int:
    npml = np.atleast_1d(np.asarray(_abi._get(sim, "npml", [0, 0, 0]), dtype=np.int64)).ravel()
    per = np.atleast_1d(np.asarray(_abi._get(sim, "periodic", [False, False, False]), dtype=bool)).ravel()
    nz_pml = int(npml[-1] if npml.size == 3 else npml[0])
    pz = bool(per[-1] if per.size == 3 else per[0])
    if pz:
        raise _abi.OrfError("orf:invalidInput", "z slabs need a non-periodic z axis")
    return nz_pml


def slab_sim(sim, s: Slab) -> dict:
    """The sim of one slab's job: planes [s.lo, s.hi) of sim, its source and
    monitors in the job's 1-based indices (a z-normal source plane outside
    the job becomes a zero source at one of its own planes; a z-normal
    monitor is kept only by the slab owning its plane)."""
    g = _abi._get
    out = dict(sim) if isinstance(sim, dict) else {k: getattr(sim, k) for k in dir(sim) if not k.startswith("_")}
    out.pop("progress", None)
    z = np.asarray(g(sim, "z"), dtype=np.float64).ravel()
    out["z"] = z[s.lo:s.hi]
    eps = g(sim, "eps")
    out["eps"] = {c: np.asfortranarray(np.asarray(g(eps, c), dtype=np.float64)[:, :, s.lo:s.hi]) for c in "xyz"}
    src = dict(g(sim, "source")) if isinstance(g(sim, "source"), dict) else dict(vars(g(sim, "source")))
    ax = int(src["axis"]) - 1
    nx, ny = np.asarray(g(sim, "x")).size, np.asarray(g(sim, "y")).size
    n = (nx, ny, s.n)
    na, nb = n[(ax + 1) % 3], n[(ax + 2) % 3]
    if ax == 2:
        loc = int(src["index"]) - 1 - s.lo
        if not (1 <= loc <= s.n - 1):
            # a plane of its own outside the grid's CPML, with zero profiles
            npml = _npml_z(sim)
            nzg = z.size
            gz = min(max(s.z0, npml), nzg - npml - 1)
            src.update(index=gz - s.lo + 1, Ea=0.0, Eb=0.0, Ha=0.0, Hb=0.0)
        else:
            src["index"] = loc + 1
    else:
        for name in ("Ea", "Eb", "Ha", "Hb"):
            v = src.get(name)
            if v is None:
                continue
            a = np.asarray(v, dtype=np.float64)
            if a.size == 1:
                continue
            full = (n[(ax + 1) % 3], z.size) if ax == 0 else (z.size, n[(ax + 2) % 3])
            a = a.reshape(full, order="F")
            src[name] = a[:, s.lo:s.hi] if ax == 0 else a[s.lo:s.hi, :]
            assert src[name].shape == (na, nb)
    out["source"] = src
    mons = g(sim, "monitors", [])
    if isinstance(mons, dict):
        mons = [mons]
    keep = []
    for mq in mons:
        axm, idx = int(g(mq, "axis")), int(g(mq, "index")) - 1
        if axm == 3:
            if s.z0 <= idx < s.z1:
                keep.append(dict(axis=3, index=idx - s.lo + 1))
        else:
            keep.append(dict(axis=axm, index=idx + 1))
    out["monitors"] = keep
    out["shutoff"] = 0.0
    return out


class _DevPlane:
    """A device plane as an object torch.as_tensor can view without a copy."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SlabJob:
    """The device-resident job of one slab (orf_job3d_create_slab)."""

    def __init__(self, sim, s: Slab, nz: int, ctx: Context):
        self.lib = _lib.load()
        self.slab = s
        self.ctx = ctx
        self.sim = slab_sim(sim, s)
        self.m = _abi.marshal_sim3d(self.sim)
        h = C.c_void_p()
        _lib.check(self.lib.orf_job3d_create_slab(ctx.handle, C.byref(self.m.struct), s.lo, nz, C.byref(h)),
                   "slab job create")
        self.handle = h
        self.steps_enqueued = 0
        self.single = self.m.struct.precision == _abi.ORF_SINGLE

    def plane(self, buffer: int, field: int, k: int):
        """(device address, element count, typestr) of local plane k."""
        p, nb = C.c_void_p(), C.c_size_t()
        _lib.check(self.lib.orf_job3d_plane(self.handle, buffer, field, k, C.byref(p), C.byref(nb)), "plane")
        es = 4 if self.single else 8
        return int(p.value), nb.value // es, "<f4" if self.single else "<f8"

    def step(self, n: int = 1) -> None:
        _lib.check(self.lib.orf_job3d_step(self.handle, int(n)), "step")
        self.steps_enqueued += int(n)

    def fields(self) -> list[np.ndarray]:
        nx, ny, nzl = self.m.meta["n"]
        arrs = [np.zeros((nx, ny, nzl), order="F") for _ in range(6)]
        ptrs = (C.POINTER(C.c_double) * 6)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        _lib.check(self.lib.orf_job_get_fields(self.handle, ptrs, 6), "get_fields")
        return arrs

    def finish(self) -> dict:
        o, bufs = _abi.alloc_out3d(self.m)
        _lib.check(self.lib.orf_job3d_finish(self.handle, C.byref(o)), "finish")
        return _abi.finish_out3d(self.m, o, bufs)

    def close(self) -> None:
        if self.handle:
            self.lib.orf_job_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def halo_views(job: SlabJob, buffer: int) -> dict:
    """torch views of the planes a slab sends and receives in one buffer:
    keys ('send_up' | 'recv_below' | 'send_down' | 'recv_above', field)."""
    import torch

    s = job.slab
    dev = torch.device("cuda", job.ctx.device)
    v = {}

    def view(k, f):
        p, cnt, ts = job.plane(buffer, f, k)
        return torch.as_tensor(_DevPlane(p, cnt, ts), device=dev)

    if s.has_above:
        for f in SEND_UP:
            v[("send_up", f)] = view(s.n - 2, f)
        for f in SEND_DOWN:
            v[("recv_above", f)] = view(s.n - 1, f)
    if s.has_below:
        for f in SEND_DOWN:
            v[("send_down", f)] = view(1, f)
        for f in SEND_UP:
            v[("recv_below", f)] = view(0, f)
    return v


class LocalTransport:
    """Swap between slabs held by one process on one device: device copies
    on the stream the jobs run on (their shared context's)."""

    def exchange(self, views: list[dict]) -> None:
        for r in range(len(views) - 1):
            lo, hi = views[r], views[r + 1]
            for f in SEND_UP:
                hi[("recv_below", f)].copy_(lo[("send_up", f)])
            for f in SEND_DOWN:
                lo[("recv_above", f)].copy_(hi[("send_down", f)])


class DistTransport:
    """Swap between the slabs of the ranks of a torch.distributed group, one
    slab per rank (rank r holds slab r): point-to-point sends and receives
    of whole planes, all of one step in one batch (NCCL groups them, so no
    order of the calls can deadlock).  Works on any backend with
    point-to-point support (NCCL on GPUs, gloo on CPU tensors)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def exchange(self, views: list[dict]) -> None:
        (v,) = views
        d, r = self.dist, self.rank
        peer = (lambda q: d.get_global_rank(self.group, q)) if self.group is not None else (lambda q: q)
        ops = []
        if r + 1 < self.world:
            ops += [d.P2POp(d.isend, v[("send_up", f)], peer(r + 1), self.group) for f in SEND_UP]
            ops += [d.P2POp(d.irecv, v[("recv_above", f)], peer(r + 1), self.group) for f in SEND_DOWN]
        if r > 0:
            ops += [d.P2POp(d.isend, v[("send_down", f)], peer(r - 1), self.group) for f in SEND_DOWN]
            ops += [d.P2POp(d.irecv, v[("recv_below", f)], peer(r - 1), self.group) for f in SEND_UP]
        if ops:
            for w in d.batch_isend_irecv(ops):
                w.wait()


def _flux(mon: dict, d: float) -> np.ndarray:
    """1/2 Re sum(Ea Hb* - Eb Ha*) dA over a monitor plane (fdtd3D.m:26)."""
    s = np.real(mon["Ea"] * np.conj(mon["Hb"]) - mon["Eb"] * np.conj(mon["Ha"]))
    return 0.5 * d * d * s.sum(axis=(0, 1))


def assemble(sim, slabs: list[Slab], outs: list[dict]) -> dict:
    """The whole grid's out struct from the slabs' outs (every slab's, in
    slab order): z-normal monitors from their owner, x- / y-normal planes
    from the own rows of every slab."""
    g = _abi._get
    mons = g(sim, "monitors", [])
    if isinstance(mons, dict):
        mons = [mons]
    x = np.asarray(g(sim, "x"), dtype=np.float64).ravel()
    d = float(x[1] - x[0])
    cursor = [0] * len(slabs)   # next monitor of each slab's out, in sim order
    res_mon, flux = [], []
    for mq in mons:
        axm, idx = int(g(mq, "axis")), int(g(mq, "index")) - 1
        if axm == 3:
            r = next(s.rank for s in slabs if s.z0 <= idx < s.z1)
            m = outs[r]["mon"][cursor[r]]
            res_mon.append(m)
            flux.append(outs[r]["flux"][cursor[r]])
            cursor[r] += 1
        else:
            parts = []
            for s in slabs:
                m = outs[s.rank]["mon"][cursor[s.rank]]
                cursor[s.rank] += 1
                a, b = s.z0 - s.lo, s.z1 - s.lo
                parts.append({k: (m[k][:, a:b, :] if axm == 1 else m[k][a:b, :, :]) for k in ("Ea", "Eb", "Ha", "Hb")})
            ax = 1 if axm == 1 else 0
            m = {k: np.asfortranarray(np.concatenate([p[k] for p in parts], axis=ax)) for k in ("Ea", "Eb", "Ha", "Hb")}
            res_mon.append(m)
            flux.append(_flux(m, d))
    o0 = outs[0]
    nL = o0["lambdas"].size
    fl = np.asfortranarray(np.array(flux).reshape(len(mons), nL)) if mons else np.zeros((0, nL), order="F")
    return {"flux": fl, "mon": res_mon, "converged": False, "steps": o0["steps"], "time": o0["time"],
            "wallTime": max(o["wallTime"] for o in outs), "lambdas": o0["lambdas"].copy()}


def own_fields(job: SlabJob) -> list[np.ndarray]:
    """A slab's fields on its own planes (the ghost planes dropped)."""
    s = job.slab
    a, b = s.z0 - s.lo, s.z1 - s.lo
    return [f[:, :, a:b] for f in job.fields()]


def _n_steps(sim) -> int:
    g = _abi._get
    x = np.asarray(g(sim, "x"), dtype=np.float64).ravel()
    S = float(g(sim, "courant", 0.99 / math.sqrt(3.0))) * float(x[1] - x[0])
    r = float(g(sim, "maxTime", 1e4)) / S
    return max(0, int(math.ceil(r - 1e-9)))


def _check_shutoff(sim) -> None:
    if float(_abi._get(sim, "shutoff", 1e-10)) != 0.0:
        raise _abi.OrfError("orf:invalidInput",
                            "a run split into z slabs has a fixed step count: set sim.shutoff = 0")


class SlabRun:
    """A 3D run as nslabs z slabs on one GPU (one process): the slab jobs
    share one context and stream, and the swap after every step is device
    copies on that stream.  The own planes update as in a distributed run
    on nslabs GPUs, so this checks that form against the single-grid run on
    one device."""

    def __init__(self, sim, nslabs: int, device: int = 0):
        import torch

        _check_shutoff(sim)
        self.sim = sim
        nz = np.asarray(_abi._get(sim, "z")).size
        self.slabs = split_z(nz, nslabs, _npml_z(sim))
        self.stream = torch.cuda.Stream(device=device)
        self.ctx = Context(device, stream=self.stream.cuda_stream)
        self.jobs = [SlabJob(sim, s, nz, self.ctx) for s in self.slabs]
        self.views = [[halo_views(j, b) for j in self.jobs] for b in (0, 1)]
        self.transport = LocalTransport()
        self.nsteps = _n_steps(sim)

    def run(self) -> None:
        """Enqueue every step of the run and its swaps (no host wait)."""
        import torch

        with torch.cuda.stream(self.stream):
            for q in range(self.nsteps):
                for j in self.jobs:
                    j.step(1)
                self.transport.exchange(self.views[(q + 1) % 2])

    def reset(self) -> None:
        for j in self.jobs:
            _lib.check(j.lib.orf_job_reset(j.handle), "reset")
            j.steps_enqueued = 0

    def finish(self) -> dict:
        self.stream.synchronize()
        return assemble(self.sim, self.slabs, [j.finish() for j in self.jobs])

    def close(self) -> None:
        for j in self.jobs:
            j.close()
        self.jobs = []
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None


def fdtd3D_slabs(sim, nslabs: int, device: int = 0, return_jobs: bool = False):
    """out = fdtd3D_slabs(sim, nslabs): fdtd3D(sim) computed as nslabs z
    slabs on one GPU (SlabRun).  return_jobs: also the slab jobs and their
    context, left open for the caller (fields of the own planes)."""
    r = SlabRun(sim, nslabs, device)
    r.run()
    out = r.finish()
    if return_jobs:
        return out, r.jobs, r.ctx
    r.close()
    return out


def sim_signature(sim) -> str:
    """A digest of everything a slab run's ranks must agree on: the grid,
    its permittivity, the source, monitors, wavelengths and step count."""
    import hashlib

    g = _abi._get
    h = hashlib.sha256()

    def put(v):
        a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
        h.update(str(a.shape).encode())
        h.update(a.tobytes())

    for k in ("x", "y", "z", "lambdas"):
        put(g(sim, k))
    eps = g(sim, "eps")
    for c in "xyz":
        put(g(eps, c))
    src = g(sim, "source")
    for k in ("axis", "index", "Ea", "Eb", "Ha", "Hb", "neff", "lambda0", "bw"):
        v = g(src, k)
        put(0.0 if v is None else np.real(v))
    mons = g(sim, "monitors", [])
    if isinstance(mons, dict):
        mons = [mons]
    put([[int(g(m, "axis")), int(g(m, "index"))] for m in mons] or [[0, 0]])
    put(np.atleast_1d(np.asarray(g(sim, "npml", [0, 0, 0]), dtype=np.float64)))
    put(np.atleast_1d(np.asarray(g(sim, "periodic", [False] * 3), dtype=np.float64)))
    put([_n_steps(sim), float(g(sim, "courant", 0.99 / math.sqrt(3.0))),
         1.0 if str(g(sim, "precision", "double")).lower() == "single" else 0.0])
    return h.hexdigest()


def check_same_sim(sim, group=None) -> None:
    """Every rank of the group must hold the same sim before the slabs are
    cut: one all_gather_object of a digest, on the host, before any device
    work (a mismatch would swap planes of different runs)."""
    import torch.distributed as dist

    sig = sim_signature(sim)
    sigs = [None] * dist.get_world_size(group)
    dist.all_gather_object(sigs, sig, group=group)
    bad = [r for r, v in enumerate(sigs) if v != sigs[0]]
    if bad:
        raise _abi.OrfError("orf:invalidInput",
                            f"the ranks hold different sims (ranks {bad} differ from rank 0): every rank of a z-slab "
                            "run must pass the same sim")


def fdtd3D_distributed(sim, group=None, device: int | None = None, return_job: bool = False):
    """out = fdtd3D_distributed(sim): fdtd3D(sim) on the ranks of a
    torch.distributed group (NCCL), rank r running z slab r on its GPU.
    Every rank returns the whole out struct (the slabs' outs are gathered
    with one all_gather_object after the run)."""
    import torch
    import torch.distributed as dist

    _check_shutoff(sim)
    tr = DistTransport(group)
    check_same_sim(sim, group)
    nz = np.asarray(_abi._get(sim, "z")).size
    slabs = split_z(nz, tr.world, _npml_z(sim))
    s = slabs[tr.rank]
    dev = torch.cuda.current_device() if device is None else device
    stream = torch.cuda.Stream(device=dev)
    ctx = Context(dev, stream=stream.cuda_stream)
    job = SlabJob(sim, s, nz, ctx)
    views = [halo_views(job, b) for b in (0, 1)]
    nsteps = _n_steps(sim)
    with torch.cuda.stream(stream):
        for q in range(nsteps):
            job.step(1)
            tr.exchange([views[(q + 1) % 2]])
    stream.synchronize()
    mine = job.finish()
    outs = [None] * tr.world
    dist.all_gather_object(outs, mine, group=group)
    out = assemble(sim, slabs, outs)
    if return_job:
        return out, job, ctx
    job.close()
    ctx.close()
    return out
