"""orf.fdtd2D / orf.fdtd2DTE / orf.fdtd3D on the B200 engine.

Host-side mirror of the reference's MATLAB interface (toolbox/+orf/fdtd2D.m,
fdtd2DTE.m:33-34, fdtd3D.m): the same sim fields with the same defaults and
1-based indices, the same out fields (flux, DFT lines, TE/TM aliases,
converged, steps, time, wallTime), the same progress/cancel behaviour (an
exception raised in sim['progress'] stops the run and propagates unchanged,
tests/TestGUISupport.m:39-43) and the same fdtd2D:notConverged warning.
Everything numeric runs in liborf_fdtd.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np

from . import _abi, _lib


class Context:
    """An orf_ctx: one device, one CUDA stream, tuning knobs and kernel timing."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self._lib.orf_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h)),
                   "orf_ctx_create")
        self.handle = h
        self.device = device

    def set_tuning(self, tsteps: int = 0, variant: int = 0, use_graph: bool = True) -> None:
        t = _abi.OrfTuning(tsteps, variant, 1 if use_graph else 0, 0)
        _lib.check(self._lib.orf_ctx_set_tuning(self.handle, C.byref(t)), "orf_ctx_set_tuning")

    def autotune2d(self, sims, steps: int = 0) -> dict:
        """Time every 2D kernel variant and fused step depth on one sim (or a
        batch of sims, run batched) and keep the fastest in this context
        (orf_autotune2d); returns the choice."""
        sims = sims if isinstance(sims, (list, tuple)) else [sims]
        ms = [_abi.marshal_sim2d(s) for s in sims]
        arr = (_abi.OrfSim2D * len(ms))(*[m.struct for m in ms])
        t = _abi.OrfTuning()
        _lib.check(self._lib.orf_autotune2d(self.handle, len(ms), arr, int(steps), C.byref(t)), "autotune2d")
        return {"tsteps": t.tsteps, "variant": t.variant, "use_graph": bool(t.use_graph)}

    def set_wait_injection(self, stall_plane: int = -1, wait_ns: int = 0) -> None:
        """Bounds of the 3D kernel's device-side plane waits (wait_ns per
        wait; 0 = one second) and the failure-detection test hook: with
        stall_plane >= 0, 3D jobs created afterwards on this context never
        load that z-plane of their tiles, so the wait runs out and the run
        ends with orf:deviceTimeout (orf_ctx_set_wait_injection)."""
        _lib.check(self._lib.orf_ctx_set_wait_injection(self.handle, int(stall_plane), int(wait_ns)),
                   "orf_ctx_set_wait_injection")

    def set_timing(self, on: bool) -> None:
        _lib.check(self._lib.orf_ctx_set_timing(self.handle, 1 if on else 0))

    def stats(self) -> dict:
        s = _abi.OrfKernelStats()
        _lib.check(self._lib.orf_ctx_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def reset_stats(self) -> None:
        _lib.check(self._lib.orf_ctx_reset_stats(self.handle))

    def close(self) -> None:
        if self.handle:
            # releases this reference; jobs and servers keep the context alive
            self._lib.orf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _warn_nc(out: dict, name: str) -> None:
    if not out["converged"]:
        warnings.warn(f"{name}:notConverged: maxTime reached before the field energy fell below the shutoff",
                      _abi.NotConvergedWarning, stacklevel=3)


def fdtd2D(sim, ctx: Context | None = None) -> dict:
    """out = fdtd2D(sim): 2D TE/TM FDTD (fdtd2D.m:1-29) on the GPU."""
    lib = _lib.load()
    m = _abi.marshal_sim2d(sim)
    o, bufs = _abi.alloc_out2d(m)
    cb, box = _abi.make_progress(_abi._get(sim, "progress"))
    fn = cb or _abi.PROGRESS_FN(0)
    if ctx is None:
        st = lib.orf_fdtd2d_run(C.byref(m.struct), C.byref(o), fn, None)
    else:
        st = lib.orf_fdtd2d_run_ctx(ctx.handle, C.byref(m.struct), C.byref(o), fn, None)
    if box and "exc" in box:
        raise box["exc"]
    _lib.check(st, "fdtd2D")
    out = _abi.finish_out2d(m, o, bufs)
    _warn_nc(out, "fdtd2D")
    return out


def fdtd2DTE(sim, ctx: Context | None = None) -> dict:
    """fdtd2D with sim.pol = "TE" (fdtd2DTE.m:33-34)."""
    sim = dict(sim) if isinstance(sim, dict) else dict(vars(sim))
    sim["pol"] = "TE"
    return fdtd2D(sim, ctx)


def fdtd3D(sim, ctx: Context | None = None) -> dict:
    """out = fdtd3D(sim): 3D Yee FDTD (fdtd3D.m:1-29) on the GPU."""
    lib = _lib.load()
    m = _abi.marshal_sim3d(sim)
    o, bufs = _abi.alloc_out3d(m)
    cb, box = _abi.make_progress(_abi._get(sim, "progress"))
    fn = cb or _abi.PROGRESS_FN(0)
    if ctx is None:
        st = lib.orf_fdtd3d_run(C.byref(m.struct), C.byref(o), fn, None)
    else:
        st = lib.orf_fdtd3d_run_ctx(ctx.handle, C.byref(m.struct), C.byref(o), fn, None)
    if box and "exc" in box:
        raise box["exc"]
    _lib.check(st, "fdtd3D")
    out = _abi.finish_out3d(m, o, bufs)
    _warn_nc(out, "fdtd3D")
    return out


def plan2d(sim, tsteps: int = 0, variant: int = 0) -> dict:
    """The tiles a 2D run of sim would use (orf_plan2d; host only, no
    device): {"tsteps", "variant", "n_interior", "n_frame", "tiles"}, tiles
    as a dict of int arrays (kind, li0, lk0, lx, lz, oi0, ok0, ow, oh, flags),
    interior tiles first, indices 0-based."""
    lib = _lib.load()
    m = _abi.marshal_sim2d(sim)
    t = _abi.OrfTuning(int(tsteps), int(variant), 1, 0)
    ni, nf, T, v = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
    _lib.check(lib.orf_plan2d(C.byref(m.struct), C.byref(t), None, 0, C.byref(ni), C.byref(nf), C.byref(T),
                              C.byref(v)), "orf_plan2d")
    n = ni.value + nf.value
    arr = (_abi.OrfTile2D * max(1, n))()
    _lib.check(lib.orf_plan2d(C.byref(m.struct), C.byref(t), arr, n, C.byref(ni), C.byref(nf), C.byref(T),
                              C.byref(v)), "orf_plan2d")
    tiles = {k: np.array([getattr(arr[q], k) for q in range(n)], dtype=np.int64) for k, _ in _abi.OrfTile2D._fields_}
    return {"tsteps": T.value, "variant": v.value, "n_interior": ni.value, "n_frame": nf.value, "tiles": tiles}


def plan3d(sim) -> dict:
    """The tiles a 3D run of sim would use (orf_plan3d; host only):
    {"n_interior", "n_cpml", "tiles"}, tiles as a dict of int arrays (kind,
    i0, j0, tw, th, k0, k1, tma, tma_x, tma_index_x), interior tiles first."""
    lib = _lib.load()
    m = _abi.marshal_sim3d(sim)
    ni, nc = C.c_int32(), C.c_int32()
    _lib.check(lib.orf_plan3d(C.byref(m.struct), None, 0, C.byref(ni), C.byref(nc)), "orf_plan3d")
    n = ni.value + nc.value
    arr = (_abi.OrfTile3D * max(1, n))()
    _lib.check(lib.orf_plan3d(C.byref(m.struct), arr, n, C.byref(ni), C.byref(nc)), "orf_plan3d")
    tiles = {k: np.array([getattr(arr[q], k) for q in range(n)], dtype=np.int64) for k, _ in _abi.OrfTile3D._fields_}
    return {"n_interior": ni.value, "n_cpml": nc.value, "tiles": tiles}


def fdtd2D_batch(sims, ctx: Context | None = None, progress=None, autotune: bool = False) -> list[dict]:
    """Run many 2D sims (same precision; TE and TM may mix) together: one
    persistent-kernel launch per fused step block advances every instance of
    a kernel configuration (orf_batch2d_run).
    Returns the list of out structs, in order."""
    lib = _lib.load()
    ms = [_abi.marshal_sim2d(s) for s in sims]
    if not ms:
        return []
    arr = (_abi.OrfSim2D * len(ms))(*[m.struct for m in ms])
    outs = _abi.alloc_out2d_many(ms)
    oarr = (_abi.OrfOut2D * len(ms))(*[o for o, _ in outs])
    own = ctx is None
    if own:
        ctx = Context(0)
    if autotune:
        # tune on a sample of up to 32 instances, run batched; every instance
        # then uses that choice
        step = max(1, len(ms) // 32)
        sample = ms[::step][:32]
        sarr = (_abi.OrfSim2D * len(sample))(*[m.struct for m in sample])
        t = _abi.OrfTuning()
        _lib.check(lib.orf_autotune2d(ctx.handle, len(sample), sarr, 1000, C.byref(t)), "autotune2d")
        ctx.tuned = {"tsteps": t.tsteps, "variant": t.variant}   # the choice, for reports
    cb, box = _abi.make_progress(progress)
    st = lib.orf_batch2d_run(ctx.handle, len(ms), arr, oarr, cb or _abi.PROGRESS_FN(0), None)
    if own:
        ctx.close()
    if box and "exc" in box:
        raise box["exc"]
    _lib.check(st, "fdtd2D_batch")
    res = []
    for q, m in enumerate(ms):
        out = _abi.finish_out2d(m, oarr[q], outs[q][1])
        res.append(out)
    return res


class Job:
    """Device-resident run: fields and DFT sums stay on the GPU between
    advance() calls (orf_job_* in include/orf_fdtd.h)."""

    def __init__(self, sim, ctx: Context, dims: int = 2):
        self.lib = _lib.load()
        self.ctx = ctx
        self.dims = dims
        self.m = _abi.marshal_sim2d(sim) if dims == 2 else _abi.marshal_sim3d(sim)
        h = C.c_void_p()
        fn = self.lib.orf_job2d_create if dims == 2 else self.lib.orf_job3d_create
        _lib.check(fn(ctx.handle, C.byref(self.m.struct), C.byref(h)), "job create")
        self.handle = h

    def advance(self, nsteps: int) -> None:
        _lib.check(self.lib.orf_job_advance(self.handle, int(nsteps)), "advance")

    def sync(self) -> None:
        _lib.check(self.lib.orf_job_sync(self.handle), "sync")

    def reset(self) -> None:
        _lib.check(self.lib.orf_job_reset(self.handle), "reset")

    @property
    def steps(self) -> int:
        return int(self.lib.orf_job_steps_done(self.handle))

    @property
    def cells(self) -> int:
        return int(self.lib.orf_job_cells(self.handle))

    def fields(self) -> list[np.ndarray]:
        """Current fields in the reference layout: 2D [P, A, B]; 3D [Ex Ey Ez Hx Hy Hz]."""
        if self.dims == 2:
            nx, nz = self.m.meta["nx"], self.m.meta["nz"]
            per = bool(self.m.struct.periodic_z)
            shapes = [(nx, nz), (nx, nz if per else nz - 1), (nx - 1, nz)]
        else:
            shapes = [tuple(self.m.meta["n"])] * 6
        arrs = [np.zeros(s, order="F") for s in shapes]
        ptrs = (C.POINTER(C.c_double) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        _lib.check(self.lib.orf_job_get_fields(self.handle, ptrs, len(arrs)), "get_fields")
        return arrs

    def checkpoint(self) -> bytes:
        """The run's state between chunks (fields, CPML psi, DFT sums, step
        counters) as bytes (orf_job_checkpoint)."""
        n = C.c_size_t(0)
        _lib.check(self.lib.orf_job_checkpoint_size(self.handle, C.byref(n)), "checkpoint")
        buf = C.create_string_buffer(n.value)
        _lib.check(self.lib.orf_job_checkpoint(self.handle, buf, n.value), "checkpoint")
        return buf.raw

    def restore(self, state: bytes) -> None:
        """Load a checkpoint of a run of the same sim (maxTime may differ);
        advancing then continues that run exactly (orf_job_restore)."""
        buf = C.create_string_buffer(bytes(state), len(state))
        _lib.check(self.lib.orf_job_restore(self.handle, buf, len(state)), "restore")

    def finish(self) -> dict:
        if self.dims == 2:
            o, bufs = _abi.alloc_out2d(self.m)
            _lib.check(self.lib.orf_job2d_finish(self.handle, C.byref(o)), "finish")
            return _abi.finish_out2d(self.m, o, bufs)
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


class Server:
    """Continuous-batching server (orf_serve_* in include/orf_fdtd.h).

    submit() copies a 2D or 3D sim into the queue and returns a ticket; each
    step() admits queued jobs while their device memory fits the budget,
    advances every resident job by up to macro_steps time steps (jobs of one
    kernel configuration share launches) and retires finished jobs.  result()
    returns the out struct of a finished ticket, info() its timing record
    (submit/admit/done on the server clock, seconds)."""

    def __init__(self, ctx: Context | None = None, max_device_bytes: int = 0, max_jobs: int = 0,
                 macro_steps: int = 0):
        self.lib = _lib.load()
        self.ctx = ctx or Context(0)
        cfg = _abi.OrfServeCfg(int(max_device_bytes), int(max_jobs), int(macro_steps))
        h = C.c_void_p()
        _lib.check(self.lib.orf_serve_open(self.ctx.handle, C.byref(cfg), C.byref(h)), "orf_serve_open")
        self.handle = h
        self._jobs: dict[int, tuple] = {}

    def submit(self, sim, dims: int = 2) -> int:
        t = C.c_int64()
        if dims == 2:
            m = _abi.marshal_sim2d(sim)
            o, bufs = _abi.alloc_out2d(m)
            _lib.check(self.lib.orf_serve_submit2d(self.handle, C.byref(m.struct), C.byref(o), C.byref(t)),
                       "serve submit")
        else:
            m = _abi.marshal_sim3d(sim)
            o, bufs = _abi.alloc_out3d(m)
            _lib.check(self.lib.orf_serve_submit3d(self.handle, C.byref(m.struct), C.byref(o), C.byref(t)),
                       "serve submit")
        # the out struct and its buffers must outlive the job
        self._jobs[int(t.value)] = (dims, m, o, bufs)
        return int(t.value)

    def step(self) -> None:
        _lib.check(self.lib.orf_serve_step(self.handle), "serve step")

    def pending(self) -> tuple[int, int]:
        q, r = C.c_int32(), C.c_int32()
        _lib.check(self.lib.orf_serve_pending(self.handle, C.byref(q), C.byref(r)))
        return int(q.value), int(r.value)

    def clock(self) -> float:
        return float(self.lib.orf_serve_clock(self.handle))

    def preempt(self, ticket: int) -> None:
        """Move a resident job's state to host memory and queue it again at
        the end; it continues where it stopped (orf_serve_preempt)."""
        _lib.check(self.lib.orf_serve_preempt(self.handle, int(ticket)), "serve preempt")

    def info(self, ticket: int) -> dict | None:
        """Timing record of a finished ticket, None while it is queued or resident."""
        i = _abi.OrfServeJobInfo()
        st = self.lib.orf_serve_poll(self.handle, int(ticket), C.byref(i))
        if st == _abi.ORF_EBUSY:
            return None
        _lib.check(st, "serve poll")
        return {k: getattr(i, k) for k, _ in i._fields_}

    def result(self, ticket: int) -> dict:
        """out struct of a finished ticket (raises the job's error if it failed)."""
        inf = self.info(ticket)
        if inf is None:
            raise _abi.OrfError("orf:busy", f"ticket {ticket} has not finished", _abi.ORF_EBUSY)
        dims, m, o, bufs = self._jobs[int(ticket)]
        st = int(inf["status"])
        if st != 0:
            raise _abi.OrfError(_abi.STATUS_IDS.get(st, "orf:error"),
                                f"served job {ticket} failed with {_abi.STATUS_NAMES.get(st, st)}", st)
        return _abi.finish_out2d(m, o, bufs) if dims == 2 else _abi.finish_out3d(m, o, bufs)

    def drain(self, max_rounds: int = 10**7) -> None:
        """step() until nothing is queued or resident."""
        for _ in range(max_rounds):
            q, r = self.pending()
            if q == 0 and r == 0:
                return
            self.step()
        raise RuntimeError("serve drain did not finish")

    def close(self) -> None:
        if self.handle:
            self.lib.orf_serve_close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count() -> int:
    return int(_lib.load().orf_device_count())
