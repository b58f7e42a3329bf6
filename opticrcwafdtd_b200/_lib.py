"""Loader of liborf_fdtd.so, the CUDA engine behind include/orf_fdtd.h.

The library is built in-tree (python -m opticrcwafdtd_b200.build).  There is
no fallback: if it is missing or cannot load, every call raises
OrfError('orf:libraryMissing').
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
# ORF_FDTD_LIB selects another build of the library (the checked build
# lib/liborf_fdtd_check.so, for instance)
LIB_PATH = os.environ.get("ORF_FDTD_LIB") or os.path.join(_HERE, "lib", "liborf_fdtd.so")
_lib = None

P = C.POINTER
_SIGS = {
    "orf_abi_version": (C.c_int32, []),
    "orf_status_string": (C.c_char_p, [C.c_int32]),
    "orf_last_error": (C.c_int32, [C.c_char_p, C.c_size_t]),
    "orf_device_count": (C.c_int32, []),
    "orf_ctx_create": (C.c_int32, [C.c_int32, C.c_void_p, P(C.c_void_p)]),
    "orf_ctx_destroy": (C.c_int32, [C.c_void_p]),
    "orf_ctx_set_tuning": (C.c_int32, [C.c_void_p, P(_abi.OrfTuning)]),
    "orf_ctx_set_timing": (C.c_int32, [C.c_void_p, C.c_int32]),
    "orf_ctx_get_stats": (C.c_int32, [C.c_void_p, P(_abi.OrfKernelStats)]),
    "orf_ctx_set_wait_injection": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64]),
    "orf_ctx_reset_stats": (C.c_int32, [C.c_void_p]),
    "orf_out2d_sizes": (C.c_int32, [P(_abi.OrfSim2D), P(C.c_int64), P(C.c_int64), P(C.c_int64), P(C.c_int64)]),
    "orf_fdtd2d_run": (C.c_int32, [P(_abi.OrfSim2D), P(_abi.OrfOut2D), _abi.PROGRESS_FN, C.c_void_p]),
    "orf_fdtd2d_run_ctx": (C.c_int32, [C.c_void_p, P(_abi.OrfSim2D), P(_abi.OrfOut2D), _abi.PROGRESS_FN, C.c_void_p]),
    "orf_fdtd2d_run_noalloc": (C.c_int32, [P(_abi.OrfSim2D), P(_abi.OrfOut2D), C.c_void_p]),
    "orf_job2d_create": (C.c_int32, [C.c_void_p, P(_abi.OrfSim2D), P(C.c_void_p)]),
    "orf_job3d_create": (C.c_int32, [C.c_void_p, P(_abi.OrfSim3D), P(C.c_void_p)]),
    "orf_job3d_create_slab": (C.c_int32, [C.c_void_p, P(_abi.OrfSim3D), C.c_int32, C.c_int32, P(C.c_void_p)]),
    "orf_job3d_step": (C.c_int32, [C.c_void_p, C.c_int64]),
    "orf_job3d_plane": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, P(C.c_void_p),
                                    P(C.c_size_t)]),
    "orf_job_advance": (C.c_int32, [C.c_void_p, C.c_int64]),
    "orf_job_sync": (C.c_int32, [C.c_void_p]),
    "orf_job_reset": (C.c_int32, [C.c_void_p]),
    "orf_job_steps_done": (C.c_int64, [C.c_void_p]),
    "orf_job_cells": (C.c_int64, [C.c_void_p]),
    "orf_job2d_finish": (C.c_int32, [C.c_void_p, P(_abi.OrfOut2D)]),
    "orf_job3d_finish": (C.c_int32, [C.c_void_p, P(_abi.OrfOut3D)]),
    "orf_job_get_fields": (C.c_int32, [C.c_void_p, P(C.POINTER(C.c_double)), C.c_int32]),
    "orf_job_destroy": (C.c_int32, [C.c_void_p]),
    "orf_job_checkpoint_size": (C.c_int32, [C.c_void_p, P(C.c_size_t)]),
    "orf_job_checkpoint": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "orf_job_restore": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "orf_out3d_sizes": (C.c_int32, [P(_abi.OrfSim3D), P(C.c_int32), P(C.c_int32)]),
    "orf_fdtd3d_run": (C.c_int32, [P(_abi.OrfSim3D), P(_abi.OrfOut3D), _abi.PROGRESS_FN, C.c_void_p]),
    "orf_fdtd3d_run_ctx": (C.c_int32, [C.c_void_p, P(_abi.OrfSim3D), P(_abi.OrfOut3D), _abi.PROGRESS_FN, C.c_void_p]),
    "orf_batch2d_run": (C.c_int32, [C.c_void_p, C.c_int32, P(_abi.OrfSim2D), P(_abi.OrfOut2D), _abi.PROGRESS_FN,
                                    C.c_void_p]),
    "orf_autotune2d": (C.c_int32, [C.c_void_p, C.c_int32, P(_abi.OrfSim2D), C.c_int32, P(_abi.OrfTuning)]),
    "orf_plan2d": (C.c_int32, [P(_abi.OrfSim2D), P(_abi.OrfTuning), P(_abi.OrfTile2D), C.c_int32, P(C.c_int32),
                               P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
    "orf_plan3d": (C.c_int32, [P(_abi.OrfSim3D), P(_abi.OrfTile3D), C.c_int32, P(C.c_int32), P(C.c_int32)]),
    "orf_serve_open": (C.c_int32, [C.c_void_p, P(_abi.OrfServeCfg), P(C.c_void_p)]),
    "orf_serve_submit2d": (C.c_int32, [C.c_void_p, P(_abi.OrfSim2D), P(_abi.OrfOut2D), P(C.c_int64)]),
    "orf_serve_submit3d": (C.c_int32, [C.c_void_p, P(_abi.OrfSim3D), P(_abi.OrfOut3D), P(C.c_int64)]),
    "orf_serve_step": (C.c_int32, [C.c_void_p]),
    "orf_serve_poll": (C.c_int32, [C.c_void_p, C.c_int64, P(_abi.OrfServeJobInfo)]),
    "orf_serve_pending": (C.c_int32, [C.c_void_p, P(C.c_int32), P(C.c_int32)]),
    "orf_serve_preempt": (C.c_int32, [C.c_void_p, C.c_int64]),
    "orf_eps3d": (C.c_int32, [C.c_void_p, P(C.c_double), P(C.c_double), P(C.c_double), C.c_int32, C.c_int32,
                              C.c_int32, C.c_double, C.c_int32, C.c_int32, P(C.c_double), C.c_int32, C.c_void_p,
                              P(C.c_double), P(C.c_double), P(C.c_double)]),
    "orf_serve_clock": (C.c_double, [C.c_void_p]),
    "orf_fdfd2d_factor": (C.c_int32, [C.c_void_p, P(_abi.OrfFdfd2D), P(C.c_void_p)]),
    "orf_fdfd2d_solve": (C.c_int32, [C.c_void_p, P(C.c_double), P(C.c_double), C.c_int32]),
    "orf_fdfd2d_info": (C.c_int32, [C.c_void_p, P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
    "orf_fdfd2d_release": (None, [C.c_void_p]),
    "orf_serve_close": (C.c_int32, [C.c_void_p]),
    "orf_check_violations": (C.c_int32, [P(C.c_uint64), C.c_int32]),
}


def exported_names() -> list[str]:
    return list(_SIGS)


def load():
    """Load the engine library (raises OrfError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise _abi.OrfError("orf:libraryMissing",
                            f"{LIB_PATH} is not built; run python -m opticrcwafdtd_b200.build", 6)
    try:
        lib = C.CDLL(LIB_PATH)
    except OSError as e:
        raise _abi.OrfError("orf:libraryMissing", f"cannot load {LIB_PATH}: {e}", 6) from e
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    load().orf_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    if status != 0:
        ident = _abi.STATUS_IDS.get(status, "orf:error")
        raise _abi.OrfError(ident, f"{what}: {last_error()}" if what else last_error(), status)
