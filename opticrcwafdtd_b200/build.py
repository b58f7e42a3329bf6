"""Build liborf_fdtd.so (the CUDA engine) in-tree for sm_100a.

    python -m opticrcwafdtd_b200.build          # incremental
    python -m opticrcwafdtd_b200.build --check  # the checked build, lib/liborf_fdtd_check.so
    python -m opticrcwafdtd_b200.build --clean

Every translation unit under csrc/ is compiled by nvcc with
-gencode arch=compute_100a,code=sm_100a (objects in csrc/_build/, in
parallel), then linked into opticrcwafdtd_b200/lib/liborf_fdtd.so with the
CUDA runtime linked statically, so the library has no dependency beyond the
driver: a MATLAB MEX gateway or any C program can load it.  The checked
build (check=True) compiles the same sources with -DORF_CHECK into
csrc/_build_check/ and lib/liborf_fdtd_check.so: its 2D step kernels test
every global access against its buffer and count what fails
(orf_check_violations).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "liborf_fdtd.so")
CHECK_LIB = os.path.join(LIBDIR, "liborf_fdtd_check.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int = 0, check: bool = False) -> str:
    obj_dir = OBJ + "_check" if check else OBJ
    lib = CHECK_LIB if check else LIB
    flags = NVCC_FLAGS + (["-DORF_CHECK"] if check else [])
    os.makedirs(obj_dir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = _headers()
    cc = nvcc()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        cmd = [cc, *ARCH, *flags, "-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(f"compiled {os.path.basename(s)}", file=sys.stderr)
        return o

    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            list(ex.map(compile_one, todo))
    if todo or _stale(lib, objs):
        cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs, "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


def clean() -> None:
    for d in (OBJ, OBJ + "_check"):
        shutil.rmtree(d, ignore_errors=True)
    for f in (LIB, CHECK_LIB):
        if os.path.exists(f):
            os.remove(f)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--check", action="store_true", help="the checked build (-DORF_CHECK)")
    a = ap.parse_args()
    if a.clean:
        clean()
    print(build(verbose=a.v, check=a.check))
