"""The GPU permittivity generator (orf_eps3d) against the host one: the same
shapes, sub-sampling and averaging order, so the same bits."""
import time

import numpy as np
import pytest

from opticrcwafdtd_b200 import Context, epsComponents3D

pytestmark = pytest.mark.gpu


def _shapes(rng):
    R = rng.uniform(0.05, 0.14, (3, 4))
    R[1, 2] = 0.0                                   # a missing pillar
    return [
        ["box", [-np.inf, np.inf, -np.inf, np.inf, -np.inf, 0.2, 1.46]],
        ["box", [0.1, 0.45, 0.05, 0.33, 0.25, 0.5, 2.1]],
        ["cyl", [0.6, 0.4, 0.13, 0.3, 0.55, 3.0]],
        ["cone", [0.2, 0.7, 0.05, 0.17, 0.1, 0.45, 1.8]],
        ["polygon", dict(xy=[[0.4, 0.6], [0.75, 0.65], [0.55, 0.9]], z1=0.05, z2=0.4, n=2.5)],
        ["lattice", dict(x0=0.15, y0=0.12, period=0.3, R=R, z1=0.3, z2=0.55, n=2.4)],
        ["lattice", dict(x0=0.3, y0=0.3, period=0.35, R=[[0.1, 0.12], [0.08, 0.14]], z1=0.05, z2=0.25, n=1.9,
                         dRdz=-0.1)],
    ]


@pytest.mark.parametrize("method", ["directional", "kottke"])
@pytest.mark.parametrize("nsub", [1, 2, 4, 5])
@pytest.mark.parametrize("periodic", [False, True])
def test_gpu_eps_matches_host_bitwise(nsub, periodic, method):
    rng = np.random.default_rng(7)
    d = 0.025
    x = (np.arange(40) + 0.5) * d
    y = (np.arange(36) + 0.5) * d
    z = np.arange(26) * d
    per = [40 * d, 36 * d] if periodic else None
    sh = _shapes(rng)
    host = epsComponents3D(x, y, z, 1.0, sh, NSub=nsub, Period=per, Method=method)
    ctx = Context(0)
    dev = epsComponents3D(x, y, z, 1.0, sh, NSub=nsub, Period=per, Method=method, device=ctx)
    ctx.close()
    for k in "xyz":
        assert dev[k].flags["F_CONTIGUOUS"]
        assert np.array_equal(dev[k], host[k]), (k, np.max(np.abs(dev[k] - host[k])))


def test_gpu_eps_pillar_lattice():
    """A 300 x 300 x 150 pillar lattice (the C3 workload at half size)."""
    d = 0.02
    x = (np.arange(300) + 0.5) * d
    y = x.copy()
    z = np.arange(150) * d
    rng = np.random.default_rng(3)
    R = rng.uniform(0.06, 0.18, (15, 15))
    shapes = [["box", [-np.inf, np.inf, -np.inf, np.inf, -np.inf, 0.9, 1.46]],
              ["lattice", dict(x0=0.2, y0=0.2, period=0.4, R=R, z1=0.9, z2=1.5, n=2.4)]]
    t0 = time.perf_counter()
    host = epsComponents3D(x, y, z, 1.0, shapes)
    t1 = time.perf_counter()
    dev = epsComponents3D(x, y, z, 1.0, shapes, device=True)
    t2 = time.perf_counter()
    for k in "xyz":
        assert np.array_equal(dev[k], host[k])
    print(f"host {t1 - t0:.2f} s, GPU {t2 - t1:.3f} s")
