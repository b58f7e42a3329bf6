"""Size-independent checks at the benchmark sizes (2D TM 4000 x 1500, 3D
600 x 600 x 300), where the oracle would take too long:
  - the tiling changes nothing: runs with different interior variants and
    fused step depths (different tile grids, frame widths and launch
    sequences) give bitwise identical fields;
  - linearity in the source amplitude: doubling the source doubles the
    fields to 1e-6 of the largest field value (exact except where gradual
    underflow, which rounds absolutely, enters);
  - FP32 stays within 1e-4 (relative L2) of FP64."""
import numpy as np
import pytest

from opticrcwafdtd_b200 import Context, Job, workloads

pytestmark = pytest.mark.gpu


def _fields(sim, dims, steps, tsteps=0, variant=0):
    ctx = Context(0)
    if tsteps or variant:
        ctx.set_tuning(tsteps=tsteps, variant=variant)
    job = Job(sim, ctx, dims=dims)
    job.advance(steps)
    f = job.fields()
    job.close()
    ctx.close()
    return f


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _linear(a, b, scale):
    assert scale > 0
    assert np.max(np.abs(b - 2 * a)) <= 1e-6 * 2 * scale


def test_pixel_region_full_size_tiling_linearity_precision():
    steps = 1000
    sim = workloads.pixel_region_sim(precision="single", steps=30000)
    f1 = _fields(sim, 2, steps)
    for a, b in zip(f1, _fields(sim, 2, steps, tsteps=4, variant=2)):
        assert np.isfinite(a).all()
        assert np.array_equal(a, b)
    s2 = dict(sim, source=dict(sim["source"], profile=2 * np.asarray(sim["source"]["profile"])))
    scale = max(np.max(np.abs(a)) for a in f1)
    for a, b in zip(f1, _fields(s2, 2, steps)):
        _linear(a, b, scale)
    for a, b in zip(f1, _fields(dict(sim, precision="double"), 2, steps)):
        assert _rel(a, b) < 1e-4


def test_pillar_lattice_full_size_linearity_precision():
    steps = 150
    sim = workloads.pillar_lattice_sim(steps=10000, precision="single")
    f1 = _fields(sim, 3, steps)
    src = dict(sim["source"])
    for k in ("Ea", "Eb", "Ha", "Hb"):
        v = np.asarray(src[k], dtype=float)
        src[k] = float(2 * v) if v.ndim == 0 else 2 * v
    f2 = _fields(dict(sim, source=src), 3, steps)
    scale = max(np.max(np.abs(a)) for a in f1)
    for q in range(6):
        assert np.isfinite(f1[q]).all()
        _linear(f1[q], f2[q], scale)
    del f2
    f64 = _fields(dict(sim, precision="double"), 3, steps)
    for a, b in zip(f1, f64):
        assert _rel(a, b) < 1e-4
