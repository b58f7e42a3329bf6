"""3D waveguide mode source on the GPU: wgModes2D on a plane of the 3D grid
feeds the TF/SF plane of fdtd3D (tests/TestFDTD3D.m:36-58, 100-127)."""
import numpy as np
import pytest

import opticrcwafdtd_b200 as orf
from tests import cases

pytestmark = pytest.mark.gpu


def test_strip_mode_source_and_dispersion():
    sim, prof, ms_eps = cases.strip3d_sim()
    cases.check_strip3d(orf.fdtd3D(sim), sim, prof, ms_eps)


def test_strip_single_precision_matches_double():
    """Flux ratios of the FP32 run within 1e-4 of FP64 (TestFDTD3D.m:119-127)."""
    o1 = orf.fdtd3D(cases.strip3d_sim("double")[0])
    o2 = orf.fdtd3D(cases.strip3d_sim("single")[0])
    r1 = o1["flux"][:, 0] / o1["flux"][1, 0]
    r2 = o2["flux"][:, 0] / o2["flux"][1, 0]
    assert np.max(np.abs(r2 - r1)) <= 1e-4
