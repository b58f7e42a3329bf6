"""CPU oracle for the Yee FDTD hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
leg may import this package, and only as the checker.  The product package
(opticrcwafdtd_b200) never imports it.

Parity status: the FDTD restatement (fdtd_oracle.cpp) is pinned against the
reference's own physics tests at their tolerances (tests/TestFDTD2D.m,
TestFDTD3D.m, TestCPO.m); bit-level parity with the closed P-code reference
(toolbox/+orf/fdtd2D.p, fdtd3D.p) is unpinned because it cannot run here.
"""
from .oracle import fdtd2D, fdtd2DTE, fdtd3D, load, pulse, max_threads  # noqa: F401
from .tmm import tmm  # noqa: F401
from .geometry_ref import epsFromBoxes_ref  # noqa: F401
