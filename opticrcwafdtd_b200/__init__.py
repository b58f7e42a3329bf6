"""opticrcwafdtd_b200 -- B200-native Yee FDTD engine for OpticRCWAFDTD's
orf.fdtd2D / orf.fdtd2DTE / orf.fdtd3D (toolbox/+orf/fdtd2D.m, fdtd3D.m), and
its 2D frequency-domain solver orf.fdfd2D (toolbox/+orf/fdfd2D.m).

The time loop runs in liborf_fdtd.so (hand-written sm_100a CUDA behind the C
ABI in include/orf_fdtd.h).  This package is the host-side mirror of the
reference's MATLAB interface: same sim/out fields, same index conventions
(1-based), same error identifiers.  There is no CPU fallback: a call fails
with OrfError('orf:noDevice' / 'orf:libraryMissing') when the CUDA library or
a GPU is missing.
"""
from ._abi import NotConvergedWarning, OrfError  # noqa: F401
from .geometry import epsCellMean, epsComponents2D, epsComponents3D, epsFromBoxes  # noqa: F401
from .modes import slabModes, wgModes2D  # noqa: F401
from .coupler import (apodizedGrating, bestFiberCoupling, fiberCoupling, gratingCouplerTE,  # noqa: F401
                      gratingCouplerTE_batch)

__version__ = "0.1.0"
from .fdtd import Context, Job, Server, device_count, fdtd2D, fdtd2D_batch, fdtd2DTE, fdtd3D  # noqa: F401,E402
from .fdfd import FDFD2D, fdfd2D  # noqa: F401,E402
from .slab3d import SlabRun, fdtd3D_distributed, fdtd3D_slabs  # noqa: F401,E402
