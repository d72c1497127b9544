"""glmmhdturb_b200 -- B200 (sm_100a) GLM-MHD / CT-MHD time step of GLMMHDTurb.

The compute lives in libglmmhd_b200.so (C ABI: include/glmmhd_b200.h).  This package is the
host-side mirror of the reference's step API:

    glmmhdturb_b200.turb          glmmhd_turb.jl step functions, CFL, diagnostics, forcing
    glmmhdturb_b200.ctmhd         ct_mhd.jl CTMHD.step! / divB_max
    glmmhdturb_b200.march_bridge  march_bridge/MarchBridge.jl
    glmmhdturb_b200.Solver        a configured engine over device tensors
"""
from ._lib import GmtError, build, lib, version  # noqa: F401
from .solver import Ensemble, Solver  # noqa: F401

__all__ = ["Solver", "Ensemble", "GmtError", "build", "lib", "version"]
