"""B200-native Blaze fluid step: hand-written sm_100a CUDA kernels behind a
C ABI (include/blaze_b200.h), with a Python host API named after the
reference's FluidSolver."""
from ._abi import (BLZ_BC_FREE_SURFACE, BLZ_BC_REF_COMPAT, BLZ_GS_PLANE, BLZ_GS_RB3D,  # noqa: F401
                   BlzParams, BlzStepStats)
from .scenes import PCG32, SceneSettings, Timer, fire_scene, family_scene, plume_scene, read_part, write_part  # noqa: F401


def __getattr__(name):
    # The solver binds the CUDA library on first use, so that scenes and the
    # ABI structs import on machines without the built library.
    if name in ("FluidSolver",):
        from .solver import FluidSolver
        return FluidSolver
    if name in ("BlazeError",):
        from ._lib import BlazeError
        return BlazeError
    raise AttributeError(name)
