"""The drop-in FluidSolver (blaze_b200/shim/FluidSolver_blaze.cu, compiled
against the reference's own FluidSolver.h) driven like the reference's
main.cu frame loop, with T read back through getTempGrid() the way the
reference's renderer reads it ((*grid)->at(i,j,k)).  It must equal the
direct C-ABI path bit for bit."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from blaze_b200 import Timer, plume_scene, write_part

pytestmark = pytest.mark.gpu


def shim_lib():
    from blaze_b200 import build
    if not os.path.exists(build.SHIM_LIB):
        pytest.skip("drop-in shim not built (needs the reference headers at build time)")
    lib = C.CDLL(build.SHIM_LIB)
    from blaze_b200 import _abi
    lib.blz_shim_create.restype = C.c_void_p
    lib.blz_shim_create.argtypes = [C.POINTER(_abi.BlzParams), C.c_char_p, C.c_char_p, C.c_int]
    lib.blz_shim_frame.argtypes = [C.c_void_p]
    lib.blz_shim_read_temp.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    lib.blz_shim_destroy.argtypes = [C.c_void_p]
    return lib


def test_drop_in_matches_c_abi():
    lib = shim_lib()
    from blaze_b200 import FluidSolver
    scn, parts = plume_scene(n=32, seed=5, particles=700)
    scn.reset_pressure = 0                        # the reference keeps p between frames
    scn.maxIterSolve = 30
    p = scn.to_params()
    frames = 4
    with tempfile.TemporaryDirectory() as d:
        write_part(os.path.join(d, "plume.part"), parts)
        h = lib.blz_shim_create(C.byref(p), d.encode(), b"plume.part", 0)
        for _ in range(frames):
            lib.blz_shim_frame(h)
        t_shim = np.empty(p.field_shape("T"), np.float32)
        assert lib.blz_shim_read_temp(h, t_shim.ctypes.data_as(C.POINTER(C.c_float))) == 0
        lib.blz_shim_destroy(h)
    tmr = Timer()
    s = FluidSolver(tmr, scn, particles=parts)
    for _ in range(frames):
        s.addSource()
        s.step()
        tmr.iter += 1
        tmr.time += scn.dt
    t_abi = s.get("T")
    s.close()
    assert np.abs(t_abi).max() > 0.1
    np.testing.assert_array_equal(t_shim, t_abi)
