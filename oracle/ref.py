"""ctypes wrapper of the reference's own CUDA build (oracle/_ref/libblaze_ref.so).

TEST INFRASTRUCTURE ONLY: used by the parity tests, by
tests/golden/make_golden.py and by bench.py's reference timing arm.  Needs a
CUDA device.  Fields use the reference layout shaped (z, y, x).
"""
import ctypes as C
import os

import numpy as np

from blaze_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libblaze_ref.so")

STAGES = {"cooldown": 0, "drag": 1, "vorticity": 2, "buoyancy": 3, "wind": 4, "turbulence": 5,
          "divergence": 6, "gs": 7, "gradient": 8, "advect": 9}

_lib = None


def available():
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle ref, needs the reference sources)")
        lib = C.CDLL(LIB)
        P = C.POINTER(_abi.BlzParams)
        F = C.POINTER(C.c_float)
        for name, res, args in [
            ("ref_create", C.c_void_p, [P]), ("ref_destroy", None, [C.c_void_p]),
            ("ref_set_time", None, [C.c_void_p, C.c_int, C.c_float]),
            ("ref_set_max_iter", None, [C.c_void_p, C.c_int]),
            ("ref_set_particles", C.c_int, [C.c_void_p, F, C.c_int]),
            ("ref_add_source", C.c_int, [C.c_void_p]), ("ref_step", C.c_int, [C.c_void_p]),
            ("ref_project", C.c_int, [C.c_void_p]), ("ref_stage", C.c_int, [C.c_void_p, C.c_int]),
            ("ref_get_field", C.c_int, [C.c_void_p, C.c_int, F]),
            ("ref_set_field", C.c_int, [C.c_void_p, C.c_int, F]),
            ("ref_perlin", C.c_int, [F, C.c_int, C.c_float, C.c_int, F]),
            ("ref_noise", C.c_int, [C.POINTER(_abi.BlzNoiseArgs), F, C.c_int, F]),
            ("ref_render_create", C.c_void_p, [C.c_void_p, C.POINTER(_abi.BlzRenderParams)]),
            ("ref_render", C.c_int, [C.c_void_p, C.c_void_p, F]),
            ("ref_render_get", C.c_int, [C.c_void_p, F]),
            ("ref_render_destroy", None, [C.c_void_p]),
        ]:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference harness: {what} failed ({rc})")


class RefSolver:
    """The reference's FluidSolver on the current CUDA device."""

    def __init__(self, params):
        self.lib = load()
        self.p = params.copy()
        self.h = self.lib.ref_create(C.byref(self.p))
        if not self.h:
            raise RuntimeError("ref_create failed")

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_time(self, it, time):
        self.lib.ref_set_time(self.h, it, time)

    def set_max_iter(self, n):
        """maxIterSolve of the following solves."""
        self.lib.ref_set_max_iter(self.h, int(n))

    def set_particles(self, rec8):
        a = np.ascontiguousarray(rec8, np.float32).reshape(-1, 8)
        _chk(self.lib.ref_set_particles(self.h, a.ctypes.data_as(C.POINTER(C.c_float)), len(a)), "set_particles")

    def add_source(self):
        _chk(self.lib.ref_add_source(self.h), "addSource")

    def step(self):
        _chk(self.lib.ref_step(self.h), "step")

    def project(self):
        _chk(self.lib.ref_project(self.h), "project")

    def stage(self, name):
        _chk(self.lib.ref_stage(self.h, STAGES[name]), name)

    def get(self, name):
        f = _abi.FIELD_NAMES[name]
        out = np.empty(self.p.field_shape(f), np.float32)
        _chk(self.lib.ref_get_field(self.h, f, out.ctypes.data_as(C.POINTER(C.c_float))), f"get {name}")
        return out

    def set(self, name, arr):
        f = _abi.FIELD_NAMES[name]
        a = np.ascontiguousarray(arr, np.float32)
        assert a.shape == self.p.field_shape(f)
        _chk(self.lib.ref_set_field(self.h, f, a.ctypes.data_as(C.POINTER(C.c_float))), f"set {name}")


def perlin(pos3, scale, seed):
    a = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
    out = np.empty(len(a), np.float32)
    _chk(load().ref_perlin(a.ctypes.data_as(C.POINTER(C.c_float)), len(a), scale, seed,
                           out.ctypes.data_as(C.POINTER(C.c_float))), "perlin")
    return out


class RefRenderer:
    """The reference's RenderEngine on a RefSolver's temperature field."""

    def __init__(self, sim, rp):
        self.sim, self.rp = sim, rp
        self.lib = sim.lib
        self.h = self.lib.ref_render_create(sim.h, C.byref(rp))
        if not self.h:
            raise RuntimeError("ref_render_create failed")

    def render(self):
        """Renders the solver's current T; returns device milliseconds."""
        ms = C.c_float()
        _chk(self.lib.ref_render(self.sim.h, self.h, C.byref(ms)), "render")
        return ms.value

    def image(self):
        out = np.empty((self.rp.height, self.rp.width, 3), np.float32)
        _chk(self.lib.ref_render_get(self.h, out.ctypes.data_as(C.POINTER(C.c_float))), "render_get")
        return out

    def close(self):
        if self.h:
            self.lib.ref_render_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def noise(args, pos3):
    """The reference library's noise function args.func (a BlzNoiseArgs) at
    positions pos3, computed by the reference build on the GPU."""
    a = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
    out = np.empty(len(a), np.float32)
    _chk(load().ref_noise(C.byref(args), a.ctypes.data_as(C.POINTER(C.c_float)), len(a),
                          out.ctypes.data_as(C.POINTER(C.c_float))), "noise")
    return out
