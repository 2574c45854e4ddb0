"""ctypes wrapper of the CPU oracle (oracle/lib/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker; never by the product path.

All field arrays use the reference layout shaped (z, y, x); ``dtype`` is
float64 (the FP64 oracle) or float32 (the reference's own arithmetic).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "liboracle.so")

from blaze_b200 import _abi  # noqa: E402  (shares the blz_params struct)

_lib = None


def build(force=False):
    srcs = [os.path.join(HERE, f) for f in ("blaze_oracle.cpp", "render_oracle.cpp")]
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE, "lib/liboracle.so"] + (["-B"] if force else []), check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        P = C.POINTER(_abi.BlzParams)
        for suf, ct in (("f64", C.c_double), ("f32", C.c_float)):
            R = C.POINTER(ct)
            sig = {
                "add_source": [P, C.POINTER(C.c_float), C.c_int, R, R, R, R, C.POINTER(C.c_float), R],
                "forces": [P, C.c_float, R, R, R, R, R],
                "divergence": [P, R, R, R, R],
                "gs_sweeps": [P, R, R, C.c_int],
                "solve": [P, R, R, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)],
                "residual": [P, R, R, C.POINTER(C.c_double), C.POINTER(C.c_double)],
                "gradient": [P, R, R, R, R],
                "advect": [P, R, R, R, R, R],
                "step": [P, C.c_float, R, R, R, R, R, R, C.POINTER(C.c_int), C.POINTER(C.c_double),
                         C.POINTER(C.c_double), R],
            }
            for name, args in sig.items():
                fn = getattr(lib, f"orc_{name}_{suf}")
                fn.restype = None
                fn.argtypes = args
        F = C.POINTER(C.c_float)
        lib.orc_tex_sample.restype = None
        lib.orc_tex_sample.argtypes = [F, C.c_int, C.c_int, C.c_int, F, C.c_int, F, C.c_int]
        lib.orc_render.restype = None
        lib.orc_render.argtypes = [C.POINTER(_abi.BlzRenderParams), P, F, F, C.c_int]
        lib.orc_perlin.restype = C.c_float
        lib.orc_perlin.argtypes = [C.c_float] * 4 + [C.c_int]
        lib.orc_noise.restype = C.c_int
        lib.orc_noise_set_lattice_patterns.restype = C.c_int
        lib.orc_noise_set_lattice_patterns.argtypes = [C.POINTER(C.c_ulonglong), C.c_int]
        lib.orc_noise.argtypes = [C.POINTER(_abi.BlzNoiseArgs), C.c_void_p, C.c_longlong, C.c_void_p]
        lib.orc_num_threads.restype = C.c_int
        if hasattr(lib, "orc_set_num_threads"):
            lib.orc_set_num_threads.restype = None
            lib.orc_set_num_threads.argtypes = [C.c_int]
        _lib = lib
    return _lib


def _ptr(a):
    ct = C.c_double if a.dtype == np.float64 else C.c_float
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(ct))


def _suf(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


class State:
    """Fields of one simulation held on the host for the oracle."""

    def __init__(self, params, dtype=np.float64):
        self.p = params
        self.dtype = np.dtype(dtype)
        z = lambda f: np.zeros(params.field_shape(f), self.dtype)
        self.T, self.U, self.V, self.W = z("T"), z("U"), z("V"), z("W")
        self.P, self.RHS = z("P"), z("RHS")
        # the density scalar of target mode (params.density_field)
        self.DENSITY = z("DENSITY") if params.density_field else None
        self.iterations, self.residual, self.rhs_norm = 0, 0.0, 0.0

    def fields(self):
        out = {"T": self.T, "U": self.U, "V": self.V, "W": self.W, "P": self.P, "RHS": self.RHS}
        if self.DENSITY is not None:
            out["DENSITY"] = self.DENSITY
        return out

    def _dn(self):
        return None if self.DENSITY is None else _ptr(self.DENSITY)

    def load(self, **arrays):
        for k, v in arrays.items():
            getattr(self, k)[...] = v

    def _fn(self, name):
        return getattr(load(), f"orc_{name}_{_suf(self.dtype)}")

    def add_source(self, rec8, density=None):
        """density: per-particle density for the density scalar (None: 1)."""
        a = np.ascontiguousarray(rec8, np.float32).reshape(-1, 8)
        d = None if density is None else np.ascontiguousarray(density, np.float32).reshape(-1)
        self._fn("add_source")(C.byref(self.p), a.ctypes.data_as(C.POINTER(C.c_float)), len(a),
                               _ptr(self.T), _ptr(self.U), _ptr(self.V), _ptr(self.W),
                               None if d is None else d.ctypes.data_as(C.POINTER(C.c_float)), self._dn())

    def forces(self, time):
        self._fn("forces")(C.byref(self.p), time, _ptr(self.T), _ptr(self.U), _ptr(self.V), _ptr(self.W),
                           self._dn())

    def divergence(self):
        self._fn("divergence")(C.byref(self.p), _ptr(self.U), _ptr(self.V), _ptr(self.W), _ptr(self.RHS))

    def gs_sweeps(self, n):
        self._fn("gs_sweeps")(C.byref(self.p), _ptr(self.RHS), _ptr(self.P), n)

    def solve(self):
        it, r, b = C.c_int(), C.c_double(), C.c_double()
        self._fn("solve")(C.byref(self.p), _ptr(self.RHS), _ptr(self.P), C.byref(it), C.byref(r), C.byref(b))
        self.iterations, self.residual, self.rhs_norm = it.value, r.value, b.value
        return it.value, r.value, b.value

    def residual_norms(self):
        r, b = C.c_double(), C.c_double()
        self._fn("residual")(C.byref(self.p), _ptr(self.RHS), _ptr(self.P), C.byref(r), C.byref(b))
        return r.value, b.value

    def gradient(self):
        self._fn("gradient")(C.byref(self.p), _ptr(self.P), _ptr(self.U), _ptr(self.V), _ptr(self.W))

    def advect(self):
        self._fn("advect")(C.byref(self.p), _ptr(self.T), _ptr(self.U), _ptr(self.V), _ptr(self.W), self._dn())

    def project(self):
        self.divergence()
        out = self.solve()
        self.gradient()
        return out

    def step(self, time):
        it, r, b = C.c_int(), C.c_double(), C.c_double()
        self._fn("step")(C.byref(self.p), time, _ptr(self.T), _ptr(self.U), _ptr(self.V), _ptr(self.W),
                         _ptr(self.P), _ptr(self.RHS), C.byref(it), C.byref(r), C.byref(b), self._dn())
        self.iterations, self.residual, self.rhs_norm = it.value, r.value, b.value
        return it.value, r.value, b.value


def perlin(x, y, z, scale, seed):
    return load().orc_perlin(x, y, z, scale, seed)


def noise(args, pos3, lattice_patterns=()):
    """The noise library's function args.func (a BlzNoiseArgs) restated
    (noise_oracle.cpp), at positions pos3 (n x 3 float32).  lattice_patterns
    selects, per value-noise lattice blend and lattice point, the other
    contraction of the hash sum (the test hook
    orc_noise_set_lattice_patterns; empty is the standalone form)."""
    a = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
    out = np.empty(len(a), np.float32)
    lib = load()
    pats = (C.c_ulonglong * max(1, len(lattice_patterns)))(*lattice_patterns)
    if lib.orc_noise_set_lattice_patterns(pats, len(lattice_patterns)) != 0:
        raise ValueError("at most 16 lattice patterns")
    try:
        rc = lib.orc_noise(C.byref(args), a.ctypes.data, len(a), out.ctypes.data)
    finally:
        lib.orc_noise_set_lattice_patterns(pats, 0)
    if rc != 0:
        raise ValueError(f"orc_noise: bad arguments ({rc})")
    return out


def num_threads():
    return load().orc_num_threads()


def set_num_threads(n):
    """Threads of the oracle's later parallel loops (OpenMP); False when the
    built library predates this call."""
    lib = load()
    if not hasattr(lib, "orc_set_num_threads"):
        return False
    lib.orc_set_num_threads(int(n))
    return True


def tex_sample(T, pos3, quant=3):
    """The texture sampler of the reference's renderer restated (trilinear,
    clamped, weights quantised per `quant`, render_oracle.cpp; 3 is the rule
    measured on B200) on T shaped (z, y, x) at texel coordinates pos3 (n, 3)."""
    T = np.ascontiguousarray(T, np.float32)
    pos = np.ascontiguousarray(pos3, np.float32).reshape(-1, 3)
    out = np.empty(len(pos), np.float32)
    D, H, W = T.shape
    load().orc_tex_sample(_ptr(T), W, H, D, _ptr(pos), len(pos), _ptr(out), quant)
    return out


def render(rp, grid, T, quant=3):
    """The reference's render pass restated (render_oracle.cpp): image of T
    (z, y, x) shaped (height, width, 3), row 0 at the top."""
    T = np.ascontiguousarray(T, np.float32)
    out = np.empty((rp.height, rp.width, 3), np.float32)
    load().orc_render(C.byref(rp), C.byref(grid), _ptr(T), _ptr(out), quant)
    return out
