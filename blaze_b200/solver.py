"""Python host API over libblaze_b200.so, named after the reference's
``class FluidSolver`` (src/FluidSolver.h:38-110).

    tmr = Timer(); scn = SceneSettings(...)
    solver = FluidSolver(tmr, scn)
    solver.setParticles(rec8)            # Parser::sourceParticleParse output
    while ...:
        solver.addSource(); solver.step()
        tmr.iter += 1; tmr.time += scn.dt

All compute runs in the CUDA library; this module only moves host arrays and
handles.  Field arrays use the reference layout, shaped (z, y, x).
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import BlazeError, check, load


class FluidSolver:
    def __init__(self, tmr, scn, particles=None, stream=None, density=None):
        self._lib = load()
        self.tmr = tmr
        self.scn = scn
        self.params = scn.to_params()
        h = C.c_void_p()
        check(self._lib.blz_create(C.byref(self.params), C.byref(h)))
        self._h = h
        self.last_stats = _abi.BlzStepStats()
        if stream is not None:
            check(self._lib.blz_set_stream(self._h, C.c_void_p(stream)), self._h)
        if particles is not None:
            self.setParticles(particles, density)

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.blz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- reference interface ----------------------------------------------------
    def setParticles(self, rec8, density=None):
        """Particle records (8 floats each).  With the density scalar on
        (scn.density_field), `density` gives each particle's density (default:
        the scene's extra["particle_density"], else 1 per particle)."""
        a = np.ascontiguousarray(rec8, dtype=np.float32).reshape(-1, 8)
        if not self.params.density_field:
            check(self._lib.blz_set_particles(self._h, a.ctypes.data_as(C.POINTER(C.c_float)), len(a)), self._h)
            return
        if density is None:
            density = getattr(self.scn, "extra", {}).get("particle_density")
        d = None
        if density is not None:
            d = np.ascontiguousarray(density, dtype=np.float32).reshape(-1)
            if len(d) != len(a):
                raise BlazeError(_abi.BLZ_ERR_ARG, f"{len(d)} densities for {len(a)} particles")
        check(self._lib.blz_set_particles_ex(self._h, a.ctypes.data_as(C.c_void_p),
                                             None if d is None else d.ctypes.data_as(C.c_void_p), len(a)), self._h)

    def addSource(self):
        check(self._lib.blz_add_source(self._h), self._h)

    def step(self, time=None):
        t = self.tmr.time if time is None else time
        check(self._lib.blz_step(self._h, C.c_float(t), C.byref(self.last_stats)), self._h)
        return self.last_stats.as_dict()

    def getTempGrid(self):
        """Device pointer of T's current front buffer (what the reference's
        Grid object behind getTempGrid() reads through at(i,j,k))."""
        return self._lib.blz_field_ptr(self._h, _abi.FIELD_T)

    # -- stages ---------------------------------------------------------------------
    def forces(self, time=None):
        t = self.tmr.time if time is None else time
        check(self._lib.blz_forces(self._h, C.c_float(t)), self._h)

    def divergence(self):
        check(self._lib.blz_divergence(self._h), self._h)

    def solve(self):
        check(self._lib.blz_solve(self._h, C.byref(self.last_stats)), self._h)
        return self.last_stats.as_dict()

    def sweeps(self, n):
        check(self._lib.blz_sweeps(self._h, int(n)), self._h)

    def tight_solve(self, tol, max_sweeps, omega):
        """The pressure system solved in FP64 to relative residual tol (SOR,
        training targets); returns (sweeps, FP64 relative residual)."""
        n, r = C.c_int(), C.c_double()
        check(self._lib.blz_tight_solve(self._h, float(tol), int(max_sweeps), float(omega), C.byref(n), C.byref(r)),
              self._h)
        return n.value, r.value

    def gradient(self):
        check(self._lib.blz_gradient(self._h), self._h)

    def project(self):
        check(self._lib.blz_project(self._h, C.byref(self.last_stats)), self._h)
        return self.last_stats.as_dict()

    def advect(self):
        check(self._lib.blz_advect(self._h), self._h)

    def residual(self):
        r, b = C.c_double(), C.c_double()
        check(self._lib.blz_residual(self._h, C.byref(r), C.byref(b)), self._h)
        return r.value, b.value

    # -- fields -----------------------------------------------------------------------
    def get(self, name, out=None):
        f = _abi.FIELD_NAMES[name] if isinstance(name, str) else name
        shape = self.params.field_shape(f)
        if out is None:
            out = np.empty(shape, np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.shape == shape
        check(self._lib.blz_get_field(self._h, f, out.ctypes.data_as(C.c_void_p), 0), self._h)
        return out

    def set(self, name, arr):
        f = _abi.FIELD_NAMES[name] if isinstance(name, str) else name
        a = np.ascontiguousarray(arr, dtype=np.float32)
        if a.shape != self.params.field_shape(f):
            raise BlazeError(_abi.BLZ_ERR_ARG, f"field {name}: shape {a.shape} != {self.params.field_shape(f)}")
        check(self._lib.blz_set_field(self._h, f, a.ctypes.data_as(C.c_void_p), 0), self._h)

    def field_ptr(self, name):
        f = _abi.FIELD_NAMES[name] if isinstance(name, str) else name
        return self._lib.blz_field_ptr(self._h, f)

    def get_device(self, name, dev_ptr):
        """Copy a field to caller-owned device memory (device pointer as int)."""
        f = _abi.FIELD_NAMES[name] if isinstance(name, str) else name
        check(self._lib.blz_get_field(self._h, f, C.c_void_p(dev_ptr), 1), self._h)

    def set_device(self, name, dev_ptr):
        f = _abi.FIELD_NAMES[name] if isinstance(name, str) else name
        check(self._lib.blz_set_field(self._h, f, C.c_void_p(dev_ptr), 1), self._h)

    def kernel_launches(self):
        return self._lib.blz_kernel_launches(self._h)

    # -- learned warm start ---------------------------------------------------------------
    def set_warm_start(self, net):
        """Attach a WarmStartUNet (dims equal to the grid's) or detach with
        None; the solver keeps a reference so the network outlives it."""
        check(self._lib.blz_set_warm_start(self._h, net.handle if net is not None else None), self._h)
        self._warm = net
