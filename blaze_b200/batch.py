"""Batched simulations: Python handle over the ``blz_batch_*`` entry points.

    sims = [FluidSolver(Timer(), s, particles=p) for s, p in batch_scenes(64, seed=4)]
    batch = Batch(sims)
    for f in range(frames):
        batch.add_source()
        stats = batch.step([f * s.scn.dt for s in sims])

No counterpart in the reference, which runs one FluidSolver per process.
"""
import ctypes as C

from . import _abi
from ._lib import check, load


class Batch:
    def __init__(self, solvers):
        self._lib = load()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = C.c_void_p()
        check(self._lib.blz_batch_create(arr, len(self.solvers), C.byref(h)))
        self._h = h
        self._stats = (_abi.BlzStepStats * len(self.solvers))()

    def close(self):
        if getattr(self, "_h", None):
            self._lib.blz_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return self._lib.blz_batch_stream(self._h)

    def add_source(self):
        check(self._lib.blz_batch_add_source(self._h))

    def step(self, times=None):
        """One frame of every solver; returns their solve statistics."""
        t = None
        if times is not None:
            t = (C.c_float * len(self.solvers))(*[float(x) for x in times])
        check(self._lib.blz_batch_step(self._h, t, self._stats))
        return [s.as_dict() for s in self._stats]

    def solve(self):
        check(self._lib.blz_batch_solve(self._h, self._stats))
        return [s.as_dict() for s in self._stats]

    def set_sweep(self, planes, paired=False):
        """-1: autotune (default); 0: the segment kernel; planes > 0: temporal
        blocking with tiles of that many planes (paired: the paired-FP32
        stencil).  Every choice gives the same bits; the stats' sweep_variant
        reports the one in use (1, 2, 4, 8 planes per thread, or 100 (scalar)
        or 200 (paired) + planes per tile)."""
        check(self._lib.blz_batch_set_sweep(self._h, int(planes), 1 if paired else 0))

    def last_ms(self):
        return float(self._lib.blz_batch_last_ms(self._h))

    def kernel_launches(self):
        return int(self._lib.blz_batch_kernel_launches(self._h))
