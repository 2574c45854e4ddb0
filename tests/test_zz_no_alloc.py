"""blz_residual_noalloc: the FP64 residual for callers that cannot allocate
device memory (a host that owns all device memory through its own pool, or
code that must not let cudaMalloc/cudaFree synchronise the device).  It must
give the same norms as the solver's blz_residual on the same rhs and
pressure, on two calls in a row (the static scratch is reused), under both
boundary modes and several wall/open patterns, and refuse grids deeper than
its 4096-plane scratch.  Widths the solver cannot hold (odd) are checked
against the FP64 oracle's residual instead.

Tolerance: relative difference <= 1e-6, the bar of the other FP64 residual
tests (both sides evaluate the stencil the same way and differ only in the
order of the FP64 sums).  Collected last so a failure here leaves every other
test already run.
"""
import ctypes as C

import numpy as np
import pytest

from blaze_b200 import BLZ_BC_FREE_SURFACE, BLZ_BC_REF_COMPAT, SceneSettings, Timer

pytestmark = pytest.mark.gpu

REL = 1e-6

BOUNDS = [(1, 0, 1, 0, 1, 1), (0, 1, 1, 1, 0, 0), (1, 1, 1, 1, 1, 1)]


def _noalloc(lib, p, rhs_d, p_d, out):
    import torch
    from blaze_b200 import _abi
    torch.cuda.synchronize()
    rc = lib.blz_residual_noalloc(C.byref(p), C.c_void_p(rhs_d.data_ptr()), C.c_void_p(p_d.data_ptr()),
                                  C.c_void_p(out.data_ptr()), None)
    assert rc == _abi.BLZ_OK, lib.blz_last_error(None)
    torch.cuda.synchronize()
    return out.cpu().tolist()


@pytest.mark.parametrize("bounds", BOUNDS, ids=["open_top_xhi", "open_xlo_z", "walls"])
@pytest.mark.parametrize("bc", [BLZ_BC_REF_COMPAT, BLZ_BC_FREE_SURFACE], ids=["ref_compat", "free_surface"])
def test_noalloc_residual_matches_solver_residual(bc, bounds):
    import torch
    from blaze_b200 import FluidSolver, _lib
    lib = _lib.load()
    dims = (40, 24, 18)
    scn = SceneSettings(gridRes=dims, dx=1.0 / 40, dt=1.0 / 24, closedBounds=bounds, bc_mode=bc)
    p = scn.to_params()
    rng = np.random.default_rng(17)
    s = FluidSolver(Timer(), scn)
    n = dims[0] * dims[1] * dims[2]
    rhs_d = torch.empty(n, dtype=torch.float32, device="cuda")
    p_d = torch.empty(n, dtype=torch.float32, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call in range(2):
        s.set("RHS", rng.standard_normal(p.field_shape("RHS")).astype(np.float32))
        s.set("P", (call + 1) * rng.standard_normal(p.field_shape("P")).astype(np.float32))
        r_ref, b_ref = s.residual()                       # the existing entry point
        s.get_device("RHS", rhs_d.data_ptr())
        s.get_device("P", p_d.data_ptr())
        r, b = _noalloc(lib, p, rhs_d, p_d, out)
        assert r == pytest.approx(r_ref, rel=REL) and b == pytest.approx(b_ref, rel=REL), (call, r, r_ref, b, b_ref)
    s.close()


@pytest.mark.parametrize("bc", [BLZ_BC_REF_COMPAT, BLZ_BC_FREE_SURFACE], ids=["ref_compat", "free_surface"])
def test_noalloc_residual_odd_width_matches_oracle(bc):
    """An odd width (which the colour-packed solver refuses) against the FP64
    oracle's residual of the same arrays."""
    import torch
    from blaze_b200 import _lib
    from oracle import oracle
    lib = _lib.load()
    dims = (21, 16, 11)
    scn = SceneSettings(gridRes=dims, dx=1.0 / 21, dt=1.0 / 24, closedBounds=(0, 1, 1, 0, 1, 0), bc_mode=bc)
    p = scn.to_params()
    rng = np.random.default_rng(23)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call in range(2):
        rhs = rng.standard_normal(p.field_shape("RHS")).astype(np.float32)
        pr = ((call + 1) * rng.standard_normal(p.field_shape("P"))).astype(np.float32)
        ref = oracle.State(p, np.float64)
        ref.RHS[...] = rhs
        ref.P[...] = pr
        r_ref, b_ref = ref.residual_norms()
        r, b = _noalloc(lib, p, torch.from_numpy(rhs.ravel()).cuda(), torch.from_numpy(pr.ravel()).cuda(), out)
        assert r == pytest.approx(r_ref, rel=REL) and b == pytest.approx(b_ref, rel=REL), (call, r, r_ref, b, b_ref)


def test_noalloc_rejects_depth_beyond_scratch():
    from blaze_b200 import _abi, _lib
    lib = _lib.load()
    p = SceneSettings(gridRes=(8, 8, 4097)).to_params()
    dummy = C.c_void_p(256)                               # never dereferenced: rejected first
    rc = lib.blz_residual_noalloc(C.byref(p), dummy, dummy, dummy, None)
    assert rc == _abi.BLZ_ERR_ARG
    assert b"4096" in lib.blz_last_error(None)
