"""Known-answer tests of the CPU oracle, written from the mathematics of each
stage (the reference ships no tests or fixtures).  CPU only."""
import math

import numpy as np
import pytest

from blaze_b200 import SceneSettings, BLZ_BC_FREE_SURFACE, BLZ_GS_PLANE, BLZ_GS_RB3D
from conftest import rel_l2


def params(n=(16, 12, 10), **kw):
    s = SceneSettings(gridRes=n, dx=1.0 / 16, dt=1.0 / 24, domainBboxMax=(n[0] / 16, n[1] / 16, n[2] / 16))
    for k, v in kw.items():
        setattr(s, k, v)
    return s.to_params()


def test_cubic_pulse_single_particle(oracle_mod):
    """A lone particle deposits value * (1 - x^2 (3 - 2x)), x = distance/radius
    (Grid.h:309-335), into T; V receives the negated y velocity (y flip)."""
    p = params((16, 16, 16))
    st = oracle_mod.State(p)
    dx = p.dx
    pos = (8.3 * dx, 7.6 * dx, 8.1 * dx)
    rec = np.array([[*pos, 0.0, 0.7, 0.0, 4 * dx, 2.0]], np.float32)
    st.add_source(rec)
    r = 2 * dx
    oy = 1.0 - float(rec[0, 1])                   # world -> object y (flip)
    for (i, j, k) in [(8, 8, 8), (7, 8, 8), (8, 7, 9), (9, 9, 8), (6, 8, 8)]:
        d = math.dist((float(rec[0, 0]), oy, float(rec[0, 2])), ((i + .5) * dx, (j + .5) * dx, (k + .5) * dx))
        x = d / r
        want = 2.0 * (1 - x * x * (3 - 2 * x)) if d <= r else 0.0
        want = want if abs(want) > 1e-5 else 0.0
        assert st.T[k, j, i] == pytest.approx(want, rel=1e-6, abs=1e-9)
    assert st.V.min() < 0 and st.V.max() <= 0        # +y world velocity is -V
    assert np.all(st.U == 0) and np.all(st.W == 0)


def test_small_pscale_skipped(oracle_mod):
    p = params()
    st = oracle_mod.State(p)
    rec = np.array([[0.3, 0.3, 0.3, 1.0, 1.0, 1.0, 0.5 * p.dx, 1.0]], np.float32)
    st.add_source(rec)
    assert not any(np.any(a) for a in (st.T, st.U, st.V, st.W))


def test_divergence_of_linear_field(oracle_mod):
    """U = a*x, V = b*y, W = c*z has div = a + b + c; with open faces the rhs
    is -div/dx everywhere, with walls the boundary flux is removed."""
    p = params(closedBounds=(0, 0, 0, 0, 0, 0))
    st = oracle_mod.State(p)
    W, H, D = p.width, p.height, p.depth
    a, b, c = 0.3, -0.2, 0.7
    st.U[...] = a * np.arange(W + 1)[None, None, :] * p.dx
    st.V[...] = b * np.arange(H + 1)[None, :, None] * p.dx
    st.W[...] = c * np.arange(D + 1)[:, None, None] * p.dx
    st.divergence()
    np.testing.assert_allclose(st.RHS, -(a + b + c), rtol=1e-12)
    p2 = params(closedBounds=(1, 1, 1, 1, 1, 1))
    st2 = oracle_mod.State(p2)
    st2.U[...], st2.V[...], st2.W[...] = st.U, st.V, st.W
    st2.divergence()
    interior = st2.RHS[1:-1, 1:-1, 1:-1]
    np.testing.assert_allclose(interior, -(a + b + c), rtol=1e-12)
    # xMin wall: the U(0) flux term is dropped -> -(U(1)/dx + ...)
    want = -(a * 1 + b + c)
    np.testing.assert_allclose(st2.RHS[1:-1, 1:-1, 0], want, rtol=1e-12)


@pytest.mark.parametrize("scheme", [0, 1, 2], ids=["rk3", "euler", "rk2"])
def test_advection_uniform_flow_shifts_cubic_exactly(oracle_mod, scheme):
    """RK3, forward Euler and RK2 in a uniform field all backtrace by exactly
    dt*u, and the Lagrange tricubic reproduces a cubic polynomial:
    T(x) -> T(x - dt*u) in the interior (Grid.h:148-222,
    FluidSolver.cu:392-456)."""
    n = (24, 20, 18)
    p = params(n, advect_scheme=scheme)
    st = oracle_mod.State(p)
    W, H, D = n
    u0, v0, w0 = 0.9, -0.6, 0.4                     # cells moved: dt*u/dx < 1
    st.U[...] = u0
    st.V[...] = v0
    st.W[...] = w0
    dx, dt = p.dx, p.dt

    def poly(x, y, z):
        # positive on the grid, so T's per-stage clamp at 0 never acts
        return 50.0 + 0.3 * x + 0.05 * x * x + 0.001 * x ** 3 + 0.2 * y - 0.001 * y * y * z + 0.02 * z ** 2

    k, j, i = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    st.T[...] = poly(i + 0.5, j + 0.5, k + 0.5)
    T0 = st.T.copy()
    st.advect()
    sx, sy, sz = dt * u0 / dx, dt * v0 / dx, dt * w0 / dx
    want = poly(i + 0.5 - sx, j + 0.5 - sy, k + 0.5 - sz)
    sl = (slice(3, -3), slice(3, -3), slice(3, -3))
    np.testing.assert_allclose(st.T[sl], want[sl], rtol=1e-12, atol=1e-10)
    assert not np.allclose(st.T[sl], T0[sl])
    # the velocity itself is uniform and stays uniform
    np.testing.assert_allclose(st.U[2:-2, 2:-2, 2:-2], u0, rtol=1e-13)


def test_buoyancy_constant_temperature(oracle_mod):
    p = params(buoyancy=2.0)
    st = oracle_mod.State(p)
    st.T[...] = 1.5
    st.forces(0.0)
    np.testing.assert_allclose(st.V, p.dt * (2.0 * 1.5 * p.gravity), rtol=1e-12)


def test_vorticity_zero_for_uniform_flow(oracle_mod):
    p = params((16, 16, 16), vorticityConf=0.5)
    st = oracle_mod.State(p)
    st.U[...] = 0.4
    st.V[...] = -0.1
    st.forces(0.0)
    np.testing.assert_allclose(st.U, 0.4, rtol=1e-13)
    np.testing.assert_allclose(st.V, -0.1, rtol=1e-13)


def test_wind_only_touches_slabs(oracle_mod):
    p = params((16, 12, 10), windAmp=0.5, windDir=0, windTurbAmp=0.0)
    st = oracle_mod.State(p)
    st.forces(0.0)
    W = p.width
    target = 0.5 * p.dt                           # u*(1-dt) + amp*(+1)*dt from 0
    for i in (0, 1, W - 1, W):
        np.testing.assert_allclose(st.U[:, :, i], target, rtol=1e-12)
    assert np.all(st.U[:, :, 2:W - 1] == 0)
    assert np.all(st.V == 0) and np.all(st.W == 0)


def test_perlin_properties(oracle_mod):
    # zero at lattice points, bounded, continuous
    assert oracle_mod.perlin(3.0, 5.0, 7.0, 1.0, 123) == 0.0
    rng = np.random.default_rng(0)
    vals = [oracle_mod.perlin(*rng.uniform(0, 50, 3), 0.25, 123) for _ in range(2000)]
    assert max(abs(v) for v in vals) <= 1.5
    assert np.std(vals) > 0.05
    a = oracle_mod.perlin(10.3, 4.2, 8.9, 0.5, 123)
    b = oracle_mod.perlin(10.3 + 1e-4, 4.2, 8.9, 0.5, 123)
    assert abs(a - b) < 1e-3


@pytest.mark.parametrize("order", [BLZ_GS_RB3D, BLZ_GS_PLANE])
def test_free_surface_projection_is_divergence_free(oracle_mod, order):
    """FREE_SURFACE: solving to a tight residual and subtracting the gradient
    leaves a discretely divergence-free velocity."""
    n = (12, 10, 8)
    p = params(n, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=BLZ_BC_FREE_SURFACE, gs_order=order,
               maxIterSolve=20000, tol=1e-10, check_every=50)
    st = oracle_mod.State(p)
    rng = np.random.default_rng(1)
    for f in ("U", "V", "W"):
        getattr(st, f)[...] = rng.standard_normal(getattr(st, f).shape)
    it, r, b = st.project()
    assert r / b <= 1e-10 and it < 20000
    st.divergence()
    assert np.max(np.abs(st.RHS)) < 1e-7 * 1.0 / p.dx


def test_ref_compat_closed_box_converges(oracle_mod):
    """All walls: the Neumann system is compatible, so the residual falls."""
    n = (12, 10, 8)
    p = params(n, closedBounds=(1, 1, 1, 1, 1, 1), maxIterSolve=5000, tol=1e-8, check_every=50)
    st = oracle_mod.State(p)
    rng = np.random.default_rng(2)
    for f in ("U", "V", "W"):
        getattr(st, f)[...] = rng.standard_normal(getattr(st, f).shape)
    st.divergence()
    it, r, b = st.solve()
    assert r / b <= 1e-8


def test_gs_sweep_reduces_residual_monotonically(oracle_mod):
    n = (16, 12, 10)
    p = params(n, closedBounds=(1, 1, 1, 0, 1, 1), bc_mode=BLZ_BC_FREE_SURFACE)
    st = oracle_mod.State(p)
    st.RHS[...] = np.random.default_rng(3).standard_normal(st.RHS.shape)
    last = st.residual_norms()[0]
    for _ in range(5):
        st.gs_sweeps(3)
        r = st.residual_norms()[0]
        assert r < last
        last = r


def test_fp32_and_fp64_oracles_agree(oracle_mod):
    """The FP32 instantiation (the reference's own arithmetic) stays within
    FP32 rounding of the FP64 one over a full step."""
    from blaze_b200 import plume_scene
    scn, parts = plume_scene(n=16, seed=4, particles=300)
    scn.maxIterSolve = 10
    scn.vorticityConf = 0.3
    p = scn.to_params()
    a, b = oracle_mod.State(p, np.float64), oracle_mod.State(p, np.float32)
    for s in (a, b):
        s.add_source(parts)
        s.step(0.0)
        s.add_source(parts)
        s.step(p.dt)
    for f in ("T", "U", "V", "W", "P"):
        assert rel_l2(getattr(b, f), getattr(a, f)) < 2e-5, f


def test_density_scalar_restates_temperature_buoyancy(oracle_mod):
    """Target mode's density scalar (no reference counterpart): splatted with
    each particle's density it follows T's sourcing rules, so with density =
    temperature per particle the scalar equals T; and buoyancy
    V += dt (beta T - alpha rho) g then equals the temperature-only buoyancy
    with beta - alpha.  Advection carries it as it carries T."""
    from blaze_b200 import SceneSettings
    rng = np.random.default_rng(3)
    n = 12
    scn = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, buoyancy=1.3, density_field=1, buoyancy_alpha=0.4)
    p = scn.to_params()
    rec = np.zeros((60, 8), np.float32)
    rec[:, :3] = rng.uniform(0.1, 0.9, (60, 3))
    rec[:, 6] = 3.0 / n
    rec[:, 7] = rng.uniform(0.2, 1.5, 60)
    st = oracle_mod.State(p, np.float64)
    st.add_source(rec, density=rec[:, 7])
    np.testing.assert_array_equal(st.DENSITY, st.T)
    st.forces(0.0)
    q = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, buoyancy=1.3 - 0.4).to_params()
    ref = oracle_mod.State(q, np.float64)
    ref.add_source(rec)
    ref.forces(0.0)
    # beta and alpha are float32 parameters: 1.3f - 0.4f and 0.9f differ by 3e-8
    np.testing.assert_allclose(st.V, ref.V, rtol=1e-7, atol=1e-12)
    st.U[...] = rng.standard_normal(st.U.shape) * 0.3
    st.advect()
    np.testing.assert_array_equal(st.DENSITY, st.T)
