"""Parity of the CUDA path (through the C ABI) with the FP64 oracle on seeded
inputs, stage by stage and over whole steps.

Tolerance (FP32 kernels against the FP64 restatement): relative L2 error
<= 5e-6 and max-abs error <= 5e-5 * max(1, max|oracle|) per field for one
stage; looser where stated (many GS sweeps, ten chaotic steps).
"""
import numpy as np
import pytest

from blaze_b200 import (BLZ_BC_FREE_SURFACE, BLZ_BC_REF_COMPAT, BLZ_GS_PLANE, BLZ_GS_RB3D,
                        SceneSettings, Timer, plume_scene)
from conftest import max_abs, rel_l2

pytestmark = pytest.mark.gpu

STAGE_REL, STAGE_ABS = 5e-6, 5e-5


def scene(dims=(24, 19, 13), **kw):
    W, H, D = dims
    s = SceneSettings(gridRes=dims, dx=1.0 / 20, dt=1.0 / 24, domainBboxMin=(-0.3, 0.1, 0.2),
                      domainBboxMax=(-0.3 + W / 20, 0.1 + H / 20, 0.2 + D / 20),
                      closedBounds=(1, 0, 1, 0, 1, 1), maxIterSolve=30)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def random_state(p, seed):
    rng = np.random.default_rng(seed)
    return {
        "T": rng.uniform(0.0, 2.0, p.field_shape("T")),
        "U": 0.5 * rng.standard_normal(p.field_shape("U")),
        "V": 0.5 * rng.standard_normal(p.field_shape("V")),
        "W": 0.5 * rng.standard_normal(p.field_shape("W")),
        "P": rng.standard_normal(p.field_shape("P")),
        "RHS": rng.standard_normal(p.field_shape("RHS")),
    }


def pair(scn, seed, fields=("T", "U", "V", "W", "P", "RHS")):
    """A GPU solver and an FP64 oracle state loaded with the same inputs."""
    from blaze_b200 import FluidSolver
    from oracle import oracle
    p = scn.to_params()
    st = random_state(p, seed)
    gpu = FluidSolver(Timer(), scn)
    ref = oracle.State(p, np.float64)
    for f in fields:
        x = st[f].astype(np.float32)
        gpu.set(f, x)
        getattr(ref, f)[...] = x
    return gpu, ref


def assert_close(gpu, ref, fields, rel=STAGE_REL, absol=STAGE_ABS):
    for f in fields:
        g = gpu.get(f)
        r = getattr(ref, f)
        scale = max(1.0, float(np.max(np.abs(r))))
        e_rel, e_abs = rel_l2(g, r), max_abs(g, r) / scale
        assert e_rel <= rel and e_abs <= absol, f"{f}: rel_l2 {e_rel:.3e} scaled max {e_abs:.3e}"


def test_perlin_bit_exact():
    """Gradient noise on the GPU equals the oracle's FP32 value bit for bit,
    including the float-rounded lattice hash (cuda_noise.cuh:120-124)."""
    import ctypes as C
    from blaze_b200 import _lib
    from oracle import oracle
    rng = np.random.default_rng(5)
    pos = np.concatenate([rng.uniform(-20, 300, (3000, 3)), rng.uniform(0, 25000, (1000, 3)),
                          np.floor(rng.uniform(0, 64, (200, 3)))]).astype(np.float32)
    for scale, seed in ((0.25, 123), (1.6, 456), (0.125, 789), (1.0, 123)):
        out = np.empty(len(pos), np.float32)
        lib = _lib.load()
        _lib.check(lib.blz_perlin(pos.ctypes.data_as(C.POINTER(C.c_float)), len(pos), scale, seed,
                                  out.ctypes.data_as(C.POINTER(C.c_float))))
        want = np.array([oracle.perlin(*p, scale, seed) for p in pos], np.float32)
        np.testing.assert_array_equal(out, want)


def test_source_splat():
    scn = scene()
    from blaze_b200 import FluidSolver
    from oracle import oracle
    rng = np.random.default_rng(11)
    p = scn.to_params()
    n = 400
    lo = np.array(scn.domainBboxMin) - 0.05
    hi = np.array(scn.domainBboxMax) + 0.05
    rec = np.zeros((n, 8), np.float32)
    rec[:, :3] = rng.uniform(lo, hi, (n, 3))
    rec[:, 3:6] = rng.standard_normal((n, 3)) * (rng.uniform(size=(n, 1)) < 0.7)
    rec[:, 6] = rng.uniform(0.0, 5.0, n) * p.dx          # some below the dx/2 cut
    rec[:, 7] = rng.uniform(-0.5, 2.0, n)
    base = random_state(p, 12)
    gpu = FluidSolver(Timer(), scn)
    ref = oracle.State(p, np.float64)
    for f in ("T", "U", "V", "W"):
        gpu.set(f, base[f].astype(np.float32))
        getattr(ref, f)[...] = base[f].astype(np.float32)
    gpu.setParticles(rec)
    gpu.addSource()
    ref.add_source(rec)
    # atomics reorder the float sums: 1e-5 relative is the bar here
    assert_close(gpu, ref, ("T", "U", "V", "W"), rel=1e-5, absol=1e-4)
    # second frame: accumulators were re-zeroed
    gpu.addSource()
    ref.add_source(rec)
    assert_close(gpu, ref, ("T", "U", "V", "W"), rel=1e-5, absol=1e-4)


@pytest.mark.parametrize("kw", [
    dict(vorticityConf=0.4),
    dict(buoyancy=1.7),
    dict(windAmp=0.3, windDir=0, windSpeed=0.7, windTurbAmp=0.5, windTurbScale=0.3),
    dict(windAmp=0.2, windDir=3, windSpeed=0.2, windTurbAmp=0.8, windTurbScale=0.5),
    dict(turbulence_amp=0.5, turbulence_scale=4.0),
    dict(turbulence_amp=0.8, turbulence_scale=2.5, turbMaskTempRamp=(0.2, 1.5), turbMaskVelRamp=(0.1, 0.9)),
    dict(coolingRate=0.35, drag=0.2),
    dict(vorticityConf=0.5, buoyancy=1.0, windAmp=0.2, windTurbAmp=0.3, windTurbScale=0.4,
         turbulence_amp=0.5, turbulence_scale=4.0, coolingRate=0.1),
], ids=["vorticity", "buoyancy", "wind_x", "wind_z", "turbulence", "turbulence_ramps", "cool_drag", "all"])
def test_forces(kw):
    gpu, ref = pair(scene(**kw), 21)
    gpu.forces(1.37)
    ref.forces(1.37)
    assert_close(gpu, ref, ("T", "U", "V", "W"))


@pytest.mark.parametrize("bounds", [(1, 1, 1, 1, 1, 1), (1, 0, 1, 0, 1, 1), (0, 0, 0, 0, 0, 0), (0, 1, 1, 0, 0, 1)])
def test_divergence(bounds):
    gpu, ref = pair(scene(closedBounds=bounds), 31)
    gpu.divergence()
    ref.divergence()
    assert_close(gpu, ref, ("RHS",))


@pytest.mark.parametrize("order", [BLZ_GS_RB3D, BLZ_GS_PLANE])
@pytest.mark.parametrize("bc", [BLZ_BC_REF_COMPAT, BLZ_BC_FREE_SURFACE])
@pytest.mark.parametrize("dims", [(24, 19, 13), (22, 9, 11), (64, 8, 6)], ids=["w24", "w22", "w64"])
def test_gs_sweeps(order, bc, dims):
    """W % 8 == 0 takes the 4-cells-per-thread kernel, other even W the
    one-cell kernel; both must equal the oracle's sweeps."""
    gpu, ref = pair(scene(dims=dims, gs_order=order, bc_mode=bc, maxIterSolve=30), 41)
    gpu.solve()
    ref.gs_sweeps(30)
    assert_close(gpu, ref, ("P",), rel=2e-5, absol=2e-4)


def test_residual_fp64():
    gpu, ref = pair(scene(bc_mode=BLZ_BC_FREE_SURFACE), 51)
    r, b = gpu.residual()
    rr, bb = ref.residual_norms()
    assert r == pytest.approx(rr, rel=1e-6) and b == pytest.approx(bb, rel=1e-6)


def test_solve_to_tolerance_matches_oracle_schedule():
    scn = scene(dims=(32, 24, 20), bc_mode=BLZ_BC_FREE_SURFACE, tol=1e-4, maxIterSolve=3000, check_every=10)
    gpu, ref = pair(scn, 61)
    st = gpu.solve()
    it, r, b = ref.solve()
    assert st["converged"] and st["rel_residual"] <= 1e-4
    assert abs(st["iterations"] - it) <= 10
    assert_close(gpu, ref, ("P",), rel=2e-4, absol=2e-3)


@pytest.mark.parametrize("bc", [BLZ_BC_REF_COMPAT, BLZ_BC_FREE_SURFACE])
@pytest.mark.parametrize("bounds", [(1, 1, 1, 1, 1, 1), (1, 0, 1, 0, 1, 1), (0, 0, 0, 0, 0, 0)])
def test_gradient(bc, bounds):
    gpu, ref = pair(scene(closedBounds=bounds, bc_mode=bc), 71)
    gpu.gradient()
    ref.gradient()
    assert_close(gpu, ref, ("U", "V", "W"))


@pytest.mark.parametrize("scheme", [0, 1, 2], ids=["rk3", "euler", "rk2"])
def test_advect(scheme):
    gpu, ref = pair(scene(advect_scheme=scheme), 81)
    gpu.advect()
    ref.advect()
    assert_close(gpu, ref, ("T", "U", "V", "W"))


@pytest.mark.parametrize("bc,defect", [(BLZ_BC_REF_COMPAT, 0), (BLZ_BC_FREE_SURFACE, 0), (BLZ_BC_FREE_SURFACE, 1)],
                         ids=["ref_compat", "free_surface", "free_surface_defect"])
def test_full_steps_against_oracle(bc, defect):
    """Whole frames (sourcing + step) of a 32^3 plume with every force on,
    after 1 and after 10 steps; with defect correction the sweeps run on the
    correction to the previous pressure (the same iterates in exact
    arithmetic as the oracle's sweeps of p)."""
    from blaze_b200 import FluidSolver
    from oracle import oracle
    scn, parts = plume_scene(n=32, seed=9, particles=800)
    scn.bc_mode = bc
    scn.defect_correction = defect
    scn.windAmp, scn.windTurbAmp, scn.windTurbScale, scn.windSpeed = 0.1, 0.3, 0.5, 0.3
    scn.turbulence_amp, scn.turbulence_scale = 0.3, 4.0
    scn.maxIterSolve = 40
    p = scn.to_params()
    tmr = Timer()
    gpu = FluidSolver(tmr, scn, particles=parts)
    ref = oracle.State(p, np.float64)
    for n in range(10):
        gpu.addSource()
        gpu.step(tmr.time)
        ref.add_source(parts)
        ref.step(tmr.time)
        tmr.iter += 1
        tmr.time += scn.dt
        if n == 0:
            assert_close(gpu, ref, ("T", "U", "V", "W", "P"), rel=2e-5, absol=2e-4)
    assert_close(gpu, ref, ("T", "U", "V", "W", "P"), rel=2e-3, absol=2e-2)


def test_step_is_deterministic():
    from blaze_b200 import FluidSolver
    scn, parts = plume_scene(n=32, seed=3, particles=600)
    out = []
    for _ in range(2):
        tmr = Timer()
        s = FluidSolver(tmr, scn, particles=parts)
        for _ in range(3):
            s.addSource()
            s.step()
            tmr.time += scn.dt
        out.append({f: s.get(f) for f in ("T", "U", "V", "W", "P")})
        s.close()
    for f in out[0]:
        np.testing.assert_array_equal(out[0][f], out[1][f])


def test_error_codes_on_gpu():
    from blaze_b200 import FluidSolver, BlazeError
    scn = scene()
    s = FluidSolver(Timer(), scn)
    bad = np.zeros((1, 8), np.float32)
    bad[0, 0] = np.nan
    with pytest.raises(BlazeError) as e:
        s.setParticles(bad)
    assert e.value.code == -4
    with pytest.raises(BlazeError) as e:
        s.setParticles(np.zeros((scn.sourceMaxParticleCount + 1, 8), np.float32))
    assert e.value.code == -2
    with pytest.raises(BlazeError):
        s.set("T", np.zeros((3, 3, 3), np.float32))


def test_device_loop_matches_host_loop():
    """The graph-run solve (conditional WHILE node deciding on the device)
    follows the host loop's schedule exactly: same sweep count, same checks,
    bitwise the same pressure."""
    from blaze_b200 import FluidSolver
    out = []
    for dl in (0, 1):
        scn = scene(dims=(32, 24, 20), bc_mode=BLZ_BC_FREE_SURFACE, tol=1e-4, maxIterSolve=3000,
                    check_every=10, device_loop=dl)
        gpu, _ = pair(scn, 63)
        st = gpu.solve()
        assert st["device_loop"] == dl
        out.append((st["iterations"], st["residual_checks"], st["converged"], gpu.get("P")))
        gpu.close()
    assert out[0][:3] == out[1][:3]
    np.testing.assert_array_equal(out[0][3], out[1][3])


def test_device_loop_hits_the_cap():
    from blaze_b200 import FluidSolver
    scn = scene(dims=(32, 24, 20), bc_mode=BLZ_BC_FREE_SURFACE, tol=1e-12, maxIterSolve=40, check_every=10)
    gpu, _ = pair(scn, 64)
    st = gpu.solve()
    assert st["device_loop"] == 1 and st["iterations"] == 40 and not st["converged"]
    assert st["residual_checks"] == 5


def test_sweep_variants_are_bitwise_identical():
    """Every launch shape of the segment sweep kernel, and every temporal-
    blocking pass (variants 6-10: TMA-staged, paired FP32), gives the same
    bits."""
    ref = None
    for v in range(11):
        gpu, _ = pair(scene(dims=(64, 20, 18), bc_mode=BLZ_BC_FREE_SURFACE, sweep_variant=v), 65)
        gpu.sweeps(7)
        p = gpu.get("P")
        gpu.close()
        if ref is None:
            ref = p
        else:
            np.testing.assert_array_equal(p, ref, err_msg=f"variant {v}")


def test_fixed_sweeps_match_oracle():
    gpu, ref = pair(scene(dims=(40, 16, 12), bc_mode=BLZ_BC_FREE_SURFACE), 66)
    gpu.sweeps(12)
    ref.gs_sweeps(12)
    assert_close(gpu, ref, ("P",), rel=2e-5, absol=2e-4)


def test_sweep_variants_identical_full_width_rows():
    """W = 256: a warp spans a whole packed row (32 segments of 4)."""
    ref = None
    for v in range(11):
        gpu, _ = pair(scene(dims=(256, 6, 8), bc_mode=BLZ_BC_FREE_SURFACE, sweep_variant=v), 67)
        gpu.sweeps(5)
        p = gpu.get("P")
        gpu.close()
        assert np.isfinite(p).all()
        if ref is None:
            ref = p
        else:
            np.testing.assert_array_equal(p, ref, err_msg=f"variant {v}")


@pytest.mark.parametrize("dims,bc", [((64, 200, 70), BLZ_BC_FREE_SURFACE), ((256, 40, 40), BLZ_BC_FREE_SURFACE),
                                     ((384, 20, 12), BLZ_BC_REF_COMPAT), ((128, 48, 33), BLZ_BC_FREE_SURFACE),
                                     ((256, 512, 64), BLZ_BC_FREE_SURFACE)])
def test_temporal_blocking_equals_plain_sweeps(dims, bc):
    """The two-sweeps-per-pass kernels (variants 6-10, 9 with TMA-staged rhs
    and input planes, 10 with the stencil on paired FP32 instructions:
    several row bands and z chunks here; 256 x 512 x 64 has 32 row bands and
    chunks of 16 planes, so its steady steps run in long stretches) give the
    plain segment kernel's bits."""
    out = {}
    for v in (0, 6, 7, 8, 9, 10):
        gpu, _ = pair(scene(dims=dims, bc_mode=bc, sweep_variant=v), 68)
        gpu.sweeps(10)
        out[v] = gpu.get("P")
        gpu.close()
    assert np.isfinite(out[0]).all() and np.abs(out[0]).max() > 0
    for v in (6, 7, 8, 9, 10):
        np.testing.assert_array_equal(out[v], out[0], err_msg=f"variant {v}")


# ---------------------------------------------------------------------------
# Target mode's density scalar (no reference counterpart): sourcing,
# buoyancy V += dt (beta T - alpha rho) g and advection against the oracle.
# ---------------------------------------------------------------------------
def dens_pair(scn, seed):
    """pair() plus a random density field on both sides."""
    gpu, ref = pair(scn, seed)
    rng = np.random.default_rng(seed + 1000)
    d = rng.uniform(0.0, 1.5, ref.DENSITY.shape).astype(np.float32)
    gpu.set("DENSITY", d)
    ref.DENSITY[...] = d
    return gpu, ref


def test_density_source_splat():
    from blaze_b200 import FluidSolver
    from oracle import oracle
    scn = scene(density_field=1, buoyancy_alpha=0.05)
    p = scn.to_params()
    rng = np.random.default_rng(13)
    n = 300
    rec = np.zeros((n, 8), np.float32)
    rec[:, :3] = rng.uniform(np.array(scn.domainBboxMin) - 0.05, np.array(scn.domainBboxMax) + 0.05, (n, 3))
    rec[:, 6] = rng.uniform(0.0, 5.0, n) * p.dx
    rec[:, 7] = rng.uniform(-0.5, 2.0, n)
    dens = rng.uniform(0.0, 1.0, n).astype(np.float32)
    dens[::7] = 0.0                                   # skipped channel
    gpu = FluidSolver(Timer(), scn)
    ref = oracle.State(p, np.float64)
    gpu.setParticles(rec, dens)
    gpu.addSource()
    ref.add_source(rec, density=dens)
    assert np.abs(ref.DENSITY).max() > 0.1
    assert_close(gpu, ref, ("T", "DENSITY"), rel=1e-5, absol=1e-4)
    # without explicit densities every particle carries 1
    gpu2 = FluidSolver(Timer(), scn)
    ref2 = oracle.State(p, np.float64)
    gpu2.setParticles(rec)
    gpu2.addSource()
    ref2.add_source(rec)
    assert_close(gpu2, ref2, ("DENSITY",), rel=1e-5, absol=1e-4)


@pytest.mark.parametrize("beta,alpha", [(1.0, 0.05), (0.0, 0.7), (1.5, -0.3)])
def test_density_buoyancy(beta, alpha):
    gpu, ref = dens_pair(scene(buoyancy=beta, density_field=1, buoyancy_alpha=alpha, vorticityConf=0.2), 23)
    gpu.forces(0.4)
    ref.forces(0.4)
    assert_close(gpu, ref, ("T", "U", "V", "W", "DENSITY"))


def test_density_advect():
    gpu, ref = dens_pair(scene(density_field=1, buoyancy_alpha=0.05), 83)
    gpu.advect()
    ref.advect()
    assert_close(gpu, ref, ("T", "U", "V", "W", "DENSITY"))


def test_density_off_is_the_reference_step():
    """density_field = 1 with alpha = 0 changes no field of the reference's
    step: the scalar is carried alongside, bit for bit the same T, U, V, W, P."""
    from blaze_b200 import FluidSolver
    out = []
    for dens in (0, 1):
        scn, parts = plume_scene(n=32, seed=4, particles=600)
        scn.density_field, scn.buoyancy_alpha = dens, 0.0
        tmr = Timer()
        with FluidSolver(tmr, scn, particles=parts) as s:
            for _ in range(3):
                s.addSource()
                s.step(tmr.time)
                tmr.time += scn.dt
            out.append({f: s.get(f) for f in ("T", "U", "V", "W", "P")})
    for f in out[0]:
        np.testing.assert_array_equal(out[0][f], out[1][f], err_msg=f)


def test_tight_solve_reaches_the_fp64_solution():
    """blz_tight_solve (FP64 SOR, training targets) returns the pressure
    system's solution: its FP64 relative residual meets tol, and the result
    equals the FP64 oracle's converged Gauss-Seidel solution within FP32
    rounding."""
    from oracle import oracle
    scn = scene(dims=(16, 16, 8), bc_mode=BLZ_BC_FREE_SURFACE, tol=1e-12, maxIterSolve=200000, check_every=200)
    gpu, ref = pair(scn, 91)
    sweeps, rel = gpu.tight_solve(1e-10, 20000, 1.8)
    assert rel <= 1e-10 and 0 < sweeps <= 20000
    it, r, b = ref.solve()
    assert r / b <= 1e-12
    p = gpu.get("P")
    assert rel_l2(p, ref.P) <= 1e-6 and max_abs(p, ref.P) <= 1e-6 * np.abs(ref.P).max()


def _smooth_rhs(p, scale):
    """A low-frequency right-hand side: its solution is smooth and large
    against ||b||, the case where FP32 storage of p sets a residual floor."""
    D, H, W = p.field_shape("RHS")
    z, y, x = np.meshgrid((np.arange(D) + 0.5) / D, (np.arange(H) + 0.5) / H, (np.arange(W) + 0.5) / W,
                          indexing="ij")
    return (scale * np.sin(np.pi * x) * np.sin(np.pi * z) * (1.0 + 0.3 * np.cos(np.pi * y))).astype(np.float32)


def test_defect_correction_passes_the_fp32_floor():
    """On a smooth 32^3 problem the FP32 iterate stalls near its rounding
    floor (2e-7 ||p|| / ||b||, a few 1e-5 here) while the defect-correction
    solve reaches relative residual 1e-7, and its pressure p + delta is the
    FP64 oracle's solution to within FP32 rounding of p."""
    from blaze_b200 import FluidSolver
    from oracle import oracle
    out = {}
    for defect in (0, 1):
        scn = SceneSettings(gridRes=(32, 32, 32), dx=1.0 / 32, dt=1.0 / 24, closedBounds=(1, 1, 1, 0, 1, 1),
                            bc_mode=BLZ_BC_FREE_SURFACE, tol=1e-7, maxIterSolve=20000, check_every=100,
                            defect_correction=defect)
        p = scn.to_params()
        rhs = _smooth_rhs(p, 10.0)
        with FluidSolver(Timer(), scn) as s:
            s.set("RHS", rhs)
            st = s.solve()
            out[defect] = (st, s.get("P"))
    plain, corr = out[0][0], out[1][0]
    assert not plain["converged"], plain
    assert corr["converged"] and corr["rel_residual"] <= 1e-7, corr
    ref = oracle.State(p, np.float64)
    ref.RHS[...] = rhs
    q = p.copy()
    q.tol, q.max_iter, q.check_every = 1e-11, 400000, 1000
    ref.p = q
    _, r, b = ref.solve()
    assert r / b <= 1e-11
    got = out[1][1]
    assert rel_l2(got, ref.P) <= 1e-6, rel_l2(got, ref.P)


def test_defect_correction_gradient_and_device_loop():
    """The device-loop solve with defect correction follows the host loop
    exactly (sweeps, checks, bits of p), and the gradient of p + delta
    matches the oracle's gradient of its own solution."""
    from blaze_b200 import FluidSolver
    out = []
    for dl in (0, 1):
        scn = scene(dims=(32, 24, 20), bc_mode=BLZ_BC_FREE_SURFACE, tol=1e-5, maxIterSolve=4000, check_every=10,
                    device_loop=dl, defect_correction=1)
        gpu, ref = pair(scn, 93)
        st = gpu.solve()
        gpu.gradient()
        out.append((st["iterations"], st["residual_checks"], st["converged"], gpu.get("P"), gpu.get("U")))
        if dl:
            q = scn.to_params()
            q.tol, q.max_iter = 0.0, st["iterations"]
            ref.p = q
            ref.solve()
            ref.gradient()
            assert_close(gpu, ref, ("P", "U", "V", "W"), rel=2e-4, absol=2e-3)
        gpu.close()
    assert out[0][:3] == out[1][:3]
    np.testing.assert_array_equal(out[0][3], out[1][3])
    np.testing.assert_array_equal(out[0][4], out[1][4])


_TUNE_CHILD = r"""
import sys, json
sys.path.insert(0, sys.argv[1])
from blaze_b200 import FluidSolver, SceneSettings, Timer, BLZ_BC_FREE_SURFACE
scn = SceneSettings(gridRes=(256, 40, 40), dx=1.0 / 20, bc_mode=BLZ_BC_FREE_SURFACE, maxIterSolve=8)
with FluidSolver(Timer(), scn) as s:
    st = s.solve()
print(json.dumps({"variant": st["sweep_variant"]}))
"""


def test_sweep_autotuner_choice_persists(tmp_path):
    """The tuner's choice goes to the cache file (BLZ_TUNE_CACHE); a later
    process with an entry for its device and grid takes that entry instead of
    tuning (the last entry for a key wins)."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cache = tmp_path / "tune.txt"
    env = dict(os.environ, BLZ_TUNE_CACHE=str(cache))
    env.pop("BLZ_SWEEP_VARIANT", None)

    def child():
        r = subprocess.run([sys.executable, "-c", _TUNE_CHILD, root], env=env, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        return json.loads(r.stdout.strip().splitlines()[-1])["variant"]

    first = child()
    lines = cache.read_text().split("\n")
    key, v = lines[0].split()
    assert int(v) == first and key.endswith("|256|40|40|11|11")
    forced = (first + 1) % 11
    with open(cache, "a") as f:
        f.write(f"{key} {forced}\n")
    assert child() == forced
