"""Batched simulations against the same simulations stepped one by one: every
field of every grid, and every solve's sweep count and residual, must be
identical bit for bit (the batch runs the single-grid kernels' per-cell code
and stopping rule)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("T", "U", "V", "W", "P")


def _make(scenes):
    from blaze_b200 import FluidSolver, Timer
    return [FluidSolver(Timer(), s, particles=p) for s, p in scenes]


def _scenes(turbulence=False):
    from blaze_b200.scenes import batch_scenes
    dims = [(16, 16, 16), (24, 16, 16), (32, 24, 16), (16, 32, 24), (40, 16, 24)]
    sc = batch_scenes(5, seed=11, tol=1e-4, max_iter=4000, check_every=10, dims=dims)
    if turbulence:
        sc[1][0].turbulence_amp, sc[1][0].turbulence_scale = 0.3, 4.0
    return sc


@pytest.mark.parametrize("turbulence", [False, True], ids=["frame-graph", "direct"])
def test_batch_equals_single(turbulence):
    from blaze_b200.batch import Batch
    frames = 4
    single = _make(_scenes(turbulence))
    single_stats = [[] for _ in single]
    for f in range(frames):
        for i, s in enumerate(single):
            s.addSource()
            single_stats[i].append(s.step(f / 24.0))
    batched = _make(_scenes(turbulence))
    batch = Batch(batched)
    batch_stats = []
    for f in range(frames):
        batch.add_source()
        batch_stats.append(batch.step([f / 24.0] * len(batched)))
    assert batch.kernel_launches() > 0
    batch.close()
    for i in range(len(single)):
        assert all(st["iterations"] > 0 and st["rhs_norm"] > 0 for st in single_stats[i]), i
        for f in range(frames):
            a, b = single_stats[i][f], batch_stats[f][i]
            assert a["iterations"] == b["iterations"] and a["residual_checks"] == b["residual_checks"], (i, f, a, b)
            assert a["residual"] == b["residual"] and a["converged"] == b["converged"]
        for name in FIELDS:
            assert np.array_equal(single[i].get(name), batched[i].get(name)), (i, name)
    for s in single + batched:
        s.close()


def test_batch_solve_only():
    from blaze_b200.batch import Batch
    sims = _make(_scenes())
    for s in sims:
        s.addSource()
        s.forces(0.0)
        s.divergence()
    batch = Batch(sims)
    stats = batch.solve()
    assert all(st["converged"] for st in stats)
    for s, st in zip(sims, stats):
        r, b = s.residual()
        assert b > 0 and st["iterations"] > 0
        assert r / b <= 1e-4 and abs(r - st["residual"]) <= 1e-12 * max(r, 1e-30)
    batch.close()


def test_batch_rejects_mismatched_solvers():
    import ctypes as C
    from blaze_b200 import FluidSolver, Timer, _lib
    from blaze_b200.scenes import batch_scenes
    lib = _lib.load()
    sc = batch_scenes(2, seed=3, tol=1e-4, max_iter=400, dims=[(16, 16, 16)])
    sc[1][0].check_every = 10
    sims = [FluidSolver(Timer(), s) for s, _ in sc]
    arr = (C.c_void_p * 2)(*[s._h.value for s in sims])
    h = C.c_void_p()
    assert lib.blz_batch_create(arr, 2, C.byref(h)) == -2
    sc2 = batch_scenes(1, seed=3, tol=1e-4, max_iter=400, dims=[(20, 16, 16)])
    s2 = FluidSolver(Timer(), sc2[0][0])
    arr2 = (C.c_void_p * 1)(s2._h.value)
    assert lib.blz_batch_create(arr2, 1, C.byref(h)) == -2          # width % 8 != 0
    for s in sims + [s2]:
        s.close()


@pytest.mark.parametrize("turbulence", [False, True], ids=["frame-graph", "direct"])
def test_batch_with_warm_start_equals_single(turbulence):
    """Solvers with an attached network (one per grid size, shared by the
    solvers of that size) warm-start inside the batch exactly as alone: same
    sweeps, residuals and fields, bit for bit."""
    from blaze_b200.batch import Batch
    from blaze_b200.unet import WarmStartUNet, init_params
    frames = 3
    params = init_params(2)
    nets = {}

    def net_for(dims):
        if dims not in nets:
            nets[dims] = WarmStartUNet(dims, params, kappa=0.5)
            nets[dims].set_smoothing(8)
        return nets[dims]

    runs = []
    for batched in (False, True):
        sims = _make(_scenes(turbulence))
        for s in sims:
            s.set_warm_start(net_for(tuple(s.scn.gridRes)))
        stats = []
        if batched:
            batch = Batch(sims)
            for f in range(frames):
                batch.add_source()
                stats.append(batch.step([f / 24.0] * len(sims)))
            batch.close()
        else:
            for f in range(frames):
                row = []
                for s in sims:
                    s.addSource()
                    row.append(s.step(f / 24.0))
                stats.append(row)
        runs.append((stats, [{k: s.get(k) for k in FIELDS} for s in sims]))
        for s in sims:
            s.close()
    (sa, fa), (sb, fb) = runs
    for f in range(frames):
        for i in range(len(sa[f])):
            a, b = sa[f][i], sb[f][i]
            assert a["warm_started"] == 1 and b["warm_started"] == 1
            assert a["iterations"] == b["iterations"] and a["residual"] == b["residual"], (f, i, a, b)
    for i in range(len(fa)):
        for name in FIELDS:
            assert np.array_equal(fa[i][name], fb[i][name]), (i, name)
    for n in nets.values():
        n.close()


# Temporal blocking in a batch: one band (16^2 rows), two bands with a ragged
# second one (96 rows of 80 per tile), 8-row tiles of 48 quads (width 384),
# an odd depth, and a small grid.
TB_DIMS = [(16, 16, 16), (64, 96, 40), (384, 20, 12), (48, 40, 31), (32, 24, 16)]


def _tb_scenes():
    from blaze_b200.scenes import batch_scenes
    return [batch_scenes(1, seed=20 + i, tol=1e-4, max_iter=4000, check_every=20, dims=[d])[0]
            for i, d in enumerate(TB_DIMS)]


def _run_frames(sims, frames, batch_planes=None, paired=False):
    from blaze_b200.batch import Batch
    stats = []
    if batch_planes is None:
        for f in range(frames):
            row = []
            for s in sims:
                s.addSource()
                row.append(s.step(f / 24.0))
            stats.append(row)
        return stats
    batch = Batch(sims)
    batch.set_sweep(batch_planes, paired)
    for f in range(frames):
        batch.add_source()
        stats.append(batch.step([f / 24.0] * len(sims)))
    batch.close()
    return stats


@pytest.mark.parametrize("planes,paired", [(-1, False), (0, False), (8, False), (16, False), (32, False),
                                           (8, True), (32, True)])
def test_batch_sweep_kernels_equal_single(planes, paired):
    """Every sweep kernel of the batch (autotuned, segment, temporal blocking
    with 8, 16 or 32 planes per tile, scalar or paired-FP32 stencil) gives
    each grid the sweeps, residuals and fields of its own solve, bit for
    bit."""
    frames = 3
    single = _make(_tb_scenes())
    sa = _run_frames(single, frames)
    batched = _make(_tb_scenes())
    sb = _run_frames(batched, frames, planes, paired)
    for f in range(frames):
        for i in range(len(single)):
            a, b = sa[f][i], sb[f][i]
            assert a["iterations"] > 0 and a["iterations"] == b["iterations"], (planes, f, i, a, b)
            assert a["residual"] == b["residual"] and a["converged"] == b["converged"], (planes, f, i)
            if planes > 0:
                assert b["sweep_variant"] == (200 if paired else 100) + planes
            elif planes == 0:
                assert b["sweep_variant"] in (1, 2, 4, 8)
    for i in range(len(single)):
        for name in FIELDS:
            assert np.array_equal(single[i].get(name), batched[i].get(name)), (planes, i, name)
    for s in single + batched:
        s.close()


def test_batch_temporal_blocking_needs_four_sweep_checks():
    """check_every = 10 (not a multiple of 4) leaves only the segment kernel."""
    from blaze_b200.batch import Batch
    from blaze_b200.scenes import batch_scenes
    sims = _make(batch_scenes(2, seed=3, tol=1e-4, max_iter=400, check_every=10, dims=[(16, 16, 16)]))
    batch = Batch(sims)
    with pytest.raises(RuntimeError):
        batch.set_sweep(16)
    batch.set_sweep(0)
    batch.close()
    for s in sims:
        s.close()
