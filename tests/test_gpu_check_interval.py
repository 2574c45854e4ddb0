"""The automatic residual-check interval (blz_params.check_every < 0): the
stopping test is unchanged, only how often it runs; every frame still ends
at FP64 relative residual <= tol."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CANDIDATES = {20, 40, 80, 160, 320}


def _run(check_every, frames=5):
    from blaze_b200 import family_scene
    from blaze_b200.scenes import Timer
    from blaze_b200.solver import FluidSolver
    scn, parts = family_scene(n=64, seed=5, tol=1e-4, max_iter=32000, check_every=check_every)
    tmr = Timer()
    stats = []
    with FluidSolver(tmr, scn, parts) as s:
        for _ in range(frames):
            s.addSource()
            stats.append(s.step())
            tmr.iter += 1
            tmr.time += scn.dt
        T = s.get("T")
    return stats, T


def test_auto_interval_keeps_the_stopping_rule():
    stats, T = _run(-1)
    assert all(st["converged"] and st["rel_residual"] <= 1e-4 for st in stats)
    assert stats[0]["check_interval"] == 20                      # no history yet
    assert all(st["check_interval"] in CANDIDATES for st in stats)
    assert all(st["device_loop"] == 1 for st in stats)
    # each interval minimises (N / c) r + c / 2 for the previous frame's N, so
    # it grows with the sweep count
    for prev, st in zip(stats, stats[1:]):
        if prev["iterations"] >= 600:
            assert st["check_interval"] >= 40
    fixed, T20 = _run(20)
    assert all(st["converged"] for st in fixed)
    # the two runs stop at different sweep counts, both within tol: the
    # temperature fields stay close
    assert np.linalg.norm(T - T20) <= 1e-2 * np.linalg.norm(T20)
