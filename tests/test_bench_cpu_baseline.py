"""bench.py's cpu_baseline leg on CPU: the FP64 oracle timed on a bounded
sample of a frame with all host threads, plus a few sweeps on one thread,
and the thread count restored afterwards (no GPU)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpu_baseline_reports_all_core_and_one_core_sweeps():
    sys.path.insert(0, ROOT)
    import bench
    from blaze_b200.scenes import family_scene
    from oracle import oracle
    scn, parts = family_scene(n=32, seed=3, tol=1e-4, max_iter=4000, check_every=20)
    cores = oracle.num_threads()
    r = bench.cpu_baseline(scn, parts, 1000.0)
    assert oracle.num_threads() == cores
    assert r["kind"] == "port" and r["unit"] == "steps/s" and r["cores"] == cores
    assert r["value"] > 0 and r["ms_per_sweep"] > 0 and r["ms_per_sweep_1core"] > 0
    assert abs(r["value_1core_sweeps_only"] * r["ms_per_sweep_1core"] * 1e-3 * 1000.0 - 1.0) < 1e-9
    assert "on one core" in r["sample"]
