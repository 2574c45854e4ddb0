"""The CUDA path against the reference's own CUDA build, live, on the golden
cases (same seeded inputs, same stage).  Needs a GPU and oracle/_ref.

Tolerance as for the oracle fixtures: relative L2 1e-5 and max-abs
1e-4 * max(1, max|ref|) per stage, 1e-4 / 1e-3 after three whole frames;
racy reference faces (gradient open-face copy across blocks) are excluded.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402
from conftest import max_abs, rel_l2  # noqa: E402
from test_oracle_golden import racy_face_mask  # noqa: E402

pytestmark = pytest.mark.gpu


def run_ours(name):
    from blaze_b200 import FluidSolver, Timer
    ovr, stage, seed, time, outs = cases.CASES[name]
    scn = cases.scene(**ovr)
    p = scn.to_params()
    tmr = Timer(0, time)
    s = FluidSolver(tmr, scn)
    for k, v in cases.inputs(p, seed).items():
        s.set(k, v)
    if stage == "source":
        s.setParticles(cases.particles(p, seed))
        s.addSource()
    elif stage == "step":
        s.setParticles(cases.particles(p, seed))
        for n in range(cases.STEP_FRAMES):
            s.addSource()
            s.step(n * p.dt)
    elif stage in ("vorticity", "buoyancy", "wind", "turbulence"):
        s.forces(time)
    elif stage == "divergence":
        s.divergence()
    elif stage == "gs":
        s.solve()
    elif stage == "gradient":
        s.gradient()
    elif stage == "advect":
        s.advect()
    out = {f: s.get(f) for f in outs}
    s.close()
    return out, p


@pytest.fixture(scope="module")
def reference_outputs(tmp_path_factory):
    """All cases run once through the reference build, in a subprocess: the
    reference's error handling calls exit(), which must not end pytest."""
    import subprocess
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build not present")
    out = tmp_path_factory.mktemp("refcases")
    res = subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_golden.py"), str(out)],
                         capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, "reference build failed:\n" + res.stdout[-3000:] + res.stderr[-3000:]
    return out


@pytest.mark.parametrize("name", list(cases.CASES))
def test_cuda_path_matches_reference_build(name, reference_outputs):
    want = dict(np.load(os.path.join(str(reference_outputs), f"{name}.npz")))
    got, p = run_ours(name)
    tol_rel, tol_abs = (1e-5, 1e-4) if cases.CASES[name][1] != "step" else (1e-4, 1e-3)
    for f, g in want.items():
        m = racy_face_mask(p, f) if cases.CASES[name][1] == "gradient" else np.zeros(g.shape, bool)
        scale = max(1.0, float(np.max(np.abs(g))))
        e_rel = rel_l2(got[f][~m], g[~m])
        e_abs = max_abs(got[f][~m], g[~m]) / scale
        assert e_rel <= tol_rel and e_abs <= tol_abs, f"{name}/{f}: rel {e_rel:.2e} scaled max {e_abs:.2e}"
