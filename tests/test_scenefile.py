"""The .blz loader and the animated-source file naming (Parser.h:41-188);
the frame loop itself on a GPU."""
import json
import os

import numpy as np
import pytest

from blaze_b200.scenefile import load_blz, run
from blaze_b200 import plume_scene, write_part


def write_scene(tmp, animated, n=32):
    scn = {
        "sceneName": "unit", "particleFile": "src/plume_0001.part", "sourceAnimated": int(animated),
        "sourceRange": [1.0, 3.0, 1.0], "sourceMaxParticleCount": 1000, "renderFile": "r.exr",
        "renderRange": [1, 4, 1], "maxIterSolve": 25, "dx": 1.0 / n, "dt": 1.0 / 24,
        "gridRes": [n, n, n], "renderRes": [64, 64], "domainBboxMin": [0.0, 0.0, 0.0],
        "domainBboxMax": [1.0, 1.0, 1.0], "closedBounds": [1, 1, 1, 0, 1, 1], "density": 0.1,
        "gravity": -9.8, "coolingRate": 0.2, "buoyancy": 1.5, "vorticityConf": 0.3, "drag": 0.0,
        "windAmp": 0.0, "windSpeed": 0.4, "windTurbAmp": 0.0, "windTurbScale": 0.6, "windDir": 2,
        "turbulenceAmp": 0.5, "turbulenceScale": 4.0, "turbMaskTempRamp": [0.1, 0.3],
        "turbMaskVelRamp": [0.0, 10.0], "lightCount": 0,
    }
    path = os.path.join(tmp, "unit.blz")
    with open(path, "w") as f:
        json.dump(scn, f)
    os.makedirs(os.path.join(tmp, "src"), exist_ok=True)
    return path


def test_load_blz_fields(tmp_path):
    path = write_scene(str(tmp_path), animated=True)
    sc = load_blz(path)
    s = sc.settings
    assert s.gridRes == (32, 32, 32) and s.maxIterSolve == 25
    assert s.closedBounds == (1, 1, 1, 0, 1, 1)
    assert s.turbulence_amp == 0.5 and s.turbulence_scale == 4.0 and s.windDir == 2
    assert s.coolingRate == pytest.approx(0.2) and s.sourceMaxParticleCount == 1000
    assert sc.source_range == (1, 3) and sc.render_range == (1, 4)
    assert sc.particle_file(7) == os.path.join(str(tmp_path), "src", "plume_0007.part")
    p = s.to_params()
    assert p.max_iter == 25 and p.tol == 0.0


def test_static_source_file_name(tmp_path):
    sc = load_blz(write_scene(str(tmp_path), animated=False))
    assert sc.particle_file(5) == os.path.join(str(tmp_path), "src", "plume_0001.part")


@pytest.mark.gpu
def test_frame_loop_runs_animated_scene(tmp_path):
    path = write_scene(str(tmp_path), animated=True)
    _, parts = plume_scene(n=32, seed=2, particles=400)
    for frame in (1, 2, 3):
        shifted = parts.copy()
        shifted[:, 1] += 0.01 * frame
        write_part(os.path.join(str(tmp_path), "src", f"plume_{frame:04d}.part"), shifted)
    seen = []
    stats = run(load_blz(path), on_frame=lambda it, s, st: seen.append((it, float(s.get("T").max()))))
    assert [it for it, _ in seen] == [1, 2, 3, 4]
    assert len(stats) == 4 and all(st["iterations"] == 25 for st in stats)
    assert seen[-1][1] > 0.1
