"""Blaze scene files (.blz JSON) and the frame loop that drives them.

``load_blz`` reads the solver fields the reference's Parser::sceneParse reads
(src/Parser.h:41-171) into a SceneSettings; renderer fields are kept in
``extra`` (``render.render_params_from_blz`` turns them into the renderer's
parameters).  ``particle_file`` applies the reference's animated-source
naming (src/Parser.h:181-188), and ``run`` is the frame loop of
src/main.cu:89-106, rendering the frames in renderRange when asked:

    python -m blaze_b200.scenefile scene.blz [--frames N] [--render]
"""
import argparse
import json
import os
import sys

from . import _abi
from .scenes import SceneSettings, Timer, read_part

# .blz key -> SceneSettings field, for the scalar solver parameters.
_SCALARS = {
    "maxIterSolve": "maxIterSolve", "dx": "dx", "dt": "dt", "density": "density", "gravity": "gravity",
    "coolingRate": "coolingRate", "buoyancy": "buoyancy", "vorticityConf": "vorticityConf", "drag": "drag",
    "windAmp": "windAmp", "windSpeed": "windSpeed", "windTurbAmp": "windTurbAmp",
    "windTurbScale": "windTurbScale", "windDir": "windDir", "turbulenceAmp": "turbulence_amp",
    "turbulenceScale": "turbulence_scale", "sourceMaxParticleCount": "sourceMaxParticleCount",
}


class SceneFile:
    """A parsed .blz scene: solver settings plus the source and frame ranges."""

    def __init__(self, settings, scene_dir, particle_file, animated, source_range, render_range, raw):
        self.settings = settings
        self.scene_dir = scene_dir
        self.particle_file_name = particle_file
        self.animated = animated
        self.source_range = source_range
        self.render_range = render_range
        self.raw = raw

    def particle_file(self, frame):
        """Path of the particle cache the reference reads for `frame`: an
        animated source replaces the last 10 characters of particleFile
        ("_0001.part") by "_%04d.part" of the frame (Parser.h:181-188)."""
        if self.animated:
            stem = self.particle_file_name[:-10]
            return os.path.join(self.scene_dir, f"{stem}_{frame:04d}.part")
        return os.path.join(self.scene_dir, self.particle_file_name)


def load_blz(path):
    with open(path) as f:
        d = json.load(f)
    s = SceneSettings()
    s.gridRes = tuple(int(v) for v in d["gridRes"])
    s.domainBboxMin = tuple(float(v) for v in d["domainBboxMin"])
    s.domainBboxMax = tuple(float(v) for v in d["domainBboxMax"])
    s.closedBounds = tuple(int(bool(v)) for v in d["closedBounds"])
    for key, field in _SCALARS.items():
        if key in d:
            cur = getattr(s, field)
            setattr(s, field, type(cur)(d[key]))
    s.turbMaskTempRamp = tuple(float(v) for v in d.get("turbMaskTempRamp", s.turbMaskTempRamp))
    s.turbMaskVelRamp = tuple(float(v) for v in d.get("turbMaskVelRamp", s.turbMaskVelRamp))
    # the reference's solve: maxIterSolve sweeps, warm started, Neumann faces
    s.tol, s.bc_mode, s.reset_pressure = 0.0, _abi.BLZ_BC_REF_COMPAT, 0
    s.extra = {k: v for k, v in d.items() if k not in _SCALARS}
    source_range = (int(float(d["sourceRange"][0])), int(float(d["sourceRange"][1])))
    render_range = (int(float(d["renderRange"][0])), int(float(d["renderRange"][1])))
    scene_dir = os.path.dirname(os.path.realpath(path))
    return SceneFile(s, scene_dir, d["particleFile"], bool(int(d["sourceAnimated"])), source_range,
                     render_range, d)


def run(scene, frames=None, on_frame=None, render=False):
    """The reference's frame loop (main.cu:89-106): frames run from
    sourceRange.x to renderRange.y; while iter <= sourceRange.y a frame
    sources particles first; a static source's file is read once
    (FluidSolver.cu:775-794); with `render`, a frame inside renderRange is
    rendered and written under the reference's file name (main.cu:96-99).
    Returns the per-frame step statistics."""
    from .solver import FluidSolver
    tmr = Timer(iter=scene.source_range[0], time=0.0)
    last = scene.render_range[1] if frames is None else scene.source_range[0] + frames - 1
    stats = []
    loaded = False
    engine = None
    if render:
        from .render import RenderEngine, render_params_from_blz
        engine = RenderEngine(tmr, scene.settings, render_params_from_blz(scene.raw))
    try:
        with FluidSolver(tmr, scene.settings) as solver:
            while tmr.iter <= last:
                if tmr.iter <= scene.source_range[1]:
                    if scene.animated or not loaded:
                        solver.setParticles(read_part(scene.particle_file(tmr.iter)))
                        loaded = True
                    solver.addSource()
                st = solver.step()
                if engine is not None and scene.render_range[0] <= tmr.iter <= scene.render_range[1]:
                    st["ms_render"] = engine.render(solver)
                    st["render_file"] = engine.writeToDisk(scene)
                stats.append(st)
                if on_frame is not None:
                    on_frame(tmr.iter, solver, st)
                tmr.iter += 1
                tmr.time += scene.settings.dt
    finally:
        if engine is not None:
            engine.close()
    return stats


def main(argv=None):
    ap = argparse.ArgumentParser(description="Run a Blaze .blz scene through the B200 fluid step")
    ap.add_argument("scene")
    ap.add_argument("--frames", type=int, default=None)
    ap.add_argument("--render", action="store_true", help="render frames in renderRange (main.cu:96-99)")
    a = ap.parse_args(argv)
    sc = load_blz(a.scene)
    for n, st in enumerate(run(sc, a.frames, render=a.render)):
        print(f"frame {sc.source_range[0] + n:04d}: {st['ms_total']:.2f} ms, "
              f"{st['iterations']} sweeps, rel. residual {st['rel_residual']:.2e}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
