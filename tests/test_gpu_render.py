"""The CUDA renderer (render.cu) against the oracle's restatement of the
reference's render pass (oracle/render_oracle.cpp) and against the
reference's own RenderEngine (src/RenderEngine.cu, built from its sources
into oracle/_ref and run on the same GPU).

Tolerances:
  texture sampler: per-axis weights exactly the fraction rounded half up to
    1/256; corner weights multiples of 1/256 summing to one; general samples
    within 2 max|T| / 256 of the oracle's model of the filter (a corner
    weight off by one 1/256 unit) and 2e-4 max|T| on average.
  images (relative L2 over the image):
  image vs oracle: RENDER_TOL.  The two march the same samples in FP32;
    they differ by the GPU's fused multiply-adds in ray positions (which can
    move a sample across a 1/256 filter-weight step) and by expf rounding.
  image vs the reference build: bit for bit.  Both sample through the same
    texture hardware and use the same fast-math intrinsics (the reference's
    documented build flags) in the same order; the empty-space skipping of
    the CUDA path only drops samples the cutoff test rejects.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RENDER_TOL = 5e-3
SAMPLER_QUANT = 3


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


def _blob(n, seed=0):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.arange(n) + 0.5,) * 3, indexing="ij")
    T = np.zeros((n, n, n))
    for _ in range(3):
        c = rng.uniform(0.3, 0.7, 3) * n
        r = rng.uniform(0.08, 0.16) * n
        T += rng.uniform(0.8, 2.0) * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * r * r))
    return (T * (1.0 + 0.2 * rng.standard_normal(T.shape))).clip(0).astype(np.float32)


def _setup(n=48):
    from blaze_b200.scenes import SceneSettings
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n)
    return s, s.to_params()


def _gpu_image(s, rp, T):
    import torch
    from blaze_b200.render import RenderEngine
    from blaze_b200.scenes import Timer
    with RenderEngine(Timer(), s, rp) as eng:
        t = torch.from_numpy(T).cuda()
        eng.render(t)
        return eng.image()


def _sampler(n):
    from blaze_b200.render import RenderEngine, default_render_params
    from blaze_b200.scenes import SceneSettings, Timer
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n)
    return RenderEngine(Timer(), s, default_render_params(s, 8, 8))


def _sample(eng, T, pos):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(T, np.float32)).cuda()
    p = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    out = torch.empty(len(pos), device="cuda")
    eng.sample_temp(t.data_ptr(), p.data_ptr(), len(pos), out.data_ptr())
    return out.cpu().numpy()


def test_texture_sampler_axis_weights_are_rounded_to_1_256():
    """On a ramp along one axis the filtered value minus the lower texel is
    that axis's weight: the fraction rounded half up to 1/256, exactly."""
    from oracle import oracle
    f = np.arange(4096) / 4096.0
    idx = np.arange(16, dtype=np.float32)
    with _sampler(16) as eng:
        for ax, T in enumerate((np.broadcast_to(idx[None, None, :], (16,) * 3), np.broadcast_to(idx[None, :, None], (16,) * 3),
                                np.broadcast_to(idx[:, None, None], (16,) * 3))):
            pos = np.full((4096, 3), 7.5, np.float32)
            pos[:, ax] = (5.5 + f).astype(np.float32)
            got = _sample(eng, T, pos).astype(np.float64)
            np.testing.assert_array_equal(got - 5.0, np.floor(f * 256 + 0.5) / 256)
            np.testing.assert_array_equal(got, oracle.tex_sample(T, pos, SAMPLER_QUANT))


def test_texture_sampler_corner_weights_sum_to_one():
    """A single unit texel seen from each of the eight corner positions: every
    corner weight is a multiple of 1/256 and the eight add up to one."""
    rng = np.random.default_rng(11)
    fr = rng.uniform(0, 1, (2048, 3))
    T = np.zeros((16, 16, 16), np.float32)
    T[8, 8, 8] = 1.0
    total = np.zeros(len(fr))
    with _sampler(16) as eng:
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = _sample(eng, T, np.array([8 - dx, 8 - dy, 8 - dz]) + 0.5 + fr).astype(np.float64)
                    np.testing.assert_array_equal(w * 256, np.round(w * 256))
                    total += w
    np.testing.assert_array_equal(total, 1.0)


def test_texture_sampler_matches_the_oracle_model():
    """General samples, inside and beyond the volume, against the oracle's
    model of the hardware filter (render_oracle.cpp, rule 3): within one
    1/256 corner-weight unit moved between two corners, 2 max|T| / 256."""
    from oracle import oracle
    rng = np.random.default_rng(3)
    T = rng.standard_normal((16, 16, 16)).astype(np.float32)
    pos = rng.uniform(-2.0, 18.0, (4096, 3)).astype(np.float32)
    with _sampler(16) as eng:
        got = _sample(eng, T, pos)
    err = np.abs(got - oracle.tex_sample(T, pos, SAMPLER_QUANT))
    tmax = np.abs(T).max()
    print(f"sampler vs oracle model: max {err.max():.2e}, mean {err.mean():.2e} (max|T| {tmax:.2f})")
    assert err.max() <= 2.0 * tmax / 256 and err.mean() <= 2e-4 * tmax


CASES = {
    "one_light_scatter": dict(lights=1, multi_scatter=True),
    "two_lights": dict(lights=2, multi_scatter=False),
    "no_emission": dict(lights=1, multi_scatter=True, emission=0.0),
}


@pytest.mark.parametrize("case", list(CASES))
def test_render_matches_oracle(case):
    from blaze_b200.render import default_render_params
    from oracle import oracle
    s, g = _setup(48)
    kw = dict(CASES[case])
    emission = kw.pop("emission", None)
    rp = default_render_params(s, width=80, height=56, **kw)
    if emission is not None:
        rp.emission_scale = emission
    T = _blob(48, seed=1)
    got = _gpu_image(s, rp, T)
    want = oracle.render(rp, g, T, SAMPLER_QUANT)
    assert np.isfinite(got).all() and want.max() > 0.05
    rel = _rel(got, want)
    print(f"{case}: rel L2 vs oracle {rel:.2e}, max |diff| {np.abs(got - want).max():.2e}")
    assert rel <= RENDER_TOL


@pytest.mark.parametrize("case", ["one_light_scatter", "two_lights"])
def test_render_equals_reference_build(case):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build absent")
    from blaze_b200.render import default_render_params
    s, g = _setup(48)
    rp = default_render_params(s, width=80, height=56, **CASES[case])
    T = _blob(48, seed=2)
    got = _gpu_image(s, rp, T)
    p = g.copy()
    with ref.RefSolver(p) as sim:
        sim.set("T", T)
        with ref.RefRenderer(sim, rp) as rr:
            rr.render()
            want = rr.image()
    print(f"{case}: rel L2 vs reference build {_rel(got, want):.2e}, max |diff| {np.abs(got - want).max():.2e}")
    np.testing.assert_array_equal(got, want)


def test_render_of_a_solver_equals_render_of_its_field(tmp_path):
    import torch
    from blaze_b200 import plume_scene
    from blaze_b200.render import RenderEngine, default_render_params
    from blaze_b200.solver import FluidSolver
    from blaze_b200.scenes import Timer
    scn, parts = plume_scene(n=32, seed=4, particles=800)
    tmr = Timer()
    with FluidSolver(tmr, scn, parts) as sol, RenderEngine(tmr, scn, default_render_params(scn, 40, 24)) as eng:
        for _ in range(3):
            sol.addSource()
            sol.step()
            tmr.iter += 1
            tmr.time += scn.dt
        eng.render(sol)
        a = eng.image()
        eng.render(torch.from_numpy(sol.get("T")).cuda())
        b = eng.image()
        np.testing.assert_array_equal(a, b)
        assert a.max() > 0
        path = eng.writeToDisk(str(tmp_path / "f.exr"))
        from test_render_cpu import read_exr
        np.testing.assert_array_equal(read_exr(path), a)
        assert eng.kernel_launches >= 2 and eng.last_ms > 0


def test_scene_loop_writes_the_reference_file_names(tmp_path):
    import json
    from blaze_b200 import plume_scene, write_part
    from blaze_b200.scenefile import load_blz, run
    from test_scenefile import write_scene
    path = write_scene(str(tmp_path), animated=False)
    d = json.load(open(path))
    d.update({"renderFile": "img/frame_####.png", "renderRes": [32, 24], "renderRange": [2, 3, 1],
              "cam": {"focal": 1.0, "aperture": 0.6, "rotMat": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "t": [0.5, 0.5, 2.4]},
              "primarySampleRate": 1.0 / 32, "shadowSamplingRate": 2.0 / 32, "cutoff": 1e-4, "densityScale": 8.0,
              "shadowDensityScale": 1.0, "volumeColor": [1, 1, 1], "scatteringColor": [0.8, 0.8, 0.8],
              "absorption": 0.2, "gain": 0.5, "emissionScale": 0.6,
              "shaderColorRamp": {"count": 2, "keys": [0, 1], "colors": [[0, 0, 0], [1, 0.6, 0.2]]},
              "shaderTempRange": [0.05, 2.0], "multiScatterScale": 0.5, "multiScatterDensityMask": [0.1, 1.0],
              "multiScatterColor": [1, 0.6, 0.3], "multiScatterBlurIter": 2, "lightCount": 1,
              "lights": [{"light_exposure": 0.5, "light_intensity": 1.0, "light_samples": 1,
                          "light_dir": [0.3, -1.0, -0.4], "light_color": [1, 1, 1]}]})
    json.dump(d, open(path, "w"))
    _, parts = plume_scene(n=32, seed=2, particles=400)
    write_part(os.path.join(str(tmp_path), "src", "plume_0001.part"), parts)
    stats = run(load_blz(path), render=True)
    files = [st.get("render_file") for st in stats]
    assert files == [None, os.path.join(str(tmp_path), "img", "frame_0002.png"),
                     os.path.join(str(tmp_path), "img", "frame_0003.png")]
    assert all(os.path.getsize(f) > 0 for f in files[1:])
