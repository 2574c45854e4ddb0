"""Seeded render cases shared by the render golden generator (run against the
reference's RenderEngine, src/RenderEngine.cu, built from its sources), the
CPU oracle-vs-fixture test and the GPU fixture test of the CUDA renderer.

Each case is a 32^3 field of three noisy Gaussian blobs rendered at 64 x 48
with the synthetic camera, ramp and lights of default_render_params.
"""
import numpy as np

from blaze_b200.render import default_render_params
from blaze_b200.scenes import SceneSettings

N = 32
WIDTH, HEIGHT = 64, 48


def blob(n, seed):
    """Three Gaussian blobs of temperature with 20 % multiplicative noise,
    clipped at zero: (z, y, x) float32."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.arange(n) + 0.5,) * 3, indexing="ij")
    T = np.zeros((n, n, n))
    for _ in range(3):
        c = rng.uniform(0.3, 0.7, 3) * n
        r = rng.uniform(0.08, 0.16) * n
        T += rng.uniform(0.8, 2.0) * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * r * r))
    return (T * (1.0 + 0.2 * rng.standard_normal(T.shape))).clip(0).astype(np.float32)


# name: (default_render_params keywords, overrides, field seed)
CASES = {
    "one_light_scatter": (dict(lights=1, multi_scatter=True), {}, 21),
    "two_lights": (dict(lights=2, multi_scatter=False), {}, 22),
    "three_lights_scatter": (dict(lights=3, multi_scatter=True), {"gain": 0.9}, 23),
    "no_emission": (dict(lights=1, multi_scatter=True), {"emission_scale": 0.0}, 24),
    "emission_only": (dict(lights=0, multi_scatter=False), {"cutoff": 0.0}, 25),
}


def setup(name):
    """(settings, grid params, render params, T) of one case."""
    kw, ovr, seed = CASES[name]
    s = SceneSettings(gridRes=(N, N, N), dx=1.0 / N)
    rp = default_render_params(s, width=WIDTH, height=HEIGHT, **kw)
    for k, v in ovr.items():
        setattr(rp, k, v)
    return s, s.to_params(), rp, blob(N, seed)
