"""Seeded cases of the noise library (thirdparty/cuda-noise/cuda_noise.cuh)
shared by the golden generator (run against the reference's CUDA build), the
CPU oracle-vs-fixture test and the GPU test of blz_noise.

Positions mix moderate, negative, large (lattice sums past 2^24, where the
rounding of the fused hash-input sums decides the lattice value), tiny and
lattice-aligned coordinates.
"""
import numpy as np

from blaze_b200._abi import noise_args

BASES = ["checker", "discrete", "linearvalue", "fadedvalue", "cubicvalue", "perlin", "simplex", "worley", "spots"]


def positions(seed=2024):
    rng = np.random.default_rng(seed)
    lattice = np.floor(rng.uniform(-10, 60, (200, 3))) + rng.choice([0.0, 0.5], (200, 3))
    return np.concatenate([rng.uniform(-40, 260, (1200, 3)), rng.uniform(0, 3000, (400, 3)), lattice,
                           rng.uniform(-1.5, 1.5, (200, 3))]).astype(np.float32)


def _cases():
    c = {
        "checker": dict(func="checker", scale=0.3, seed=7),
        "checker_neg": dict(func="checker", scale=1.7, seed=-3),
        "discrete": dict(func="discrete", scale=0.7, seed=11),
        "discrete_big_seed": dict(func="discrete", scale=2.5, seed=987654321),
        "linearvalue": dict(func="linearvalue", scale=1.0, seed=13),
        "linearvalue_neg_seed": dict(func="linearvalue", scale=3.0, seed=-77),
        "fadedvalue": dict(func="fadedvalue", scale=0.5, seed=17),
        "fadedvalue_unit": dict(func="fadedvalue", scale=1.0, seed=4),
        "cubicvalue": dict(func="cubicvalue", scale=0.25, seed=19),
        "cubicvalue_fine": dict(func="cubicvalue", scale=1.3, seed=0),
        "perlin": dict(func="perlin", scale=0.4, seed=99),
        "perlin_fine": dict(func="perlin", scale=1.6, seed=-5),
        "simplex": dict(func="simplex", scale=0.35, seed=5),
        "simplex_fine": dict(func="simplex", scale=1.7, seed=-12345),
        "simplex_coarse": dict(func="simplex", scale=0.05, seed=2147000000),
        "worley": dict(func="worley", scale=0.2, seed=21, size=1.0, min_num=4, max_num=4, jitter=1.0),
        "worley_var": dict(func="worley", scale=1.0, seed=-8, size=0.5, min_num=1, max_num=5, jitter=0.7),
        "worley_zero_size": dict(func="worley", scale=1.0, seed=1, size=0.0),
        "spots_step": dict(func="spots", scale=0.6, seed=23, size=0.3, min_num=0, max_num=4, jitter=1.0, shape=0),
        "spots_linear": dict(func="spots", scale=1.0, seed=29, size=0.1, min_num=0, max_num=4, jitter=1.0, shape=1),
        "spots_quadratic": dict(func="spots", scale=0.8, seed=31, size=0.2, min_num=1, max_num=3, jitter=0.5,
                                shape=2),
        "repeater_perlin": dict(func="repeater_perlin", scale=0.05, seed=1, octaves=5, lacunarity=2.0, decay=0.5),
        "repeater_perlin_bounded": dict(func="repeater_perlin_bounded", scale=0.08, seed=3, octaves=6,
                                        lacunarity=1.9, decay=0.6, threshold=0.1),
        "repeater_perlin_abs": dict(func="repeater_perlin_abs", scale=0.03, seed=37, octaves=4, lacunarity=2.2,
                                    decay=0.45),
        "repeater_simplex": dict(func="repeater_simplex", scale=0.04, seed=41, octaves=5, lacunarity=2.0, decay=0.5),
        "repeater_simplex_abs": dict(func="repeater_simplex_abs", scale=0.06, seed=43, octaves=4, lacunarity=2.5,
                                     decay=0.4),
        "repeater_simplex_bounded": dict(func="repeater_simplex_bounded", scale=0.05, seed=47, octaves=6,
                                         lacunarity=2.0, decay=0.5, threshold=0.05),
        "fractal_simplex": dict(func="fractal_simplex", scale=0.5, seed=53, du=0.01, octaves=10, lacunarity=2.0,
                                decay=0.5),
        "fractal_simplex_all": dict(func="fractal_simplex", scale=0.02, seed=59, du=0.0001, octaves=6,
                                    lacunarity=2.0, decay=0.55),
    }
    for b in BASES:
        c[f"repeater_{b}"] = dict(func="repeater", basis=b, scale=0.02, seed=61, octaves=4, lacunarity=2.0, decay=0.5)
    for bi, bo in (("perlin", "simplex"), ("simplex", "perlin"), ("worley", "linearvalue"), ("checker", "fadedvalue"),
                   ("cubicvalue", "worley"), ("linearvalue", "checker"), ("fadedvalue", "cubicvalue"),
                   ("discrete", "perlin"), ("perlin", "spots"), ("simplex", "discrete")):
        c[f"turbulence_{bi}_{bo}"] = dict(func="turbulence", basis=bi, basis_out=bo, scale=0.1, scale_out=0.3,
                                          seed=67, strength=2.5)
    c["repeater_turbulence_perlin_simplex"] = dict(func="repeater_turbulence", basis="perlin", basis_out="simplex",
                                                   scale=0.05, scale_out=0.1, seed=71, strength=3.0, octaves=3)
    c["repeater_turbulence_worley_spots"] = dict(func="repeater_turbulence", basis="worley", basis_out="spots",
                                                 scale=0.1, scale_out=0.2, seed=73, strength=1.5, octaves=2)
    return c


CASES = _cases()


def args(name):
    kw = dict(CASES[name])
    return noise_args(kw.pop("func"), **kw)
