"""Seeded stage cases shared by the golden-fixture generator (run against the
reference's CUDA build), the CPU oracle-vs-fixture test and the live GPU
comparison of the CUDA path with the reference build.

Grids are 16 x 16 x 8: the reference's Gauss-Seidel kernel then runs as a
single 16x16 thread block, which makes its plane-by-plane schedule
deterministic (FluidSolver.cu:517-599, launch 839-841), and every dim meets
its launch-shape rules (multiples of 16 in x, y and of 8 in z).
"""
import numpy as np

from blaze_b200 import BLZ_BC_REF_COMPAT, BLZ_GS_PLANE, SceneSettings

DIMS = (16, 16, 8)


def scene(**kw):
    W, H, D = DIMS
    s = SceneSettings(gridRes=DIMS, dx=1.0 / 16, dt=1.0 / 24, domainBboxMin=(-0.2, 0.3, 0.1),
                      domainBboxMax=(-0.2 + W / 16, 0.3 + H / 16, 0.1 + D / 16),
                      closedBounds=(1, 1, 1, 0, 1, 1), maxIterSolve=20,
                      bc_mode=BLZ_BC_REF_COMPAT, gs_order=BLZ_GS_PLANE, sourceMaxParticleCount=4096)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def inputs(params, seed):
    rng = np.random.default_rng(seed)
    return {
        "T": rng.uniform(0.0, 2.0, params.field_shape("T")).astype(np.float32),
        "U": (0.5 * rng.standard_normal(params.field_shape("U"))).astype(np.float32),
        "V": (0.5 * rng.standard_normal(params.field_shape("V"))).astype(np.float32),
        "W": (0.5 * rng.standard_normal(params.field_shape("W"))).astype(np.float32),
        "P": rng.standard_normal(params.field_shape("P")).astype(np.float32),
        "RHS": rng.standard_normal(params.field_shape("RHS")).astype(np.float32),
    }


def particles(params, seed, n=300):
    rng = np.random.default_rng(seed)
    lo = np.array(params.domain_min, np.float64)
    hi = np.array(params.domain_max, np.float64)
    rec = np.zeros((n, 8), np.float32)
    rec[:, :3] = rng.uniform(lo + 0.1, hi - 0.1, (n, 3))
    rec[:, 3:6] = rng.standard_normal((n, 3)) * (rng.uniform(size=(n, 1)) < 0.6)
    rec[:, 6] = rng.uniform(1.0, 5.0, n) * params.dx
    rec[:, 7] = rng.uniform(0.2, 2.0, n)
    return rec


# name: (scene overrides, stage, input seed, time, output fields)
CASES = {
    "source": (dict(), "source", 101, 0.0, ("T", "U", "V", "W")),
    "vorticity": (dict(vorticityConf=0.4), "vorticity", 102, 0.0, ("U", "V", "W")),
    "buoyancy": (dict(buoyancy=1.7), "buoyancy", 103, 0.0, ("V",)),
    "wind_x": (dict(windAmp=0.3, windDir=0, windSpeed=0.7, windTurbAmp=0.5, windTurbScale=0.3),
               "wind", 104, 1.37, ("U", "V", "W")),
    "wind_z": (dict(windAmp=0.2, windDir=3, windSpeed=0.2, windTurbAmp=0.8, windTurbScale=0.5),
               "wind", 105, 0.61, ("U", "V", "W")),
    "turbulence": (dict(turbulence_amp=0.5, turbulence_scale=4.0), "turbulence", 106, 0.9, ("U", "V", "W")),
    "turbulence_ramps": (dict(turbulence_amp=0.8, turbulence_scale=2.5, turbMaskTempRamp=(0.2, 1.5),
                              turbMaskVelRamp=(0.1, 0.9)), "turbulence", 107, 2.2, ("U", "V", "W")),
    "divergence": (dict(closedBounds=(1, 0, 1, 0, 0, 1)), "divergence", 108, 0.0, ("RHS",)),
    "gs_plane": (dict(maxIterSolve=20), "gs", 109, 0.0, ("P",)),
    "gradient_walls": (dict(closedBounds=(1, 1, 1, 1, 1, 1)), "gradient", 110, 0.0, ("U", "V", "W")),
    "gradient_open": (dict(closedBounds=(0, 0, 0, 0, 0, 0)), "gradient", 111, 0.0, ("U", "V", "W")),
    "advect": (dict(), "advect", 112, 0.0, ("T", "U", "V", "W")),
    "step": (dict(buoyancy=1.0, vorticityConf=0.3, windAmp=0.1, windTurbAmp=0.3, windTurbScale=0.5,
                  windSpeed=0.3, turbulence_amp=0.3, turbulence_scale=4.0, maxIterSolve=20),
             "step", 113, 0.0, ("T", "U", "V", "W", "P")),
}

STEP_FRAMES = 3


def load_inputs_into(setter, params, seed):
    for k, v in inputs(params, seed).items():
        setter(k, v)
