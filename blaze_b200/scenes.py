"""Scene settings, particle records and the seeded synthetic scenes.

``SceneSettings`` keeps the solver fields of the reference's POD
(src/SceneSettings.h:32-71) under the same names; ``to_params`` maps it to the
C ABI's ``blz_params``.  Particle records are the reference's ``.part``
format (src/Parser.h:196-209): little-endian float32 records of 8 values,
pos.xyz (world), vel.xyz, pscale, temperature.

The synthetic scenes stand in for the reference's demo caches (which are not
distributed with it): every particle position and attribute comes from a
PCG32 stream (O'Neill's published permuted congruential generator) seeded by
the caller, so the same bytes feed the CUDA path, the oracle and the
reference build.
"""
from dataclasses import dataclass, field
import math
import os

import numpy as np

from . import _abi

MASK64 = (1 << 64) - 1


class PCG32:
    """PCG-XSH-RR 64/32 (M. O'Neill, 2014)."""

    MULT = 6364136223846793005

    def __init__(self, seed, seq=0xDA3E39CB94B95BDB):
        self.inc = ((seq << 1) | 1) & MASK64
        self.state = 0
        self.next_u32()
        self.state = (self.state + (seed & MASK64)) & MASK64
        self.next_u32()

    def next_u32(self):
        old = self.state
        self.state = (old * self.MULT + self.inc) & MASK64
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * (self.next_u32() * (1.0 / 4294967296.0))

    def integer(self, lo, hi):
        """Uniform integer in [lo, hi]."""
        return lo + self.next_u32() % (hi - lo + 1)


@dataclass
class SceneSettings:
    """Solver subset of the reference's SceneSettings (same field names)."""
    gridRes: tuple = (64, 64, 64)
    dx: float = 1.0 / 64
    dt: float = 1.0 / 24
    domainBboxMin: tuple = (0.0, 0.0, 0.0)
    domainBboxMax: tuple = (1.0, 1.0, 1.0)
    closedBounds: tuple = (1, 1, 1, 1, 1, 1)     # xMin, xMax, yMin, yMax, zMin, zMax
    maxIterSolve: int = 200
    density: float = 0.1
    gravity: float = -9.8
    buoyancy: float = 0.0
    coolingRate: float = 0.0
    vorticityConf: float = 0.0
    drag: float = 0.0
    windDir: int = 0
    windAmp: float = 0.0
    windSpeed: float = 0.0
    windTurbAmp: float = 0.0
    windTurbScale: float = 1.0
    turbulence_amp: float = 0.0
    turbulence_scale: float = 1.0
    turbMaskTempRamp: tuple = (1e30, 2e30)         # both masks == 1
    turbMaskVelRamp: tuple = (-1.0, 0.0)
    sourceMaxParticleCount: int = 1 << 16
    # Solver controls with no reference counterpart.
    tol: float = 0.0
    check_every: int = 10
    bc_mode: int = _abi.BLZ_BC_REF_COMPAT
    gs_order: int = _abi.BLZ_GS_RB3D
    reset_pressure: int = 0
    temporal_block: int = 0
    device_loop: int = 1
    sweep_variant: int = -1
    advect_scheme: int = _abi.BLZ_ADVECT_RK3
    # Target mode: a smoke density scalar with buoyancy weight alpha
    # (V += dt (beta T - alpha rho) g); the reference has neither.
    density_field: int = 0
    buoyancy_alpha: float = 0.0
    # Solve for the correction to the previous pressure with an FP64 defect
    # (removes the FP32 floor of the residual; see blz_params).
    defect_correction: int = 0
    extra: dict = field(default_factory=dict)

    def to_params(self):
        p = _abi.BlzParams()
        p.width, p.height, p.depth = (int(v) for v in self.gridRes)
        p.dx, p.dt = self.dx, self.dt
        p.domain_min[:] = list(self.domainBboxMin)
        p.domain_max[:] = list(self.domainBboxMax)
        p.closed_bounds[:] = [int(b) for b in self.closedBounds]
        p.density, p.gravity, p.buoyancy = self.density, self.gravity, self.buoyancy
        p.cooling_rate, p.vorticity_conf, p.drag = self.coolingRate, self.vorticityConf, self.drag
        p.wind_dir, p.wind_amp, p.wind_speed = self.windDir, self.windAmp, self.windSpeed
        p.wind_turb_amp, p.wind_turb_scale = self.windTurbAmp, self.windTurbScale
        p.turbulence_amp, p.turbulence_scale = self.turbulence_amp, self.turbulence_scale
        p.turb_mask_temp_ramp[:] = list(self.turbMaskTempRamp)
        p.turb_mask_vel_ramp[:] = list(self.turbMaskVelRamp)
        p.max_iter, p.tol, p.check_every = self.maxIterSolve, self.tol, self.check_every
        p.bc_mode, p.gs_order, p.reset_pressure = self.bc_mode, self.gs_order, self.reset_pressure
        p.max_particles, p.temporal_block = self.sourceMaxParticleCount, self.temporal_block
        p.device_loop, p.sweep_variant = self.device_loop, self.sweep_variant
        p.advect_scheme = self.advect_scheme
        p.density_field, p.buoyancy_alpha = int(self.density_field), float(self.buoyancy_alpha)
        p.defect_correction = int(self.defect_correction)
        return p


class Timer:
    """Frame counter and simulation time (src/Timer.h:35-36)."""

    def __init__(self, iter=0, time=0.0):
        self.iter = iter
        self.time = time


# ---------------------------------------------------------------------------
# .part records
# ---------------------------------------------------------------------------
def write_part(path, rec8):
    np.ascontiguousarray(rec8, dtype="<f4").reshape(-1, 8).tofile(path)


def read_part(path):
    """Parser::sourceParticleParse: whole 32-byte records only."""
    raw = np.fromfile(path, dtype="<f4")
    n = raw.size // 8
    return raw[: n * 8].reshape(n, 8).astype(np.float32)


# ---------------------------------------------------------------------------
# Seeded synthetic scenes
# ---------------------------------------------------------------------------
# Particle pscale in cells.  The reference sums overlapping cubic pulses of
# radius pscale/2 (Grid.h:309-335), so the splatted temperature of a ball of
# particles is roughly (particles per cell) x (pulse volume) x (mean pulse
# weight 0.2).  At the configs' density (2000 particles in a ball of radius 6
# cells, 2.2 per cell) 1.5 cells gives a splatted temperature of about 1, the
# configured source value; 4 cells would give about 25 and a far stronger
# buoyancy than the scene describes.
PSCALE_CELLS = 1.5


def _cell_to_world(s, c):
    """World position of grid-cell coordinates given with y up (world axes)."""
    return [s.domainBboxMin[a] + c[a] * s.dx for a in range(3)]


def sphere_particles(rng, s, centre_cells, radius_cells, count, temp=(1.0, 1.0), pscale_cells=PSCALE_CELLS):
    """`count` particles uniform in a ball (rejection sampling), velocity 0."""
    cx, cy, cz = _cell_to_world(s, centre_cells)
    r = radius_cells * s.dx
    out = np.zeros((count, 8), np.float32)
    n = 0
    while n < count:
        x, y, z = (rng.uniform(-1.0, 1.0) for _ in range(3))
        if x * x + y * y + z * z > 1.0:
            continue
        out[n] = (cx + r * x, cy + r * y, cz + r * z, 0.0, 0.0, 0.0,
                  pscale_cells * s.dx, rng.uniform(*temp))
        n += 1
    return out


def disc_particles(rng, s, centre_cells, radius_cells, count, temp=(1.0, 1.0), pscale_cells=PSCALE_CELLS,
                   thickness_cells=2.0):
    """`count` particles uniform in a horizontal disc (world y up)."""
    cx, cy, cz = _cell_to_world(s, centre_cells)
    r = radius_cells * s.dx
    out = np.zeros((count, 8), np.float32)
    for n in range(count):
        a = rng.uniform(0.0, 2.0 * math.pi)
        rr = r * math.sqrt(rng.uniform())
        y = cy + thickness_cells * s.dx * rng.uniform()
        out[n] = (cx + rr * math.cos(a), y, cz + rr * math.sin(a), 0.0, 0.0, 0.0,
                  pscale_cells * s.dx, rng.uniform(*temp))
    return out


def plume_scene(n=64, seed=1, particles=2000, alpha=None):
    """Smoke plume: n^3, dx = 1/n, dt = 1/24, one ball of radius 6 cells at
    cells (n/2, n/8, n/2) (y up), T = 1, beta = 1, epsilon = 0.3, no noise,
    walls except a free-surface top, 80 sweeps from p = 0.  alpha (target
    mode): carry the density scalar (density 1 per particle) with buoyancy
    weight alpha (the configuration's 0.05)."""
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, dt=1.0 / 24,
                      closedBounds=(1, 1, 1, 0, 1, 1), maxIterSolve=80, buoyancy=1.0,
                      vorticityConf=0.3, reset_pressure=1)
    if alpha is not None:
        s.density_field, s.buoyancy_alpha = 1, float(alpha)
    rng = PCG32(seed)
    parts = sphere_particles(rng, s, (n / 2, n / 8, n / 2), 6.0, particles)
    s.sourceMaxParticleCount = max(particles, 1)
    return s, parts


def fire_scene(n=128, seed=2, per_disc=5000, density_field=0, alpha=0.0):
    """Fire and smoke: n^3, four discs of radius 8 cells on the floor with
    5000 particles each, T ~ U[0.5, 1.5], pseudo-curl noise amplitude 0.5 with
    a 4-cell period, wind 0.2 cells/step along +x, epsilon = 0.5, walls except
    the top, RBGS to relative residual 1e-4 with a cap of 400 sweeps.  Every
    particle's density ~ U[0.2, 1.0] (its own PCG32 stream, so the records do
    not depend on it) is in extra["particle_density"]; density_field carries
    it as the density scalar (target mode) with buoyancy weight alpha."""
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, dt=1.0 / 24,
                      closedBounds=(1, 1, 1, 0, 1, 1), maxIterSolve=400, tol=1e-4,
                      buoyancy=1.0, vorticityConf=0.5, turbulence_amp=0.5, turbulence_scale=4.0,
                      windDir=0, windAmp=0.2 * (1.0 / n) / (1.0 / 24), windSpeed=0.0)
    rng = PCG32(seed)
    parts = []
    for _ in range(4):
        c = (rng.uniform(0.2 * n, 0.8 * n), 2.0, rng.uniform(0.2 * n, 0.8 * n))
        parts.append(disc_particles(rng, s, c, 8.0, per_disc, temp=(0.5, 1.5)))
    parts = np.concatenate(parts)
    s.sourceMaxParticleCount = len(parts)
    drng = PCG32(seed, seq=0x5EED0D3E5)
    s.extra = {"particle_density": np.array([drng.uniform(0.2, 1.0) for _ in range(len(parts))], np.float32)}
    s.density_field, s.buoyancy_alpha = int(density_field), float(alpha)
    return s, parts


# Vorticity confinement of the plume family, given at the 64^3 resolution of
# the smoke-plume scene.  The reference's confinement force,
# epsilon * dx * (grad|omega| x omega) (FluidSolver.cu:229-238), takes the
# unnormalised gradient, so at a fixed flow it grows as 1/dx: the same epsilon
# is 4x stronger at 256^3 than at 64^3, and there the plumes run away within
# 10-20 frames (measured: peak speed 3.7 -> 1e3 cells/step over frames 10-17
# of seed 119, plain RBGS).  Scaling epsilon by 64/n keeps the force of the
# 64^3 scene.
FAMILY_EPSILON_64 = 0.3


def family_scene(n=256, seed=3, bc_mode=_abi.BLZ_BC_FREE_SURFACE, tol=1e-4, max_iter=4000,
                 check_every=20):
    """One seeded member of the plume family used for warm-start training and
    for the 256^3 benchmark: 1-6 balls of radius 4-16 cells on the lower half
    of the domain, wind 0-0.4 cells/step along +x, beta = 1, epsilon = 0.3 at
    64^3 scaled by 64/n (0.075 at 256^3), walls except a free-surface top;
    RBGS warm-started from the previous frame's pressure to relative residual
    `tol`."""
    rng = PCG32(seed)
    nsrc = rng.integer(1, 6)
    wind = rng.uniform(0.0, 0.4)
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, dt=1.0 / 24,
                      closedBounds=(1, 1, 1, 0, 1, 1), maxIterSolve=max_iter, tol=tol,
                      check_every=check_every, buoyancy=1.0, vorticityConf=FAMILY_EPSILON_64 * 64.0 / n,
                      windDir=0, windAmp=wind * (1.0 / n) / (1.0 / 24), bc_mode=bc_mode)
    parts = []
    for _ in range(nsrc):
        r = rng.uniform(4.0, 16.0)
        c = (rng.uniform(r + 2, n - r - 2), rng.uniform(r + 2, 0.5 * n), rng.uniform(r + 2, n - r - 2))
        count = int(min(40000, max(500, round(2000 * (r / 6.0) ** 3))))
        parts.append(sphere_particles(rng, s, c, r, count))
    parts = np.concatenate(parts)
    s.sourceMaxParticleCount = len(parts)
    s.extra = {"sources": nsrc, "wind_cells_per_step": wind}
    return s, parts


BATCH_DIMS = [(48, 48, 48), (64, 64, 64), (96, 96, 96), (128, 64, 64), (64, 128, 64)]


def batch_scenes(count=64, seed=4, tol=1e-4, max_iter=20000, check_every=20, dims=None):
    """`count` independent plume scenes for batched runs: grid dims drawn
    uniformly from `dims` (default 48^3, 64^3, 96^3, 128x64x64, 64x128x64),
    1-3 balls of radius 3-8 cells in the lower half, epsilon ~ U[0.1, 0.6],
    beta = 1, walls except a free-surface top, RBGS warm-started to relative
    residual `tol`.  dx = 1/W.  Returns [(SceneSettings, particles)]."""
    rng = PCG32(seed)
    dims = dims or BATCH_DIMS
    out = []
    for _ in range(count):
        W, H, D = dims[rng.integer(0, len(dims) - 1)]
        dx = 1.0 / W
        s = SceneSettings(gridRes=(W, H, D), dx=dx, dt=1.0 / 24, closedBounds=(1, 1, 1, 0, 1, 1),
                          domainBboxMax=(W * dx, H * dx, D * dx),
                          maxIterSolve=max_iter, tol=tol, check_every=check_every, buoyancy=1.0,
                          vorticityConf=rng.uniform(0.1, 0.6), bc_mode=_abi.BLZ_BC_FREE_SURFACE)
        parts = []
        for _ in range(rng.integer(1, 3)):
            r = rng.uniform(3.0, min(8.0, min(W, H, D) / 4.0))
            c = (rng.uniform(r + 1, W - r - 1), rng.uniform(r + 1, 0.5 * H), rng.uniform(r + 1, D - r - 1))
            count_p = int(min(8000, max(200, round(2000 * (r / 6.0) ** 3))))
            parts.append(sphere_particles(rng, s, c, r, count_p))
        parts = np.concatenate(parts)
        s.sourceMaxParticleCount = len(parts)
        out.append((s, parts))
    return out


def large_fire_scene(n=384, seed=5, defect_correction=1):
    """Large fire (384^3 by default), dx = 1/n, dt = 1/24: a ground disc of
    radius 40 cells with 30000 particles, and two spheres of radius 10 cells
    (9259 particles each, the plume family's density) moving along seeded
    straight paths at 1 cell per frame; T ~ U[1, 2]; curl noise amplitude 0.8
    with an 8-cell period; wind 0.3 cells/step along +x; epsilon at the
    family's 64^3 strength (0.3 * 64 / n); walls except a free-surface top;
    RBGS to FP64 relative residual 1e-4 (defect correction on by default: at
    384^3 the FP32 floor of a plain iterate is above 1e-4).

    Returns (SceneSettings, frame_particles): frame_particles(f) gives the
    records of frame f (the disc is the same every frame, the spheres have
    moved f cells along their paths), as the per-frame .part files of an
    animated source (write_animated_source) hold them."""
    s = SceneSettings(gridRes=(n, n, n), dx=1.0 / n, dt=1.0 / 24, closedBounds=(1, 1, 1, 0, 1, 1),
                      maxIterSolve=60000, tol=1e-4, check_every=-1, buoyancy=1.0,
                      vorticityConf=FAMILY_EPSILON_64 * 64.0 / n, turbulence_amp=0.8, turbulence_scale=8.0,
                      windDir=0, windAmp=0.3 * (1.0 / n) / (1.0 / 24), bc_mode=_abi.BLZ_BC_FREE_SURFACE,
                      defect_correction=defect_correction)
    rng = PCG32(seed)
    disc = disc_particles(rng, s, (n / 2, 2.0, n / 2), 40.0, 30000, temp=(1.0, 2.0))
    paths = []
    for _ in range(2):
        r = 10.0
        start = np.array([rng.uniform(r + 20, n - r - 20), rng.uniform(r + 4, 0.3 * n), rng.uniform(r + 20, n - r - 20)])
        a = rng.uniform(0.0, 2.0 * math.pi)
        rise = rng.uniform(-0.3, 0.3)
        v = np.array([math.cos(a), rise, math.sin(a)])
        v /= np.linalg.norm(v)                       # 1 cell per frame
        ball = sphere_particles(rng, s, (0.0, 0.0, 0.0), r, int(round(2000 * (r / 6.0) ** 3)), temp=(1.0, 2.0))
        paths.append((start, v, ball))
    n_parts = len(disc) + sum(len(b) for _, _, b in paths)
    s.sourceMaxParticleCount = n_parts
    s.extra = {"paths": [(p.tolist(), v.tolist()) for p, v, _ in paths]}

    def frame_particles(f):
        out = [disc]
        for start, v, ball in paths:
            c = np.clip(start + f * v, 10.0 + 1.0, n - 11.0)            # stays inside the domain
            moved = ball.copy()
            moved[:, :3] += np.array(_cell_to_world(s, c), np.float32) - np.array(_cell_to_world(s, (0, 0, 0)),
                                                                                   np.float32)
            out.append(moved)
        return np.concatenate(out)

    return s, frame_particles


def write_animated_source(directory, stem, frame_particles, frames):
    """The per-frame particle caches of an animated source, named as the
    reference's parser looks them up (<stem>_%04d.part, src/Parser.h:181-188);
    returns the particleFile value of frame 1 for a .blz scene."""
    os.makedirs(directory, exist_ok=True)
    for f in frames:
        write_part(os.path.join(directory, f"{stem}_{f:04d}.part"), frame_particles(f))
    return f"{stem}_0001.part"
