"""Seeded synthetic dam-break scenes.

The reference seeds particles with FluidGPU.fillBlock (fluid-gpu.js:107-128):
a lattice at 0.5-cell spacing, Math.random() jitter, mass 1, zero velocity and
affine.  Math.random() is unseeded, so scenes here come from a counter-based
splitmix64 stream instead (Steele, Lea & Flood 2014, "Fast splittable
pseudorandom number generators"): value i of stream `seed` is
mix64(seed + (i + 1) * 0x9E3779B97F4A7C15), and its top 24 bits make a
uniform float in [0, 1).  The same arrays feed the oracle and the GPU.

Workloads (grid in cells, particle counts exact):
  dam_break_64       64^3, 65,536 particles: 16x32x16 cells from cell 2,
                     2x2x2 per cell, jitter +-0.25 cell, 200 substeps.
  dam_break_1m       128^3, 1,048,576 particles: a block 40% of the width and
                     60% of the height from cell 2, z-depth filled row-major
                     until the count is reached; diffuse pool 262,144.
  dam_break_sphere_8m 256x128x256, 8,388,608 particles: a dam block plus a
                     radius-20-cell sphere falling at 2 cells per substep;
                     diffuse pool 1,048,576.
  batch_mix          64 independent scenes, counts log-uniform in
                     [4,096, 524,288], cubic grids of edge 32/48/64/96/128,
                     dam blocks of 20-60% of each axis, 200 substeps.
  serve_job          served jobs: counts log-uniform in [8,192, 2,097,152],
                     grid edge 32-192 at 8 particles per cell in the dam
                     block, 50-500 substeps; Poisson arrivals.
"""
import math

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed, n, offset=0):
    """n consecutive outputs (uint64) of the counter-based splitmix64 stream."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + i * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed, n, offset=0):
    """n uniforms in [0,1) as float64 (exact multiples of 2^-24)."""
    return (splitmix64(seed, n, offset) >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)


def lattice_block(lo, counts, n, spacing=0.5):
    """First n points of a lattice (x fastest, then y, then z) with points at
    lo + spacing * (i + 0.5), like fillBlock's half-cell lattice."""
    nx, ny, nz = counts
    assert n <= nx * ny * nz, "block too small for the requested count"
    k = np.arange(n, dtype=np.int64)
    ix, iy, iz = k % nx, (k // nx) % ny, k // (nx * ny)
    return np.stack([lo[0] + spacing * (ix + 0.5), lo[1] + spacing * (iy + 0.5),
                     lo[2] + spacing * (iz + 0.5)], axis=1)


def jitter(points, seed, amplitude):
    """Add U(-amplitude, amplitude) per axis; returns float32."""
    u = uniform01(seed, points.size).reshape(points.shape)
    return (points + (u - 0.5) * (2.0 * amplitude)).astype(np.float32)


class Scene:
    """Particle arrays in the reference layouts plus the grid dims."""

    def __init__(self, grid, pos3, vel3=None, name="scene", substeps=200, diffuse_max=0):
        self.grid = tuple(int(g) for g in grid)
        n = pos3.shape[0]
        self.n = n
        self.pos = np.zeros((n, 4), np.float32)
        self.pos[:, :3] = pos3
        self.vel = np.zeros((n, 4), np.float32)
        if vel3 is not None:
            self.vel[:, :3] = vel3
        self.affine = np.zeros((n, 9), np.float32)
        self.mass = np.ones(n, np.float32)
        self.name = name
        self.substeps = substeps
        self.diffuse_max = diffuse_max

    @property
    def cells(self):
        return self.grid[0] * self.grid[1] * self.grid[2]


def dam_break(grid, block_lo, block_counts, n, seed=0, amplitude=0.25, name="dam_break",
              substeps=200, diffuse_max=0):
    pts = lattice_block(block_lo, block_counts, n)
    return Scene(grid, jitter(pts, seed, amplitude), name=name, substeps=substeps,
                 diffuse_max=diffuse_max)


def dam_break_64(seed=0):
    """64^3 grid, 65,536 particles (16x32x16 cells x 8 per cell), 200 substeps."""
    return dam_break((64, 64, 64), (2.0, 2.0, 2.0), (32, 64, 32), 65536, seed,
                     name="dam_break_64", substeps=200)


def dam_break_1m(seed=0):
    """128^3 grid, 1,048,576 particles, diffuse pool 262,144, 500 substeps."""
    n = 1048576
    nx = int(0.4 * 128 / 0.5)   # 102 half-cell columns (40% of the width)
    ny = int(0.6 * 128 / 0.5)   # 153 half-cell rows (60% of the height)
    nz = -(-n // (nx * ny))
    return dam_break((128, 128, 128), (2.0, 2.0, 2.0), (nx, ny, nz), n, seed,
                     name="dam_break_1m", substeps=500, diffuse_max=262144)


def sphere_points(center, radius, spacing=0.5):
    r = int(math.ceil(radius / spacing))
    a = (np.arange(-r, r) + 0.5) * spacing
    X, Y, Z = np.meshgrid(a, a, a, indexing="ij")
    m = X * X + Y * Y + Z * Z <= radius * radius
    p = np.stack([Z[m], Y[m], X[m]], axis=1)[:, ::-1]
    return p + np.asarray(center, np.float64)


def dam_break_sphere_8m(seed=0, dt=0.3):
    """256x128x256 grid, 8,388,608 particles: dam block + falling sphere."""
    n = 8388608
    sph = sphere_points((192.0, 80.0, 128.0), 20.0)
    nb = n - sph.shape[0]
    nx, ny = int(0.4 * 256 / 0.5), int(0.6 * 128 / 0.5)
    nz = -(-nb // (nx * ny))
    blk = lattice_block((2.0, 2.0, 2.0), (nx, ny, nz), nb)
    pts = np.concatenate([blk, sph], axis=0)
    pos = jitter(pts, seed, 0.25)
    vel = np.zeros((n, 3), np.float32)
    vel[nb:, 1] = np.float32(-2.0 / dt)
    return Scene((256, 128, 256), pos, vel, name="dam_break_sphere_8m", substeps=100,
                 diffuse_max=1048576)


def small_box(grid=(24, 20, 22), n=3000, seed=1, lo=(2.0, 2.0, 2.0), counts=None, name="small"):
    """A small dam break for quick parity tests (jitter +-0.25 cell)."""
    if counts is None:
        nx = max(2, int((grid[0] * 0.5 - lo[0]) / 0.5))
        ny = max(2, int((grid[1] * 0.7 - lo[1]) / 0.5))
        nz = -(-n // (nx * ny))
        counts = (nx, ny, nz)
    return dam_break(grid, lo, counts, n, seed, name=name)


BATCH_EDGES = (32, 48, 64, 96, 128)


def batch_scene(seed, index, n_min=4096, n_max=524288, edges=BATCH_EDGES):
    """One scene of the batched mix: particle count log-uniform in [n_min,
    n_max], a cubic grid with edge drawn from `edges`, and a dam block from
    cell 2 whose extent is U[0.2, 0.6] of each axis, filled with the count at
    uniform random (seeded) positions — particles per cell = n / block cells,
    so small blocks with large counts are overpacked."""
    u = uniform01(seed * 1000003 + index, 5)
    n = int(round(math.exp(math.log(n_min) + u[0] * (math.log(n_max) - math.log(n_min)))))
    edge = edges[min(int(u[1] * len(edges)), len(edges) - 1)]
    ext = [max(1.0, math.floor((0.2 + 0.4 * f) * edge)) for f in u[2:5]]
    ext = [min(e, edge - 4.0) for e in ext]
    r = uniform01(seed * 1000003 + index + 7919, 3 * n).reshape(n, 3)
    pos = (2.0 + r * np.asarray(ext)).astype(np.float32)
    sc = Scene((edge, edge, edge), pos, name=f"batch_{index}", substeps=200)
    sc.block_cells = int(ext[0] * ext[1] * ext[2])
    return sc


def batch_mix(count=64, seed=0, **kw):
    """The batched workload: `count` independent scenes (batch_scene)."""
    return [batch_scene(seed, i, **kw) for i in range(count)]


def serve_job(seed, index, n_min=8192, n_max=2097152, steps_min=50, steps_max=500):
    """One job of the served workload: particle count log-uniform in [n_min,
    n_max]; a cubic grid whose edge (32..192, a multiple of 8) makes a dam
    block of 40% x 60% x 40% of the domain hold the particles at 8 per cell
    (2 x 2 x 2 lattice, jitter +-0.25 cell); substeps uniform in
    [steps_min, steps_max].  Returns (scene, substeps)."""
    u = uniform01(seed * 1000033 + index, 2)
    n = int(round(math.exp(math.log(n_min) + u[0] * (math.log(n_max) - math.log(n_min)))))
    edge = int(math.ceil((n / (8 * 0.4 * 0.6 * 0.4)) ** (1.0 / 3.0) / 8.0) * 8)
    edge = min(192, max(32, edge))
    nx = int(0.4 * edge / 0.5)
    ny = int(0.6 * edge / 0.5)
    nz = -(-n // (nx * ny))
    sc = dam_break((edge, edge, edge), (2.0, 2.0, 2.0), (nx, ny, nz), n, seed * 7919 + index,
                   name=f"job_{index}")
    steps = steps_min + min(int(u[1] * (steps_max - steps_min + 1)), steps_max - steps_min)
    return sc, steps


def poisson_arrivals(rate, count, seed):
    """Arrival times (s) of a Poisson process of `rate` jobs/s."""
    u = uniform01(seed * 1000037 + 17, count)
    gaps = -np.log1p(-u) / rate
    return np.cumsum(gaps) - gaps[0]


WORKLOADS = {"dam_break_64": dam_break_64, "dam_break_1m": dam_break_1m,
             "dam_break_sphere_8m": dam_break_sphere_8m}
