"""Seeded synthetic MPM workloads with the shapes of the benchmark configurations.

No public dataset is involved: every scene is a jittered particle lattice drawn from
``numpy.random.default_rng(seed)``.  Materials are given as (kind, kwargs) pairs so
the same description drives the CUDA path (genesis_b200.materials.MPM) and the CPU
oracle.

  elastic_cube    1 Elastic cube, 32,768 particles (32^3 jittered lattice in [0.4,0.6]^3),
                  grid_density 64 (65^3 nodes), dt 1e-4, gravity -9.8 z
  mixed_500k      4 boxes x 125,000 particles (50^3 lattices, edge 0.25): Liquid, Sand,
                  Snow, ElastoPlastic; grid_density 128 (129^3 nodes), dt 5e-5, v ~ N(0, 0.5)
  batch_scenes    256 independent scenes, N log-uniform in [2e3, 2e5], grid density
                  32/64/96, material uniform over the five, E log-uniform in [1e4, 1e6]
  diff_elastic    1 Elastic scene, 64 density, 20,000 lattice particles, per-particle
                  E = 1e5 exp(0.5 N(0,1)), 200 substeps at dt 1e-4
  serving_stream  Poisson arrivals of rollouts, N log-uniform [1e3, 5e5], grid density
                  32..128, substeps U[100, 2000], material mix of mixed_500k
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MATERIAL_KINDS = ("elastic", "elastoplastic", "liquid", "sand", "snow")


@dataclass
class SceneDesc:
    name: str
    grid_density: float
    particle_size: float
    dt: float  # substep dt
    n_substeps: int
    pos: np.ndarray  # [N,3] float64
    vel: np.ndarray  # [N,3] float64
    mat_idx: np.ndarray  # [N] int
    materials: list  # [(kind, kwargs)]
    lower_bound: tuple = (0.0, 0.0, 0.0)
    upper_bound: tuple = (1.0, 1.0, 1.0)
    gravity: tuple = (0.0, 0.0, -9.8)
    E_particle: np.ndarray | None = None  # optional per-particle Young's modulus
    meta: dict = field(default_factory=dict)

    @property
    def n_particles(self) -> int:
        return int(self.pos.shape[0])

    @property
    def grid_res(self) -> int:
        return int(round(self.grid_density * self.upper_bound[0]) - round(self.grid_density * self.lower_bound[0]) + 1)


def jittered_lattice(rng, n_side, lower, spacing, jitter=0.25):
    """n_side^3 (or n_side tuple) lattice of cell centres lower + (i + 0.5) * spacing, with
    uniform jitter of +-jitter * spacing per component."""
    ns = (n_side,) * 3 if np.isscalar(n_side) else tuple(n_side)
    axes = [np.asarray(lower[d], dtype=np.float64) + (np.arange(ns[d]) + 0.5) * spacing for d in range(3)]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    if jitter:
        g = g + rng.uniform(-jitter * spacing, jitter * spacing, size=g.shape)
    return g


def elastic_cube(seed: int = 0, n_side: int = 32, n_substeps: int = 1000) -> SceneDesc:
    rng = np.random.default_rng(seed)
    spacing = 0.2 / n_side
    pos = jittered_lattice(rng, n_side, (0.4, 0.4, 0.4), spacing)
    n = pos.shape[0]
    return SceneDesc(
        name=f"elastic_cube_{n}",
        grid_density=64,
        particle_size=spacing,
        dt=1e-4,
        n_substeps=n_substeps,
        pos=pos,
        vel=np.zeros((n, 3)),
        mat_idx=np.zeros(n, dtype=np.int64),
        materials=[("elastic", dict(E=1e5, nu=0.3, rho=1000.0))],
    )


MIXED_MATERIALS = [
    ("liquid", dict(E=1e5, nu=0.2)),
    ("sand", dict(friction_angle=45)),
    ("snow", dict(yield_lower=2.5e-2, yield_higher=7.5e-3)),
    ("elastoplastic", dict(von_mises_yield_stress=1e4)),
]


def mixed_500k(seed: int = 1, n_side: int = 50, n_substeps: int = 2000, grid_density: int = 128) -> SceneDesc:
    """Four boxes of n_side^3 particles (edge n_side * 0.005) placed in the four xy quadrants."""
    rng = np.random.default_rng(seed)
    spacing = 0.005 * (50.0 / n_side) if n_side != 50 else 0.005
    edge = n_side * spacing
    dx = 1.0 / grid_density
    lo, hi = 3 * dx + dx, 1.0 - 3 * dx - dx
    pos, mat = [], []
    for q in range(4):
        qx, qy = q % 2, q // 2
        x0 = rng.uniform(lo + qx * 0.5 * (hi - lo), lo + (qx + 1) * 0.5 * (hi - lo) - edge)
        y0 = rng.uniform(lo + qy * 0.5 * (hi - lo), lo + (qy + 1) * 0.5 * (hi - lo) - edge)
        z0 = rng.uniform(lo, hi - edge)
        pos.append(jittered_lattice(rng, n_side, (x0, y0, z0), spacing))
        mat.append(np.full(n_side**3, q, dtype=np.int64))
    pos = np.concatenate(pos)
    n = pos.shape[0]
    vel = rng.normal(0.0, 0.5, size=(n, 3))
    return SceneDesc(
        name=f"mixed_{n}",
        grid_density=grid_density,
        particle_size=spacing,
        dt=5e-5,
        n_substeps=n_substeps,
        pos=pos,
        vel=vel,
        mat_idx=np.concatenate(mat),
        materials=list(MIXED_MATERIALS),
    )


def _scene_of(rng, n, density, kind, E, dt, n_substeps, name):
    n_side = int(np.ceil(n ** (1.0 / 3.0)))
    dx = 1.0 / density
    avail = 1.0 - 8 * dx  # keep clear of the 3 dx padding
    spacing = min(0.5 / density, 0.6 * avail / n_side)
    edge = n_side * spacing
    lower = rng.uniform(4 * dx, 1.0 - 4 * dx - edge, size=3)
    lat = jittered_lattice(rng, n_side, lower, spacing)
    keep = np.sort(rng.choice(lat.shape[0], size=n, replace=False))
    pos = lat[keep]
    kw = dict(E=float(E))
    return SceneDesc(
        name=name,
        grid_density=density,
        particle_size=spacing,
        dt=dt,
        n_substeps=n_substeps,
        pos=pos,
        vel=rng.normal(0.0, 0.2, size=(n, 3)),
        mat_idx=np.zeros(n, dtype=np.int64),
        materials=[(kind, kw)],
    )


def batch_scenes(seed: int = 2, n_scenes: int = 256, n_substeps: int = 500, n_range=(2e3, 2e5),
                 densities=(32, 64, 96)) -> list[SceneDesc]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        density = int(rng.choice(densities))
        kind = MATERIAL_KINDS[int(rng.integers(0, 5))]
        E = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        dt = min(1e-4, 2e-2 / density)
        out.append(_scene_of(rng, n, density, kind, E, dt, n_substeps, f"batch_{i}"))
    return out


def diff_elastic(seed: int = 3, n: int = 20000, n_substeps: int = 200) -> SceneDesc:
    """The block starts 1.5 mm above the padded floor (3 dx = 0.047 m) so that with a
    downward initial velocity it impacts and deforms during the rollout; both gradients
    (initial velocity and per-particle E) are then non-trivial."""
    rng = np.random.default_rng(seed)
    spacing = 0.00625
    dims = (25, 25, 32) if n == 20000 else (int(np.ceil(n ** (1 / 3))),) * 3
    lat = jittered_lattice(rng, dims, (0.42, 0.42, 0.0484), spacing)[:n]
    E = 1e5 * np.exp(0.5 * rng.normal(size=n))
    return SceneDesc(
        name=f"diff_elastic_{n}",
        grid_density=64,
        particle_size=spacing,
        dt=1e-4,
        n_substeps=n_substeps,
        pos=lat,
        vel=np.zeros((n, 3)),
        mat_idx=np.zeros(n, dtype=np.int64),
        materials=[("elastic", dict(E=1e5, nu=0.3, rho=1000.0))],
        E_particle=E,
        meta=dict(target=np.array([0.55, 0.5, 0.25]), v0=np.array([0.5, 0.0, -1.0])),
    )


@dataclass
class Request:
    rid: int
    arrival: float  # seconds since stream start
    scene: SceneDesc


def serving_stream(seed: int = 4, n_requests: int = 2000, rate: float = 10.0, n_range=(1e3, 5e5),
                   densities=(32, 64, 96, 128), substeps_range=(100, 2000)) -> list[Request]:
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        density = int(rng.choice(densities))
        mi = int(rng.integers(0, 4))
        kind, kw = MIXED_MATERIALS[mi]
        steps = int(rng.integers(substeps_range[0], substeps_range[1] + 1))
        dt = min(5e-5, 2e-2 / density)
        sc = _scene_of(rng, n, density, kind, 1e5 if kind == "liquid" else 1e6, dt, steps, f"req_{i}")
        sc.materials = [(kind, dict(kw))]
        out.append(Request(i, t, sc))
    return out


def make_materials(scene: SceneDesc, module):
    """Instantiate scene.materials with ``module`` = genesis_b200.materials.MPM."""
    cls = {
        "elastic": module.Elastic,
        "elastoplastic": module.ElastoPlastic,
        "liquid": module.Liquid,
        "sand": module.Sand,
        "snow": module.Snow,
        "muscle": module.Muscle,
    }
    return [cls[k](**kw) for k, kw in scene.materials]
