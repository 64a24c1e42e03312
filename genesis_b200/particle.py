"""Shape-to-particle samplers used by the emitter (genesis/utils/particle.py:174-298).

Only the 'random' and 'regular' samplers exist; the reference's 'pbs' samplers run an
external prebuilt executable that is not part of this build, so 'pbs' requests are
sampled as 'regular', as for morphs.  Cylinders, spheres and shells are cut out of the
box sample by radius, as in the reference.
"""

from __future__ import annotations

import numpy as np

from .exceptions import GenesisException
from .morphs import n_particles_1D, n_particles_3D


def _sampler(sampler):
    return "regular" if "pbs" in sampler else sampler


def _box_to_particles(p_size, pos, size, sampler, rng=None):
    """utils/particle.py:174-202."""
    size = np.asarray(size, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    lower, upper = pos - size / 2, pos + size / 2
    if sampler == "random":
        rng = rng or np.random.default_rng()
        return rng.uniform(low=lower, high=upper, size=(n_particles_3D(p_size, size), 3))
    if sampler == "regular":
        axes = [
            np.linspace(lower[d] + 0.5 * p_size, upper[d] - 0.5 * p_size, n_particles_1D(p_size, size[d]))
            for d in range(3)
        ]
        return np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape((-1, 3))
    raise GenesisException(f"Unsupported sampler method: {sampler}.")


def box_to_particles(p_size=0.01, pos=(0, 0, 0), size=(1, 1, 1), sampler="random", rng=None):
    return _box_to_particles(p_size, pos, size, _sampler(sampler), rng)


def cylinder_to_particles(p_size=0.01, pos=(0, 0, 0), radius=0.5, height=1.0, sampler="random", rng=None):
    """Cylinder along z: the box [2r, 2r, h] minus the points farther than r from the axis."""
    p = _box_to_particles(p_size, pos, (2 * radius, 2 * radius, height), _sampler(sampler), rng)
    r = np.linalg.norm(p[:, :2] - np.asarray(pos, dtype=np.float64)[:2], axis=1)
    return p[r <= radius]


def sphere_to_particles(p_size=0.01, pos=(0, 0, 0), radius=0.5, sampler="random", rng=None):
    p = _box_to_particles(p_size, pos, (2 * radius,) * 3, _sampler(sampler), rng)
    return p[np.linalg.norm(p - np.asarray(pos, dtype=np.float64), axis=1) <= radius]


def shell_to_particles(p_size=0.01, pos=(0, 0, 0), inner_radius=0.5, outer_radius=0.7, sampler="random", rng=None):
    p = _box_to_particles(p_size, pos, (2 * outer_radius,) * 3, _sampler(sampler), rng)
    r = np.linalg.norm(p - np.asarray(pos, dtype=np.float64), axis=1)
    return p[(r <= outer_radius) & (r >= inner_radius)]
