"""gs.force_fields: external acceleration fields of the MPM grid op (engine/force_fields.py).

Each class keeps the reference's constructor arguments, properties and activate() /
deactivate() / active (a field starts inactive, force_fields.py:18-32).  scene.add_force_field
registers one before build; at build the MPM solver packs every field into a device table of
mpm_force_field rows, which the grid op applies per active node after gravity (v += acc dt,
legacy_coupler.py:377-379).  activate() / deactivate() after build write the row's flag on the
device.  Turbulence's Perlin permutation tables are made here exactly as PerlinNoiseField makes
them (force_fields.py:447-460: numpy's legacy generator seeded with seed + axis, shuffling
arange(256)).  Noise draws from a counter-based hash instead of ti.random's stream; Custom (a
gstaichi function) cannot be compiled here and is refused.
"""

from __future__ import annotations

import numpy as np

from . import _native as nat
from .exceptions import GenesisException


class ForceField:
    """Base class (force_fields.py:9-46)."""

    _kind = None

    def __init__(self):
        self._active = False
        self._solver = None  # the built scene's MPM solver
        self._row = -1

    def activate(self):
        self._set_active(True)

    def deactivate(self):
        self._set_active(False)

    def _set_active(self, on):
        self._active = bool(on)
        if self._solver is not None and self._row >= 0:
            self._solver.runtime.set_force_field_active(self._row, self._active)

    @property
    def active(self):
        return self._active

    def _row_struct(self, perm_offset):
        f = nat.ForceField()
        f.kind = self._kind
        f.active = 1 if self._active else 0
        f.falloff_max = float("inf")
        f.perm_offset = perm_offset
        self._fill(f)
        return f

    def _perm(self):
        return None

    def _fill(self, f):
        raise NotImplementedError


def _vec3(x, name):
    a = np.array(x, dtype=np.float64)
    if a.shape != (3,):
        raise ValueError(f"{name} must have shape (3,)")
    return a


class Constant(ForceField):
    """acc = direction * strength everywhere (force_fields.py:49-82)."""

    _kind = nat.FF_CONSTANT

    def __init__(self, direction=(1, 0, 0), strength=1.0):
        super().__init__()
        d = _vec3(direction, "direction")
        self._direction = d / np.linalg.norm(d)
        self._strength = strength

    def _fill(self, f):
        for i in range(3):
            f.vec[i] = float(self._direction[i] * self._strength)

    @property
    def direction(self):
        return self._direction

    @property
    def strength(self):
        return self._strength


class Wind(ForceField):
    """direction * strength inside the cylinder of `radius` about the line through `center`
    along `direction` (force_fields.py:85-144)."""

    _kind = nat.FF_WIND

    def __init__(self, direction=(1, 0, 0), strength=1.0, radius=1, center=(0, 0, 0)):
        super().__init__()
        d = _vec3(direction, "direction")
        self._center = _vec3(center, "center")
        self._direction = d / np.linalg.norm(d)
        self._strength = strength
        self._radius = radius

    def _fill(self, f):
        for i in range(3):
            f.vec[i] = float(self._direction[i] * self._strength)
            f.dir[i] = float(self._direction[i])
            f.center[i] = float(self._center[i])
        f.radius = float(self._radius)

    @property
    def direction(self):
        return self._direction

    @property
    def strength(self):
        return self._strength

    @property
    def radius(self):
        return self._radius

    @property
    def center(self):
        return self._center


class Point(ForceField):
    """strength towards (negative: away from) `position`, with flow and a distance falloff
    (force_fields.py:147-198)."""

    _kind = nat.FF_POINT

    def __init__(self, strength=1.0, position=(0, 0, 0), falloff_pow=0.0, flow=1.0):
        super().__init__()
        self._strength = strength
        self._position = _vec3(position, "position")
        self._falloff_pow = falloff_pow
        self._flow = flow

    def _fill(self, f):
        for i in range(3):
            f.vec[i] = float(self._position[i])
        f.strength = float(self._strength)
        f.falloff_pow = float(self._falloff_pow)
        f.flow = float(self._flow)

    @property
    def strength(self):
        return self._strength

    @property
    def position(self):
        return self._position


class Drag(ForceField):
    """-linear v - quadratic |v| v (force_fields.py:201-229)."""

    _kind = nat.FF_DRAG

    def __init__(self, linear=0.0, quadratic=0.0):
        super().__init__()
        self._linear = linear
        self._quadratic = quadratic

    def _fill(self, f):
        f.linear = float(self._linear)
        f.quadratic = float(self._quadratic)

    @property
    def linear(self):
        return self._linear

    @property
    def quadratic(self):
        return self._quadratic


class Noise(ForceField):
    """strength (2 u - 1), u uniform in [0, 1)^3 per node and substep (force_fields.py:232-260);
    the draws come from a counter-based hash keyed by `seed` (an addition: the reference draws
    ti.random)."""

    _kind = nat.FF_NOISE

    def __init__(self, strength=1.0, seed=0):
        super().__init__()
        self._strength = strength
        self._seed = int(seed) & 0xFFFFFFFF

    def _fill(self, f):
        f.strength = float(self._strength)
        f.seed = self._seed

    @property
    def strength(self):
        return self._strength


class Vortex(ForceField):
    """Rotation about the z axis through `center` with radial pull, falloff and damping
    (force_fields.py:263-369)."""

    _kind = nat.FF_VORTEX

    def __init__(self, direction=(0.0, 0.0, 1.0), center=(0.0, 0.0, 0.0), strength_perpendicular=20.0,
                 strength_radial=0.0, falloff_pow=2.0, falloff_min=0.01, falloff_max=np.inf, damping=0.0):
        super().__init__()
        d = _vec3(direction, "direction")
        self._center = _vec3(center, "center")
        self._direction = d / np.linalg.norm(d)
        self._damping = damping
        self._strength_perpendicular = strength_perpendicular
        self._strength_radial = strength_radial
        self._falloff_pow = falloff_pow
        self._falloff_min = falloff_min
        self._falloff_max = falloff_max

    def _fill(self, f):
        for i in range(3):
            f.center[i] = float(self._center[i])
            f.dir[i] = float(self._direction[i])
        f.strength = float(self._strength_perpendicular)
        f.strength2 = float(self._strength_radial)
        f.falloff_pow = float(self._falloff_pow)
        f.falloff_min = float(self._falloff_min)
        f.falloff_max = float(self._falloff_max)
        f.damping = float(self._damping)

    @property
    def direction(self):
        return self._direction

    @property
    def center(self):
        return self._center

    @property
    def strength_perpendicular(self):
        return self._strength_perpendicular

    @property
    def strength_radial(self):
        return self._strength_radial

    @property
    def falloff_pow(self):
        return self._falloff_pow

    @property
    def falloff_min(self):
        return self._falloff_min

    @property
    def falloff_max(self):
        return self._falloff_max


def perlin_permutation(seed, seed_offset, wrap_size=256):
    """PerlinNoiseField's table (force_fields.py:447-460): arange(wrap_size), shuffled by numpy's
    legacy generator seeded with seed + seed_offset when a seed is given, written twice."""
    p = np.arange(wrap_size, dtype=np.int32)
    if seed is not None:
        np.random.RandomState(seed + seed_offset).shuffle(p)
    return np.concatenate([p, p])


class Turbulence(ForceField):
    """strength times three Perlin noise fields (one per axis), with flow
    (force_fields.py:372-421)."""

    _kind = nat.FF_TURBULENCE

    def __init__(self, strength=1.0, frequency=3, flow=0.0, seed=None):
        super().__init__()
        self._strength = strength
        self._frequency = frequency
        self._flow = flow
        self._seed = seed

    def _perm(self):
        return np.concatenate([perlin_permutation(self._seed, k) for k in range(3)])

    def _fill(self, f):
        f.strength = float(self._strength)
        f.frequency = float(self._frequency)
        f.flow = float(self._flow)

    @property
    def strength(self):
        return self._strength

    @property
    def frequency(self):
        return self._frequency


class Custom(ForceField):
    """A user gstaichi function f(pos, vel, t, i) (force_fields.py:424-438): there is no gstaichi
    here to compile it, so a scene refuses it."""

    def __init__(self, func):
        super().__init__()
        self.get_acc = func


def pack(fields):
    """(rows, perm): the mpm_force_field rows of `fields` in order and the concatenated
    permutation tables they index."""
    rows, perms, off = [], [], 0
    for f in fields:
        p = f._perm()
        rows.append(f._row_struct(off if p is not None else 0))
        if p is not None:
            perms.append(p)
            off += p.size
    return rows, (np.concatenate(perms) if perms else None)
