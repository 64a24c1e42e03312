"""gs.materials.MPM.* with the reference constructors, defaults and properties.

Each class restates its reference counterpart's parameters
(genesis/engine/materials/MPM/{base,elastic,elasto_plastic,liquid,sand,snow,muscle}.py);
the constitutive arithmetic itself runs in the CUDA kernel (csrc/constitutive.cuh),
selected by ``kind`` from a device material table.
"""

from __future__ import annotations

import math

import numpy as np

from .. import _native as nat
from ..exceptions import GenesisException

_SAMPLERS = ("pbs", "random", "regular")


class Base:
    """Base MPM material (materials/MPM/base.py:8-135)."""

    _kind = None

    def __init__(self, E=1e6, nu=0.2, rho=1000.0, lam=None, mu=None, sampler=None):
        if sampler is None:
            sampler = "pbs"
        if not (sampler in _SAMPLERS or str(sampler).startswith("pbs-")):
            raise GenesisException(
                f"Particle sampler must be either 'pbs(-[0-9]+)', 'random' or 'regular. Got '{sampler}'."
            )
        self._E = E
        self._nu = nu
        self._rho = rho
        self._sampler = sampler
        self._default_Jp = 1.0
        # base.py:61-70
        self._mu = E / (2.0 * (1.0 + nu)) if mu is None else mu
        self._lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)) if lam is None else lam
        self._idx = None

    # materials are deduplicated by value when registered (base.py:92-101, mpm_solver.py:240-251)
    def __eq__(self, other):
        if self.__class__ is other.__class__:
            for key in self.__dict__:
                if key not in ("_id", "_idx", "_sampler") and key.startswith("_"):
                    if self.__dict__[key] != other.__dict__.get(key):
                        return False
            return True
        return False

    __hash__ = object.__hash__

    def __repr__(self):
        return f"<gs.materials.MPM.{type(self).__name__}(E={self._E}, nu={self._nu}, rho={self._rho})>"

    # ---------------------------------------------------------------- native
    def _native(self, p_vol: float) -> nat.Material:
        m = nat.Material()
        m.kind = self._kind
        m.flags = 0
        m.mu = float(self._mu)
        m.lam = float(self._lam)
        # mass = particle_volume * rho evaluated in float32 (mpm_solver.py:785)
        m.mass = float(np.float32(p_vol) * np.float32(self._rho))
        m.default_Jp = float(self._default_Jp)
        m.clamp_lo = 0.0
        m.clamp_hi = 0.0
        m.vm_threshold = 0.0
        m.sand_c1 = 0.0
        m.sand_alpha = 0.0
        m.muscle_stiffness = 0.0
        return m

    @property
    def idx(self):
        return self._idx

    @property
    def E(self):
        """Young's modulus."""
        return self._E

    @property
    def nu(self):
        """Poisson ratio."""
        return self._nu

    @property
    def mu(self):
        """The second Lame parameter."""
        return self._mu

    @property
    def lam(self):
        """The first Lame parameter."""
        return self._lam

    @property
    def rho(self):
        """The rest density."""
        return self._rho

    @property
    def sampler(self):
        """Particle sampler ('pbs', 'regular', 'random')."""
        return self._sampler

    @property
    def default_Jp(self):
        return self._default_Jp


class Elastic(Base):
    """Corotated (default) or Neo-Hookean elasticity (materials/MPM/elastic.py:8-88)."""

    _kind = nat.MAT_ELASTIC

    def __init__(self, E=3e5, nu=0.2, rho=1000.0, lam=None, mu=None, sampler=None, model="corotation"):
        super().__init__(E, nu, rho, lam, mu, sampler)
        if model not in ("corotation", "neohooken"):
            raise GenesisException(f"Unrecognized constitutive model: {model}")
        self._model = model

    def _native(self, p_vol):
        m = super()._native(p_vol)
        if self._model == "neohooken":
            m.flags |= nat.MATF_NEOHOOKEAN
        return m

    @property
    def model(self):
        """Stress model ('corotation', 'neohooken')."""
        return self._model


class ElastoPlastic(Base):
    """Von Mises or singular-value-clamp plasticity (materials/MPM/elasto_plastic.py:8-113)."""

    _kind = nat.MAT_ELASTOPLASTIC

    def __init__(
        self,
        E=1e6,
        nu=0.2,
        rho=1000.0,
        lam=None,
        mu=None,
        sampler=None,
        yield_lower=2.5e-2,
        yield_higher=4.5e-3,
        use_von_mises=True,
        von_mises_yield_stress=10000.0,
    ):
        super().__init__(E, nu, rho, lam, mu, sampler)
        self._yield_lower = yield_lower
        self._yield_higher = yield_higher
        self._use_von_mises = use_von_mises
        self._von_mises_yield_stress = von_mises_yield_stress

    def _native(self, p_vol):
        m = super()._native(p_vol)
        if self._use_von_mises:
            m.flags |= nat.MATF_VON_MISES
            # elasto_plastic.py:75: von_mises_yield_stress / (2 * mu) folded in float64
            m.vm_threshold = float(self._von_mises_yield_stress / (2 * self._mu)) if self._mu else float("inf")
        m.clamp_lo = float(1 - self._yield_lower)
        m.clamp_hi = float(1 + self._yield_higher)
        return m

    @property
    def yield_lower(self):
        return self._yield_lower

    @property
    def yield_higher(self):
        return self._yield_higher

    @property
    def use_von_mises(self):
        return self._use_von_mises

    @property
    def von_mises_yield_stress(self):
        return self._von_mises_yield_stress


class Liquid(Base):
    """Weakly compressible fluid (materials/MPM/liquid.py:8-64)."""

    _kind = nat.MAT_LIQUID

    def __init__(self, E=1e6, nu=0.2, rho=1000.0, lam=None, mu=None, viscous=False, sampler=None):
        super().__init__(E, nu, rho, lam, mu, sampler)
        self._viscous = viscous
        if not viscous:
            self._mu = 0.0

    @property
    def viscous(self):
        return self._viscous


class Sand(Base):
    """Drucker-Prager sand (materials/MPM/sand.py:9-89)."""

    _kind = nat.MAT_SAND

    def __init__(self, E=1e6, nu=0.2, rho=1000.0, lam=None, mu=None, sampler="random", friction_angle=45):
        super().__init__(E, nu, rho, lam, mu, sampler)
        self._default_Jp = 0.0
        self.friction_angle = float(np.deg2rad(friction_angle))
        sin_phi = math.sin(self.friction_angle)
        self.alpha = math.sqrt(2 / 3) * 2 * sin_phi / (3 - sin_phi)

    def _native(self, p_vol):
        m = super()._native(p_vol)
        m.sand_c1 = float((3 * self._lam + 2 * self._mu) / (2 * self._mu))
        m.sand_alpha = float(self.alpha)
        return m


class Snow(ElastoPlastic):
    """Snow: clamp plasticity with hardening (materials/MPM/snow.py:8-81)."""

    _kind = nat.MAT_SNOW

    def __init__(self, E=1e6, nu=0.2, rho=1000.0, lam=None, mu=None, sampler="random", yield_lower=2.5e-2,
                 yield_higher=4.5e-3):
        super().__init__(E=E, nu=nu, rho=rho, lam=lam, mu=mu, sampler=sampler, yield_lower=yield_lower,
                         yield_higher=yield_higher, use_von_mises=False)


class Muscle(Elastic):
    """Actuated elastic material (materials/MPM/muscle.py:8-75): the Elastic stress plus
    stiffness * actu * F_tmp (d d^T) F_tmp^T, with stiffness = E, per-particle actuation
    actu (set per muscle group) and fibre direction d."""

    def __init__(self, E=1e6, nu=0.2, rho=1000.0, lam=None, mu=None, sampler=None, model="neohooken", n_groups=1):
        super().__init__(E, nu, rho, lam, mu, sampler, model)
        self._stiffness = E  # muscle.py:54: Young's modulus is the muscle stiffness
        self._n_groups = int(n_groups)

    def _native(self, p_vol):
        m = super()._native(p_vol)
        m.flags |= nat.MATF_MUSCLE
        m.muscle_stiffness = float(self._stiffness)
        return m

    @property
    def stiffness(self):
        """Muscle stiffness."""
        return self._stiffness

    @property
    def n_groups(self):
        """Number of muscle groups."""
        return self._n_groups


__all__ = ["Base", "Elastic", "ElastoPlastic", "Liquid", "Sand", "Snow", "Muscle"]
