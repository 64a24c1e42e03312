"""gs.materials.Rigid (genesis/engine/materials/rigid.py:9-130), with the reference's
constructor, defaults and checks.  Only the coupling parameters act on this path: a rigid
entity is a kinematic collider of the MPM grid op (there is no rigid-body solver here)."""

from __future__ import annotations

import logging

from ..exceptions import GenesisException

log = logging.getLogger("genesis_b200")


class Rigid:
    def __init__(self, rho=200.0, friction=None, needs_coup=True, coup_friction=0.1, coup_softness=0.002,
                 coup_restitution=0.0, sdf_cell_size=0.005, sdf_min_res=32, sdf_max_res=128, gravity_compensation=0):
        if friction is not None and (friction < 1e-2 or friction > 5.0):
            raise GenesisException("`friction` must be in the range [1e-2, 5.0] for simulation stability.")
        if coup_friction < 0:
            raise GenesisException("`coup_friction` must be non-negative.")
        if coup_softness < 0:
            raise GenesisException("`coup_softness` must be non-negative.")
        if coup_restitution < 0 or coup_restitution > 1:
            raise GenesisException("`coup_restitution` must be in the range [0, 1].")
        if coup_restitution != 0:
            log.warning("Non-zero `coup_restitution` could lead to instability. Use with caution.")
        if sdf_min_res < 16:
            raise GenesisException("`sdf_min_res` must be at least 16.")
        if sdf_min_res > sdf_max_res:
            raise GenesisException("`sdf_min_res` must be smaller than or equal to `sdf_max_res`.")
        self._rho = rho
        self._friction = None if friction is None else float(friction)
        self._needs_coup = bool(needs_coup)
        self._coup_friction = float(coup_friction)
        self._coup_softness = float(coup_softness)
        self._coup_restitution = float(coup_restitution)
        self._sdf_cell_size = sdf_cell_size
        self._sdf_min_res = sdf_min_res
        self._sdf_max_res = sdf_max_res
        self._gravity_compensation = gravity_compensation

    @property
    def rho(self):
        return self._rho

    @property
    def friction(self):
        return self._friction

    @property
    def needs_coup(self):
        return self._needs_coup

    @property
    def coup_friction(self):
        return self._coup_friction

    @property
    def coup_softness(self):
        return self._coup_softness

    @property
    def coup_restitution(self):
        return self._coup_restitution

    @property
    def gravity_compensation(self):
        return self._gravity_compensation

    @property
    def sdf_cell_size(self):
        return self._sdf_cell_size

    @property
    def sdf_min_res(self):
        return self._sdf_min_res

    @property
    def sdf_max_res(self):
        return self._sdf_max_res
