"""gs.materials: the MPM family (gs.materials.MPM.*) and Rigid, whose entities enter this
build as kinematic colliders coupled in the MPM grid op."""

from . import MPM
from .rigid import Rigid

__all__ = ["MPM", "Rigid"]
