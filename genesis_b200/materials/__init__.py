"""gs.materials: the MPM family (gs.materials.MPM.*), and Rigid and Tool, whose entities enter
this build as kinematic colliders coupled in the MPM grid op."""

from . import MPM
from .rigid import Rigid
from .tool import Tool

__all__ = ["MPM", "Rigid", "Tool"]
