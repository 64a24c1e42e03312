"""gs.materials: only the MPM family is on this path (gs.materials.MPM.*)."""

from . import MPM

__all__ = ["MPM"]
