"""gs.materials.Tool (genesis/engine/materials/tool.py:7-40): a kinematic tool whose mesh's
signed-distance grid pushes MPM material in the grid op."""

from __future__ import annotations

from ..exceptions import GenesisException


class Tool:
    def __init__(self, friction=0.0, coup_softness=0.01, collision=True, sdf_res=128):
        if friction < 0:
            raise GenesisException("`friction` must be non-negative.")
        if coup_softness < 0:
            raise GenesisException("`coup_softness` must be non-negative.")
        if int(sdf_res) < 2 or int(sdf_res) > 1024:
            raise GenesisException("`sdf_res` must be in [2, 1024].")
        self._friction = float(friction)
        self._coup_softness = float(coup_softness)
        self._collision = bool(collision)
        self._sdf_res = int(sdf_res)

    @property
    def friction(self):
        return self._friction

    @property
    def coup_softness(self):
        return self._coup_softness

    @property
    def collision(self):
        return self._collision

    @property
    def sdf_res(self):
        return self._sdf_res
