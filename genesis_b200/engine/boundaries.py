"""CubeBoundary (genesis/engine/boundaries/boundaries.py:11-49).  The boundary's
arithmetic runs inside the grid-op and g2p kernels; this object carries its bounds."""

from __future__ import annotations

import numpy as np


class CubeBoundary:
    def __init__(self, lower, upper, restitution=0.0):
        self.restitution = restitution
        self.upper = np.array(upper, dtype=np.float32)
        self.lower = np.array(lower, dtype=np.float32)
        assert (self.upper >= self.lower).all()

    def is_inside(self, pos):
        return bool(np.all(pos < self.upper) and np.all(pos > self.lower))

    def impose_pos_vel(self, pos, vel):
        """Host restatement for small arrays (vel component toward an outside wall is zeroed, pos clamped)."""
        pos = np.array(pos, dtype=np.float32, copy=True)
        vel = np.array(vel, dtype=np.float32, copy=True)
        for i in range(3):
            up = (pos[..., i] >= self.upper[i]) & (vel[..., i] >= 0)
            dn = (~up) & (pos[..., i] <= self.lower[i]) & (vel[..., i] <= 0)
            vel[..., i] = np.where(up | dn, vel[..., i] * -self.restitution, vel[..., i])
        return np.clip(pos, self.lower, self.upper), vel

    def __repr__(self):
        return f"CubeBoundary(lower={self.lower}, upper={self.upper}, restitution={self.restitution})"
