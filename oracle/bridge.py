"""Build oracle inputs from a genesis_b200.workloads.SceneDesc -- test infrastructure only."""

from __future__ import annotations

import numpy as np

from . import mpm_ref as R


def from_desc(desc, dtype=np.float64, gravity=None):
    p = R.Params(
        grid_density=desc.grid_density,
        lower_bound=desc.lower_bound,
        upper_bound=desc.upper_bound,
        particle_size=desc.particle_size,
        dt=desc.dt,
        gravity=desc.gravity if gravity is None else gravity,
        dtype=dtype,
    )
    mats = [R.make_material(k, **kw) for k, kw in desc.materials]
    st = R.make_state(desc.pos, mats, desc.mat_idx, dtype, v=desc.vel)
    return p, mats, st
