"""Build oracle inputs from a genesis_b200.workloads.SceneDesc -- test infrastructure only."""

from __future__ import annotations

import numpy as np

from . import mpm_ref as R


def from_desc(desc, dtype=np.float64, gravity=None, model_dtype=None):
    """Oracle inputs for `desc` computed in `dtype`.  model_dtype: the precision whose gs.EPS
    the model uses (EPS = max(1e-15, finfo.eps), genesis/__init__.py:205-206; it enters the
    grid mass threshold and Matrix.norm(EPS) of the plastic return mappings).  Default: the
    arithmetic dtype, as gs.init(precision=...) sets both.  from_desc(d, float64,
    model_dtype=float32) is the reference's precision-32 model evaluated in float64."""
    p = R.Params(
        grid_density=desc.grid_density,
        lower_bound=desc.lower_bound,
        upper_bound=desc.upper_bound,
        particle_size=desc.particle_size,
        dt=desc.dt,
        gravity=desc.gravity if gravity is None else gravity,
        dtype=dtype,
    )
    if model_dtype is not None:
        p.eps = max(1e-15, float(np.finfo(model_dtype).eps))
    mats = [R.make_material(k, **kw) for k, kw in desc.materials]
    st = R.make_state(desc.pos, mats, desc.mat_idx, dtype, v=desc.vel)
    return p, mats, st
