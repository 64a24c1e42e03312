"""Generate the golden fixtures of this directory from the float64 numpy oracle
(oracle/mpm_ref.py) -- the reference itself (gstaichi) cannot run here, so the fixtures pin
the oracle and give the CUDA path fixed vectors to meet.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz

Each fixture is one seeded scene: its inputs (positions, velocities, material indices,
active mask, the materials as JSON, grid/time constants), the grid mass and momentum
totals after the first p2g, and the full particle state (x, v, C, F, Jp) after 1, 10 and
100 substeps, all float64.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from genesis_b200 import workloads as W  # noqa: E402
from oracle import mpm_ref as R  # noqa: E402

SNAPSHOTS = (1, 10, 100)


def scenes():
    out = {}
    out["elastic_cube"] = W.elastic_cube(n_side=5)
    neo = W.elastic_cube(seed=5, n_side=5)
    neo.materials = [("elastic", dict(E=1e5, nu=0.3, rho=1000.0, model="neohooken"))]
    out["elastic_neohookean"] = neo
    out["mixed"] = W.mixed_500k(n_side=5, grid_density=32)
    act = W.mixed_500k(seed=7, n_side=5, grid_density=32)
    act.meta["active"] = (np.arange(act.n_particles) % 3 != 0)
    out["mixed_partly_active"] = act
    for i, d in enumerate(W.batch_scenes(seed=9, n_scenes=3, n_range=(80, 200), densities=(32, 64))):
        out[f"batch_{i}"] = d
    return out


def run(d):
    p = R.Params(grid_density=d.grid_density, lower_bound=d.lower_bound, upper_bound=d.upper_bound,
                 particle_size=d.particle_size, dt=d.dt, gravity=d.gravity, dtype=np.float64)
    mats = [R.make_material(k, **dict(kw)) for k, kw in d.materials]
    active = d.meta.get("active")
    st = R.make_state(d.pos, mats, d.mat_idx, np.float64, v=d.vel, active=active)
    gm, gp, _, _ = R.p2g(p, mats, st)
    rec = dict(grid_mass=np.array(gm.sum()), grid_momentum=gp.reshape(-1, 3).sum(0))
    done = 0
    for n in SNAPSHOTS:
        st = R.run(p, mats, st, n - done)
        done = n
        for k in ("x", "v", "C", "F", "Jp"):
            rec[f"{k}_{n}"] = st[k]
    return rec


def main():
    for name, d in scenes().items():
        rec = run(d)
        meta = dict(name=name, grid_density=d.grid_density, lower_bound=list(d.lower_bound),
                    upper_bound=list(d.upper_bound), particle_size=d.particle_size, dt=d.dt,
                    gravity=list(d.gravity), materials=[[k, kw] for k, kw in d.materials], snapshots=list(SNAPSHOTS))
        active = d.meta.get("active")
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), meta=np.array(json.dumps(meta)), pos=d.pos, vel=d.vel,
            mat_idx=d.mat_idx, active=np.ones(d.n_particles, bool) if active is None else active, **rec)
        print(name, d.n_particles)


if __name__ == "__main__":
    main()
