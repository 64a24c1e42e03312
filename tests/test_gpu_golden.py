"""The CUDA path against the committed golden fixtures (tests/golden/): grid sums after the
first p2g and particle state after 1, 10 and 100 substeps.  The three batch fixtures run
together as instances of one runtime.  Positions are held to max(1e-5 m, 2x the float32
CPU restatement's own deviation from the fixture)."""

import glob
import json
import os

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")


def _desc(z):
    meta = json.loads(str(z["meta"]))
    return W.SceneDesc(
        name=meta["name"], grid_density=meta["grid_density"], particle_size=meta["particle_size"], dt=meta["dt"],
        n_substeps=100, pos=z["pos"], vel=z["vel"], mat_idx=z["mat_idx"],
        materials=[(k, dict(kw)) for k, kw in meta["materials"]], lower_bound=tuple(meta["lower_bound"]),
        upper_bound=tuple(meta["upper_bound"]), gravity=tuple(meta["gravity"]))


def _f32_dev(z, n):
    from oracle import cref
    from oracle import mpm_ref as R

    d = _desc(z)
    p = R.Params(grid_density=d.grid_density, lower_bound=d.lower_bound, upper_bound=d.upper_bound,
                 particle_size=d.particle_size, dt=d.dt, gravity=d.gravity, dtype=np.float32)
    mats = [R.make_material(k, **dict(kw)) for k, kw in d.materials]
    st = R.make_state(d.pos, mats, d.mat_idx, np.float32, v=d.vel, active=z["active"])
    o, _ = cref.substeps(p, mats, st, n)
    return np.abs(o["x"] - z[f"x_{n}"]).max()


def _run(zs):
    from genesis_b200.engine.runtime import runtime_from_descs

    rt = runtime_from_descs([_desc(z) for z in zs])
    act = np.concatenate([z["active"] for z in zs])
    off = np.nonzero(~act)[0]
    if off.size:
        rt.set_particles_active(torch.as_tensor(off, dtype=torch.int32), torch.zeros(off.size, dtype=torch.uint8))
    return rt


@pytest.mark.parametrize("name", ["elastic_cube", "elastic_neohookean", "mixed", "mixed_partly_active"])
def test_cuda_path_meets_golden(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    rt = _run([z])
    rt.sort()
    rt.p2g()
    mm, _ = rt.grid_views()
    torch.cuda.synchronize()
    assert np.isclose(float(mm[..., 3].double().sum()), float(z["grid_mass"]), rtol=1e-6)
    mom = mm[..., :3].double().reshape(-1, 3).sum(0).cpu().numpy()
    assert np.allclose(mom, z["grid_momentum"], rtol=1e-5, atol=1e-9 * float(z["grid_mass"]))
    rt = _run([z])  # fresh state
    done = 0
    for n in (1, 10, 100):
        rt.substeps(n - done)
        done = n
        st = rt.get_state()
        x = st["pos"].cpu().numpy()
        tol = max(1e-5, 2 * _f32_dev(z, n))
        assert np.abs(x - z[f"x_{n}"]).max() < tol, (n, tol)
        assert np.abs(st["Jp"].cpu().numpy() - z[f"Jp_{n}"]).max() < max(1e-4, 100 * tol)
        act = z["active"]
        assert np.array_equal(x[~act], z["pos"][~act].astype(np.float32))  # inactive: untouched


def test_batched_instances_meet_golden():
    zs = [np.load(p) for p in sorted(glob.glob(os.path.join(HERE, "batch_*.npz")))]
    assert len(zs) == 3
    rt = _run(zs)
    rt.substeps(100)
    x = rt.get_state()["pos"].cpu().numpy()
    offs = rt.instance_offsets
    for i, z in enumerate(zs):
        n = len(z["pos"])
        tol = max(1e-5, 2 * _f32_dev(z, 100))
        assert np.abs(x[offs[i]: offs[i] + n] - z["x_100"]).max() < tol, i
