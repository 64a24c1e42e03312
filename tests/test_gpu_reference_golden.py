"""The CUDA path against fixtures made by running the REFERENCE's own MPM code
(tests/golden/ref_*.npz, from make_reference_golden.py: Genesis's mpm_solver.py,
legacy_coupler.py, boundaries.py and materials/MPM/*.py executed unchanged on a numpy
stand-in for gstaichi, float64).

* every material variant's return mapping (F_new, Jp_new) and stress, read back after one
  p2g from particles whose stencils do not overlap (so each grid node's momentum is one
  particle's stress contribution);
* whole substeps over 9 material variants (random F, C, Jp, velocity; inactive particles;
  muscle actuation) and a cube thrown at the floor: grid mass/momentum after the first p2g
  and the full state after each snapshot.

Tolerances (float32 kernels against the float64 reference): positions 1e-5 of the 1 m domain
after every snapshot; velocities 1e-5 m/s; F and Jp 1e-5; grid mass and momentum totals 1e-6
relative, per node 1e-5 of the largest node; F_new 2e-6 and Jp_new 2e-6 relative to the
largest entry of each variant, stress (through the momentum it scatters) 1e-5 relative to
each particle's largest node.
"""

import json
import os

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")


def _dense(rt):
    from genesis_b200.engine.runtime import block_major_to_dense

    mm, _ = rt.grid_views()
    torch.cuda.synchronize()
    return block_major_to_dense(mm.cpu().numpy().astype(np.float64), rt.specs[0], int(rt._insts[0].blk_base))


def _weights(fx):
    return [0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2]


def test_material_functions_and_stress_match_reference():
    from genesis_b200.engine.runtime import runtime_from_descs

    z = np.load(os.path.join(HERE, "ref_functions.npz"))
    meta = json.loads(str(z["meta"]))
    variants = meta["variants"]
    nv, n = len(variants), len(z["m0_F_tmp"])
    density, psize, dt = 96, 0.01, 1e-4
    dx = 1.0 / density
    # isolated particles: bases 6 cells apart, so no two stencils share a node and no two
    # particles share a 4^3 grid block (each chunk's fixed-point scale is its one particle's)
    ks = np.stack(np.meshgrid(*[np.arange(1, 16)] * 3, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(3)
    sel = rng.permutation(len(ks))[: nv * n]
    pos = (6 * ks[sel] + 1.0) * dx + rng.uniform(-0.2 * dx, 0.2 * dx, size=(nv * n, 3))
    mat_idx = np.repeat(np.arange(nv), n)
    d = W.SceneDesc(name="ref_functions", grid_density=density, particle_size=psize, dt=dt, n_substeps=1, pos=pos,
                    vel=np.zeros((nv * n, 3)), mat_idx=mat_idx, materials=[(k, dict(kw)) for k, kw in variants],
                    gravity=(0.0, 0.0, 0.0))
    rt = runtime_from_descs([d], use_graphs=False)
    F0 = np.concatenate([z[f"m{v}_F_tmp"] for v in range(nv)])
    Jp0 = np.concatenate([z[f"m{v}_Jp"] for v in range(nv)])
    rt.set_state(pos=pos, C_=np.zeros((nv * n, 3, 3)), F=F0, Jp=Jp0)
    mus = [v for v, (k, _) in enumerate(variants) if k == "muscle"]
    for v in mus:
        idx = np.arange(v * n, (v + 1) * n)
        rt.set_muscle_group(idx, np.zeros(n, dtype=np.int64))
        rt.set_actu_by_group(idx, z[f"m{v}_actu"][:, None])
        rt.set_muscle_direction(idx, z[f"m{v}_mdir"])
    rt.sort()
    rt.p2g()
    st = rt.get_state(("F", "Jp"))
    torch.cuda.synchronize()
    F = st["F"].cpu().numpy().astype(np.float64)
    Jp = st["Jp"].cpu().numpy().astype(np.float64)
    grid = _dense(rt)
    lo = np.round(density * np.asarray(d.lower_bound)).astype(int)
    scale = -dt * (psize**3 * 1e3) * 4 * density * density
    for v in range(nv):
        sl = slice(v * n, (v + 1) * n)
        want_F, want_Jp, want_s = z[f"m{v}_F_new"], z[f"m{v}_Jp_new"], z[f"m{v}_stress"]
        eF = np.abs(F[sl] - want_F).max() / max(1.0, np.abs(want_F).max())
        eJ = np.abs(Jp[sl] - want_Jp).max() / max(1.0, np.abs(want_Jp).max())
        assert eF < 2e-6 and eJ < 2e-6, (variants[v], eF, eJ)
        # stress: node momentum = w * (scale * stress) @ dpos (v = 0, C = 0)
        xi = pos[sl] * density
        base = np.floor(xi - 0.5).astype(int)
        fx = xi - base
        w = _weights(fx)
        got, want = [], []
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    off = np.array([i, j, k])
                    wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
                    dpos = (off - fx) * dx
                    want.append(wt[:, None] * np.einsum("nab,nb->na", scale * want_s, dpos))
                    node = base + off - lo
                    got.append(grid[node[:, 0], node[:, 1], node[:, 2], :3])
        got, want = np.stack(got), np.stack(want)  # [27, n, 3]
        es = (np.abs(got - want).max(axis=(0, 2)) / np.abs(want).max(axis=(0, 2))).max()  # per particle
        assert es < 1e-5, (variants[v], es)


def _scene(name):
    from genesis_b200.engine.runtime import runtime_from_descs

    z = np.load(os.path.join(HERE, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    d = W.SceneDesc(name=name, grid_density=meta["grid_density"], particle_size=meta["particle_size"], dt=meta["dt"],
                    n_substeps=meta["snapshots"][-1], pos=z["pos"], vel=z["vel"], mat_idx=z["mat_idx"],
                    materials=[(k, dict(kw)) for k, kw in meta["materials"]],
                    lower_bound=tuple(meta["lower_bound"]), upper_bound=tuple(meta["upper_bound"]),
                    gravity=tuple(meta["gravity"]))
    rt = runtime_from_descs([d], sort_interval=4)
    rt.set_state(pos=z["pos"], vel=z["vel"], C_=z["C"], F=z["F"], Jp=z["Jp"], active=z["active"].astype(np.uint8))
    if "muscle_idx" in z.files:
        idx = z["muscle_idx"]
        rt.set_muscle_group(idx, z["muscle_group"])
        rt.set_actu_by_group(idx, np.tile(z["muscle_actu"], (len(idx), 1)))
        rt.set_muscle_direction(idx, z["muscle_dir"])
    return z, meta, rt


@pytest.mark.parametrize("name", ["ref_mixed", "ref_cube"])
def test_first_p2g_grid_matches_reference(name):
    z, meta, rt = _scene(name)
    rt.sort()
    rt.p2g()
    g = _dense(rt)
    gm, gp = z["grid_mass"], z["grid_mom"]
    assert abs(g[..., 3].sum() - gm.sum()) <= 1e-6 * gm.sum()
    mscale = np.abs(gp).sum()
    assert np.abs(g[..., :3].reshape(-1, 3).sum(0) - gp.reshape(-1, 3).sum(0)).max() <= 1e-6 * mscale
    assert np.abs(g[..., 3] - gm).max() <= 1e-5 * gm.max()
    assert np.abs(g[..., :3] - gp).max() <= 1e-5 * np.abs(gp).max()


@pytest.mark.parametrize("name", ["ref_mixed", "ref_cube"])
def test_substeps_match_reference(name):
    z, meta, rt = _scene(name)
    done = 0
    act = z["active"]
    for n in meta["snapshots"]:
        rt.substeps(n - done)
        done = n
        st = rt.get_state()
        torch.cuda.synchronize()
        got = {k: st[k].cpu().numpy().astype(np.float64) for k in ("pos", "vel", "F", "Jp")}
        ex = np.abs(got["pos"] - z[f"x_{n}"]).max()
        ev = np.abs(got["vel"] - z[f"v_{n}"]).max()
        eF = np.abs(got["F"] - z[f"F_{n}"]).max()
        eJ = np.abs(got["Jp"] - z[f"Jp_{n}"]).max()
        print(f"{name} after {n}: |dx| {ex:.2e} |dv| {ev:.2e} |dF| {eF:.2e} |dJp| {eJ:.2e}")
        assert ex < 1e-5 and ev < 1e-5 and eF < 1e-5 and eJ < 1e-5, (n, ex, ev, eF, eJ)
        assert np.array_equal(got["pos"][~act], z["pos"][~act].astype(np.float32).astype(np.float64))
    assert rt.status() == 0
