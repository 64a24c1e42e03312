"""Kinematic rigid colliders coupled in the grid op (legacy_coupler.py:131-343, 385-397) on
the GPU: trajectories and reaction forces match the float64 oracle; colliders move with
their velocity."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu


def _scene(morph, substeps=10, n_envs=0, exact_box=False, **rigid_kw):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-4 * substeps, substeps=substeps, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.01),
        b200_options=gs.options.B200Options(exact_box_sdf=exact_box),
    )
    block = scene.add_entity(gs.morphs.Box(lower=(0.45, 0.45, 0.33), upper=(0.55, 0.55, 0.43)),
                             material=gs.materials.MPM.Elastic(E=2e4))
    rigid = scene.add_entity(morph, material=gs.materials.Rigid(**rigid_kw))
    scene.build(n_envs=n_envs)
    return scene, block, rigid


def _oracle(block, collider, v0, n_substeps):
    from oracle import cref
    from oracle import mpm_ref as R

    x = block.get_particles_pos().cpu().numpy().astype(np.float64)
    n = len(x)
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-4, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile(v0, (n, 1)))
    st["colliders"] = [collider]
    out, rc = cref.substeps(p, mats, st, n_substeps)
    assert rc == 0
    return out


@pytest.mark.parametrize("kind", ["sphere", "box", "box_exact", "plane"])
def test_block_on_rigid_collider_matches_oracle(kind):
    """box: the reference's sampled signed-distance grid (rigid_geom.py:147-193, trilinear
    lookups utils/sdf_decomp.py:102-276); box_exact: B200Options(exact_box_sdf=True)."""
    from genesis_b200.engine.rigid import box_sdf_grid
    from oracle import mpm_ref as R

    if kind == "sphere":
        morph = gs.morphs.Sphere(pos=(0.5, 0.5, 0.25), radius=0.06)
        col = R.Collider("sphere", np.array([0.5, 0.5, 0.25]), np.eye(3), np.array([0.06, 0, 0]), friction=0.3)
    elif kind in ("box", "box_exact"):
        morph = gs.morphs.Box(pos=(0.52, 0.5, 0.2), size=(0.3, 0.3, 0.2), euler=(0, 10, 0))
        Rm = gs.morphs._quat_to_R(np.asarray(morph.quat))
        half = np.array([0.15, 0.15, 0.1])
        if kind == "box_exact":
            col = R.Collider("box", np.array([0.52, 0.5, 0.2]), Rm, half, friction=0.3)
        else:
            val, grad, scale, cell, vmax = box_sdf_grid(half)
            col = R.Collider("sdf", np.array([0.52, 0.5, 0.2]), Rm, np.zeros(3), friction=0.3, sdf=val, sdf_scale=scale,
                             sdf_grad=grad, sdf_cell=cell, sdf_max=vmax)
    else:
        morph = gs.morphs.Plane(pos=(0.5, 0.5, 0.3), normal=(0.2, 0.0, 1.0))
        nrm = np.array([0.2, 0.0, 1.0]) / np.linalg.norm([0.2, 0.0, 1.0])
        col = R.Collider("plane", np.array([0.5, 0.5, 0.3]), np.eye(3), nrm, friction=0.3)
    scene, block, rigid = _scene(morph, exact_box=kind == "box_exact", coup_friction=0.3)
    v0 = (0.0, 0.0, -2.0)
    block.set_particles_vel(torch.tensor(v0).expand(block.n_particles, 3))
    o = _oracle(block, col, v0, 40)
    away = R.Collider(col.kind, np.array([0.5, 0.5, -5.0]), col.rot, col.data, sdf=col.sdf, sdf_scale=col.sdf_scale,
                      sdf_grad=col.sdf_grad, sdf_cell=col.sdf_cell, sdf_max=col.sdf_max)
    free = _oracle(block, away, v0, 40)
    assert np.abs(o["x"] - free["x"]).max() > 1e-4  # the collider changed the trajectory (10x the tolerance)
    for _ in range(4):
        scene.step()
    g = block.get_particles_pos().cpu().numpy()
    assert np.abs(g - o["x"]).max() < 1e-5
    f = rigid.get_coupling_force().cpu().numpy()
    # the last step's mean force; the oracle accumulated all 40 substeps
    assert f[2] < 0 and np.isfinite(f).all()


def test_collider_moves_with_its_velocity_and_resets():
    scene, block, rigid = _scene(gs.morphs.Sphere(pos=(0.3, 0.3, 0.2), radius=0.05))
    rigid.set_dofs_velocity([0.5, 0.0, 0.2, 0.0, 0.0, 4.0])
    scene.step()  # 10 substeps of 1e-4 s
    assert torch.allclose(rigid.get_pos().cpu(), torch.tensor([0.3005, 0.3, 0.2002]), atol=1e-6)
    q = rigid.get_quat().cpu().numpy()
    assert np.isclose(2 * np.arctan2(q[3], q[0]), 4.0 * 1e-3, atol=1e-6)
    rigid.set_pos((0.6, 0.6, 0.2))
    assert torch.allclose(rigid.get_pos().cpu(), torch.tensor([0.6, 0.6, 0.2]))
    scene.reset()
    assert torch.allclose(rigid.get_pos().cpu(), torch.tensor([0.3, 0.3, 0.2]))
    assert torch.equal(rigid.get_dofs_velocity().cpu(), torch.zeros(6))


def test_colliders_per_environment():
    scene, block, rigid = _scene(gs.morphs.Plane(pos=(0.5, 0.5, 0.3)), n_envs=2)
    rigid.set_pos(torch.tensor([[0.5, 0.5, 0.3], [0.5, 0.5, 0.2]]))
    block.set_particles_vel(torch.tensor([0.0, 0.0, -2.5]).expand(block.n_particles, 3))
    for _ in range(20):
        scene.step()
    z = block.get_particles_pos()[..., 2].min(dim=1).values.cpu()
    assert z[0] > 0.3 - 1.5 / 64 and z[1] < z[0] - 0.01  # env 1's floor is lower


def test_block_on_rigid_mesh_matches_oracle(tmp_path):
    """A rigid Mesh (a tilted, off-origin icosphere, convex: its collision geom is its hull) through
    the reference's sampled grid (rigid_geom.py:147-193): the grid mpm_sdf_grid samples against
    the float64 signed-distance oracle at its nodes, then a block landing on it against the C
    restatement through the same grid."""
    from genesis_b200 import mesh
    from oracle import mpm_ref as R
    from oracle import sdf_ref

    v, f = mesh.icosphere(subdivisions=2, radius=0.5)
    v = v + np.array([0.1, -0.05, 0.0])  # off the mesh origin: the grid is centred on the bounds
    path = tmp_path / "ball.obj"
    with open(path, "w") as fh:
        for q in v:
            fh.write(f"v {q[0]:.9f} {q[1]:.9f} {q[2]:.9f}\n")
        for t in f:
            fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    morph = gs.morphs.Mesh(file=str(path), scale=0.14, pos=(0.49, 0.5, 0.26), euler=(0, 15, 10))
    # the hull's top (z ~ 0.33) sits just under the falling block (z >= 0.335), inside its grid
    scene, block, rigid = _scene(morph, coup_friction=0.3)
    val, grad, scale, cell, vmax = rigid._grid
    centre = rigid._data
    res = np.array(val.shape)
    # the sampled distances at a random subset of the nodes against the oracle's exact ones
    rng = np.random.default_rng(0)
    idx = rng.integers(0, res, size=(400, 3))
    pts = centre + (idx - (res - 1) / 2) * cell
    exact = sdf_ref.signed_distance(pts, morph.vertices, morph.faces)
    assert np.abs(val[idx[:, 0], idx[:, 1], idx[:, 2]] - exact).max() < 2e-6
    Rm = gs.morphs._quat_to_R(np.asarray(morph.quat))
    col = R.Collider("sdf", np.array(morph.pos), Rm, centre.astype(np.float64), friction=0.3,
                     sdf=val.astype(np.float64), sdf_scale=scale, sdf_grad=grad.astype(np.float64), sdf_cell=cell,
                     sdf_max=vmax)
    v0 = (0.0, 0.0, -2.0)
    block.set_particles_vel(torch.tensor(v0).expand(block.n_particles, 3))
    o = _oracle(block, col, v0, 40)
    away = R.Collider("sdf", np.array([0.5, 0.5, -5.0]), Rm, col.data, sdf=col.sdf, sdf_scale=scale,
                      sdf_grad=col.sdf_grad, sdf_cell=cell, sdf_max=vmax)
    free = _oracle(block, away, v0, 40)
    assert np.abs(o["x"] - free["x"]).max() > 1e-4  # the mesh changed the trajectory (10x the tolerance)
    for _ in range(4):
        scene.step()
    g = block.get_particles_pos().cpu().numpy()
    print(f"\n[rigid mesh] grid {tuple(res)}, cell {cell:.4f}: max|dx| vs oracle {np.abs(g - o['x']).max():.2e}")
    assert np.abs(g - o["x"]).max() < 1e-5
