"""Render fields on the GPU (mpm_solver.py:743-766): particle render buffers and
skinned visual vertices, checked against the same arithmetic on the host."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu


def _scene(n_envs=0):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64),
    )
    cube = scene.add_entity(gs.morphs.Box(lower=(0.4, 0.4, 0.4), upper=(0.6, 0.6, 0.6)),
                            material=gs.materials.MPM.Elastic(E=1e5, nu=0.3))
    ball = scene.add_entity(gs.morphs.Sphere(pos=(0.3, 0.7, 0.3), radius=0.08),
                            material=gs.materials.MPM.ElastoPlastic())
    sand = scene.add_entity(gs.morphs.Box(lower=(0.7, 0.2, 0.1), upper=(0.8, 0.3, 0.2)),
                            material=gs.materials.MPM.Sand())
    scene.build(n_envs=n_envs)
    return scene, cube, ball, sand


def test_render_fields_match_host_arithmetic():
    scene, cube, ball, sand = _scene(n_envs=2)
    assert cube.n_vverts == 8 and ball.n_vverts == 642 and sand.n_vverts == 0  # sand is not skinned
    sand.set_particles_active(torch.zeros(sand.n_particles, dtype=torch.uint8))
    for _ in range(3):
        scene.step()
    solver = scene.sim.mpm_solver
    solver.update_render_fields()
    st = scene.get_state()[3]
    pos, vel, act = st.pos.cpu().numpy(), st.vel.cpu().numpy(), st.active.cpu().numpy()
    pr = {k: v.cpu().numpy() for k, v in solver.particles_render.items()}
    nowhere = np.array([2333333.0, 6666666.0, 5201314.0], dtype=np.float32)
    assert np.array_equal(pr["active"].astype(bool), act)
    assert np.array_equal(pr["pos"][act], pos[act]) and (pr["pos"][~act] == nowhere).all()
    assert np.array_equal(pr["vel"][act], vel[act])
    idx = solver._vv_idx.cpu().numpy()
    w = solver._vv_w.cpu().numpy()
    vv = np.einsum("vk,bvkd->bvd", w.astype(np.float64), pos[:, idx].astype(np.float64))
    got = solver.vverts_render["pos"].cpu().numpy()
    assert got.shape == (2, 650, 3)
    assert np.abs(got - vv).max() < 1e-5
    assert solver.vverts_render["active"].cpu().numpy().all()


def test_vverts_follow_a_rigid_translation():
    scene, cube, ball, sand = _scene()
    solver = scene.sim.mpm_solver
    solver.update_render_fields()
    v0 = solver.vverts_render["pos"][0, : cube.n_vverts].clone()
    assert torch.allclose(v0.cpu(), torch.as_tensor(cube.vverts, dtype=torch.float32), atol=1e-5)
    cube.set_particles_pos(cube.get_particles_pos() + torch.tensor([0.05, -0.02, 0.01], device="cuda"))
    solver.update_render_fields()
    v1 = solver.vverts_render["pos"][0, : cube.n_vverts]
    assert torch.allclose(v1 - v0, torch.tensor([0.05, -0.02, 0.01], device="cuda"), atol=1e-5)
