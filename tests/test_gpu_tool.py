"""Tool entities on the GPU (tool_entity/mesh.py:80-176, legacy_coupler.py:346-350): the
voxel signed-distance grid of mpm_sdf_voxelize against the float64 oracle, an MPM block
pushed by a moving, spinning tool against the C restatement, the tool's kinematics and its
floor, and tools in differentiable scenes."""

import os

import numpy as np
import pytest
import torch

import genesis_b200 as gs
from genesis_b200 import mesh

pytestmark = pytest.mark.gpu


def _write_obj(path, v, f):
    with open(path, "w") as fh:
        for q in v:
            fh.write(f"v {q[0]:.9f} {q[1]:.9f} {q[2]:.9f}\n")
        for t in f:
            fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    return path


@pytest.mark.parametrize("shape", ["box", "sphere", "cylinder"])
def test_voxelize_matches_oracle(shape):
    from oracle import sdf_ref

    from genesis_b200.engine.tool import sdf_voxels

    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    if shape == "box":
        v, f = mesh.box_mesh((0.7, 0.5, 0.9))
    elif shape == "sphere":
        v, f = mesh.icosphere(subdivisions=2, radius=0.45)
    else:
        v, f = mesh.cylinder_mesh(radius=0.3, height=1.0, sections=24)
    res = 21
    g = sdf_voxels(v, f, res, "cuda").cpu().numpy().astype(np.float64)
    o = sdf_ref.sdf_voxels(v, f, res)
    assert np.abs(g - o).max() < 2e-5
    assert (g < 0).sum() > 0 and (g > 0).sum() > 0


def _scene(tmp_path, n_envs=0, tool_pos=(0.5, 0.5, 0.3), friction=0.4, **tool_opts):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.01),
        **tool_opts,
    )
    block = scene.add_entity(gs.morphs.Box(lower=(0.42, 0.42, 0.36), upper=(0.58, 0.58, 0.46)),
                             material=gs.materials.MPM.Elastic(E=2e4))
    v, f = mesh.cylinder_mesh(radius=0.5, height=0.25, sections=32)
    path = _write_obj(os.path.join(tmp_path, "disc.obj"), v, f)
    tool = scene.add_entity(gs.morphs.Mesh(file=path, scale=0.4, pos=tool_pos, euler=(0, 20, 0)),
                            material=gs.materials.Tool(friction=friction, sdf_res=64))
    scene.build(n_envs=n_envs)
    return scene, block, tool


def _oracle(block, tool, rt, v0, lin, ang, n_substeps, tool_pos=None):
    from oracle import cref
    from oracle import mpm_ref as R

    from genesis_b200.engine.rigid import quat_to_R

    x = block.get_particles_pos().cpu().numpy().astype(np.float64).reshape(-1, 3)
    n = len(x)
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-4, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile(v0, (n, 1)))
    res = tool.material.sdf_res
    vox = rt.sdf_voxels[: res ** 3].cpu().numpy().astype(np.float64).reshape(res, res, res)
    pos = np.asarray(tool.morph.pos if tool_pos is None else tool_pos, dtype=np.float64)
    st["colliders"] = [R.Collider("tool", pos, quat_to_R(tool.morph.quat), np.zeros(3), np.asarray(lin, float),
                                  np.asarray(ang, float), friction=tool.material.friction,
                                  softness=tool.material.coup_softness, restitution=0.0, sdf=vox,
                                  sdf_scale=tool._sdf_scale, floor=0.0)]
    out, rc = cref.substeps(p, mats, st, n_substeps)
    assert rc == 0
    return out


def test_moving_tool_pushes_block_matches_oracle(tmp_path):
    scene, block, tool = _scene(tmp_path)
    rt = scene._sim.mpm_solver.runtime
    v0, lin, ang = (0.0, 0.0, -1.5), (0.0, 0.0, 0.4), (0.0, 0.0, 3.0)
    block.set_particles_vel(torch.tensor(v0).expand(block.n_particles, 3))
    tool.set_velocity(vel=lin, ang=ang)
    o = _oracle(block, tool, rt, v0, lin, ang, 40)
    free = _oracle(block, tool, rt, v0, lin, ang, 40, tool_pos=(0.5, 0.5, -5.0))
    assert np.abs(o["x"] - free["x"]).max() > 1e-4  # the tool changed the trajectory (10x the tolerance)
    for _ in range(4):
        scene.step()
    g = block.get_particles_pos().cpu().numpy()
    assert np.abs(g - o["x"]).max() < 1e-5
    gv = block.get_particles_vel().cpu().numpy()
    assert np.abs(gv - o["v"]).max() < 2e-3
    st = tool.get_state()
    assert np.allclose(st.pos.cpu().numpy()[0], o["colliders"][0].pos, atol=1e-6)


def test_tool_kinematics_floor_and_environments(tmp_path):
    scene, block, tool = _scene(tmp_path, n_envs=2, tool_pos=(0.3, 0.3, 0.001))
    tool.set_velocity(vel=torch.tensor([[0.5, 0.0, -2.0], [0.0, 0.2, 1.0]]), ang=(0.0, 0.0, 4.0))
    q0 = tool.get_state().quat.cpu().numpy()
    scene.step()  # 10 substeps of 1e-4 s
    st = tool.get_state()
    pos = st.pos.cpu().numpy()
    assert np.allclose(pos[0], [0.3005, 0.3, 0.0], atol=1e-6)  # clamped to the floor height
    assert np.allclose(pos[1], [0.3, 0.3002, 0.002], atol=1e-6)
    assert np.allclose(st.vel.cpu().numpy(), [[0.5, 0.0, -2.0], [0.0, 0.2, 1.0]])
    # quat = exp(ang dt) quat0: the relative rotation is 4e-3 rad about z in both environments
    from genesis_b200.engine.rigid import quat_to_R

    for e in range(2):
        Rrel = quat_to_R(st.quat.cpu().numpy()[e]) @ quat_to_R(q0[e]).T
        assert np.isclose(np.arctan2(Rrel[1, 0], Rrel[0, 0]), 4e-3, atol=1e-6)


def test_tool_floor_height_from_options(tmp_path):
    scene, block, tool = _scene(tmp_path, tool_pos=(0.3, 0.3, 0.2),
                                tool_options=gs.options.ToolOptions(floor_height=0.15))
    tool.set_velocity(vel=(0.0, 0.0, -100.0))
    scene.step()
    assert np.isclose(tool.get_state().pos.cpu().numpy()[0, 2], 0.15)


def test_differentiable_scene_takes_tools(tmp_path):
    """A differentiable scene with a tool builds and steps; the tool's inputs become step inputs
    (their gradients are checked in tests/test_gpu_tool_grad.py)."""
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, requires_grad=True))
    scene.add_entity(gs.morphs.Box(lower=(0.4, 0.4, 0.4), upper=(0.5, 0.5, 0.5)), material=gs.materials.MPM.Elastic())
    v, f = mesh.cylinder_mesh()
    path = _write_obj(os.path.join(tmp_path, "t.obj"), v, f)
    tool = scene.add_entity(gs.morphs.Mesh(file=path, scale=0.1, pos=(0.5, 0.5, 0.2)), material=gs.materials.Tool())
    scene.build()
    tool.set_velocity(vel=(0.0, 0.0, 0.5))
    scene.step()
    assert np.allclose(tool.get_state().pos.cpu().numpy()[0], [0.5, 0.5, 0.2 + 0.5e-3], atol=1e-6)


def test_scene_state_holds_tools_and_reset_restores_them(tmp_path):
    """The scene's state carries the tool solver's state at solvers_state[0] (one
    ToolEntityState per tool, states/solvers.py:114-133); scene.reset(state) puts the tools
    back where that state had them."""
    scene, block, tool = _scene(tmp_path, n_envs=2)
    tool.set_velocity(vel=(0.1, 0.0, 0.2), ang=(0.0, 1.0, 0.0))
    scene.step()
    s1 = scene.get_state()
    ts = s1.solvers_state[0]
    assert len(ts) == 1 and s1.solvers_state[3] is not None
    assert torch.allclose(ts[0].pos, tool.get_state().pos)
    pos1, quat1 = ts[0].pos.clone(), ts[0].quat.clone()
    x1 = block.get_particles_pos().clone()
    for _ in range(3):
        scene.step()
    assert not torch.allclose(tool.get_state().pos, pos1)
    scene.reset(s1)
    st = tool.get_state()
    assert torch.allclose(st.pos, pos1, atol=1e-7)
    assert torch.allclose(st.quat, quat1, atol=1e-6)
    assert torch.allclose(block.get_particles_pos(), x1)
    scene.reset()  # the built poses
    assert np.allclose(tool.get_state().pos.cpu().numpy(), [[0.5, 0.5, 0.3]] * 2, atol=1e-7)
