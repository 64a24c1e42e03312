"""The adjoint through tools (mpm_substep_adjoint_colliders behind a differentiable gs.Scene):
gradients with respect to a tool's position (set_position before the first step), its velocity
in every step (set_velocity, as tests/test_grad.py:20-103 gives it) and the block's initial
velocity, against the float64 oracle (oracle/mpm_adjoint.py: rollout_colliders, itself checked
against central differences in tests/test_oracle_adjoint_tools.py).

The scene: an Elastic block falling onto a disc-shaped tool that rises into it (30 substeps,
the tool in contact for most of them).  Tolerance: every gradient within 2e-3 of the largest
gradient of its kind (float32 kernels against the float64 oracle over a contact rollout).
"""

import os

import numpy as np
import pytest
import torch

import genesis_b200 as gs
from genesis_b200 import mesh

pytestmark = pytest.mark.gpu

SUB, DT, STEPS = 5, 1e-3, 6
E_BLOCK = 2e4


def _write_obj(path, v, f):
    with open(path, "w") as fh:
        for q in v:
            fh.write(f"v {q[0]:.9f} {q[1]:.9f} {q[2]:.9f}\n")
        for t in f:
            fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    return path


def _scene(tmp_path, n_envs=0):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=DT, substeps=SUB, gravity=(0, 0, -9.8), requires_grad=True),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.01),
    )
    block = scene.add_entity(gs.morphs.Box(lower=(0.45, 0.45, 0.2), upper=(0.53, 0.53, 0.26)),
                             material=gs.materials.MPM.Elastic(E=E_BLOCK, nu=0.3))
    v, f = mesh.cylinder_mesh(radius=0.5, height=0.25, sections=32)
    path = _write_obj(os.path.join(tmp_path, "disc.obj"), v, f)
    tool = scene.add_entity(gs.morphs.Mesh(file=path, scale=0.2, pos=(0.49, 0.49, 0.17), euler=(0, 15, 0)),
                            material=gs.materials.Tool(friction=0.4, sdf_res=48))
    scene.build(n_envs=n_envs) if n_envs else scene.build()
    return scene, block, tool


def _run(scene, block, tool, p0, vb, v_steps, W):
    """The differentiable run: returns (loss, dL/dp0, dL/dvb, [dL/dv_i])."""
    p0 = torch.tensor(p0, dtype=torch.float32, device="cuda", requires_grad=True)
    vb = torch.tensor(vb, dtype=torch.float32, device="cuda", requires_grad=True)
    vs = [torch.tensor(v, dtype=torch.float32, device="cuda", requires_grad=True) for v in v_steps]
    tool.set_position(p0)
    block.set_velocity(vb)
    for i in range(STEPS):
        tool.set_velocity(vel=vs[i])
        scene.step()
    pos = scene.get_state().solvers_state[3].pos
    loss = (pos * torch.as_tensor(W, dtype=torch.float32, device="cuda")).sum()
    loss.backward()
    assert scene._sim.mpm_solver.runtime.status() == 0
    return float(loss), p0.grad.cpu().numpy(), vb.grad.cpu().numpy(), [v.grad.cpu().numpy() for v in vs]


def _oracle(scene, block, tool, p0, vb, v_steps, W):
    from oracle import mpm_adjoint as A
    from oracle import mpm_ref as R

    from genesis_b200.engine.rigid import quat_to_R

    rt = scene._sim.mpm_solver.runtime
    x0 = np.asarray(block.init_particles, dtype=np.float64)
    n = len(x0)
    p = R.Params(grid_density=64, particle_size=0.01, dt=DT / SUB, dtype=np.float64)
    mats = [R.make_material("elastic", E=E_BLOCK, nu=0.3)]
    st = R.make_state(x0, mats, np.zeros(n, np.int64), np.float64, v=np.tile(vb, (n, 1)))
    mu, lam = np.full(n, mats[0].mu), np.full(n, mats[0].lam)
    res = tool.material.sdf_res
    vox = rt.sdf_voxels[: res ** 3].cpu().numpy().astype(np.float64).reshape(res, res, res)
    col = R.Collider("tool", np.asarray(p0, dtype=np.float64), quat_to_R(tool.morph.quat), np.zeros(3),
                     friction=tool.material.friction, softness=tool.material.coup_softness, restitution=0.0,
                     sdf=vox, sdf_scale=tool._sdf_scale, floor=0.0)
    lin = np.repeat(np.asarray(v_steps, dtype=np.float64), SUB, axis=0)[:, None, :]
    loss, v_bar, pos_bar, lin_bar = A.rollout_colliders(p, mats, st, mu, lam, [col], lin, W)
    free = A.rollout_colliders(p, mats, st, mu, lam, [col], lin + np.array([0.0, 0.0, -50.0]), W, grad=False)
    return loss, free, pos_bar[0], v_bar.sum(0), lin_bar[:, 0].reshape(STEPS, SUB, 3).sum(1)


def test_tool_position_and_velocity_gradients_match_oracle(tmp_path):
    scene, block, tool = _scene(tmp_path)
    rng = np.random.default_rng(3)
    W = rng.normal(size=(block.n_particles, 3))
    p0 = np.array([0.49, 0.49, 0.17])
    vb = np.array([0.1, 0.0, -1.0])
    v_steps = [np.array([0.05 * i, 0.0, 1.0]) for i in range(STEPS)]
    lg, gp, gvb, gvs = _run(scene, block, tool, p0, vb, v_steps, W)
    lo, lfree, op, ovb, ovs = _oracle(scene, block, tool, p0, vb, v_steps, W)
    assert abs(lo - lfree) > 1e-3 * abs(lo)  # the tool changed the outcome
    ep = np.abs(gp - op).max() / np.abs(op).max()
    eb = np.abs(gvb - ovb).max() / np.abs(ovb).max()
    gvs, ovs = np.stack(gvs), np.asarray(ovs)
    es = np.abs(gvs - ovs).max() / np.abs(ovs).max()
    print(f"\n[grad] tool: loss {lg:.6e} (oracle {lo:.6e}); dL/d(tool pos) {gp} (oracle {op}), rel. err {ep:.1e}; "
          f"dL/d(tool vel per step) rel. err {es:.1e}; dL/d(block vel) rel. err {eb:.1e}")
    assert abs(lg - lo) <= 1e-4 * abs(lo)
    assert np.abs(ovs).max() > 1e-3 * np.abs(ovb).max()  # the tool's velocity matters
    assert ep <= 2e-3 and es <= 2e-3 and eb <= 2e-3


def test_tool_gradients_per_environment(tmp_path):
    """Two environments, one tool velocity per environment ([2, 3] inputs): each environment's
    rows get the gradient of its own half of the loss, equal to the one-environment run."""
    scene, block, tool = _scene(tmp_path, n_envs=2)
    rng = np.random.default_rng(3)
    n = block.n_particles
    W1 = rng.normal(size=(n, 3))
    p0 = torch.tensor([[0.49, 0.49, 0.17], [0.49, 0.49, 0.17]], device="cuda", requires_grad=True)
    vs = [torch.tensor([[0.05 * i, 0.0, 1.0], [0.05 * i, 0.0, 1.0]], device="cuda", requires_grad=True)
          for i in range(STEPS)]
    tool.set_position(p0)
    block.set_velocity(torch.tensor([0.1, 0.0, -1.0], device="cuda"))
    for i in range(STEPS):
        tool.set_velocity(vel=vs[i])
        scene.step()
    pos = scene.get_state().solvers_state[3].pos  # [2, n, 3]
    W = torch.as_tensor(np.stack([W1, 0.5 * W1]), dtype=torch.float32, device="cuda")
    (pos * W).sum().backward()
    g = p0.grad.cpu().numpy()
    assert np.abs(g[1] - 0.5 * g[0]).max() <= 1e-5 * np.abs(g[0]).max()
    gv = np.stack([v.grad.cpu().numpy() for v in vs])
    assert np.abs(gv[:, 1] - 0.5 * gv[:, 0]).max() <= 1e-5 * np.abs(gv[:, 0]).max()
    lo, _, op, _, ovs = _oracle(scene, block, tool, np.array([0.49, 0.49, 0.17]), np.array([0.1, 0.0, -1.0]),
                                [np.array([0.05 * i, 0.0, 1.0]) for i in range(STEPS)], W1)
    assert np.abs(g[0] - op).max() <= 2e-3 * np.abs(op).max()
    assert np.abs(gv[:, 0] - np.asarray(ovs)).max() <= 2e-3 * np.abs(np.asarray(ovs)).max()
