"""Differentiable scenes (SimOptions(requires_grad=True)) through gs.Scene, the way the
reference's scripts use them (tests/test_grad.py, examples/differentiable_push.py): inputs given
with set_position / set_velocity / set_actuation as tensors that require grad, a loss over the
states queried after every step, loss.backward().  Gradients against float64 central
differences of the C restatement run step by step with the same inputs."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu

SUB, DT, P_SIZE = 10, 1e-3, 0.01
GOAL = np.array([0.52, 0.48, 0.2])


def _scene(material):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=DT, substeps=SUB, gravity=(0, 0, -9.8), requires_grad=True),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=P_SIZE),
    )
    ent = scene.add_entity(gs.morphs.Box(pos=(0.5, 0.5, 0.15), size=(0.08, 0.08, 0.08)), material=material)
    scene.build()
    return scene, ent


def _oracle_loss(offsets, pos, vel_by_step, n_steps, mat_kw, kind="elastic", actu_by_step=None, groups=None,
                 shape=False):
    """Sum over steps of |mean position - GOAL|^2 (shape=True: of the mean of |x - GOAL|^2, which
    internal forces such as a muscle's can change), float64 C restatement."""
    from oracle import cref
    from oracle import mpm_ref as R

    p = R.Params(grid_density=64, particle_size=P_SIZE, dt=DT / SUB, dtype=np.float64)
    mats = [R.make_material(kind, **mat_kw)]
    n = len(offsets)
    st = R.make_state(offsets + pos, mats, np.zeros(n, np.int64), np.float64, v=np.zeros((n, 3)))
    loss = 0.0
    for s in range(n_steps):
        if s in vel_by_step:
            st["v"] = np.tile(vel_by_step[s], (n, 1))
        if actu_by_step is not None:
            st["actu"] = np.asarray(actu_by_step[min(s, len(actu_by_step) - 1)])[groups]
            st["mdir"] = np.tile([0.0, 0.0, 1.0], (n, 1))
        st, rc = cref.substeps(p, mats, st, SUB)
        assert rc == 0
        if shape:
            loss += float(((st["x"] - GOAL) ** 2).sum(1).mean())
        else:
            loss += float(((st["x"].mean(0) - GOAL) ** 2).sum())
    return loss


def test_position_and_velocity_inputs_with_a_trajectory_loss():
    mat_kw = dict(E=2e4, nu=0.3, rho=1000.0)
    scene, ent = _scene(gs.materials.MPM.Elastic(**mat_kw))
    offsets = ent.init_particles - np.asarray(ent.morph.pos)
    pos = gs.tensor([0.5, 0.5, 0.15], requires_grad=True)  # as the reference's scripts create inputs
    v0 = torch.tensor([0.3, -0.2, -1.0], device="cuda", requires_grad=True)
    v3 = torch.tensor([-0.4, 0.1, 0.5], device="cuda", requires_grad=True)
    ent.set_position(pos)
    ent.set_velocity(v0)
    goal = torch.tensor(GOAL, dtype=torch.float32, device="cuda")
    loss = 0.0
    for s in range(6):
        if s == 3:
            ent.set_velocity(v3)  # an input in the middle of the rollout
        scene.step()
        st = scene.get_state().solvers_state[3]
        loss = loss + ((st.pos[0].mean(0) - goal) ** 2).sum()
    loss.backward()
    vals = {"pos": pos.detach().cpu().numpy().astype(np.float64), "v0": v0.detach().cpu().numpy().astype(np.float64),
            "v3": v3.detach().cpu().numpy().astype(np.float64)}
    L = lambda a: _oracle_loss(offsets, a["pos"], {0: a["v0"], 3: a["v3"]}, 6, mat_kw)
    assert abs(float(loss.detach()) - L(vals)) <= 1e-4 * L(vals)
    for name, t, h in (("pos", pos, 1e-5), ("v0", v0, 1e-4), ("v3", v3, 1e-4)):
        g = t.grad.cpu().numpy()
        for c in range(3):
            ap, am = {k: v.copy() for k, v in vals.items()}, {k: v.copy() for k, v in vals.items()}
            ap[name][c] += h
            am[name][c] -= h
            fd = (L(ap) - L(am)) / (2 * h)
            print(f"\n[accuracy] scene grad {name}[{c}]: adjoint {g[c]:.6e}  fp64 FD {fd:.6e}")
            assert abs(g[c] - fd) <= 2e-2 * max(abs(fd), 1e-3 * np.abs(g).max()), (name, c, g[c], fd)


def test_muscle_actuation_per_step():
    mat_kw = dict(E=5e4, nu=0.45, rho=1000.0, n_groups=2)
    scene, ent = _scene(gs.materials.MPM.Muscle(**mat_kw))
    n = ent.n_particles
    groups = (ent.init_particles[:, 0] > 0.5).astype(np.int64)
    ent.set_muscle(muscle_group=torch.tensor(groups, device="cuda"),
                   muscle_direction=torch.tensor([[0.0, 0.0, 1.0]] * n, device="cuda"))
    offsets = ent.init_particles - np.asarray(ent.morph.pos)
    acts = [torch.tensor([0.3, -0.2], device="cuda", requires_grad=True) for _ in range(3)]
    goal = torch.tensor(GOAL, dtype=torch.float32, device="cuda")
    loss = 0.0
    for s in range(5):
        if s < 3:
            ent.set_actuation(acts[s])  # held from step 2 on
        scene.step()
        loss = loss + ((ent.get_particles_pos() - goal) ** 2).sum(1).mean()  # the muscle changes the shape
    loss.backward()
    a_np = [a.detach().cpu().numpy().astype(np.float64) for a in acts]
    kw = {k: v for k, v in mat_kw.items() if k != "n_groups"}
    L = lambda aa: _oracle_loss(offsets, np.array([0.5, 0.5, 0.15]), {0: np.zeros(3)}, 5, kw, kind="muscle",
                                actu_by_step=aa, groups=groups, shape=True)
    for s in range(3):
        g = acts[s].grad.cpu().numpy()
        for k in range(2):
            ap = [a.copy() for a in a_np]
            am = [a.copy() for a in a_np]
            ap[s][k] += 1e-3
            am[s][k] -= 1e-3
            fd = (L(ap) - L(am)) / 2e-3
            print(f"\n[accuracy] scene grad actuation step {s} group {k}: adjoint {g[k]:.6e}  fp64 FD {fd:.6e}")
            assert abs(g[k] - fd) <= 3e-2 * max(abs(fd), 1e-2 * np.abs(g).max()), (s, k, g[k], fd)


def test_differentiable_scene_limits():
    scene, ent = _scene(gs.materials.MPM.Elastic(E=2e4))
    scene.step()
    with pytest.raises(gs.GenesisException):
        ent.set_position(torch.zeros(3, device="cuda"))
    for cpic in (False, True):
        gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
        s2 = gs.Scene(sim_options=gs.options.SimOptions(dt=DT, substeps=SUB, requires_grad=True),
                      mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1),
                                                        enable_CPIC=cpic))
        s2.add_entity(gs.morphs.Box(pos=(0.5, 0.5, 0.3), size=(0.1, 0.1, 0.1)), material=gs.materials.MPM.Sand())
        s2.add_entity(gs.morphs.Box(pos=(0.5, 0.5, 0.1), size=(0.3, 0.3, 0.05)), material=gs.materials.Rigid())
        if cpic:
            with pytest.raises(gs.GenesisException):  # no adjoint of the particle-level coupling
                s2.build()
        else:  # a rigid collider is differentiated with respect to the node velocities
            s2.build()
            s2.step()


def test_gradients_with_environments():
    """Two identical environments and one velocity input applied to both: the loss sums the two,
    so the gradient is twice the one-environment gradient (the tape addresses particles through
    the environments' runtime ids)."""

    def run(n_envs):
        gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
        scene = gs.Scene(
            sim_options=gs.options.SimOptions(dt=DT, substeps=SUB, gravity=(0, 0, -9.8), requires_grad=True),
            mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                              particle_size=P_SIZE),
        )
        ent = scene.add_entity(gs.morphs.Box(pos=(0.5, 0.5, 0.15), size=(0.08, 0.08, 0.08)),
                               material=gs.materials.MPM.Elastic(E=2e4))
        scene.build(n_envs=n_envs)
        v = torch.tensor([0.3, -0.2, -1.0], device="cuda", requires_grad=True)
        ent.set_velocity(v)
        goal = torch.tensor(GOAL, dtype=torch.float32, device="cuda")
        loss = 0.0
        for _ in range(4):
            scene.step()
            pos = scene.get_state().solvers_state[3].pos  # [B, N, 3]
            loss = loss + ((pos.mean(1) - goal) ** 2).sum()
        loss.backward()
        return v.grad.cpu().numpy()

    g1, g2 = run(0), run(2)
    assert np.allclose(g2, 2 * g1, rtol=1e-4, atol=1e-9), (g1, g2)


def test_reset_between_optimisation_iterations():
    """forward, backward, scene.reset(), forward, backward (an optimisation loop): the second
    iteration with the same input gives the same gradient, and a changed input a different one."""
    scene, ent = _scene(gs.materials.MPM.Elastic(E=2e4))
    goal = torch.tensor(GOAL, dtype=torch.float32, device="cuda")

    def iteration(v):
        vv = gs.tensor(v, requires_grad=True)
        ent.set_velocity(vv)
        loss = 0.0
        for _ in range(3):
            scene.step()
            loss = loss + ((ent.get_particles_pos().mean(0) - goal) ** 2).sum()
        loss.backward()
        scene.reset()
        return vv.grad.cpu().numpy(), float(loss.detach())

    g1, l1 = iteration([0.2, 0.0, -0.5])
    g2, l2 = iteration([0.2, 0.0, -0.5])
    g3, _ = iteration([0.0, 0.4, 0.5])
    assert np.allclose(g1, g2, rtol=1e-5, atol=1e-9) and abs(l1 - l2) <= 1e-6 * l1
    assert not np.allclose(g1, g3, rtol=1e-3)
