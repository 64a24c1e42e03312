"""The reference's own MPM test scenarios run through this package, with their assertions
(the parts that involve only MPM and rigid colliders; the PBD cloth, SPH water and FEM box of
the same scenes belong to other solvers)."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu


def test_deformable_parallel_mpm_cube():
    """tests/test_deformable_physics.py:110-222 (test_deformable_parallel), its MPM cube: an
    Elastic cube (rho 200) dropped on a frictionless coupled ground plane in two environments,
    1,500 steps of 10 substeps; it moves, stays above the ground and comes to rest."""
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=2e-3, substeps=10),
        mpm_options=gs.options.MPMOptions(lower_bound=(0.5, -0.1, -0.05), upper_bound=(0.7, 0.1, 0.3)),
    )
    scene.add_entity(morph=gs.morphs.Plane(), material=gs.materials.Rigid(needs_coup=True, coup_friction=0.0))
    cube = scene.add_entity(morph=gs.morphs.Box(pos=(0.6, 0.0, 0.1), size=(0.1, 0.1, 0.1)),
                            material=gs.materials.MPM.Elastic(rho=200),
                            surface=gs.surfaces.Default(color=(0.9, 0.8, 0.2, 1.0)))
    scene.build(n_envs=2)
    init = cube.get_particles_pos().clone()
    scene.get_state()
    for _ in range(1500):
        scene.step()
    final = cube.get_particles_pos()
    assert float((init - final).abs().sum()) > 0.1
    assert float(final[..., 2].min()) > -1e-5
    vel = cube.get_particles_vel()
    print(f"\n[reference scenario] max |v| after 1500 steps: {float(vel.abs().max()):.2e}")
    assert torch.allclose(vel, torch.zeros_like(vel), atol=1e-4)


@pytest.mark.parametrize("material_type", [gs.materials.MPM.Liquid, gs.materials.MPM.Sand, gs.materials.MPM.Snow,
                                           gs.materials.MPM.Elastic])
def test_fluid_emitter_mpm(material_type):
    """tests/test_hybrid.py:86-154 (test_fluid_emitter) with its MPM materials and two
    environments: a ground plane added without a material (a Rigid entity by default), an
    emitter of 5,000 particles, emit_omni, then five circular droplets with a step after each.
    The reference asserts only that this runs; here the emitted particles also stay finite and
    inside the domain."""
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=4e-3, substeps=10),
        mpm_options=gs.options.MPMOptions(lower_bound=(0.0, -1.5, 0.0), upper_bound=(1.0, 1.5, 4.0)),
    )
    scene.add_entity(gs.morphs.Plane())
    emitter = scene.add_emitter(material=material_type(), max_particles=5000,
                                surface=gs.surfaces.Glass(color=(0.7, 0.85, 1.0, 0.7)))
    scene.build(n_envs=2)
    emitter.emit_omni()
    for _ in range(5):
        emitter.emit(droplet_shape="circle", droplet_size=0.25)
        scene.step()
    scene.step()
    ent = emitter.entity
    act = ent.get_particles_active()
    pos = ent.get_particles_pos()
    assert act.shape[0] == 2 and int(act[0].sum()) > 0 and torch.equal(act[0], act[1])
    live = pos[act]
    assert bool(torch.isfinite(live).all())
    assert float(live[:, 2].min()) >= 0.0 and float(live[:, 0].max()) <= 1.0


def _legacy_coupling(substeps):
    substep_dt, horizon_substeps = 4e-4, 100
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=substep_dt * substeps, substeps=substeps),
        mpm_options=gs.options.MPMOptions(lower_bound=(-0.5, -1.0, 0.0), upper_bound=(0.5, 1.0, 1)),
    )
    scene.add_entity(morph=gs.morphs.Plane())
    box = scene.add_entity(material=gs.materials.Rigid(rho=1.0), morph=gs.morphs.Box(pos=(0.0, -0.25, 0.1),
                                                                                     size=(0.2, 0.2, 0.2)))
    liquid = scene.add_entity(material=gs.materials.MPM.Liquid(), morph=gs.morphs.Box(pos=(0.0, 0.0, 0.2),
                                                                                      size=(0.3, 0.3, 0.3)))
    scene.build()
    impulse = torch.zeros(3, device="cuda")
    for _ in range(horizon_substeps // substeps):
        scene.step()
        impulse += box.get_coupling_force()[:3] * substep_dt * substeps  # mean force over the step x its time
    return liquid.get_particles_pos(), impulse.cpu().numpy()


def test_rigid_mpm_legacy_coupling():
    """tests/test_hybrid.py:285-360 (test_rigid_mpm_legacy_coupling) for a kinematic box: the
    reference checks that the liquid pushes the box along -y and that the result does not depend
    on how the same substep dt is grouped into steps.  The box here does not move (no rigid
    dynamics), so the push is read as the impulse the liquid gave it, and the grouping check is
    made on the liquid's particles and that impulse."""
    p1, j1 = _legacy_coupling(1)
    p10, j10 = _legacy_coupling(10)
    print(f"\n[reference scenario] impulse on the box: substeps 1 {j1}, substeps 10 {j10}")
    assert j1[1] < 0 and j10[1] < 0  # pushed along -y
    assert torch.allclose(p1, p10, atol=1e-5)
    assert np.allclose(j1, j10, rtol=1e-3, atol=1e-6)


@pytest.mark.parametrize("n_envs", [0, 2])
def test_muscle_worm(n_envs, tmp_path):
    """tests/test_deformable_physics.py:15-107 (test_muscle) with MPM.Muscle: a worm on a
    high-friction coupled plane, four muscle groups (upper/lower x fore/hind) along +y, 200
    steps with the hind-lower group actuated sinusoidally.  The reference's worm mesh is an
    asset file; an elongated ellipsoid of the same footprint written by the test stands in.
    The reference only runs it; here the worm also stays finite and above the plane, and its
    actuated groups move relative to an unactuated copy."""
    from genesis_b200 import mesh

    v, f = mesh.icosphere(3, 1.0)
    v = v * np.array([0.6, 2.0, 0.5])  # scaled by 0.1 below: 0.12 x 0.4 x 0.1 m
    obj = tmp_path / "worm.obj"
    obj.write_text("".join(f"v {a} {b} {c}\n" for a, b, c in v) + "".join(f"f {i+1} {j+1} {k+1}\n" for i, j, k in f))

    def run(actuate):
        gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
        scene = gs.Scene(
            sim_options=gs.options.SimOptions(dt=5e-4, substeps=10, gravity=(0, 0, -9.8)),
            mpm_options=gs.options.MPMOptions(lower_bound=(-1.0, -1.0, -0.2), upper_bound=(1.0, 1.0, 1.0)),
        )
        scene.add_entity(morph=gs.morphs.Plane(), material=gs.materials.Rigid(coup_friction=5.0))
        worm = scene.add_entity(
            morph=gs.morphs.Mesh(file=str(obj), pos=(0.3, 0.3, 0.051), scale=0.1),
            material=gs.materials.MPM.Muscle(E=5e5, nu=0.45, rho=10000.0, n_groups=4),
            surface=gs.surfaces.Default(diffuse_texture=gs.textures.ImageTexture(image_path="worm.png")),
        )
        scene.build(n_envs=n_envs) if n_envs > 0 else scene.build()
        pos = worm.get_state().pos[0].cpu().numpy()
        n_units = worm.n_particles
        pmax, pmin = pos.max(0), pos.min(0)
        rng_ = pmax - pmin
        upper = pos[:, 2] > pmin[2] + rng_[2] * 0.3
        fore = pos[:, 1] < pmin[1] + rng_[1] * 0.6
        group = np.zeros(n_units, dtype=int)
        group[upper & ~fore] = 1
        group[~upper & fore] = 2
        group[~upper & ~fore] = 3
        worm.set_muscle(muscle_group=group, muscle_direction=np.array([[0.0, 1.0, 0.0]] * n_units, dtype=np.float32))
        scene.reset()
        for i in range(200):
            a = np.array([0.0, 0.0, 0.0, (1.0 * (0.5 + np.sin(0.005 * np.pi * i))) if actuate else 0.0])
            worm.set_actuation(np.tile(a, (n_envs, 1)) if n_envs > 1 else a)
            scene.step()
        return worm.get_particles_pos(), group

    p_act, group = run(True)
    p_rest, _ = run(False)
    p_act = p_act if n_envs == 0 else p_act[0]
    p_rest = p_rest if n_envs == 0 else p_rest[0]
    assert bool(torch.isfinite(p_act).all()) and float(p_act[:, 2].min()) > -1e-5
    moved = (p_act - p_rest).norm(dim=1).cpu().numpy()
    print(f"\n[reference scenario] worm: mean displacement by actuation, group 3 {moved[group == 3].mean():.2e} m")
    assert moved[group == 3].mean() > 1e-4


def _stirrer_obj(tmp_path):
    """A stand-in for the reference's meshes/stirrer.obj (not shipped here): a paddle whose
    largest extent is its local y, so that euler (90, 0, 0) stands it upright."""
    from genesis_b200 import mesh

    v, f = mesh.box_mesh((0.3, 1.0, 0.6))
    path = str(tmp_path / "stirrer.obj")
    with open(path, "w") as fh:
        for q in v:
            fh.write(f"v {q[0]:.9f} {q[1]:.9f} {q[2]:.9f}\n")
        for t in f:
            fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    return path


def _push(tmp_path, pos_obj, v_obj, requires_grad, v_stick=None):
    """tests/test_grad.py:20-103 (test_differentiable_push): the plane, the stirrer Tool
    (friction 8) at two starting positions, the Elastic box (rho 500) in two environments;
    returns the loss and the per-step stirrer velocities."""
    HORIZON = 10
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=2e-3, substeps=10, requires_grad=requires_grad),
        mpm_options=gs.options.MPMOptions(lower_bound=(0.0, -1.0, 0.0), upper_bound=(1.0, 1.0, 0.55)),
    )
    scene.add_entity(gs.morphs.Plane())
    stick = scene.add_entity(morph=gs.morphs.Mesh(file=_stirrer_obj(tmp_path), scale=0.6, pos=(0.5, 0.5, 0.05),
                                                  euler=(90.0, 0.0, 0.0)),
                             material=gs.materials.Tool(friction=8.0))
    obj = scene.add_entity(morph=gs.morphs.Box(lower=(0.2, 0.1, 0.05), upper=(0.4, 0.3, 0.15)),
                           material=gs.materials.MPM.Elastic(rho=500))
    scene.build(n_envs=2)
    init_pos = gs.tensor([[0.3, 0.1, 0.28], [0.3, 0.1, 0.5]], requires_grad=requires_grad)
    stick.set_position(init_pos)
    obj.set_position(pos_obj)
    obj.set_velocity(v_obj)
    goal = gs.tensor([0.5, 0.8, 0.05])
    loss = 0.0
    v_list = []
    for i in range(HORIZON):
        v_i = gs.tensor([[0.0, 1.0, 0.0], [0.0, 1.0, 0.0]], requires_grad=requires_grad)
        if v_stick is not None and i == 3:
            v_i = gs.tensor(v_stick)
        stick.set_velocity(vel=v_i)
        v_list.append(v_i)
        scene.step()
        if i == HORIZON // 2:
            mpm_particles = scene.get_state().solvers_state[3]
            loss += torch.pow(mpm_particles.pos[mpm_particles.active == 1] - goal, 2).sum()
        if i == HORIZON - 2:
            state = obj.get_state()
            loss += torch.pow(state.pos - goal, 2).sum()
    return loss, v_list, init_pos


def test_differentiable_push(tmp_path):
    """The reference's assertions (every stirrer velocity but the last has a gradient, the last
    has none), plus the object's inputs against central differences of the forward run
    (dL/dv_obj[1]) and the stirrer's velocity in step 3 against central differences too."""
    pos_obj_init = gs.tensor([0.3, 0.3, 0.1], requires_grad=True)
    v_obj_init = gs.tensor([0.0, -1.0, 0.0], requires_grad=True)
    loss, v_list, init_pos = _push(tmp_path, pos_obj_init, v_obj_init, True)
    loss.backward()
    for v_i in v_list[:-1]:
        assert (v_i.grad.abs() > gs.EPS).any()
    assert (v_list[-1].grad.abs() < gs.EPS).all()
    gp, gv = pos_obj_init.grad, v_obj_init.grad
    assert bool(torch.isfinite(gp).all()) and bool(torch.isfinite(gv).all()) and bool(torch.isfinite(init_pos.grad).all())
    assert (gp.abs() > gs.EPS).any() and (gv.abs() > gs.EPS).any() and (init_pos.grad.abs() > gs.EPS).any()
    h = 1e-2
    p0 = [0.3, 0.3, 0.1]
    lp = float(_push(tmp_path, gs.tensor(p0), gs.tensor([0.0, -1.0 + h, 0.0]), False)[0])
    lm = float(_push(tmp_path, gs.tensor(p0), gs.tensor([0.0, -1.0 - h, 0.0]), False)[0])
    fd = (lp - lm) / (2 * h)
    print(f"\n[reference scenario] push: dL/dv_obj[1] adjoint {float(gv[1]):.5e}, central difference {fd:.5e}")
    assert abs(float(gv[1]) - fd) <= 5e-2 * abs(fd)
    g3 = v_list[3].grad.cpu().numpy()
    hs = 1e-2
    vp = [[0.0, 1.0 + hs, 0.0], [0.0, 1.0, 0.0]]
    vm = [[0.0, 1.0 - hs, 0.0], [0.0, 1.0, 0.0]]
    lp = float(_push(tmp_path, gs.tensor(p0), gs.tensor([0.0, -1.0, 0.0]), False, v_stick=vp)[0])
    lm = float(_push(tmp_path, gs.tensor(p0), gs.tensor([0.0, -1.0, 0.0]), False, v_stick=vm)[0])
    fd3 = (lp - lm) / (2 * hs)
    print(f"[reference scenario] push: dL/dv_stick(step 3)[env 0, y] adjoint {g3[0, 1]:.5e}, central difference "
          f"{fd3:.5e}")
    assert abs(g3[0, 1] - fd3) <= 5e-2 * abs(fd3)
