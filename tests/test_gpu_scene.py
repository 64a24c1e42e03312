"""End-to-end through the public API (gs.init / gs.Scene / entities), on the GPU."""

import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _init():
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")


def _scene(n_envs=0, substeps=10, **b200):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")  # same particle samples per scene
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-4 * substeps, substeps=substeps, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.0125),
        b200_options=gs.options.B200Options(**b200),
    )
    cube = scene.add_entity(gs.morphs.Box(lower=(0.4, 0.4, 0.4), upper=(0.6, 0.6, 0.6)),
                            material=gs.materials.MPM.Elastic(E=1e5, nu=0.3))
    sand = scene.add_entity(gs.morphs.Box(lower=(0.2, 0.2, 0.1), upper=(0.3, 0.3, 0.2)),
                            material=gs.materials.MPM.Sand())
    scene.build(n_envs=n_envs)
    return scene, cube, sand


def test_scene_step_state_shapes_and_fall():
    scene, cube, sand = _scene()
    N = cube.n_particles + sand.n_particles
    p0 = cube.get_particles_pos().clone()
    for _ in range(3):
        scene.step()
    st = scene.get_state()
    s = st.solvers_state[3]
    assert s.pos.shape == (1, N, 3) and s.F.shape == (1, N, 3, 3) and s.Jp.shape == (1, N)
    assert s.active.dtype == torch.bool and bool(s.active.all())
    p1 = cube.get_particles_pos()
    assert p1.shape == (cube.n_particles, 3)
    assert float((p1[:, 2] - p0[:, 2]).mean()) < 0  # falls under gravity
    assert scene.sim.cur_substep_global == 30


def test_envs_identical_and_reset():
    scene, cube, sand = _scene(n_envs=3)
    s0 = scene.get_state()
    for _ in range(2):
        scene.step()
    s = scene.get_state()[3]
    assert s.pos.shape[0] == 3
    assert torch.allclose(s.pos[0], s.pos[1], atol=1e-6) and torch.allclose(s.pos[0], s.pos[2], atol=1e-6)
    scene.reset()
    r = scene.get_state()[3]
    assert torch.equal(r.pos, s0[3].pos.to(r.pos.device))


def test_plugin_substeps_match_fused_step():
    """Simulator.substep (pre_coupling / couple / post_coupling calls) == Simulator.step."""
    a, _, _ = _scene(use_cuda_graph=False)
    b, _, _ = _scene(use_cuda_graph=True)
    for f in range(10):
        a.sim.substep(0)
    b.step()
    pa, pb = a.get_state()[3].pos, b.get_state()[3].pos
    assert torch.allclose(pa, pb, atol=1e-6)


def test_set_position_target_applied_next_step():
    scene, cube, sand = _scene()
    tgt = torch.tensor([0.5, 0.5, 0.7])
    cube.set_position(tgt)
    scene.step()
    p = cube.get_particles_pos()
    assert abs(float(p.mean(0)[2]) - 0.7) < 0.01


def test_entity_active_mask():
    scene, cube, sand = _scene()
    sand.set_particles_active(torch.zeros(sand.n_particles, dtype=torch.uint8))
    ps = sand.get_particles_pos().clone()
    scene.step()
    assert torch.equal(sand.get_particles_pos(), ps)
    assert not bool(sand.get_particles_active().any())


def _host_state(scene, pinned):
    st = scene.get_state()[3]
    out = {k: getattr(st, k).cpu() for k in ("pos", "vel", "C", "F", "Jp", "active")}
    return {k: (v.pin_memory() if pinned else v) for k, v in out.items()}


def test_staged_upload_matches_synchronous_upload():
    """scene.reset from pinned host tensors (asynchronous staged copy) gives the same
    trajectory as from pageable host tensors (synchronous copy)."""
    from genesis_b200.engine.states import MPMSolverState

    res = []
    for pinned in (False, True):
        scene, cube, sand = _scene()
        scene.step()
        h = _host_state(scene, pinned)
        h["vel"] = h["vel"] + 0.1  # a state different from the scene's current one
        scene.step()
        for _ in range(2):  # twice in a row: the staging buffer is reused
            scene.reset(MPMSolverState(scene, h["pos"], h["vel"], h["C"], h["F"], h["Jp"], h["active"]))
            scene.step()
        res.append(scene.get_state()[3].pos.clone())
    assert torch.equal(res[0], res[1])


def test_async_nan_check_raises_on_a_later_call():
    from genesis_b200.engine.states import MPMSolverState

    scene, cube, sand = _scene(check_nan="async")
    scene.step()
    h = _host_state(scene, pinned=True)
    h["pos"][0, 0, 0] = float("nan")
    scene.reset(MPMSolverState(scene, h["pos"], h["vel"], h["C"], h["F"], h["Jp"], h["active"]))
    scene.step()  # does not block; the NaN is found by a later call
    torch.cuda.synchronize()
    with pytest.raises(gs.GenesisException):
        scene.get_state()
    with pytest.raises(gs.GenesisException):
        scene.check_state()  # the device status word stays set


def test_mesh_morph_entity_matches_box(tmp_path):
    """A box loaded from an OBJ file steps like the Box primitive of the same size and pose
    (same lattice up to round-off), and its file mesh is skinned."""
    hx = 0.5
    v = [[x, y, z] for x in (-hx, hx) for y in (-hx, hx) for z in (-hx, hx)]
    q = [[0, 1, 3, 2], [4, 6, 7, 5], [0, 4, 5, 1], [2, 3, 7, 6], [0, 2, 6, 4], [1, 5, 7, 3]]
    obj = tmp_path / "cube.obj"
    obj.write_text("".join(f"v {a} {b} {c}\n" for a, b, c in v) + "".join(
        "f " + " ".join(str(i + 1) for i in f) + "\n" for f in q))

    def run(morph):
        gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
        scene = gs.Scene(
            sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, gravity=(0, 0, -9.8)),
            mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                              particle_size=0.0125),
        )
        e = scene.add_entity(morph, material=gs.materials.MPM.Elastic(E=1e5, nu=0.3))
        scene.build()
        for _ in range(5):
            scene.step()
        return e, e.get_particles_pos().cpu()

    em, pm = run(gs.morphs.Mesh(file=str(obj), scale=0.2, pos=(0.5, 0.5, 0.5), euler=(0, 0, 20)))
    eb, pb = run(gs.morphs.Box(size=(0.2, 0.2, 0.2), pos=(0.5, 0.5, 0.5), euler=(0, 0, 20)))
    assert em.n_particles == eb.n_particles == 16**3
    assert torch.allclose(pm, pb, atol=1e-5)
    assert em.n_vverts == 8


def test_entity_utilities():
    """activate/deactivate, get_free, find_closest_particle and the visual-mesh ranges
    (particle_entity.py:639-651, 709-738; mpm_entity.py:571-583)."""
    scene, cube, sand = _scene(substeps=5)
    assert cube.uid != sand.uid and len(cube.uid) == 7
    assert cube.vvert_start == 0 and cube.vvert_end == cube.n_vverts == 8 and cube.n_vfaces == 12
    assert sand.n_vverts == 0 and sand.vvert_start == sand.vvert_end == 8  # Sand is not skinned
    assert bool(cube.get_free().all()) and cube.get_free().shape == (cube.n_particles,)
    cube.set_free(torch.zeros(cube.n_particles, dtype=torch.bool))
    assert not bool(cube.get_free().any()) and bool(sand.get_free().all())
    cube.set_free(torch.ones(cube.n_particles, dtype=torch.bool))
    p = cube.get_particles_pos()
    k = 123
    i = cube.find_closest_particle(p[k] + 1e-4)
    assert i.ndim == 0 and int(i) == k
    cube.deactivate()
    p0 = cube.get_particles_pos().clone()
    scene.step()
    assert not bool(cube.get_particles_active().any())
    assert torch.equal(cube.get_particles_pos(), p0)  # inactive particles are copied through
    cube.activate()
    scene.step()
    assert bool(cube.get_particles_active().all())
    assert float((cube.get_particles_pos()[:, 2] - p0[:, 2]).mean()) < 0


def test_find_closest_particle_batched():
    scene, cube, sand = _scene(n_envs=2, substeps=5)
    p = cube.get_particles_pos()
    i = cube.find_closest_particle(torch.stack([p[0, 7], p[1, 99]]))
    assert i.shape == (2,) and i.tolist() == [7, 99]


def test_cylinder_entity_steps_and_skins():
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.0125),
    )
    cyl = scene.add_entity(gs.morphs.Cylinder(pos=(0.5, 0.5, 0.3), radius=0.1, height=0.2),
                           material=gs.materials.MPM.Elastic(E=1e5, nu=0.3))
    scene.build()
    z0 = float(cyl.get_particles_pos()[:, 2].mean())
    for _ in range(5):
        scene.step()
    assert float(cyl.get_particles_pos()[:, 2].mean()) < z0
    assert cyl.n_vverts == 66 and cyl.n_vfaces == 128
    solver = cyl.solver
    solver.update_render_fields()
    vv = solver.vverts_render["pos"][0].cpu().double()
    # the skinned rim stays around the particles' centre of mass
    c = cyl.get_particles_pos().cpu().double().mean(0)
    assert float((vv.mean(0) - c).norm()) < 0.02


def test_mesh_set_entity(tmp_path):
    """Two OBJ cubes in one MeshSet entity: each keeps its particles' group id and both fall."""
    hx = 0.5
    v = [[x, y, z] for x in (-hx, hx) for y in (-hx, hx) for z in (-hx, hx)]
    q = [[0, 1, 3, 2], [4, 6, 7, 5], [0, 4, 5, 1], [2, 3, 7, 6], [0, 2, 6, 4], [1, 5, 7, 3]]
    obj = tmp_path / "cube.obj"
    obj.write_text("".join(f"v {a} {b} {c}\n" for a, b, c in v) + "".join(
        "f " + " ".join(str(i + 1) for i in f) + "\n" for f in q))
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.0125),
    )
    e = scene.add_entity(gs.morphs.MeshSet(files=[str(obj), str(obj)], poss=[(0.3, 0.5, 0.5), (0.7, 0.5, 0.5)],
                                           scale=0.1), material=gs.materials.MPM.Elastic(E=1e5, nu=0.3))
    scene.build()
    g = e.mesh_set_group_ids
    assert g.shape == (e.n_particles,) and (g == 0).sum() == (g == 1).sum() == 8**3
    z0 = e.get_particles_pos()[:, 2].clone()
    for _ in range(5):
        scene.step()
    dz = (e.get_particles_pos()[:, 2] - z0).cpu().numpy()
    assert dz[g == 0].mean() < 0 and dz[g == 1].mean() < 0
    assert e.n_vverts == 16


def test_get_frame_fills_given_tensors():
    scene, cube, sand = _scene(substeps=5)
    scene.step()
    B, n = 1, cube.n_particles
    bufs = [torch.zeros(B, n, 3), torch.zeros(B, n, 3), torch.zeros(B, n, 3, 3), torch.zeros(B, n, 3, 3),
            torch.zeros(B, n), torch.zeros(B, n, dtype=torch.bool)]
    cube.get_frame(scene.sim.cur_substep_local, *bufs)
    st = cube.get_state()
    assert torch.equal(bufs[0], st.pos.cpu()) and torch.equal(bufs[3], st.F.cpu()) and bool(bufs[5].all())
    with pytest.raises(gs.GenesisException):
        cube.get_frame(scene.sim.cur_substep_local + 1, *bufs)
