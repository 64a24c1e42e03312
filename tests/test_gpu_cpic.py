"""CPIC against rigid colliders (mpm_solver.py:357-379, 412-427; legacy_coupler.py:498-525) on
the GPU through gs.Scene: a block falling onto a fixed slab far thinner than a grid cell
matches the float64 oracle, stays on its side of the slab (it leaks through without CPIC), and
every particle remembers the side it came from.  The slab is the exact box
(B200Options(exact_box_sdf=True)), the oracle's kind 'box'."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu

SLAB = dict(pos=(0.5, 0.5, 0.3), size=(0.6, 0.6, 0.002))


def _scene(cpic, substeps=10, z0=0.33):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-4 * substeps, substeps=substeps, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.01, enable_CPIC=cpic),
        # the exact box: a 2 mm slab is below the resolution of the reference's sampled grid
        # (sdf_cell_size 5 mm), whose blended gradients near the slab's faces would stand in
        # for the side each particle remembers
        b200_options=gs.options.B200Options(exact_box_sdf=True),
    )
    block = scene.add_entity(gs.morphs.Box(lower=(0.45, 0.45, z0), upper=(0.55, 0.55, z0 + 0.1)),
                             material=gs.materials.MPM.Elastic(E=2e4))
    slab = scene.add_entity(gs.morphs.Box(**SLAB), material=gs.materials.Rigid())
    scene.build()
    block.set_particles_vel(torch.tensor([0.0, 0.0, -2.0]).expand(block.n_particles, 3))
    return scene, block, slab


def _oracle(x0, cpic, n_substeps):
    from oracle import cref
    from oracle import mpm_ref as R

    n = len(x0)
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-4, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4)]
    st = R.make_state(x0, mats, np.zeros(n, np.int64), np.float64, v=np.tile((0.0, 0.0, -2.0), (n, 1)))
    st["colliders"] = [R.Collider("box", np.array(SLAB["pos"]), np.eye(3), np.array(SLAB["size"]) / 2)]
    if cpic:
        st["cpic_normal"] = np.zeros((1, n, 3))
    out, rc = cref.substeps(p, mats, st, n_substeps)
    assert rc == 0
    return out


def test_cpic_matches_oracle():
    # the lowest particles' stencils reach under the slab from the first substep
    scene, block, slab = _scene(cpic=True, z0=0.31)
    x0 = block.get_particles_pos().cpu().numpy().astype(np.float64)
    o = _oracle(x0, True, 60)
    plain = _oracle(x0, False, 60)
    assert np.abs(o["x"] - plain["x"]).max() > 1e-4  # CPIC changed the trajectory (10x the tolerance)
    for _ in range(6):
        scene.step()
    g = block.get_particles_pos().cpu().numpy()
    assert np.abs(g - o["x"]).max() < 1e-5
    nrm = scene.sim.mpm_solver.runtime.get_cpic_normals()[0].cpu().numpy()
    assert np.abs(nrm - o["cpic_normal"][0]).max() < 1e-5


def test_cpic_keeps_the_block_on_its_side():
    scene, block, slab = _scene(cpic=True)
    for _ in range(30):
        scene.step()
    z = block.get_particles_pos()[:, 2]
    assert float(z.min()) > 0.3 - 1.5 / 64
    nrm = scene.sim.mpm_solver.runtime.get_cpic_normals()[0]
    assert bool((nrm[:, 2] > 0.99).all())  # every particle remembers the upper side
    assert float(slab.get_coupling_force()[2]) < 0  # and pushes the slab down
    scene.reset()
    assert float(scene.sim.mpm_solver.runtime.get_cpic_normals().abs().max()) == 0.0

    leak, lblock, _ = _scene(cpic=False)
    for _ in range(30):
        leak.step()
    assert float(lblock.get_particles_pos()[:, 2].min()) < 0.28  # without CPIC it passes through


def test_cpic_per_environment():
    """Each environment's particles see only their own slab (collider.instance): with two
    environments both keep the block on top, identically."""
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-3, substeps=10, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.01, enable_CPIC=True),
    )
    block = scene.add_entity(gs.morphs.Box(lower=(0.45, 0.45, 0.31), upper=(0.55, 0.55, 0.41)),
                             material=gs.materials.MPM.Elastic(E=2e4))
    scene.add_entity(gs.morphs.Box(**SLAB), material=gs.materials.Rigid())
    scene.build(n_envs=2)
    block.set_particles_vel(torch.tensor([0.0, 0.0, -2.0]).expand(2, block.n_particles, 3))
    for _ in range(20):
        scene.step()
    z = block.get_particles_pos()[..., 2]
    assert z.shape[0] == 2 and float(z.min()) > 0.3 - 1.5 / 64
    assert torch.allclose(z[0], z[1], atol=1e-6)
