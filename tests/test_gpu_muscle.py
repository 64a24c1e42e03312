"""MPM.Muscle on the GPU (materials/MPM/muscle.py, mpm_entity.py:412-530): per-group
actuation and fibre directions drive the actuation stress; the trajectory matches the
float64 oracle."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu


def _scene(n_groups=2, substeps=10):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-4 * substeps, substeps=substeps, gravity=(0, 0, 0)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.0125),
    )
    m = scene.add_entity(gs.morphs.Box(lower=(0.4, 0.4, 0.4), upper=(0.55, 0.55, 0.55)),
                         material=gs.materials.MPM.Muscle(E=1e5, n_groups=n_groups, sampler="regular"))
    scene.build()
    return scene, m


def test_muscle_groups_directions_and_actuation_match_oracle():
    from oracle import cref
    from oracle import mpm_ref as R

    scene, m = _scene()
    n = m.n_particles
    p0 = m.get_particles_pos().cpu().numpy().astype(np.float64)
    group = (p0[:, 0] > 0.475).astype(np.int64)  # two groups split along x
    d = np.zeros((n, 3))
    d[group == 0] = (0.0, 0.0, 1.0)
    d[group == 1] = (0.0, 0.6, 0.8)
    m.set_muscle(muscle_group=torch.as_tensor(group), muscle_direction=torch.as_tensor(d))
    assert torch.equal(m.get_muscle_group().cpu(), torch.as_tensor(group, dtype=torch.int32))
    m.set_actuation(torch.tensor([0.5, -0.3]))  # larger values make this soft block unstable
    scene.step()  # the buffered actuation is applied before the substeps
    a = m.get_particles_actu().cpu().numpy()
    assert np.allclose(a, np.where(group == 0, 0.5, -0.3))
    for _ in range(2):
        scene.step()
    g = m.get_particles_pos().cpu().numpy()

    p = R.Params(grid_density=64, particle_size=0.0125, dt=1e-4, gravity=(0, 0, 0), dtype=np.float64)
    mats = [R.make_material("muscle", E=1e5)]
    st = R.make_state(p0, mats, np.zeros(n, np.int64), np.float64)
    st["actu"] = np.where(group == 0, 0.5, -0.3)
    st["mdir"] = d
    o, rc = cref.substeps(p, mats, st, 30)
    assert rc == 0
    assert np.abs(o["x"] - st["x"]).max() > 1e-5  # the actuation moved the particles
    assert np.abs(g - o["x"]).max() < 1e-5


def test_unactuated_muscle_is_neo_hookean_elastic():
    scene, m = _scene(n_groups=1)
    p0 = m.get_particles_pos().clone()
    for _ in range(3):
        scene.step()
    assert torch.allclose(m.get_particles_pos(), p0, atol=1e-6)  # no gravity, no actuation: at rest


def test_actuation_needs_a_muscle():
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(mpm_options=gs.options.MPMOptions(grid_density=64))
    e = scene.add_entity(gs.morphs.Box(lower=(0.4,) * 3, upper=(0.5,) * 3), material=gs.materials.MPM.Elastic())
    scene.build()
    with pytest.raises(gs.GenesisException):
        e.set_actuation(1.0)
