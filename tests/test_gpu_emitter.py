"""Emitter and dynamic particle activation on the GPU: emitted droplets become active,
move, recycle slots, and a scene with emitted particles advances exactly like the
float64 oracle started from the same state (inactive slots untouched)."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs

pytestmark = pytest.mark.gpu


def _scene(max_particles=4000, substeps=10):
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=1e-4 * substeps, substeps=substeps, gravity=(0, 0, -9.8)),
        mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), grid_density=64,
                                          particle_size=0.01),
    )
    sand = scene.add_entity(gs.morphs.Box(lower=(0.3, 0.3, 0.06), upper=(0.5, 0.5, 0.12)),
                            material=gs.materials.MPM.Sand())
    em = scene.add_emitter(gs.materials.MPM.Liquid(), max_particles=max_particles)
    scene.build()
    return scene, sand, em


def test_emitted_particles_activate_and_fall():
    scene, sand, em = _scene()
    ent = em.entity
    assert not bool(ent.get_particles_active().any())  # a Nowhere entity starts inactive
    total = 0
    for _ in range(3):
        total += em.emit("circle", 0.06, droplet_length=0.02, pos=(0.6, 0.6, 0.6), direction=(0, 0, -1), speed=2.0)
        scene.step()
    act = ent.get_particles_active()
    assert int(act.sum()) == total > 0
    pos = ent.get_particles_pos()[act]
    vel = ent.get_particles_vel()[act]
    # droplets are emitted centred on the nozzle (z 0.59..0.61) and have moved down since
    assert torch.isfinite(pos).all() and (pos[:, 2] < 0.61 - 1e-3).all()
    assert float(vel[:, 2].mean()) < -1.9  # launched at 2 m/s downwards, still accelerating
    assert scene.check_state() == 0


def test_emitter_recycles_slots():
    scene, sand, em = _scene(max_particles=600)
    starts = []
    for _ in range(8):
        starts.append(em.next_particle)
        em.emit("square", 0.04, droplet_length=0.02, pos=(0.6, 0.6, 0.6), speed=1.0)  # 4*4*2 = 32 particles
        scene.step()
    assert starts[:3] == [0, 32, 64]
    assert int(em.entity.get_particles_active().sum()) == 8 * 32
    scene.reset()
    assert em.next_particle == 0


def test_scene_with_emitted_particles_matches_oracle():
    from oracle import cref
    from oracle import mpm_ref as R

    scene, sand, em = _scene(substeps=10)
    for _ in range(2):
        # a sphere ignores the droplet length, but a positive one is needed to emit at all
        em.emit("sphere", 0.08, droplet_length=0.08, pos=(0.6, 0.55, 0.5), speed=1.0, direction=(1, 0, -1))
        scene.step()
    s0 = scene.get_state()[3]
    host = {k: getattr(s0, k)[0].cpu().numpy() for k in ("pos", "vel", "C", "F", "Jp", "active")}
    n_sand = sand.n_particles
    mat = np.concatenate([np.zeros(n_sand, np.int64), np.ones(em.entity.n_particles, np.int64)])
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-4, gravity=(0, 0, -9.8), dtype=np.float64)
    mats = [R.make_material("sand"), R.make_material("liquid")]
    st = dict(x=host["pos"].astype(np.float64), v=host["vel"].astype(np.float64),
              C=host["C"].astype(np.float64), F=host["F"].astype(np.float64), Jp=host["Jp"].astype(np.float64),
              mat=mat, active=host["active"].astype(bool))
    o, rc = cref.substeps(p, mats, st, 10)
    assert rc == 0
    scene.step()
    g = scene.get_state()[3]
    gx = g.pos[0].cpu().numpy()
    act = host["active"].astype(bool)
    assert act.sum() > n_sand
    assert np.abs(gx[act] - o["x"][act]).max() < 1e-5
    assert np.array_equal(gx[~act], host["pos"][~act])  # inactive slots are copied through
