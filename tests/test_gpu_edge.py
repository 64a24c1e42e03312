"""Edge cases on the GPU: scenes whose particles are all inactive, a single particle,
particles on the padded wall, and a 4-million-particle scene (int32 indexing and
chunk-table sizes at scale)."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs
from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_scene_of_inactive_particles_steps():
    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(sim_options=gs.options.SimOptions(dt=1e-3, substeps=10),
                     mpm_options=gs.options.MPMOptions(grid_density=64))
    em = scene.add_emitter(gs.materials.MPM.Liquid(), max_particles=1000)
    scene.build()
    p0 = em.entity.get_particles_pos().clone()
    for _ in range(3):
        scene.step()
    assert torch.equal(em.entity.get_particles_pos(), p0)  # parked, untouched
    assert scene.check_state() == 0


def test_single_particle_falls_like_the_oracle():
    from oracle import bridge, cref

    from genesis_b200.engine.runtime import runtime_from_descs

    d = W.elastic_cube(n_side=1)
    rt = runtime_from_descs([d])
    rt.substeps(50)
    g = rt.get_state()["pos"].cpu().numpy()
    o, rc = cref.substeps(*bridge.from_desc(d, np.float64), 50)
    assert rc == 0 and np.abs(g - o["x"]).max() < 1e-6


def test_particles_on_the_padded_wall_stay_in_the_grid():
    """Particles exactly on the 3 dx padding (the boundary the g2p clamps to) keep their
    stencils inside the grid: no out-of-grid status, no fallback loss."""
    from genesis_b200 import _native as nat
    from genesis_b200.engine.runtime import runtime_from_descs

    d = W.elastic_cube(n_side=8)
    lo, hi = 3 / 64, 1 - 3 / 64
    pos = d.pos.copy()
    pos[:8, 0] = lo
    pos[8:16, 2] = lo
    pos[16:24, 1] = hi
    d.pos = pos
    d.vel = np.tile([0.0, 0.0, -1.0], (d.n_particles, 1))
    rt = runtime_from_descs([d])
    rt.substeps(20)
    assert rt.status() & (nat.MPM_STATUS_OUT_OF_GRID | nat.MPM_STATUS_NAN) == 0
    x = rt.get_state()["pos"].cpu().numpy()
    assert (x >= lo - 1e-6).all() and (x <= hi + 1e-6).all()


def test_four_million_particles():
    """4M particles (16 boxes of 250k) on a 257^3 grid: p2g conserves mass to float32
    summation, 10 substeps stay finite and inside the boundary."""
    from genesis_b200.engine.runtime import runtime_from_descs

    d = W.mixed_500k(n_side=100, grid_density=256)  # 4 x 1,000,000 particles
    assert d.n_particles == 4_000_000
    rt = runtime_from_descs([d])
    rt.sort()
    rt.p2g()
    mm, _ = rt.grid_views()
    total = float(mm[..., 3].double().sum())
    expect = sum(float(m.mass) for m in [rt._mats[i] for i in d.mat_idx[:: 1_000_000]]) * 1_000_000
    assert abs(total - expect) / expect < 1e-5
    rt.grid_op()
    rt.g2p()
    rt.substeps(10)
    x = rt.get_state(("pos",))["pos"]
    assert torch.isfinite(x).all()
    assert rt.status() == 0


def test_513_cubed_grid_free_fall_is_exact():
    """A 513^3 grid (129^3 = 2.1M blocks, 137M nodes: 64-bit node addressing) with a falling
    elastic cube: a uniform velocity field is carried exactly by p2g/g2p, so after n substeps
    every particle has moved by the semi-implicit Euler free fall g dt^2 n (n + 1) / 2."""
    from genesis_b200.engine.runtime import runtime_from_descs

    rng = np.random.default_rng(2)
    pos = W.jittered_lattice(rng, 40, (0.475, 0.475, 0.6), 0.05 / 40)
    d = W.SceneDesc(name="fall_513", grid_density=512, particle_size=0.05 / 40, dt=2e-5, n_substeps=200,
                    pos=pos, vel=np.zeros_like(pos), mat_idx=np.zeros(len(pos), np.int64),
                    materials=[("elastic", dict(E=1e5, nu=0.3, rho=1000.0))])
    rt = runtime_from_descs([d])
    assert rt.n_blocks == 129 ** 3
    n = 200
    rt.substeps(n)
    x = rt.get_state(("pos",))["pos"].cpu().numpy().astype(np.float64)
    drop = 9.8 * 2e-5 ** 2 * n * (n + 1) / 2
    assert np.abs(x[:, :2] - pos[:, :2]).max() < 2e-6
    assert np.abs((pos[:, 2] - x[:, 2]) - drop).max() < 2e-6, drop
    assert rt.status() == 0


def _empty_like(desc):
    import dataclasses

    return dataclasses.replace(desc, pos=np.zeros((0, 3)), vel=np.zeros((0, 3)), mat_idx=np.zeros(0, dtype=np.int64),
                               name="empty")


def test_empty_scene_in_a_batch_and_alone():
    """A scene without particles: alone it steps as a no-op (status clean), and between two
    others in one batch it changes nothing of theirs (ragged instance table with a zero
    particle range)."""
    from genesis_b200 import workloads as W
    from genesis_b200.engine.runtime import runtime_from_descs

    a = W.elastic_cube(n_side=12, n_substeps=20)
    b = W.mixed_500k(n_side=10, n_substeps=20)
    empty = _empty_like(a)
    rt0 = runtime_from_descs([empty])
    rt0.substeps(5)
    torch.cuda.synchronize()
    assert rt0.status() == 0 and rt0.n == 0
    alone = []
    for d in (a, b):
        rt = runtime_from_descs([d])
        rt.substeps(20)
        alone.append(rt.get_state(("pos",))["pos"].cpu().numpy())
    rt = runtime_from_descs([a, empty, b])
    rt.substeps(20)
    pos = rt.get_state(("pos",))["pos"].cpu().numpy()
    offs = rt.instance_offsets
    assert offs[1] == offs[2] == a.n_particles
    assert np.abs(pos[: a.n_particles] - alone[0]).max() <= 1e-5  # float atomics: summation order
    assert np.abs(pos[a.n_particles:] - alone[1]).max() <= 1e-5
    assert (rt.instance_status() == 0).all()
