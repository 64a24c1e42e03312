"""Emitter host logic (genesis/engine/entities/emitter.py) with a fake entity: droplet
sampling and placement, length accumulation, slot recycling, boundary checks.  No GPU."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs
from genesis_b200 import geom as gu
from genesis_b200 import particle as pu
from genesis_b200.engine.boundaries import CubeBoundary
from genesis_b200.engine.emitter import Emitter


class _Solver:
    def __init__(self):
        self.boundary = CubeBoundary(lower=(0.05,) * 3, upper=(0.95,) * 3)
        self.substep_dt = 1e-3


class _Sim:
    substeps = 10


class _Entity:
    def __init__(self, n):
        self.n_particles = n
        self.particle_size = 0.01
        self.sampler = "regular"
        self.sim = _Sim()
        self.solver = _Solver()
        self.calls = []

    def set_particles_pos(self, pos, idx):
        self.calls.append(("pos", np.asarray(pos), torch.as_tensor(idx).clone()))

    def set_particles_vel(self, vel, idx):
        self.calls.append(("vel", np.asarray(vel), torch.as_tensor(idx).clone()))

    def set_particles_active(self, act, idx):
        self.calls.append(("act", act, torch.as_tensor(idx).clone()))


def _emitter(n=2000):
    gs.init(backend=gs.gpu, seed=0, logging_level="warning")
    e = Emitter(n)
    ent = _Entity(n)
    e.set_entity(ent)
    return e, ent


def test_rotation_helpers():
    for d in ([0, 0, -1], [1, 0, 0], [0.3, -0.4, 0.5], [0, 0, 1]):
        R = gu.z_up_to_R(np.array(d, dtype=float))
        assert np.allclose(R.T @ R, np.eye(3), atol=1e-12) and np.isclose(np.linalg.det(R), 1.0)
        assert np.allclose(R[:, 2], np.asarray(d) / np.linalg.norm(d))
    R = gu.axis_angle_to_R(np.array([0.0, 0.0, 1.0]), 0.3)
    assert np.allclose(R, [[np.cos(0.3), -np.sin(0.3), 0], [np.sin(0.3), np.cos(0.3), 0], [0, 0, 1]])
    # built from cos(theta): theta and -theta give the same matrix (utils/geom.py:1445)
    assert np.allclose(gu.axis_angle_to_R(np.array([0.0, 1.0, 0.0]), -0.7), gu.axis_angle_to_R(np.array([0, 1.0, 0]), 0.7))


def test_shape_samplers():
    c = pu.cylinder_to_particles(0.01, pos=(0.1, 0.2, 0.3), radius=0.05, height=0.04, sampler="regular")
    assert (np.linalg.norm(c[:, :2] - [0.1, 0.2], axis=1) <= 0.05).all() and np.ptp(c[:, 2]) <= 0.04
    s = pu.sphere_to_particles(0.01, radius=0.05, sampler="random", rng=np.random.default_rng(1))
    assert (np.linalg.norm(s, axis=1) <= 0.05).all() and len(s) > 0
    sh = pu.shell_to_particles(0.01, inner_radius=0.04, outer_radius=0.1, sampler="regular")
    r = np.linalg.norm(sh, axis=1)
    assert (r >= 0.04).all() and (r <= 0.1).all()
    b = pu.box_to_particles(0.01, size=(0.1, 0.05, 0.02), sampler="pbs")  # pbs is sampled as regular
    assert b.shape == (10 * 5 * 2, 3)


def test_emit_places_droplet_at_nozzle_along_direction():
    e, ent = _emitter()
    n = e.emit("square", 0.05, droplet_length=0.03, pos=(0.5, 0.5, 0.8), direction=(0, 0, -1), speed=2.0)
    assert n == 5 * 5 * 3
    kinds = [c[0] for c in ent.calls]
    assert kinds == ["pos", "vel", "act"]
    pos, vel, idx = ent.calls[0][1], ent.calls[1][1], ent.calls[0][2]
    assert np.allclose(pos.mean(0), [0.5, 0.5, 0.8], atol=1e-9)
    assert np.allclose(vel, [0, 0, -2.0])
    assert torch.equal(idx, torch.arange(0, n))
    assert e.next_particle == n


def test_droplet_length_accumulates_until_one_particle_long():
    e, ent = _emitter()
    # one step moves speed * substep_dt * substeps = 0.004 < p_size 0.01: nothing until the third call
    kw = dict(pos=(0.5, 0.5, 0.5), speed=0.4)
    assert e.emit("circle", 0.04, **kw) == 0
    assert e.emit("circle", 0.04, **kw) == 0
    assert e.emit("circle", 0.04, **kw) > 0
    assert len(ent.calls) == 3


def test_slots_recycle_and_limits():
    e, ent = _emitter(n=200)
    sizes = []
    for _ in range(5):
        sizes.append(e.emit("square", 0.05, droplet_length=0.02, pos=(0.5, 0.5, 0.5)))  # 50 particles
    starts = [int(c[2][0]) for c in ent.calls if c[0] == "pos"]
    # recycled as soon as the next droplet of this size would not fit (emitter.py:190-192)
    assert sizes == [50] * 5 and starts == [0, 50, 100, 150, 0]
    with pytest.raises(gs.GenesisException):
        e.emit("square", 0.2, droplet_length=0.1, pos=(0.5, 0.5, 0.5))  # 20*20*10 > 200
    with pytest.raises(gs.GenesisException):
        e.emit("square", 0.05, droplet_length=0.02, pos=(0.5, 0.5, 0.97))  # outside the padded boundary
    with pytest.raises(gs.GenesisException):
        e.emit("triangle", 0.05)
    with pytest.raises(gs.GenesisException):
        e.emit("square", 0.05, direction=(0, 0, 0))


def test_emit_omni_radial_velocity():
    e, ent = _emitter()
    n = e.emit_omni(source_radius=0.05, pos=(0.5, 0.5, 0.5), speed=1.5)
    pos, vel = ent.calls[0][1], ent.calls[1][1]
    assert n == len(pos) > 0
    d = pos - 0.5
    assert np.allclose(np.linalg.norm(vel, axis=1), 1.5, atol=1e-5)
    assert np.allclose(vel / 1.5, d / np.linalg.norm(d, axis=1, keepdims=True), atol=1e-5)
