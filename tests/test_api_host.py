"""Host-side API logic that needs no GPU: options, materials, morphs, derived constants
and the no-CPU-fallback rule."""

import numpy as np
import pytest

import genesis_b200 as gs
from genesis_b200.engine.runtime import InstanceSpec


def test_cpu_backend_is_refused():
    with pytest.raises(gs.GenesisException):
        gs.init(backend=gs.cpu)
    with pytest.raises(gs.GenesisException):
        gs.init(precision="64")


def test_options_defaults_follow_reference():
    so = gs.options.SimOptions()
    assert so.dt == 1e-2 and so.substeps == 1 and so.substeps_local == 1
    assert gs.options.SimOptions(requires_grad=True, substeps=4).substeps_local == 4
    mo = gs.options.MPMOptions(grid_density=128)
    assert np.isclose(mo.particle_size, 0.005)
    with pytest.raises(gs.GenesisException):
        gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(0, 1, 1))
    with pytest.raises(gs.GenesisException):
        gs.options.SimOptions(bogus=1)


def test_material_classes_and_dedupe():
    M = gs.materials.MPM
    assert M.Elastic().E == 3e5
    assert M.ElastoPlastic().yield_higher == 4.5e-3
    assert M.Liquid().mu == 0.0 and M.Liquid(viscous=True).mu > 0
    assert M.Sand().default_Jp == 0.0
    assert M.Elastic(E=1e5) == M.Elastic(E=1e5)
    assert M.Elastic(E=1e5) != M.Elastic(E=2e5)
    assert M.Elastic() != M.Liquid()
    e = M.ElastoPlastic(von_mises_yield_stress=1e4)
    nm = e._native(1e-3)
    assert nm.flags & 2 and np.isclose(nm.vm_threshold, 1e4 / (2 * e.mu), rtol=1e-6)
    assert np.isclose(nm.mass, np.float32(1e-3) * np.float32(1000.0))
    with pytest.raises(gs.GenesisException):
        M.Elastic(model="bogus")


def test_box_sampler_counts():
    b = gs.morphs.Box(lower=(0.4, 0.4, 0.4), upper=(0.6, 0.6, 0.6))
    pts = b.sample(0.00625, "regular")
    assert pts.shape == (32**3, 3)
    assert np.all(pts > 0.4) and np.all(pts < 0.6)
    r = b.sample(0.01, "random", np.random.default_rng(0))
    assert r.shape == (20**3, 3)


def test_instance_spec_derived_constants():
    sp = InstanceSpec(grid_density=64, lower_bound=(0, 0, 0), upper_bound=(1, 1, 1), particle_size=0.00625, dt=1e-4,
                      gravity=(0, 0, -9.8), materials=[], n_particles=0)
    assert tuple(sp.grid_res) == (65, 65, 65)
    assert tuple(sp.nblk) == (17, 17, 17)
    assert np.allclose(sp.bnd_lo, 3 / 64) and np.allclose(sp.bnd_hi, 1 - 3 / 64)
    sp2 = InstanceSpec(grid_density=128, lower_bound=(-1, -1, 0), upper_bound=(1, 1, 1), particle_size=0.005,
                       dt=1e-4, gravity=(0, 0, -9.8), materials=[], n_particles=0)
    assert tuple(sp2.grid_res) == (257, 257, 129) and tuple(sp2.lower_cell) == (-128, -128, 0)


def test_scene_requires_init():
    from genesis_b200 import _globals

    saved = _globals.initialized
    _globals.initialized = False
    try:
        with pytest.raises(gs.GenesisException):
            gs.Scene()
    finally:
        _globals.initialized = saved


def test_check_nan_option_is_validated():
    gs.options.B200Options(check_nan="async")
    with pytest.raises(gs.GenesisException):
        gs.options.B200Options(check_nan="sometimes")


def test_muscle_material_follows_reference():
    from genesis_b200 import _native as nat

    m = gs.materials.MPM.Muscle()
    assert m.E == 1e6 and m.stiffness == 1e6 and m.n_groups == 1 and m.model == "neohooken"
    nm = m._native(1e-3)
    assert nm.kind == nat.MAT_ELASTIC and nm.flags & nat.MATF_MUSCLE and nm.flags & nat.MATF_NEOHOOKEAN
    assert nm.muscle_stiffness == 1e6
    assert isinstance(m, gs.materials.MPM.Elastic)
    assert gs.materials.MPM.Elastic()._native(1e-3).muscle_stiffness == 0.0


def test_rigid_material_and_plane_follow_reference():
    m = gs.materials.Rigid()
    assert (m.coup_friction, m.coup_softness, m.coup_restitution, m.needs_coup) == (0.1, 0.002, 0.0, True)
    for bad in (dict(coup_friction=-1), dict(coup_softness=-1), dict(coup_restitution=2), dict(friction=10.0),
                dict(sdf_min_res=8)):
        with pytest.raises(gs.GenesisException):
            gs.materials.Rigid(**bad)
    p = gs.morphs.Plane(normal=(0, 0, 2))
    assert np.allclose(p.normal, (0, 0, 1))
    from genesis_b200.engine.rigid import R_to_quat, quat_to_R

    q = np.array([0.9, 0.1, -0.3, 0.2])
    q /= np.linalg.norm(q)
    assert np.allclose(R_to_quat(quat_to_R(q)), q)


def test_sim_state_solver_order():
    """A scene's state holds one entry per solver in the reference's order
    (simulator.py:129-140), so scripts find the MPM state at solvers_state[3]."""
    import torch

    from genesis_b200.engine.states import MPM_INDEX, SOLVER_NAMES, MPMSolverState, SimState

    assert SOLVER_NAMES == ("tool", "rigid", "avatar", "mpm", "sph", "pbd", "fem", "sf")
    assert MPM_INDEX == 3
    z = torch.zeros
    mpm = MPMSolverState(None, z(1, 2, 3), z(1, 2, 3), z(1, 2, 3, 3), z(1, 2, 3, 3), z(1, 2), torch.ones(1, 2, dtype=torch.bool))
    slots = [None] * len(SOLVER_NAMES)
    slots[MPM_INDEX] = mpm
    s = SimState(None, 7, slots)
    assert s.solvers_state[3] is mpm and s[3] is mpm
    assert [i for i, st in enumerate(s) if st is not None] == [3]
    assert s.s_global == 7
    assert bool((s.solvers_state[3].active == 1).all())
    s.serializable()
    assert s.scene is None


def test_tool_solver_state_container():
    """ToolSolverState holds one entity state per tool (states/solvers.py:114-133)."""
    import torch

    from genesis_b200.engine.states import ToolSolverState
    from genesis_b200.engine.tool import ToolEntityState

    z = torch.zeros
    ts = ToolSolverState("scene")
    ts.entities = [ToolEntityState("tool", 4, z(2, 3, requires_grad=True), z(2, 4), z(2, 3), z(2, 3))]
    assert len(ts) == 1 and ts[0].s_global == 4 and ts[0].entity == "tool"
    ts.serializable()
    assert ts.scene is None and ts[0].entity is None and not ts[0].pos.requires_grad
