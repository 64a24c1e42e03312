"""CPU checks of the oracle itself (no GPU): algebraic identities, the reference's
qualitative MPM invariants, and agreement of the numpy and C restatements."""

import numpy as np
import pytest

from genesis_b200 import workloads as W
from oracle import bridge, cref
from oracle import mpm_ref as R


def _rand_F(rng, n, scale=0.2):
    return np.eye(3)[None] + scale * rng.normal(size=(n, 3, 3))


def test_svd_convention_and_reconstruction():
    rng = np.random.default_rng(0)
    F = _rand_F(rng, 2000, 0.6)
    F[:10] = -F[:10]  # det < 0 cases
    U, S, V = R.svd3(F)
    assert np.allclose(np.linalg.det(U), 1.0)
    assert np.allclose(np.linalg.det(V), 1.0)
    assert np.allclose(U @ (S[:, :, None] * np.swapaxes(V, 1, 2)), F, atol=1e-12)
    assert np.all(S[:, 0] >= np.abs(S[:, 1]) - 1e-12) and np.all(S[:, 1] >= np.abs(S[:, 2]) - 1e-12)
    assert np.all(S[:, :2] >= 0)
    neg = np.linalg.det(F) < 0
    assert np.all(S[neg, 2] < 0) and np.all(S[~neg, 2] >= 0)


def test_c_svd_matches_lapack_convention():
    """The C port's Jacobi+QR SVD and LAPACK agree on rotation-invariant outputs."""
    rng = np.random.default_rng(1)
    d = W.elastic_cube(n_side=4)
    p, mats, st = bridge.from_desc(d, np.float64)
    st["F"] = _rand_F(rng, st["x"].shape[0], 0.3)
    st["C"] = 50 * rng.normal(size=st["C"].shape)
    a = R.substep(p, mats, st)
    b, rc = cref.substeps(p, mats, st, 1)
    assert rc == 0
    for k in ("x", "v", "C", "F", "Jp"):
        assert np.allclose(a[k], b[k], rtol=1e-9, atol=1e-12), k


def test_bspline_partition_of_unity_and_first_moment():
    fx = np.random.default_rng(2).uniform(0.5, 1.5, size=(1000, 3))
    w = R._weights(fx)
    s = sum(w)
    assert np.allclose(s, 1.0)
    # sum_i w_i (i - fx) = 0 : APIC affine term carries no net momentum
    m1 = sum(w[i] * (i - fx) for i in range(3))
    assert np.allclose(m1, 0.0, atol=1e-14)


@pytest.mark.parametrize("kind", ["elastic", "elastoplastic", "liquid", "sand", "snow"])
def test_p2g_conserves_mass_and_momentum(kind):
    rng = np.random.default_rng(3)
    d = W.elastic_cube(n_side=8)
    d.materials = [(kind, {})]
    d.vel = rng.normal(0, 0.5, size=d.vel.shape)
    p, mats, st = bridge.from_desc(d, np.float64)
    st["F"] = _rand_F(rng, st["x"].shape[0], 0.05)
    st["C"] = rng.normal(size=st["C"].shape)
    gm, gp, _, _ = R.p2g(p, mats, st)
    m = R.particle_mass(p, mats[0])
    n = st["x"].shape[0]
    assert np.isclose(gm.sum(), n * m, rtol=1e-12)
    # stress contributions sum to zero (sum_i w_i dpos_i = 0); momentum = sum m v + sum m C @ 0
    assert np.allclose(gp.reshape(-1, 3).sum(0), m * st["v"].sum(0), rtol=1e-9, atol=1e-9)


def test_grid_op_gravity_and_boundary():
    d = W.elastic_cube(n_side=4)
    p, mats, st = bridge.from_desc(d, np.float64)
    res = tuple(p.grid_res)
    gm = np.zeros(res)
    gp = np.zeros(res + (3,))
    gm[10, 10, 10] = 2.0
    gp[10, 10, 10] = [2.0, 0.0, 0.0]
    gm[1, 10, 10] = 1.0
    gp[1, 10, 10] = [-1.0, 0.5, 0.0]  # outside the padded lower x wall, moving out
    gm[20, 20, 20] = 1e-9  # below EPS? (f64 EPS = 2.2e-16: still active)
    vel = R.grid_op(p, gm, gp)
    assert np.allclose(vel[10, 10, 10], [1.0, 0.0, -9.8 * p.dt])
    assert vel[1, 10, 10, 0] == 0.0 and np.isclose(vel[1, 10, 10, 1], 0.5)
    assert np.all(vel[0, 0, 0] == 0)


def test_g2p_uniform_field_is_exact():
    d = W.elastic_cube(n_side=6)
    p, mats, st = bridge.from_desc(d, np.float64)
    res = tuple(p.grid_res)
    vel = np.zeros(res + (3,))
    vel[...] = [0.1, -0.2, 0.3]
    xn, vn, Cn = R.g2p(p, st, vel)
    assert np.allclose(vn, [0.1, -0.2, 0.3])
    assert np.allclose(Cn, 0.0, atol=1e-10)
    assert np.allclose(xn, st["x"] + p.dt * vn)


def test_material_return_mappings():
    rng = np.random.default_rng(4)
    n = 500
    F = _rand_F(rng, n, 0.15)
    U, S, V = R.svd3(F)
    J = S[:, 0] * S[:, 1] * S[:, 2]
    Jp = np.ones(n)
    # von Mises: after projection the deviatoric log-strain norm is at most the yield radius
    ep = R.make_material("elastoplastic", von_mises_yield_stress=1e4)
    Fn, Sn, _ = R.update_F_S_Jp(ep, 2.2e-16, J, F, U, S, V, Jp)
    e = np.log(np.maximum(Sn, 0.05))
    eh = e - e.mean(1, keepdims=True)
    assert np.all(np.linalg.norm(eh, axis=1) <= ep.von_mises_yield_stress / (2 * ep.mu) + 1e-6)
    # snow: clamp and Jp bookkeeping keeps Jp * det(F_new) = det(F_tmp)
    sn = R.make_material("snow", yield_lower=2.5e-2, yield_higher=7.5e-3)
    Fn, Sn, Jpn = R.update_F_S_Jp(sn, 2.2e-16, J, F, U, S, V, Jp)
    assert np.all(Sn >= 1 - 2.5e-2 - 1e-12) and np.all(Sn <= 1 + 7.5e-3 + 1e-12)
    assert np.allclose(Jpn * np.linalg.det(Fn), np.linalg.det(F))
    # sand: expansion (tr >= 0) resets to identity singular values
    sd = R.make_material("sand")
    Fn, Sn, Jpn = R.update_F_S_Jp(sd, 2.2e-16, J, F, U, S, V, np.zeros(n))
    tr = np.log(np.maximum(np.abs(S), 1e-4)).sum(1)
    assert np.allclose(Sn[tr >= 0], 1.0) and np.allclose(Jpn[tr >= 0], tr[tr >= 0])
    # liquid: F_new = J^(1/3) I
    lq = R.make_material("liquid")
    Fn, _, _ = R.update_F_S_Jp(lq, 2.2e-16, J, F, U, S, V, Jp)
    assert np.allclose(Fn, np.cbrt(J)[:, None, None] * np.eye(3))


def test_material_defaults_follow_reference():
    assert R.make_material("elastic").E == 3e5  # elastic.py:40
    assert R.make_material("elastoplastic").yield_higher == 4.5e-3  # elasto_plastic.py:52
    assert R.make_material("sand").default_Jp == 0.0  # sand.py:45
    assert R.make_material("liquid").mu == 0.0  # liquid.py:47-48
    assert not R.make_material("snow").use_von_mises  # snow.py:59
    p = R.Params(grid_density=64, lower_bound=(0, 0, 0), upper_bound=(1, 1, 1))
    assert tuple(p.grid_res) == (65, 65, 65)  # mpm_solver.py:53-55
    assert np.isclose(p.particle_size, 0.01)  # options/solvers.py:490-491
    assert np.isclose(p.p_vol, 1e-6 * 1e3)
    assert R.Params(dtype=np.float32).eps == np.finfo(np.float32).eps


def test_numpy_and_c_oracles_agree_f32_and_f64():
    d = W.mixed_500k(n_side=6, grid_density=64)
    for dtype, tol in ((np.float64, 1e-12), (np.float32, 2e-5)):
        p, mats, st = bridge.from_desc(d, dtype)
        a = R.run(p, mats, st, 5)
        b, rc = cref.substeps(p, mats, st, 5, n_threads=2)
        assert rc == 0
        assert np.abs(a["x"] - b["x"]).max() < tol
        assert np.abs(a["v"] - b["v"]).max() < 100 * tol


def test_reference_invariants_cube_falls_and_stays_in_domain():
    """tests/test_deformable_physics.py:209-219 asserts the MPM cube moved and stays above
    the floor; here: it falls under gravity and never leaves the padded boundary."""
    d = W.elastic_cube(n_side=8)
    p, mats, st = bridge.from_desc(d, np.float64)
    out, rc = cref.substeps(p, mats, st, 300, n_threads=2)
    assert rc == 0
    assert out["x"][:, 2].mean() < st["x"][:, 2].mean() - 1e-4
    assert np.all(out["x"] >= p.bnd_lo - 1e-12) and np.all(out["x"] <= p.bnd_hi + 1e-12)
    assert np.all(np.isfinite(out["x"]))


def test_f32_oracle_error_is_small_over_100_substeps():
    """Inherent float32 drift of the restatement (the CUDA tolerance is set against it)."""
    d = W.elastic_cube(n_side=10)
    a, _ = cref.substeps(*bridge.from_desc(d, np.float64), 100)
    b, _ = cref.substeps(*bridge.from_desc(d, np.float32), 100)
    assert np.abs(a["x"] - b["x"]).max() < 1e-5


def _muscle_case(actu_value, n_side=8, dtype=np.float64):
    rng = np.random.default_rng(7)
    x = W.jittered_lattice(rng, n_side, (0.45, 0.45, 0.45), 0.1 / n_side)
    n = x.shape[0]
    p = R.Params(grid_density=64, dt=1e-4, gravity=(0.0, 0.0, 0.0), dtype=dtype)
    mats = [R.make_material("muscle", E=1e5)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), dtype)
    st["actu"] = np.full(n, actu_value, dtype=dtype)
    st["mdir"] = np.tile(np.array([0.0, 0.0, 1.0], dtype=dtype), (n, 1))
    return p, mats, st


def test_muscle_material_defaults_and_oracles_agree():
    """Muscle (muscle.py:35-65): an Elastic with E=1e6 and the neo-Hookean model by default;
    the numpy and C restatements of the actuation stress agree."""
    m = R.make_material("muscle")
    assert m.muscle and m.neohookean and m.stiffness == 1e6 and m.kind == R.KIND_ELASTIC
    p, mats, st = _muscle_case(2.0)
    o_np = R.run(p, mats, st, 5)
    o_c, rc = cref.substeps(p, mats, st, 5)
    assert rc == 0
    assert np.abs(o_np["x"] - o_c["x"]).max() < 1e-12
    assert np.abs(o_np["F"] - o_c["F"]).max() < 1e-9


def test_muscle_actuation_contracts_along_the_fibre():
    """A positive actuation adds tension along d = +z: the block shortens along z and not
    along x (no gravity), while an unactuated block stays at rest."""
    p, mats, st = _muscle_case(5.0)
    o, _ = cref.substeps(p, mats, st, 200)
    p0, m0, s0 = _muscle_case(0.0)
    r, _ = cref.substeps(p0, m0, s0, 200)
    ext = lambda a, d: a[:, d].max() - a[:, d].min()
    assert ext(o["x"], 2) < ext(st["x"], 2) - 1e-5
    assert abs(ext(r["x"], 2) - ext(st["x"], 2)) < 1e-9
    assert ext(o["x"], 2) < ext(o["x"], 0)


def _block_over(collider, n_side=10, z0=0.35, v0=(0.0, 0.0, -1.0), substeps=300, dtype=np.float64):
    rng = np.random.default_rng(11)
    x = W.jittered_lattice(rng, n_side, (0.45, 0.45, z0), 0.1 / n_side)
    n = x.shape[0]
    p = R.Params(grid_density=64, dt=1e-4, dtype=dtype)
    mats = [R.make_material("elastic", E=2e4)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), dtype, v=np.tile(v0, (n, 1)))
    st["colliders"] = [collider]
    out, rc = cref.substeps(p, mats, st, substeps)
    assert rc == 0
    return out, st


def test_rigid_colliders_numpy_and_c_agree():
    """The two restatements of the grid-op rigid coupling agree (sphere, tilted box,
    moving plane), including the reaction force and the advanced pose."""
    th = np.deg2rad(20)
    Rt = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    cases = [
        R.Collider("sphere", np.array([0.5, 0.5, 0.3]), np.eye(3), np.array([0.05, 0, 0]), friction=0.5),
        R.Collider("box", np.array([0.5, 0.5, 0.3]), Rt, np.array([0.2, 0.2, 0.04]), ang_vel=np.array([0, 0, 2.0])),
        R.Collider("plane", np.array([0.5, 0.5, 0.33]), np.eye(3), np.array([0, 0, 1.0]), lin_vel=np.array([0, 0, 0.3])),
    ]
    for c in cases:
        rng = np.random.default_rng(5)
        x = W.jittered_lattice(rng, 6, (0.45, 0.45, 0.345), 0.06 / 6)
        n = x.shape[0]
        p = R.Params(grid_density=64, dt=1e-4, dtype=np.float64)
        mats = [R.make_material("elastic", E=2e4)]
        st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile([0.0, 0.0, -2.0], (n, 1)))
        st["colliders"] = [c]
        a = R.run(p, mats, st, 8)
        b, rc = cref.substeps(p, mats, st, 8)
        assert rc == 0
        assert np.abs(a["x"] - b["x"]).max() < 1e-12, c.kind
        assert np.allclose(a["colliders"][0].pos, b["colliders"][0].pos)
        assert np.allclose(a["colliders"][0].rot, b["colliders"][0].rot)


def test_rigid_sphere_collider_stops_a_falling_block():
    """legacy_coupler.py:166-343: a block thrown down onto a fixed sphere does not pass
    through it; without the collider it falls below the sphere's top."""
    c = R.Collider("sphere", np.array([0.5, 0.5, 0.25]), np.eye(3), np.array([0.06, 0, 0]))
    out, st = _block_over(c, v0=(0, 0, -3.0), substeps=400)
    r = np.linalg.norm(out["x"] - c.pos, axis=1)
    assert r.min() > 0.06 - 1.5 / 64  # penetration bounded by the grid resolution
    assert out["forces"][0][2] < 0  # the block pushes the sphere down
    free, _ = _block_over(R.Collider("sphere", np.array([0.5, 0.5, -5.0]), np.eye(3), np.array([0.06, 0, 0])),
                          v0=(0, 0, -3.0), substeps=400)
    assert free["x"][:, 2].min() < 0.25


def test_rigid_collider_forms_agree():
    """A plane with normal +z through z=0.3 and a box whose top face is at z=0.3 stop a
    falling block at the same height; a tilted frictionless plane lets it slide."""
    plane = R.Collider("plane", np.array([0.5, 0.5, 0.3]), np.eye(3), np.array([0.0, 0.0, 1.0]))
    box = R.Collider("box", np.array([0.5, 0.5, 0.2]), np.eye(3), np.array([0.3, 0.3, 0.1]))
    a, _ = _block_over(plane, v0=(0, 0, -2.0))
    b, _ = _block_over(box, v0=(0, 0, -2.0))
    assert abs(a["x"][:, 2].min() - b["x"][:, 2].min()) < 2e-3
    assert 0.3 - 1.5 / 64 < a["x"][:, 2].min() < 0.31
    th = np.deg2rad(30)
    Rt = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    slope = R.Collider("plane", np.array([0.5, 0.5, 0.3]), Rt, np.array([0.0, 0.0, 1.0]), friction=0.0)
    c, st = _block_over(slope, z0=0.33, v0=(0, 0, -1.0), substeps=600)
    assert c["x"][:, 0].mean() > st["x"][:, 0].mean() + 0.005  # slid down-slope (+x)


def test_kinematic_collider_motion():
    p = R.Params(grid_density=64, dt=1e-4, dtype=np.float64)
    c = R.Collider("sphere", np.array([0.5, 0.5, 0.4]), np.eye(3), np.array([0.05, 0, 0]),
                   lin_vel=np.array([0.0, 0.0, 0.5]), ang_vel=np.array([0.0, 0.0, 3.0]))
    c2 = R.advance_colliders(p, [c])[0]
    assert np.allclose(c2.pos, [0.5, 0.5, 0.4 + 0.5e-4])
    assert np.allclose(c2.rot @ c2.rot.T, np.eye(3)) and np.isclose(np.arctan2(c2.rot[1, 0], c2.rot[0, 0]), 3e-4)


def _block_cpic(collider, cpic, n_side=10, z0=0.33, v0=(0.0, 0.0, -2.0), substeps=400, n_threads=0):
    rng = np.random.default_rng(12)
    x = W.jittered_lattice(rng, n_side, (0.45, 0.45, z0), 0.1 / n_side)
    n = x.shape[0]
    p = R.Params(grid_density=64, dt=1e-4, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile(v0, (n, 1)))
    st["colliders"] = [collider]
    if cpic:
        st["cpic_normal"] = np.zeros((1, n, 3))
    out, rc = cref.substeps(p, mats, st, substeps, n_threads=n_threads)
    assert rc == 0
    return out


def test_cpic_thin_slab_separates_its_sides():
    """mpm_solver.py:357-379, 412-427: a fixed slab far thinner than a grid cell (0.002 m
    against dx = 0.0156 m).  The grid-op coupling alone reaches only the nodes within its
    influence band, so a falling block passes through; with CPIC the nodes under the slab are
    cut off from the particles above it, which stay on their side."""
    slab = R.Collider("box", np.array([0.5, 0.5, 0.3]), np.eye(3), np.array([0.3, 0.3, 0.001]))
    leak = _block_cpic(slab, cpic=False)
    assert leak["x"][:, 2].min() < 0.28
    kept = _block_cpic(slab, cpic=True)
    assert kept["x"][:, 2].min() > 0.3 - 1.5 / 64
    assert (kept["cpic_normal"][0][:, 2] > 0.99).all()  # every particle remembers the upper side
    assert kept["forces"][0][2] < 0  # the block pushes the slab down


def test_cpic_without_crossing_is_the_plain_coupling():
    """Far from any collider nothing is separated: CPIC changes nothing."""
    far = R.Collider("sphere", np.array([0.5, 0.5, 0.1]), np.eye(3), np.array([0.03, 0, 0]))
    a = _block_cpic(far, cpic=False, substeps=100, n_threads=1)  # one thread: a fixed summation order
    b = _block_cpic(far, cpic=True, substeps=100, n_threads=1)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["v"], b["v"])
