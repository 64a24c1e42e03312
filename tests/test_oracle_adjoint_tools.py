"""The tool coupling and its adjoint, on the CPU (float64).

* The numpy tool response (oracle/mpm_ref.py: collide_tool, tool_entity/mesh.py:80-176)
  against the C restatement's (oracle/mpm_ref.c) on a block pushed by a moving, spinning tool.
* The adjoint of a rollout with a tool (oracle/mpm_adjoint.py: rollout_colliders, the tool's
  response differentiated by complex steps with respect to the node velocity, the tool's
  position and its linear velocity, chained through pos_{t+1} = pos_t + lin_vel_t dt) against
  central finite differences: every particle's initial velocity (summed per axis), the tool's
  initial position and its velocity in each of three groups of substeps (what three
  set_velocity calls give it), with the tool pressed to its floor in one case.
"""

import dataclasses

import numpy as np
import pytest

from oracle import mpm_adjoint as A
from oracle import mpm_ref as R


def sphere_tool(pos, lin_vel, ang_vel=(0.0, 0.0, 0.0), res=24, world_radius=0.06, floor=0.0, friction=0.4):
    """A Tool whose normalised mesh is a sphere of radius 0.4 (signed distances in the mesh's
    normalised units on the [-0.6, 0.6]^3 voxel grid of utils/mesh.py:179-201), scaled so that
    its world radius is world_radius."""
    g = np.linspace(-0.6, 0.6, res)
    X = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1)
    vox = np.linalg.norm(X, axis=-1) - 0.4
    scale = world_radius / 0.4
    th = 0.3
    rot = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    return R.Collider("tool", np.asarray(pos, dtype=np.float64), rot, np.zeros(3), np.asarray(lin_vel, float),
                      np.asarray(ang_vel, float), friction=friction, softness=0.01, sdf=vox,
                      sdf_scale=np.full(3, (res - 1) / 1.2 / scale), floor=floor)


def _block(seed=0, n_side=6, lo=(0.45, 0.45, 0.2)):
    rng = np.random.default_rng(seed)
    g = np.arange(n_side) * 0.01
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + np.asarray(lo)
    return x + rng.uniform(-0.002, 0.002, x.shape)


def _setup(tool_pos, floor=0.0, lin=(1.0, 0.0, 0.0)):
    x = _block()
    n = len(x)
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-3, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4, nu=0.3)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile([0.2, 0.0, -0.3], (n, 1)))
    m = mats[0]
    mu = np.full(n, m.mu)
    lam = np.full(n, m.lam)
    tool = sphere_tool(tool_pos, lin, ang_vel=(0.0, 0.0, 3.0), floor=floor)
    return p, mats, st, mu, lam, tool


def test_numpy_tool_coupling_matches_the_c_restatement():
    from oracle import cref

    p, mats, st, _, _, tool = _setup((0.40, 0.475, 0.225))
    st["colliders"] = [tool]
    out_c, rc = cref.substeps(p, mats, dict(st), 12)
    assert rc == 0
    out_n = R.run(p, mats, dict(st), 12)
    assert np.abs(out_n["x"] - out_c["x"]).max() < 1e-12
    assert np.abs(out_n["v"] - out_c["v"]).max() < 1e-9
    assert np.allclose(out_n["colliders"][0].pos, out_c["colliders"][0].pos, atol=1e-14)
    # the tool did push: without it the block's velocity stays near its initial value
    free = dict(st)
    free["colliders"] = [dataclasses.replace(tool, pos=np.array([0.1, 0.1, 0.8]))]
    out_f = R.run(p, mats, free, 12)
    assert np.abs(out_n["v"] - out_f["v"]).max() > 0.1


@pytest.mark.parametrize("case", ["push", "floor"])
def test_tool_rollout_gradient_matches_central_differences(case):
    if case == "push":
        p, mats, st, mu, lam, tool = _setup((0.40, 0.475, 0.225))
        lin = np.array([1.0, 0.0, 0.0])
    else:  # the tool sinks towards its floor at z = 0.17 and is held there
        p, mats, st, mu, lam, tool = _setup((0.475, 0.475, 0.175), floor=0.17, lin=(0.0, 0.0, -2.0))
        lin = np.array([0.0, 0.0, -2.0])
    T, groups = 9, 3
    per = T // groups
    base = np.tile(lin, (groups, 1))
    rng = np.random.default_rng(5)
    W = rng.normal(size=st["x"].shape)

    def lin_seq(g):
        return np.repeat(g, per, axis=0)[:, None, :]

    def L(st2=st, tool2=tool, g=base):
        return A.rollout_colliders(p, mats, st2, mu, lam, [tool2], lin_seq(g), W, grad=False)

    loss, v_bar, pos_bar, lin_bar = A.rollout_colliders(p, mats, st, mu, lam, [tool], lin_seq(base), W)
    assert loss == pytest.approx(L())
    grp_bar = lin_bar[:, 0].reshape(groups, per, 3).sum(1)
    if case == "floor":
        # the origin reaches the floor in the third substep and stays there, and before that
        # it sinks faster than the block falls (no node pushes into it): neither its initial
        # height nor its z velocity changes anything
        assert tool.pos[2] + 3 * lin[2] * p.dt < tool.floor < tool.pos[2] + 2 * lin[2] * p.dt
        assert np.all(grp_bar[:, 2] == 0.0) and pos_bar[0, 2] == 0.0
    # the response jumps where the influence crosses 0.1 and its normal has kinks where
    # pv +- 1e-2 crosses a voxel face: a step must not reach one (1e-5 and 1e-6 do here)
    h = 1e-7
    checks = []
    for c in range(3):
        s_p, s_m = dict(st), dict(st)
        s_p["v"] = st["v"].copy()
        s_m["v"] = st["v"].copy()
        s_p["v"][:, c] += h
        s_m["v"][:, c] -= h
        checks.append(("v0", c, v_bar[:, c].sum(), (L(st2=s_p) - L(st2=s_m)) / (2 * h)))
        tp = dataclasses.replace(tool, pos=tool.pos + h * np.eye(3)[c])
        tm = dataclasses.replace(tool, pos=tool.pos - h * np.eye(3)[c])
        checks.append(("tool pos", c, pos_bar[0, c], (L(tool2=tp) - L(tool2=tm)) / (2 * h)))
        for g in range(groups):
            gp, gm = base.copy(), base.copy()
            gp[g, c] += h
            gm[g, c] -= h
            checks.append((f"tool vel {g}", c, grp_bar[g, c], (L(g=gp) - L(g=gm)) / (2 * h)))
    scale = max(abs(c[3]) for c in checks)
    assert scale > 1e-3  # the tool moved the block
    nonzero = [c for c in checks if c[0].startswith("tool") and abs(c[3]) > 1e-3 * scale]
    assert len(nonzero) >= 4
    noise = 8 * np.finfo(np.float64).eps * abs(loss) / h  # the differences' round-off
    for name, c, got, fd in checks:
        assert abs(got - fd) <= 1e-5 * max(abs(fd), 1e-3 * scale) + noise, (name, c, got, fd)


def test_rigid_response_adjoint_matches_central_differences():
    """collider_vjp of a tilted, moving, spinning box with restitution (legacy_coupler.py:297-341;
    its pose taken as given) against central differences of collide_rigid in the node velocity."""
    rng = np.random.default_rng(7)
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-3, dtype=np.float64)
    th = 0.4
    rot = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    c = R.Collider("box", np.array([0.5, 0.5, 0.5]), rot, np.array([0.05, 0.03, 0.04]), np.array([0.2, 0.0, -0.1]),
                   np.array([0.0, 0.0, 1.0]), friction=0.3, softness=0.01, restitution=0.4)
    nodes = c.pos + rng.uniform(-0.07, 0.07, size=(300, 3))
    v = rng.normal(size=(300, 3))
    vbar = rng.normal(size=(300, 3))
    mass = np.full(300, 1e-3)
    got, pb, lb = A.collider_vjp(p, c, nodes, v, vbar, mass=mass)
    assert np.all(pb == 0) and np.all(lb == 0)
    h = 1e-7
    fd = np.zeros_like(v)
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        up = R.collide_rigid(c, p.eps, p.dt, nodes, v + e, mass)[0]
        dn = R.collide_rigid(c, p.eps, p.dt, nodes, v - e, mass)[0]
        fd[:, k] = ((up - dn) / (2 * h) * vbar).sum(1)
    hit = np.abs(got - vbar).max(1) > 1e-12  # nodes the response acted on
    assert hit.sum() > 20
    assert np.abs(got - fd).max() <= 1e-6 * np.abs(fd).max()
