"""External force fields without a GPU: the oracle against the reference's own
engine/force_fields.py (tests/golden/ref_force_fields.npz, made by running that file and the
reference's MPMSolver + LegacyCoupler under a numpy stand-in for gstaichi), and the host-side
packing of gs.force_fields into the grid op's mpm_force_field rows."""

import json
import os

import numpy as np
import pytest

from oracle import mpm_ref as R

HERE = os.path.join(os.path.dirname(__file__), "golden")


def _fx():
    z = np.load(os.path.join(HERE, "ref_force_fields.npz"))
    return z, json.loads(str(z["meta"]))


def test_force_field_accelerations_match_reference():
    z, meta = _fx()
    for k, (name, kw) in enumerate(meta["fields"]):
        f = R.make_force_field(name, **kw)
        acc = R.force_field_acc(f, z[f"f{k}_pos"], z[f"f{k}_vel"], meta["eps"])
        assert np.abs(acc - z[f"f{k}_acc"]).max() <= 1e-12 * max(1.0, np.abs(z[f"f{k}_acc"]).max()), (name, kw)


def _scene_oracle(z, meta, fields=True):
    sc = meta["scene"]
    p = R.Params(grid_density=sc["grid_density"], upper_bound=tuple(sc["upper_bound"]),
                 particle_size=sc["particle_size"], dt=sc["dt"], gravity=tuple(sc["gravity"]), dtype=np.float64)
    p.eps = meta["eps"]
    mats = [R.make_material(k, **dict(kw)) for k, kw in sc["materials"]]
    st = R.make_state(z["scene_pos"], mats, z["scene_mat_idx"], np.float64, v=z["scene_vel"])
    if fields:
        st["force_fields"] = [R.make_force_field(n, **kw) for n, kw in sc["fields"]]
    out, done = {}, 0
    for n in sc["snapshots"]:
        st = R.run(p, mats, st, n - done)
        done = n
        out[n] = st
    return out


def test_scene_under_force_fields_matches_reference():
    z, meta = _fx()
    got = _scene_oracle(z, meta)
    free = _scene_oracle(z, meta, fields=False)
    for n, st in got.items():
        assert np.abs(st["x"] - z[f"scene_x_{n}"]).max() < 1e-12
        assert np.abs(st["v"] - z[f"scene_v_{n}"]).max() < 1e-10
        assert np.abs(st["F"] - z[f"scene_F_{n}"]).max() < 1e-10
    last = meta["scene"]["snapshots"][-1]
    assert np.abs(free[last]["v"] - z[f"scene_v_{last}"]).max() > 1e-2  # the fields changed the flow


def test_force_fields_pack_into_rows():
    from genesis_b200 import _native as nat
    from genesis_b200 import force_fields as ff

    z, meta = _fx()
    objs = [getattr(ff, n)(**kw) for n, kw in meta["fields"]]
    objs[0].activate()
    rows, perm = ff.pack(objs)
    assert [r.kind for r in rows] == [nat.FF_CONSTANT, nat.FF_WIND, nat.FF_POINT, nat.FF_DRAG, nat.FF_VORTEX,
                                      nat.FF_VORTEX, nat.FF_TURBULENCE, nat.FF_TURBULENCE]
    assert rows[0].active == 1 and all(r.active == 0 for r in rows[1:])  # fields start inactive
    c = R.make_force_field(*meta["fields"][0][:1], **meta["fields"][0][1])
    assert np.allclose(list(rows[0].vec), c["direction"] * c["strength"], atol=1e-7)
    assert rows[5].falloff_max == float("inf")
    # the turbulence fields' permutation tables: the oracle's (the reference's construction)
    for k, i in enumerate((6, 7)):
        t = R.make_force_field(*meta["fields"][i][:1], **meta["fields"][i][1])
        assert rows[i].perm_offset == k * 3 * 512
        assert np.array_equal(perm[k * 1536:(k + 1) * 1536], np.concatenate(t["perms"]))


def test_custom_and_noise_rules():
    import genesis_b200 as gs
    from genesis_b200 import force_fields as ff

    with pytest.raises(ValueError):
        ff.Constant(direction=(1, 0))
    n = ff.Noise(strength=2.0, seed=5)
    rows, perm = ff.pack([n, ff.Drag(linear=1.0)])
    assert perm is None and rows[0].seed == 5 and rows[1].linear == 1.0
    f = ff.Vortex()
    assert not f.active
    f.activate()
    assert f.active
    f.deactivate()
    assert not f.active
    assert isinstance(gs.force_fields.Turbulence(seed=1), gs.force_fields.ForceField)


def test_rollout_gradient_with_force_fields_matches_central_differences():
    """The adjoint oracle (oracle/mpm_adjoint.py: the fields' v-dependence differentiated by
    complex steps) against central differences, through Drag, Vortex damping, Point and
    Turbulence flow and a constant Wind."""
    from oracle import mpm_adjoint as A

    rng = np.random.default_rng(9)
    p = R.Params(grid_density=32, upper_bound=(0.5, 0.5, 0.5), particle_size=0.01, dt=5e-4, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4, nu=0.3)]
    x = rng.uniform(0.18, 0.3, size=(80, 3))
    st = R.make_state(x, mats, np.zeros(len(x), np.int64), np.float64, v=rng.normal(0, 0.3, (len(x), 3)))
    st["force_fields"] = [
        R.make_force_field("Drag", linear=0.8, quadratic=0.5),
        R.make_force_field("Vortex", center=(0.25, 0.25, 0.0), strength_perpendicular=8.0, strength_radial=2.0,
                           falloff_min=0.02, falloff_max=0.4, damping=0.6),
        R.make_force_field("Point", strength=1.5, position=(0.3, 0.2, 0.3), falloff_pow=1.0, flow=0.7),
        R.make_force_field("Turbulence", strength=4.0, frequency=6, flow=0.9, seed=3),
        R.make_force_field("Wind", direction=(1.0, 0.0, 0.0), strength=2.0, radius=0.05, center=(0.25, 0.25, 0.25)),
    ]
    m = mats[0]
    mu, lam = np.full(len(x), m.mu), np.full(len(x), m.lam)
    W = rng.normal(size=x.shape)
    T = 6
    none = np.zeros((T, 0, 3))
    loss, vbar, _, _ = A.rollout_colliders(p, mats, st, mu, lam, [], none, W)
    h = 1e-6
    for c in range(3):
        sp, sm = dict(st), dict(st)
        sp["v"], sm["v"] = st["v"].copy(), st["v"].copy()
        sp["v"][:, c] += h
        sm["v"][:, c] -= h
        fd = (A.rollout_colliders(p, mats, sp, mu, lam, [], none, W, grad=False) -
              A.rollout_colliders(p, mats, sm, mu, lam, [], none, W, grad=False)) / (2 * h)
        assert abs(vbar[:, c].sum() - fd) <= 1e-6 * abs(fd) + 1e-8, (c, vbar[:, c].sum(), fd)
    # the fields' velocity terms matter: without them the gradient differs
    st0 = dict(st)
    st0["force_fields"] = []
    _, vb0, _, _ = A.rollout_colliders(p, mats, st0, mu, lam, [], none, W)
    assert np.abs(vb0.sum(0) - vbar.sum(0)).max() > 1e-3 * np.abs(vbar.sum(0)).max()
