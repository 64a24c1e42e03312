"""Tool entities without a GPU: the signed-distance oracle against exact distances, the C
restatement's tool coupling (a sand block lands on a static tool plate and stays on it), and
the host-side mesh normalisation and voxel scale of the tool (tool_entity/mesh.py:23-59)."""

import os

import numpy as np
import pytest

from genesis_b200 import mesh


def test_sdf_oracle_exact_for_a_box_and_close_for_a_sphere():
    from oracle import sdf_ref

    v, f = mesh.box_mesh((0.6, 0.4, 0.8))
    P = sdf_ref.lattice(12)
    d = np.abs(P) - np.array([0.3, 0.2, 0.4])
    exact = np.linalg.norm(np.maximum(d, 0), axis=1) + np.minimum(d.max(1), 0)
    assert np.abs(sdf_ref.signed_distance(P, v, f) - exact).max() < 1e-12
    v, f = mesh.icosphere(subdivisions=3, radius=0.4)
    sd = sdf_ref.signed_distance(P, v, f)
    # the polyhedron lies within 0.4 (1 - cos(edge angle / 2)) of the sphere
    assert np.abs(sd - (np.linalg.norm(P, axis=1) - 0.4)).max() < 0.01
    assert (sd[np.linalg.norm(P, axis=1) < 0.35] < 0).all()


def _tool_collider(kind_pos, res=32):
    from oracle import mpm_ref as R
    from oracle import sdf_ref

    v, f = mesh.box_mesh((1.0, 1.0, 0.1))  # a unit-extent plate, as normalised
    vox = sdf_ref.sdf_voxels(v, f, res)
    scale = np.array([0.3, 0.3, 0.3])  # the tool is 0.3 x 0.3 x 0.03
    return R.Collider("tool", np.asarray(kind_pos, dtype=np.float64), np.eye(3), np.zeros(3), friction=0.0,
                      softness=0.01, sdf=vox, sdf_scale=(res - 1) / 1.2 / scale, floor=0.0)


def test_oracle_tool_plate_holds_a_falling_block():
    from oracle import cref
    from oracle import mpm_ref as R

    x = np.stack(np.meshgrid(*[np.arange(0.45, 0.55, 0.01)] * 3, indexing="ij"), -1).reshape(-1, 3)
    n = len(x)
    p = R.Params(grid_density=64, particle_size=0.01, dt=2e-4, dtype=np.float64)
    mats = [R.make_material("elastic")]

    def run(tool_z):
        st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile([0.0, 0.0, -1.0], (n, 1)))
        st["colliders"] = [_tool_collider([0.5, 0.5, tool_z])]
        out, rc = cref.substeps(p, mats, st, 400)
        assert rc == 0
        return out

    free = run(-5.0)
    assert free["x"][:, 2].min() < 0.35  # without the plate the block falls below z = 0.35
    out = run(0.35)
    # the plate's top is at z = 0.35 + 0.015: the block lands on it
    assert out["x"][:, 2].min() > 0.36
    assert np.allclose(out["colliders"][0].pos, [0.5, 0.5, 0.35])


def test_oracle_tool_kinematics_and_floor():
    from oracle import cref
    from oracle import mpm_ref as R

    x = np.array([[0.8, 0.8, 0.8]])
    p = R.Params(grid_density=32, particle_size=0.01, dt=1e-3, dtype=np.float64)
    mats = [R.make_material("elastic")]
    st = R.make_state(x, mats, np.zeros(1, np.int64), np.float64)
    c = _tool_collider([0.3, 0.3, 0.05])
    c.lin_vel = np.array([0.1, 0.0, -1.0])
    c.ang_vel = np.array([0.0, 0.0, 2.0])
    st["colliders"] = [c]
    out, rc = cref.substeps(p, mats, st, 100)
    m = out["colliders"][0]
    assert np.allclose(m.pos, [0.31, 0.3, 0.0])  # z clamped to the floor height 0
    th = 0.2
    assert np.allclose(m.rot, [[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]], atol=1e-12)


def test_tool_mesh_normalisation_and_voxel_scale(tmp_path):
    import genesis_b200 as gs
    from genesis_b200.engine.tool import ToolEntity, normalized_mesh

    v, f = mesh.cylinder_mesh(radius=0.5, height=2.0, sections=16)
    path = os.path.join(tmp_path, "stick.obj")
    with open(path, "w") as fh:
        for q in v + np.array([3.0, 0.0, 1.0]):
            fh.write(f"v {q[0]} {q[1]} {q[2]}\n")
        for t in f:
            fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    morph = gs.morphs.Mesh(file=path, scale=0.6, pos=(0.5, 0.5, 0.2))
    nv, nf = normalized_mesh(morph)
    # centred on the bounding box and divided by its largest extent (2.0)
    assert np.allclose((nv.min(0) + nv.max(0)) / 2, 0, atol=1e-12)
    assert np.isclose((nv.max(0) - nv.min(0)).max(), 1.0)
    t = ToolEntity(None, 0, gs.materials.Tool(sdf_res=65), morph)
    assert np.allclose(t._sdf_scale, 64 / 1.2 / 0.6)
    assert np.allclose(t.vertices, nv * 0.6)
    with pytest.raises(gs.GenesisException):
        gs.materials.Tool(sdf_res=1)
