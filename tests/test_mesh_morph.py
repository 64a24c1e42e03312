"""gs.morphs.Mesh on the host: the OBJ reader, the inside test and the box-lattice sampler
(utils/particle.py:42-76, ``trimesh_to_particles_simple``).  No GPU."""

import numpy as np
import pytest

from genesis_b200 import mesh
from genesis_b200.exceptions import GenesisException
from genesis_b200.morphs import Box, Mesh


def _write_obj(path, v, f, quads=None):
    with open(path, "w") as fh:
        fh.write("# generated\no body\n")
        for p in v:
            fh.write(f"v {p[0]:.9f} {p[1]:.9f} {p[2]:.9f}\n")
        fh.write("vn 0 0 1\n")
        for t in f:
            fh.write("f " + " ".join(f"{i + 1}//1" for i in t) + "\n")
        for q in quads or []:
            fh.write("f " + " ".join(str(i - len(v)) for i in q) + "\n")  # negative indices


def _box_quads(size):
    """A box written as six quads (fanned into triangles by the reader)."""
    hx, hy, hz = np.asarray(size) / 2
    v = np.array([[x, y, z] for x in (-hx, hx) for y in (-hy, hy) for z in (-hz, hz)])
    q = [[0, 1, 3, 2], [4, 6, 7, 5], [0, 4, 5, 1], [2, 3, 7, 6], [0, 2, 6, 4], [1, 5, 7, 3]]
    return v, q


def test_obj_reader(tmp_path):
    v, q = _box_quads((0.2, 0.1, 0.3))
    p = tmp_path / "box.obj"
    _write_obj(p, v, [], quads=q)
    rv, rf = mesh.load_obj(str(p))
    assert np.allclose(rv, v) and rf.shape == (12, 3)
    with pytest.raises(ValueError):
        mesh.load_obj(str(_write_empty(tmp_path)))


def _write_empty(tmp_path):
    p = tmp_path / "empty.obj"
    p.write_text("# nothing\n")
    return p


def test_inside_exact_on_box_and_sphere():
    rng = np.random.default_rng(1)
    bv, bf = mesh.box_mesh((0.2, 0.1, 0.3))
    q = rng.uniform(-0.2, 0.2, size=(4000, 3))
    assert (mesh.points_inside(bv, bf, q) == (np.abs(q) < [0.1, 0.05, 0.15]).all(1)).all()
    sv, sf = mesh.icosphere(3, 0.1)
    p = rng.uniform(-0.12, 0.12, size=(8000, 3))
    r = np.linalg.norm(p, axis=1)
    ins = mesh.points_inside(sv, sf, p)
    # the icosphere lies between radius 0.1*cos(edge angle) and 0.1
    assert not ins[r > 0.1].any() and ins[r < 0.098].all()


def test_mesh_morph_matches_box_lattice(tmp_path):
    v, q = _box_quads((1.0, 1.0, 1.0))
    p = tmp_path / "unit.obj"
    _write_obj(p, v, [], quads=q)
    m = Mesh(file=str(p), scale=(0.2, 0.1, 0.3), pos=(0.5, 0.4, 0.3), euler=(0, 0, 30))
    b = Box(size=(0.2, 0.1, 0.3), pos=(0.5, 0.4, 0.3), euler=(0, 0, 30))
    pm, pb = m.sample(0.01, "regular"), b.sample(0.01, "regular")
    assert pm.shape == pb.shape
    assert np.allclose(np.sort(pm, axis=0), np.sort(pb, axis=0), atol=1e-12)


def test_mesh_morph_sphere_counts(tmp_path):
    sv, sf = mesh.icosphere(3, 1.0)
    p = tmp_path / "ball.obj"
    _write_obj(p, sv, sf)
    m = Mesh(file=str(p), scale=0.1, pos=(0.5, 0.5, 0.5))
    pts = m.sample(0.01, "regular")
    t = m.vertices[m.faces]
    vol = np.einsum("ij,ij->i", t[:, 0], np.cross(t[:, 1], t[:, 2])).sum() / 6.0  # enclosed volume
    size = np.ptp(m.vertices, axis=0)
    n = np.round(size / 0.01)
    cell = np.prod((size - 0.01) / (n - 1))  # the lattice spacing the sampler used per axis
    assert abs(len(pts) * cell / vol - 1.0) < 0.02
    assert (np.linalg.norm(pts - 0.5, axis=1) <= 0.1).all()
    rnd = m.sample(0.01, "random", rng=np.random.default_rng(0))
    expect = np.prod(n) * vol / np.prod(size)  # the bounds-box sample times the inside share
    assert abs(len(rnd) / expect - 1.0) < 0.05
    assert (np.linalg.norm(rnd - 0.5, axis=1) <= 0.1).all()
    pbs = m.sample(0.01, "pbs")
    assert pbs.shape == pts.shape


def test_mesh_morph_errors(tmp_path):
    with pytest.raises(GenesisException):
        Mesh(file=str(tmp_path / "missing.obj"))
    with pytest.raises(GenesisException):
        Mesh(file=str(tmp_path / "a.stl"))
    p = _write_empty(tmp_path)
    with pytest.raises(GenesisException):
        Mesh(file=str(p))


def test_cylinder_morph_and_mesh():
    from genesis_b200.morphs import Cylinder

    c = Cylinder(pos=(0.5, 0.5, 0.4), radius=0.1, height=0.2, euler=(90, 0, 0))
    pts = c.sample(0.01, "regular")
    # regular lattice of 20 x 20 x 20 cut to the disc: pi/4 of the columns
    assert abs(len(pts) / (20**3 * np.pi / 4) - 1.0) < 0.03
    R = np.array([[1, 0, 0], [0, 0, -1], [0, 1, 0]])  # 90 degrees about x
    local = (pts - [0.5, 0.5, 0.4]) @ R
    assert (np.linalg.norm(local[:, :2], axis=1) <= 0.1 + 1e-12).all() and (np.abs(local[:, 2]) < 0.1).all()
    v, f = mesh.cylinder_mesh(0.1, 0.2, sections=32)
    assert v.shape == (66, 3) and f.shape == (128, 3)
    n = np.cross(v[f][:, 1] - v[f][:, 0], v[f][:, 2] - v[f][:, 0])
    assert (np.einsum("ij,ij->i", n, v[f].mean(1)) > 0).all()  # outward winding
    q = np.random.default_rng(3).uniform(-0.12, 0.12, size=(3000, 3))
    ins = mesh.points_inside(v, f, q)
    r = np.linalg.norm(q[:, :2], axis=1)
    assert not ins[(r > 0.1) | (np.abs(q[:, 2]) > 0.1)].any()
    assert ins[(r < 0.1 * np.cos(np.pi / 32)) & (np.abs(q[:, 2]) < 0.1)].all()
    with pytest.raises(GenesisException):
        Cylinder(radius=0.0)


def test_mesh_set_samples_each_mesh_at_its_position(tmp_path):
    from genesis_b200.morphs import MeshSet

    v, q = _box_quads((1.0, 1.0, 1.0))
    a, b = tmp_path / "a.obj", tmp_path / "b.obj"
    _write_obj(a, v, [], quads=q)
    sv, sf = mesh.icosphere(2, 1.0)
    _write_obj(b, sv, sf)
    ms = MeshSet(files=[str(a), str(b)], poss=[(0.3, 0.5, 0.5), (0.7, 0.5, 0.5)], eulers=[(0, 0, 0), (0, 0, 45)],
                 scale=0.1)
    pts = ms.sample(0.01, "regular")
    g = ms.group_ids
    assert pts.shape[0] == g.shape[0] and set(g.tolist()) == {0, 1}
    assert np.allclose(pts[g == 0].mean(0), [0.3, 0.5, 0.5], atol=1e-9)  # 10^3 lattice of the cube
    assert (g == 0).sum() == 1000
    assert (np.linalg.norm(pts[g == 1] - [0.7, 0.5, 0.5], axis=1) <= 0.1).all()
    vv, vf = ms.visual_mesh()
    assert vv.shape[0] == 8 + len(sv) and vf.max() == vv.shape[0] - 1
    with pytest.raises(GenesisException):
        MeshSet(files=[str(a)], poss=[(0, 0, 0), (1, 1, 1)])
