"""Visual-vertex skinning set-up on the host (particle_entity.py:192-226) and the
primitive meshes it skins (utils/mesh.py): no GPU."""

import numpy as np

from genesis_b200 import mesh
from genesis_b200.engine.entity import skinning_supports
from genesis_b200.morphs import Box


def test_primitive_meshes():
    v, f = mesh.icosphere(3, radius=0.2)
    assert v.shape == (642, 3) and f.shape == (1280, 3)
    assert np.allclose(np.linalg.norm(v, axis=1), 0.2)
    v, f = mesh.box_mesh((0.1, 0.2, 0.3))
    assert v.shape == (8, 3) and f.shape == (12, 3)
    assert np.allclose(v.max(0), [0.05, 0.1, 0.15]) and np.allclose(v.min(0), [-0.05, -0.1, -0.15])
    n = np.cross(v[f][:, 1] - v[f][:, 0], v[f][:, 2] - v[f][:, 0])
    assert (np.einsum("ij,ij->i", n, v[f].mean(1)) > 0).all()  # outward winding


def test_supports_reproduce_vertices_and_affine_motion():
    b = Box(lower=(0.4, 0.4, 0.4), upper=(0.6, 0.6, 0.6))
    parts = b.sample(0.02, "regular")
    v, _ = mesh.box_mesh(b.size)
    v = v + np.asarray(b.pos)
    idx, w = skinning_supports(parts, v, 12)
    assert idx.shape == (8, 12) and w.shape == (8, 12)
    assert np.allclose(w.sum(1), 1.0, atol=1e-6)
    assert np.allclose(np.einsum("vk,vkd->vd", w, parts[idx]), v, atol=1e-6)
    # an affine map of the particles moves the vertices by the same map
    A = np.array([[1.1, 0.2, 0.0], [0.0, 0.9, 0.1], [0.05, 0.0, 1.0]])
    t = np.array([0.01, -0.02, 0.03])
    moved = parts @ A.T + t
    assert np.allclose(np.einsum("vk,vkd->vd", w, moved[idx]), v @ A.T + t, atol=1e-5)
