"""The sampled signed-distance grid of a Box rigid geom (the grid the reference builds for
every geom that is not a sphere or a plane, rigid_geom.py:147-193, and looks up trilinearly,
utils/sdf_decomp.py:102-276), on the CPU: its layout follows the reference's formula, its
lookups stay within the interpolation error of the exact distance, and the numpy and C
restatements of the coupling agree through it."""

import numpy as np

from genesis_b200.engine.rigid import box_sd, box_sdf_grid
from oracle import cref
from oracle import mpm_ref as R


def test_grid_layout_follows_the_reference_formula():
    half = np.array([0.15, 0.15, 0.1])
    val, grad, scale, cell, vmax = box_sdf_grid(half)
    ext = 2 * half
    grid = ext.max() * 0.2 + ext  # rigid_geom.py:154
    c = np.float32(1.1920929e-07) + np.clip(0.005, grid.max() / 127, grid.min() / 31)  # :155-158
    res = np.ceil(grid / c).astype(int) + 1  # :160
    assert val.shape == tuple(res) and grad.shape == tuple(res) + (3,)
    assert np.isclose(cell, c) and np.allclose(scale, (res - 1) / ((res - 1) * c))
    assert np.isclose(vmax, val.max())
    # the corner node is outside the box: distance to the box's corner
    g = (res - 1) * c
    assert np.isclose(val[0, 0, 0], np.linalg.norm(g / 2 - half), atol=1e-6)


def test_lookup_stays_within_interpolation_error():
    half = np.array([0.15, 0.15, 0.1])
    val, grad, scale, cell, vmax = box_sdf_grid(half)
    col = R.Collider("sdf", np.zeros(3), np.eye(3), np.zeros(3), sdf=val, sdf_scale=scale, sdf_grad=grad, sdf_cell=cell,
                     sdf_max=vmax)
    rng = np.random.default_rng(0)
    inner = 0.5 * (np.array(val.shape) - 1) / scale * 0.99  # inside the grid (outside it: the proxy)
    p = rng.uniform(-inner, inner, size=(2000, 3))
    sd, g = R.sdf_sampled(col, p, 1e-12)
    exact = box_sd(p, half)
    assert np.abs(sd - exact).max() < 0.5 * cell  # trilinear of a piecewise-linear distance
    # outside the grid the reference's proxy keeps the distance large (no coupling there)
    far, _ = R.sdf_sampled(col, np.array([[0.0, 0.0, 0.5]]), 1e-12)
    assert far[0] > vmax
    near = np.abs(exact) < 0.02
    # near the surface, away from edges and from the interior's medial planes (where two faces
    # are about equally near), the gradient is the face normal
    dist = np.sort(np.abs(np.abs(p) - half), axis=1)
    sel = near & (dist[:, 1] - dist[:, 0] > 3 * cell)
    assert sel.sum() > 50
    assert (np.linalg.norm(g[sel], axis=1) > 0.98).all()  # (interpolated unit normals rotating near an edge: 0.99)


def test_numpy_and_c_restatements_agree_through_the_grid():
    half = np.array([0.15, 0.15, 0.1])
    val, grad, scale, cell, vmax = box_sdf_grid(half)
    Rm = np.array([[np.cos(0.2), 0, np.sin(0.2)], [0, 1, 0], [-np.sin(0.2), 0, np.cos(0.2)]])
    col = R.Collider("sdf", np.array([0.52, 0.5, 0.2]), Rm, np.zeros(3), friction=0.3, sdf=val, sdf_scale=scale,
                     sdf_grad=grad, sdf_cell=cell, sdf_max=vmax)
    rng = np.random.default_rng(1)
    n = 400
    x = np.stack([rng.uniform(0.45, 0.55, n), rng.uniform(0.45, 0.55, n), rng.uniform(0.31, 0.36, n)], 1)
    p = R.Params(grid_density=64, particle_size=0.01, dt=1e-4, dtype=np.float64)
    mats = [R.make_material("elastic", E=2e4)]
    st = R.make_state(x, mats, np.zeros(n, np.int64), np.float64, v=np.tile([0.0, 0.0, -2.0], (n, 1)))
    st["colliders"] = [col]
    c_out, rc = cref.substeps(p, mats, st, 30)
    assert rc == 0
    s2 = dict(st)
    s2["colliders"] = [col]
    forces = np.zeros((1, 6))
    for _ in range(30):
        s2 = R.substep(p, mats, s2)
    assert np.abs(c_out["x"] - s2["x"]).max() < 1e-10


def test_mesh_collision_geom_and_grid_layout():
    """A rigid Mesh's collision geom (utils/mesh.py:301-400 for an object): the convex hull,
    faces oriented outwards, for a convex mesh or with convexify on and a small hull error; the
    mesh itself with convexify=False or a hull error above decompose_object_error_threshold.
    And the sampling grid's layout (rigid_geom.py:147-170) for a mesh off its origin."""
    from genesis_b200 import mesh
    from genesis_b200.engine.rigid import collision_mesh, sdf_grid_layout

    class M:  # the fields collision_mesh reads from a gs.morphs.Mesh
        def __init__(self, v, f, convexify=None, thr=0.15):
            self.vertices, self.faces = v, f
            self.convexify, self.decompose_object_error_threshold = convexify, thr

    v, f = mesh.icosphere(subdivisions=2, radius=0.4)
    hv, hf = collision_mesh(M(v, f))
    assert len(hf) == len(f)  # convex: the hull has the same faces
    tv = hv[hf]
    assert (np.einsum("ij,ij->i", np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0]), tv[:, 0]) > 0).all()
    # an L-shaped (non-convex) prism: hull volume 4/3 of the mesh's
    bv, bf = mesh.box_mesh((1.0, 1.0, 1.0))
    L = np.concatenate([bv, bv + [1.0, 0.0, 0.0], bv + [0.0, 1.0, 0.0]])
    Lf = np.concatenate([bf, bf + 8, bf + 16])
    assert collision_mesh(M(L, Lf, convexify=False))[1] is Lf
    assert collision_mesh(M(L, Lf))[1] is Lf  # hull error ~0.5 > 0.15: not convexified
    assert len(collision_mesh(M(L, Lf, thr=1.0))[1]) != len(Lf)
    centre, res, cell, grid = sdf_grid_layout(np.array([0.1, 0.2, 0.3]), np.array([0.5, 0.4, 0.9]))
    assert np.allclose(centre, [0.3, 0.3, 0.6])
    ext = np.array([0.4, 0.2, 0.6])
    g0 = ext.max() * 0.2 + ext
    c = np.float32(np.finfo(np.float32).eps) + np.clip(0.005, g0.max() / 127, g0.min() / 31)
    assert np.isclose(cell, c) and np.array_equal(res, np.ceil(g0 / c).astype(int) + 1)
