"""Test infrastructure (oracle): numpy restatement of the tool signed-distance grid.

compute_sdf_data (genesis/utils/mesh.py:179-201) samples igl.signed_distance of the
normalised tool mesh at a res^3 lattice over [-0.6, 0.6]^3.  libigl is not available here;
its published algorithm for a closed mesh is restated: the distance to the nearest triangle
(closest point by Voronoi region, Ericson, Real-Time Collision Detection 5.1.5) and the sign
of the generalised winding number (Jacobson et al. 2013; solid angles by Van Oosterom &
Strackee 1983), negative inside.  Float64, vectorised over the query points, one triangle
at a time: for small grids only.
"""

from __future__ import annotations

import numpy as np


def lattice(res, radius=0.6):
    x = np.linspace(-radius, radius, res)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    return np.stack([X, Y, Z], -1).reshape(-1, 3)


def _tri_dist2(p, a, b, c):
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ap @ ab, ap @ ac
    bp, cp = p - b, p - c
    d3, d4 = bp @ ab, bp @ ac
    d5, d6 = cp @ ab, cp @ ac
    vc = d1 * d4 - d3 * d2
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    with np.errstate(divide="ignore", invalid="ignore"):
        den = va + vb + vc
        q = a + np.outer(vb / den, ab) + np.outer(vc / den, ac)  # interior
        t_bc = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        q = np.where(((va <= 0) & (d4 - d3 >= 0) & (d5 - d6 >= 0))[:, None], b + np.outer(t_bc, c - b), q)
        t_ac = d2 / (d2 - d6)
        q = np.where(((vb <= 0) & (d2 >= 0) & (d6 <= 0))[:, None], a + np.outer(t_ac, ac), q)
        t_ab = d1 / (d1 - d3)
        q = np.where(((vc <= 0) & (d1 >= 0) & (d3 <= 0))[:, None], a + np.outer(t_ab, ab), q)
    q = np.where(((d6 >= 0) & (d5 <= d6))[:, None], c, q)
    q = np.where(((d3 >= 0) & (d4 <= d3))[:, None], b, q)
    q = np.where(((d1 <= 0) & (d2 <= 0))[:, None], a, q)
    return ((p - q) ** 2).sum(1)


def _solid_angle(p, a, b, c):
    ra, rb, rc = a - p, b - p, c - p
    la, lb, lc = (np.linalg.norm(r, axis=1) for r in (ra, rb, rc))
    det = np.einsum("ij,ij->i", ra, np.cross(rb, rc))
    den = la * lb * lc + (ra * rb).sum(1) * lc + (ra * rc).sum(1) * lb + (rb * rc).sum(1) * la
    return 2 * np.arctan2(det, den)


def signed_distance(points, vertices, faces):
    p = np.asarray(points, dtype=np.float64)
    V = np.asarray(vertices, dtype=np.float64)
    d2 = np.full(len(p), np.inf)
    w = np.zeros(len(p))
    for f in np.asarray(faces):
        a, b, c = V[f[0]], V[f[1]], V[f[2]]
        d2 = np.minimum(d2, _tri_dist2(p, a, b, c))
        w += _solid_angle(p, a, b, c)
    w /= 4 * np.pi
    return np.where(np.abs(w) > 0.5, -1.0, 1.0) * np.sqrt(d2)


def sdf_voxels(vertices, faces, res, radius=0.6):
    """[res, res, res] signed distances at the lattice of compute_sdf_data."""
    return signed_distance(lattice(res, radius), vertices, faces).reshape(res, res, res)
