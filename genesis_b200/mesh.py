"""Visual meshes of the primitive morphs, used to skin MPM entities (the reference builds
them with trimesh: genesis/engine/mesh.py:369-381, utils/mesh.py:706-723, 823-880).

box_mesh: the 8 corners and 12 triangles of an axis-aligned box.
cylinder_mesh: a closed polygonal cylinder along z (trimesh.creation.cylinder's layout).
icosphere: the unit icosahedron with every triangle split into four `subdivisions`
times and the new vertices pushed onto the sphere (subdivisions=3: 642 vertices,
1280 faces, as trimesh.creation.icosphere gives).
"""

from __future__ import annotations

import numpy as np


def box_mesh(size):
    h = np.asarray(size, dtype=np.float64) / 2
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], dtype=np.float64) * h
    # corners indexed by (x, y, z) bits: 4x + 2y + z
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    f = []
    for a, b, c, d in quads:
        f += [(a, b, c), (a, c, d)]
    return v, np.asarray(f, dtype=np.int64)


def icosphere(subdivisions=3, radius=1.0):
    t = (1.0 + 5.0**0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.asarray(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    for _ in range(int(subdivisions)):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.asarray(verts) * radius, np.asarray(f, dtype=np.int64)


def cylinder_mesh(radius=0.5, height=1.0, sections=32):
    """Closed cylinder along z centred on the origin: `sections` vertices per rim plus the
    two cap centres (2 * sections + 2 vertices, 4 * sections outward-wound triangles)."""
    a = 2.0 * np.pi * np.arange(sections) / sections
    ring = np.stack([radius * np.cos(a), radius * np.sin(a)], 1)
    h = height / 2.0
    v = np.concatenate([np.c_[ring, np.full(sections, -h)], np.c_[ring, np.full(sections, h)],
                        [[0.0, 0.0, -h], [0.0, 0.0, h]]])
    lo, hi = 2 * sections, 2 * sections + 1
    f = []
    for i in range(sections):
        j = (i + 1) % sections
        f += [(i, j, sections + j), (i, sections + j, sections + i), (lo, j, i), (hi, sections + i, sections + j)]
    return v, np.asarray(f, dtype=np.int64)


# ---------------------------------------------------------------- mesh files

def load_obj(path):
    """Vertices [V, 3] and triangles [F, 3] of a Wavefront OBJ file ('v' and 'f' records;
    polygons are fanned into triangles, 'f' indices may carry /vt/vn and be negative)."""
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v" and len(parts) >= 4:
                verts.append([float(parts[1]), float(parts[2]), float(parts[3])])
            elif parts[0] == "f" and len(parts) >= 4:
                idx = []
                for tok in parts[1:]:
                    i = int(tok.split("/")[0])
                    idx.append(i - 1 if i > 0 else len(verts) + i)
                for k in range(1, len(idx) - 1):
                    faces.append([idx[0], idx[k], idx[k + 1]])
    if not verts or not faces:
        raise ValueError(f"{path}: no vertices or faces")
    return np.asarray(verts, dtype=np.float64), np.asarray(faces, dtype=np.int64)


def _ray_crossings(tri, oy, oz):
    """x of the crossings of the lines {(t, oy[r], oz[r])} with the triangles tri [T, 3, 3]:
    a list of sorted arrays, one per line.  Triangles are binned by their y-z bounding box
    on a coarse grid so each line is tested only against the triangles of its cell."""
    y0, z0 = tri[:, :, 1], tri[:, :, 2]
    lo = np.array([min(y0.min(), oy.min()), min(z0.min(), oz.min())])
    hi = np.array([max(y0.max(), oy.max()), max(z0.max(), oz.max())])
    G = int(np.clip(np.sqrt(len(tri)) / 2, 1, 128))
    cell = (hi - lo) / G + 1e-12
    tminy = np.floor((y0.min(1) - lo[0]) / cell[0]).astype(int).clip(0, G - 1)
    tmaxy = np.floor((y0.max(1) - lo[0]) / cell[0]).astype(int).clip(0, G - 1)
    tminz = np.floor((z0.min(1) - lo[1]) / cell[1]).astype(int).clip(0, G - 1)
    tmaxz = np.floor((z0.max(1) - lo[1]) / cell[1]).astype(int).clip(0, G - 1)
    buckets = [[[] for _ in range(G)] for _ in range(G)]
    for t in range(len(tri)):
        for a in range(tminy[t], tmaxy[t] + 1):
            for b in range(tminz[t], tmaxz[t] + 1):
                buckets[a][b].append(t)
    ly = np.floor((oy - lo[0]) / cell[0]).astype(int).clip(0, G - 1)
    lz = np.floor((oz - lo[1]) / cell[1]).astype(int).clip(0, G - 1)
    out = [None] * len(oy)
    key = ly * G + lz
    for k in np.unique(key):
        rays = np.nonzero(key == k)[0]
        ts = buckets[k // G][k % G]
        if not ts:
            for r in rays:
                out[r] = np.zeros(0)
            continue
        T = tri[ts]  # [t, 3, 3]
        a, b, c = T[:, 0], T[:, 1], T[:, 2]
        # 2-D barycentrics of (oy, oz) in the y-z projection of each triangle
        d = (b[:, 1] - a[:, 1]) * (c[:, 2] - a[:, 2]) - (c[:, 1] - a[:, 1]) * (b[:, 2] - a[:, 2])
        py = oy[rays][:, None] - a[None, :, 1]
        pz = oz[rays][:, None] - a[None, :, 2]
        dd = np.where(d == 0, 1.0, d)[None, :]  # triangles seen edge-on never count as hit
        u = (py * (c[None, :, 2] - a[None, :, 2]) - (c[None, :, 1] - a[None, :, 1]) * pz) / dd
        v = ((b[None, :, 1] - a[None, :, 1]) * pz - py * (b[None, :, 2] - a[None, :, 2])) / dd
        hit = (d[None, :] != 0) & (u >= 0) & (v >= 0) & (u + v <= 1)
        x = a[None, :, 0] + u * (b[None, :, 0] - a[None, :, 0]) + v * (c[None, :, 0] - a[None, :, 0])
        for i, r in enumerate(rays):
            out[r] = np.sort(x[i][hit[i]])
    return out


def points_inside(verts, faces, pts):
    """Even-odd ray test (rays along +x) of points against a closed triangle mesh.  The rays
    are shifted by an irrational sub-tolerance offset so none passes exactly through an
    edge or a vertex."""
    tri = np.asarray(verts, dtype=np.float64)[np.asarray(faces)]
    ext = float(np.ptp(verts, axis=0).max()) or 1.0
    oy = pts[:, 1] + 1e-9 * ext * np.sqrt(2.0)
    oz = pts[:, 2] + 1e-9 * ext * np.sqrt(3.0)
    # points sharing a ray (a regular lattice) are tested once per ray
    keys, inv = np.unique(np.stack([oy, oz], 1), axis=0, return_inverse=True)
    xs = _ray_crossings(tri, keys[:, 0], keys[:, 1])
    inside = np.zeros(len(pts), dtype=bool)
    inv = np.asarray(inv).reshape(-1)
    order = np.argsort(inv, kind="stable")
    starts = np.searchsorted(inv[order], np.arange(len(keys) + 1))
    for r, x in enumerate(xs):
        sel = order[starts[r]:starts[r + 1]]
        n_after = len(x) - np.searchsorted(x, pts[sel, 0], side="right")
        inside[sel] = (n_after % 2) == 1
    return inside
