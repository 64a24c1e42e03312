"""Visual meshes of the primitive morphs, used to skin MPM entities (the reference builds
them with trimesh: genesis/engine/mesh.py:369-381, utils/mesh.py:706-723, 823-880).

box_mesh: the 8 corners and 12 triangles of an axis-aligned box.
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
