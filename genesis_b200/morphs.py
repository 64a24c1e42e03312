"""gs.morphs used by MPM entities: Box, Sphere, Cylinder, Mesh and Nowhere.

Particle sampling follows the reference's simple samplers
(genesis/utils/particle.py:174-202, ``_box_to_particles``): 'regular' places
round(size / p_size) points per axis on [lower + p/2, upper - p/2]; 'random' draws
n_particles_3D uniform points.  The reference's default 'pbs' sampler runs an external
prebuilt executable that is not part of this build; 'pbs' requests are sampled as
'regular'.
"""

from __future__ import annotations

import numpy as np

from .exceptions import GenesisException


def _quat_to_R(q):
    w, x, y, z = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
            [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
            [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
        ]
    )


def _euler_to_quat(euler_deg):
    # scipy's extrinsic x-y-z convention (options/morphs.py docstring)
    rx, ry, rz = np.deg2rad(np.asarray(euler_deg, dtype=np.float64)) / 2
    cx, sx, cy, sy, cz, sz = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry), np.cos(rz), np.sin(rz)
    return np.array(
        [
            cx * cy * cz + sx * sy * sz,
            sx * cy * cz - cx * sy * sz,
            cx * sy * cz + sx * cy * sz,
            cx * cy * sz - sx * sy * cz,
        ]
    )


def n_particles_1D(p_size=0.01, length=1.0):
    return max(1, round(length / p_size))


def n_particles_3D(p_size=0.01, size=(1.0, 1.0, 1.0)):
    return n_particles_1D(p_size, size[0]) * n_particles_1D(p_size, size[1]) * n_particles_1D(p_size, size[2])


class Morph:
    def __init__(self, pos=(0.0, 0.0, 0.0), euler=(0.0, 0.0, 0.0), quat=None, visualization=True, collision=True,
                 **_ignored):
        self.pos = tuple(float(v) for v in pos)
        self.euler = tuple(euler)
        self.quat = tuple(quat) if quat is not None else tuple(_euler_to_quat(euler))
        self.visualization = visualization
        self.collision = collision

    def _local_particles(self, p_size, sampler, rng):
        raise NotImplementedError

    def sample(self, p_size, sampler, rng=None):
        rng = rng or np.random.default_rng()
        if sampler.startswith("pbs"):
            sampler = "regular"
        local = self._local_particles(p_size, sampler, rng)
        R = _quat_to_R(self.quat)
        return (local @ R.T + np.asarray(self.pos)).astype(np.float64)


class Box(Morph):
    """Axis-aligned box given by (pos, size) or (lower, upper); the latter wins."""

    def __init__(self, pos=(0.0, 0.0, 0.0), euler=(0.0, 0.0, 0.0), quat=None, lower=None, upper=None, size=None,
                 **kw):
        if lower is not None and upper is not None:
            lower = np.asarray(lower, dtype=np.float64)
            upper = np.asarray(upper, dtype=np.float64)
            if not np.all(upper >= lower):
                raise GenesisException("Invalid lower and upper corner.")
            pos = tuple((lower + upper) / 2)
            size = tuple(upper - lower)
        elif size is None:
            raise GenesisException("Either [`pos` and `size`] or [`lower` and `upper`] should be specified.")
        super().__init__(pos=pos, euler=euler, quat=quat, **kw)
        self.size = tuple(float(s) for s in size)
        self.lower = tuple(np.asarray(self.pos) - np.asarray(self.size) / 2)
        self.upper = tuple(np.asarray(self.pos) + np.asarray(self.size) / 2)

    def _local_particles(self, p_size, sampler, rng):
        size = np.asarray(self.size)
        lower, upper = -size / 2, size / 2
        if sampler == "random":
            n = n_particles_3D(p_size, size)
            return rng.uniform(low=lower, high=upper, size=(n, 3))
        if sampler == "regular":
            axes = []
            for d in range(3):
                n = n_particles_1D(p_size, size[d])
                axes.append(np.linspace(lower[d] + 0.5 * p_size, upper[d] - 0.5 * p_size, n))
            return np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
        raise GenesisException(f"Unsupported sampler method: {sampler}.")


class Sphere(Morph):
    def __init__(self, pos=(0.0, 0.0, 0.0), euler=(0.0, 0.0, 0.0), quat=None, radius=0.5, **kw):
        super().__init__(pos=pos, euler=euler, quat=quat, **kw)
        self.radius = float(radius)

    def _local_particles(self, p_size, sampler, rng):
        r = self.radius
        if sampler == "random":
            n = max(1, round(4.0 / 3.0 * np.pi * r**3 / p_size**3))
            d = rng.normal(size=(n, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            return d * (r * rng.uniform(size=(n, 1)) ** (1.0 / 3.0))
        n = n_particles_1D(p_size, 2 * r)
        ax = np.linspace(-r + 0.5 * p_size, r - 0.5 * p_size, n)
        g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
        return g[np.linalg.norm(g, axis=1) <= r]


class Cylinder(Morph):
    """Cylinder along the local z axis, centred on pos (options/morphs.py:278-343).  Sampled as
    the box [2r, 2r, h] cut to the points within r of the axis (utils/particle.py:225-246)."""

    def __init__(self, pos=(0.0, 0.0, 0.0), euler=(0.0, 0.0, 0.0), quat=None, height=1.0, radius=0.5, **kw):
        super().__init__(pos=pos, euler=euler, quat=quat, **kw)
        self.height = float(height)
        self.radius = float(radius)
        if self.height <= 0 or self.radius <= 0:
            raise GenesisException("Cylinder height and radius must be positive.")

    def _local_particles(self, p_size, sampler, rng):
        r, h = self.radius, self.height
        size = np.array([2 * r, 2 * r, h])
        if sampler == "random":
            pts = rng.uniform(low=-size / 2, high=size / 2, size=(n_particles_3D(p_size, size), 3))
        elif sampler == "regular":
            axes = [np.linspace(-size[d] / 2 + 0.5 * p_size, size[d] / 2 - 0.5 * p_size,
                                n_particles_1D(p_size, size[d])) for d in range(3)]
            pts = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
        else:
            raise GenesisException(f"Unsupported sampler method: {sampler}.")
        return pts[np.linalg.norm(pts[:, :2], axis=1) <= r]


class Nowhere(Morph):
    """Inactive particles parked far away, activated later by an emitter (options/morphs.py: Nowhere)."""

    def __init__(self, n_particles, **kw):
        super().__init__(**kw)
        if n_particles <= 0:
            raise GenesisException("n_particles must be positive.")
        self.n_particles = int(n_particles)

    def _local_particles(self, p_size, sampler, rng):
        return np.zeros((self.n_particles, 3))

    def sample(self, p_size, sampler, rng=None):
        # the reference parks them at gu.nowhere() (utils/geom.py:1703-1705)
        return np.tile(np.array([2333333.0, 6666666.0, 5201314.0]), (self.n_particles, 1))


class Mesh(Morph):
    """Morph loaded from a Wavefront OBJ file (options/morphs.py:603-760, ``Mesh``).

    The vertices are scaled in the file's frame, then rotated by ``quat``/``euler`` and moved
    to ``pos`` (engine/mesh.py:342, particle_entity.py:265-268).  Particles are sampled the
    way the reference's ``trimesh_to_particles_simple`` does (utils/particle.py:42-76): a
    box lattice over the scaled mesh's bounds, of which the points inside the closed mesh are
    kept; inside is an exact even-odd ray test here (the reference keeps points with a
    negative winding-number signed distance, which is the same set for a closed mesh).
    `convexify` and `decompose_object_error_threshold` choose a rigid entity's collision geom
    (engine/rigid.py); the other fields of the reference's Mesh that only matter to rigid
    bodies or to the renderer (decimate, coacd_options, group_by_material, ...) are accepted
    and ignored."""

    def __init__(self, file, scale=1.0, pos=(0.0, 0.0, 0.0), euler=(0.0, 0.0, 0.0), quat=None, convexify=None,
                 decompose_object_error_threshold=0.15, **kw):
        super().__init__(pos=pos, euler=euler, quat=quat, **kw)
        from . import mesh as _mesh

        # read by rigid entities (options/morphs.py:505-565): a collision geom is the mesh's
        # convex hull unless that is convexify=False or the hull's volume error is above the
        # threshold (the reference then decomposes the mesh into convex parts)
        self.convexify = convexify
        self.decompose_object_error_threshold = float(decompose_object_error_threshold)
        self.file = str(file)
        if not self.file.lower().endswith(".obj"):
            raise GenesisException(f"Unsupported mesh file (only .obj is read): {self.file}")
        try:
            v, f = _mesh.load_obj(self.file)
        except (OSError, ValueError) as e:
            raise GenesisException(f"Cannot load mesh {self.file}: {e}") from e
        sc = np.broadcast_to(np.asarray(scale, dtype=np.float64), (3,))
        if np.any(sc <= 0):
            raise GenesisException("Mesh scale must be positive.")
        self.scale = float(sc[0]) if np.all(sc == sc[0]) else tuple(float(x) for x in sc)
        self.vertices = v * sc  # local (scaled, untransformed) frame
        self.faces = f

    def _local_particles(self, p_size, sampler, rng):
        from . import mesh as _mesh

        lo, hi = self.vertices.min(0), self.vertices.max(0)
        size, center = hi - lo, (hi + lo) / 2
        if sampler == "random":
            pts = rng.uniform(low=lo, high=hi, size=(n_particles_3D(p_size, size), 3))
        elif sampler == "regular":
            axes = [np.linspace(center[d] - size[d] / 2 + 0.5 * p_size, center[d] + size[d] / 2 - 0.5 * p_size,
                                n_particles_1D(p_size, size[d])) for d in range(3)]
            pts = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
        else:
            raise GenesisException(f"Unsupported sampler method: {sampler}.")
        return pts[_mesh.points_inside(self.vertices, self.faces, pts)]


class MeshSet(Mesh):
    """Several OBJ meshes sampled into one entity (options/morphs.py:720-723).  As the
    reference's particle entity does (particle_entity.py:239-262), every mesh is scaled and
    sampled in its own frame and its particles are moved by its entry of `poss`; `eulers`
    orient only the visual meshes (particle_entity.py:280-286).  `group_ids` gives each
    particle the index of its mesh (the entity's mesh_set_group_ids)."""

    def __init__(self, files, poss=None, eulers=None, scale=1.0, **kw):
        files = list(files)
        if not files:
            raise GenesisException("MeshSet needs at least one file.")
        poss = [tuple(p) for p in (poss if poss is not None else [(0.0, 0.0, 0.0)] * len(files))]
        eulers = [tuple(e) for e in (eulers if eulers is not None else [(0.0, 0.0, 0.0)] * len(files))]
        if len(poss) != len(files) or len(eulers) != len(files):
            raise GenesisException("MeshSet: `files`, `poss` and `eulers` must have the same length.")
        super().__init__(file=files[0], scale=scale, **kw)
        self.files = [str(f) for f in files]
        self.poss, self.eulers = poss, eulers
        self.parts = [Mesh(file=f, scale=scale) for f in self.files]
        self.group_ids = np.zeros(0, dtype=np.int64)

    def sample(self, p_size, sampler, rng=None):
        rng = rng or np.random.default_rng()
        if sampler.startswith("pbs"):
            sampler = "regular"
        out, gid = [], []
        for i, (m, pos) in enumerate(zip(self.parts, self.poss)):
            pts = m._local_particles(p_size, sampler, rng) + np.asarray(pos, dtype=np.float64)
            out.append(pts)
            gid.append(np.full(len(pts), i, dtype=np.int64))
        self.group_ids = np.concatenate(gid)
        return np.concatenate(out).astype(np.float64)

    def visual_mesh(self):
        """The meshes placed by poss and eulers, concatenated (vertices, faces)."""
        vs, fs, off = [], [], 0
        for m, pos, eul in zip(self.parts, self.poss, self.eulers):
            R = _quat_to_R(_euler_to_quat(eul))
            vs.append(m.vertices @ R.T + np.asarray(pos, dtype=np.float64))
            fs.append(m.faces + off)
            off += len(m.vertices)
        return np.concatenate(vs), np.concatenate(fs)


class Plane(Morph):
    """Infinite plane through `pos` with `normal` in its local frame (options/morphs.py:409-470);
    only meaningful for rigid entities (a collider of the MPM grid op)."""

    def __init__(self, pos=(0.0, 0.0, 0.0), euler=(0.0, 0.0, 0.0), quat=None, normal=(0.0, 0.0, 1.0), fixed=True,
                 plane_size=(1e3, 1e3), **kw):
        super().__init__(pos=pos, euler=euler, quat=quat, **kw)
        n = np.asarray(normal, dtype=np.float64)
        if np.linalg.norm(n) < 1e-12:
            raise GenesisException("Plane normal must be non-zero.")
        self.normal = tuple(n / np.linalg.norm(n))
        self.fixed = fixed
        self.plane_size = tuple(plane_size)

    def _local_particles(self, p_size, sampler, rng):
        raise GenesisException("A Plane has no particles; use it with gs.materials.Rigid.")


__all__ = ["Morph", "Box", "Sphere", "Cylinder", "Mesh", "MeshSet", "Nowhere", "Plane"]
