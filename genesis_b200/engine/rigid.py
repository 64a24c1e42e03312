"""Rigid entities as kinematic colliders of the MPM grid op.

The reference couples MPM grid nodes to rigid geoms inside mpm_grid_op
(genesis/engine/couplers/legacy_coupler.py:131-343, 385-397) and hands the momentum it
removes to its rigid-body solver.  This build has no rigid-body solver: a rigid entity's
pose and velocity are set by the caller (set_pos / set_quat / set_dofs_velocity), the
collider moves at that velocity over the substeps, and the reaction force and torque on
it are reported by get_coupling_force().  Sphere and Plane use the reference's analytic
signed distance.  A Box is coupled as the reference couples every other geom, through a
signed-distance grid sampled once at build (box_sdf_grid: the grid of rigid_geom.py:147-193,
trilinear lookups of distance and gradient in the grid op); B200Options(exact_box_sdf=True)
uses the exact box distance instead.  A Mesh is coupled the same way through the grid of its
collision geom (collision_mesh: its convex hull, or the mesh itself), sampled on the device
(mesh_sdf_grid).
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _native as nat
from .. import morphs as _morphs
from ..exceptions import GenesisException

# float32 columns of one mpm_collider row after its two int32 fields
_POS, _ROT, _DATA, _LIN, _ANG = slice(0, 3), slice(3, 12), slice(12, 15), slice(15, 18), slice(18, 21)


def box_sd(p, half):
    """Exact signed distance of points p [n, 3] to the box [-half, half] (negative inside)."""
    d = np.abs(p) - half
    return np.linalg.norm(np.maximum(d, 0.0), axis=1) + np.minimum(d.max(axis=1), 0.0)


def sdf_grid_layout(lower, upper, sdf_cell_size=0.005, sdf_min_res=32, sdf_max_res=128,
                    eps=float(np.finfo(np.float32).eps)):
    """The sampling grid the reference lays over a geom (rigid_geom.py:147-170): its vertex
    bounds' extent padded by 0.2 of the largest side, cell size sdf_cell_size clipped to
    [grid.max() / (sdf_max_res - 1), grid.min() / max(sdf_min_res - 1, 2)] plus gs.EPS,
    ceil(grid / cell) + 1 nodes per axis, centred on the bounds' centre.  Returns (centre,
    nodes per axis, cell size, grid size)."""
    lower, upper = np.asarray(lower, dtype=np.float64), np.asarray(upper, dtype=np.float64)
    centre = (upper + lower) / 2
    ext = upper - lower
    grid = ext.max() * 0.2 + ext
    cell = eps + np.clip(sdf_cell_size, grid.max() / (sdf_max_res - 1), grid.min() / max(sdf_min_res - 1, 2))
    res = np.ceil(grid / cell).astype(np.int64) + 1
    return centre, res, cell, (res - 1) * cell


def box_sdf_grid(half, sdf_cell_size=0.005, sdf_min_res=32, sdf_max_res=128, eps=float(np.finfo(np.float32).eps)):
    """The signed-distance grid the reference builds for a geom (rigid_geom.py:147-193), for a
    box mesh centred at its origin (sdf_grid_layout), the distance at every node (the box
    mesh's signed distance, which is the box's) and its central-difference gradient with a
    step of 1e-2 cell.  Returns (values [rx, ry, rz], gradients [rx, ry, rz, 3], voxel scale
    (res - 1) / grid size per axis, cell size, largest value), all float32."""
    half = np.asarray(half, dtype=np.float64)
    _, res, cell, grid = sdf_grid_layout(-half, half, sdf_cell_size, sdf_min_res, sdf_max_res, eps)
    axes = [np.linspace(-grid[d] / 2, grid[d] / 2, res[d]) for d in range(3)]
    pts = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    val = box_sd(pts, half)
    delta = cell * 1e-2
    grad = np.stack([(box_sd(pts + delta * e, half) - box_sd(pts - delta * e, half)) / (2 * delta) for e in np.eye(3)],
                    -1)
    shape = tuple(int(r) for r in res)
    return (val.reshape(shape).astype(np.float32), grad.reshape(shape + (3,)).astype(np.float32),
            ((res - 1) / grid).astype(np.float32), np.float32(cell), np.float32(val.max()))


def mesh_sdf_grid(vertices, faces, device, sdf_cell_size=0.005, sdf_min_res=32, sdf_max_res=128,
                  eps=float(np.finfo(np.float32).eps)):
    """The grid the reference samples for a mesh geom (rigid_geom.py:147-193): the layout of
    sdf_grid_layout over the vertices' bounds, the mesh's signed distance at every node
    (_compute_sd, :247-249, here mpm_sdf_grid on the device) and its central differences with a
    step of 1e-2 cell (_compute_sd_grad, :260-273: six more grids shifted by +-step).  Returns
    (values, gradients, voxel scale, cell size, largest value, grid centre) as box_sdf_grid,
    float32 numpy arrays."""
    import ctypes as C

    from .runtime import _cuda_stream_handle

    v = np.asarray(vertices, dtype=np.float64)
    centre, res, cell, grid = sdf_grid_layout(v.min(0), v.max(0), sdf_cell_size, sdf_min_res, sdf_max_res, eps)
    lib = nat.load()
    vt = torch.as_tensor(np.ascontiguousarray(v, dtype=np.float32), device=device)
    ft = torch.as_tensor(np.ascontiguousarray(faces, dtype=np.int32), device=device)
    if ft.numel() == 0 or ft.min() < 0 or ft.max() >= vt.shape[0]:
        raise GenesisException("Rigid mesh has faces that index no vertex.")
    n = int(np.prod(res))
    lower = centre - grid / 2
    delta = cell * 1e-2

    def sample(origin):
        out = torch.empty(n, dtype=torch.float32, device=device)
        o = (C.c_float * 3)(*[float(x) for x in origin])
        st = (C.c_float * 3)(*[float(cell)] * 3)
        r = (C.c_int32 * 3)(*[int(x) for x in res])
        nat.check("mpm_sdf_grid", lib.mpm_sdf_grid(C.c_void_p(vt.data_ptr()), int(vt.shape[0]),
                                                   C.c_void_p(ft.data_ptr()), int(ft.shape[0]), o, st, r,
                                                   C.c_void_p(out.data_ptr()), _cuda_stream_handle()))
        return out

    val = sample(lower)
    grad = torch.stack([(sample(lower + delta * e) - sample(lower - delta * e)) / (2 * delta) for e in np.eye(3)], -1)
    shape = tuple(int(r) for r in res)
    val_np = val.reshape(shape).cpu().numpy()
    return (val_np, grad.reshape(shape + (3,)).cpu().numpy(), ((res - 1) / grid).astype(np.float32),
            np.float32(cell), np.float32(val_np.max()), centre.astype(np.float32))


def collision_mesh(morph):
    """The geom a rigid Mesh entity collides with (utils/mesh.py:301-400 for an object): the
    convex hull of its (scaled) mesh when convexify is on (the default) and the hull's volume
    exceeds the mesh's by at most decompose_object_error_threshold; otherwise the mesh itself
    (the reference decomposes such a mesh into convex parts whose union approximates it)."""
    v, f = np.asarray(morph.vertices, dtype=np.float64), np.asarray(morph.faces, dtype=np.int64)
    if morph.convexify is False:
        return v, f
    from scipy.spatial import ConvexHull

    hull = ConvexHull(v)
    tv = v[f]
    vol = abs(np.einsum("ij,ij->i", tv[:, 0], np.cross(tv[:, 1], tv[:, 2])).sum()) / 6.0
    if vol > 0 and hull.volume / vol - 1.0 > morph.decompose_object_error_threshold:
        return v, f
    hf = hull.simplices.copy()
    c = v[hull.vertices].mean(0)  # orient every hull face outwards
    nrm = np.cross(v[hf[:, 1]] - v[hf[:, 0]], v[hf[:, 2]] - v[hf[:, 0]])
    flip = np.einsum("ij,ij->i", nrm, v[hf[:, 0]] - c) < 0
    hf[flip] = hf[flip][:, [0, 2, 1]]
    return v, hf


def quat_to_R(q):
    return _morphs._quat_to_R(np.asarray(q, dtype=np.float64))


def R_to_quat(R):
    """w-x-y-z quaternion of a rotation matrix (Shepperd's method)."""
    R = np.asarray(R, dtype=np.float64)
    tr = np.trace(R)
    if tr > 0:
        s = np.sqrt(tr + 1.0) * 2
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = np.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2]) * 2
        q = [(R[2, 1] - R[1, 2]) / s, 0.25 * s, (R[0, 1] + R[1, 0]) / s, (R[0, 2] + R[2, 0]) / s]
    elif R[1, 1] > R[2, 2]:
        s = np.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2]) * 2
        q = [(R[0, 2] - R[2, 0]) / s, (R[0, 1] + R[1, 0]) / s, 0.25 * s, (R[1, 2] + R[2, 1]) / s]
    else:
        s = np.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1]) * 2
        q = [(R[1, 0] - R[0, 1]) / s, (R[0, 2] + R[2, 0]) / s, (R[1, 2] + R[2, 1]) / s, 0.25 * s]
    q = np.asarray(q)
    return q / np.linalg.norm(q) * (1 if q[0] >= 0 else -1)


class KinematicRigidEntity:
    """A gs.materials.Rigid entity with a Box, Sphere, Plane or Mesh morph."""

    def __init__(self, scene, idx, material, morph, exact_box_sdf=False):
        self._grid = None
        self._mesh = None
        if isinstance(morph, _morphs.Sphere):
            kind, data = nat.COLLIDER_SPHERE, (morph.radius, 0.0, 0.0)
        elif isinstance(morph, _morphs.Plane):
            kind, data = nat.COLLIDER_PLANE, morph.normal
        elif isinstance(morph, _morphs.Box):
            half = tuple(np.asarray(morph.size) / 2)
            if exact_box_sdf:
                kind, data = nat.COLLIDER_BOX, half
            else:
                self._grid = box_sdf_grid(half, material.sdf_cell_size, material.sdf_min_res, material.sdf_max_res)
                kind, data = nat.COLLIDER_SDF, (0.0, 0.0, 0.0)  # the grid's centre: the box's
        elif isinstance(morph, _morphs.Mesh) and not isinstance(morph, _morphs.MeshSet):
            # sampled at build, on the device (mesh_sdf_grid); data: the grid's centre
            self._mesh = collision_mesh(morph)
            kind, data = nat.COLLIDER_SDF, (0.0, 0.0, 0.0)
        else:
            raise GenesisException("Rigid entities on this path take a Box, Sphere, Plane or Mesh morph.")
        self._scene = scene
        self._idx = idx
        self._material = material
        self._morph = morph
        self._kind = kind
        self._data = np.asarray(data, dtype=np.float64)
        self._rows = None  # collider rows in the runtime table, one per environment
        self._rt = None

    # ------------------------------------------------------------- build
    def _sdf(self, device):
        """The sampled grid's values then gradients, flattened (None for analytic geoms)."""
        if self._mesh is not None and self._grid is None:
            m = self._material
            *grid, centre = mesh_sdf_grid(self._mesh[0], self._mesh[1], device, m.sdf_cell_size, m.sdf_min_res,
                                          m.sdf_max_res)
            self._grid = tuple(grid)
            self._data = np.asarray(centre, dtype=np.float64)
        if self._grid is None:
            return None
        val, grad = self._grid[0], self._grid[1]
        return torch.as_tensor(np.concatenate([val.reshape(-1), grad.reshape(-1)]), device=device)

    def _collider(self, env, sdf_offset=0):
        c = nat.Collider()
        c.kind = self._kind
        c.instance = int(env)
        if self._grid is not None:
            val, _, scale, cell, vmax = self._grid
            for d in range(3):
                c.sdf_res3[d] = int(val.shape[d])
                c.sdf_scale[d] = float(scale[d])
            c.sdf_offset = int(sdf_offset)
            c.sdf_cell = float(cell)
            c.sdf_max = float(vmax)
        R = quat_to_R(self._morph.quat)
        for d in range(3):
            c.pos[d] = float(self._morph.pos[d])
            c.data[d] = float(self._data[d])
        for k in range(9):
            c.rot[k] = float(R.reshape(9)[k])
        m = self._material
        c.friction, c.softness, c.restitution = m.coup_friction, m.coup_softness, m.coup_restitution
        return c

    def _bind(self, runtime, rows):
        self._rt = runtime
        self._rows = torch.as_tensor(rows, dtype=torch.int64, device=runtime.device)

    def _check_built(self):
        if self._rt is None:
            raise GenesisException("Scene is not built yet.")

    def _sel(self, envs_idx):
        envs = self._scene._sanitize_envs_idx(envs_idx)
        return self._rows[envs.to(self._rows.device)]

    def _set_cols(self, cols, vals, envs_idx):
        self._check_built()
        rows = self._sel(envs_idx)
        v = torch.as_tensor(np.asarray(vals, dtype=np.float32), device=self._rt.device)
        v = v.reshape(-1, cols.stop - cols.start).expand(len(rows), -1)
        self._rt.collider_table()[rows, cols] = v

    def _get_cols(self, cols, envs_idx):
        self._check_built()
        t = self._rt.collider_table()[self._sel(envs_idx), cols]
        return t[0] if self._scene.n_envs == 0 else t

    # ------------------------------------------------------------- API
    @property
    def idx(self):
        return self._idx

    @property
    def material(self):
        return self._material

    @property
    def morph(self):
        return self._morph

    def set_pos(self, pos, envs_idx=None):
        self._set_cols(_POS, pos, envs_idx)

    def get_pos(self, envs_idx=None):
        return self._get_cols(_POS, envs_idx)

    def set_quat(self, quat, envs_idx=None):
        q = np.asarray(quat, dtype=np.float64).reshape(-1, 4)
        self._set_cols(_ROT, np.stack([quat_to_R(qq).reshape(9) for qq in q]), envs_idx)

    def get_quat(self, envs_idx=None):
        R = self._get_cols(_ROT, envs_idx).cpu().numpy().reshape(-1, 3, 3)
        q = torch.as_tensor(np.stack([R_to_quat(r) for r in R]), dtype=torch.float32)
        return q[0] if self._scene.n_envs == 0 else q

    def set_dofs_velocity(self, velocity, dofs_idx_local=None, envs_idx=None):
        """Velocity of the free base: linear (3) then angular (3), both in the world frame."""
        v = np.asarray(velocity, dtype=np.float64).reshape(-1, 6)
        if dofs_idx_local is not None:
            raise GenesisException("dofs_idx_local is not supported for kinematic colliders.")
        self._set_cols(_LIN, v[:, :3], envs_idx)
        self._set_cols(_ANG, v[:, 3:], envs_idx)

    def get_dofs_velocity(self, envs_idx=None):
        return torch.cat([self._get_cols(_LIN, envs_idx), self._get_cols(_ANG, envs_idx)], dim=-1)

    def get_coupling_force(self, envs_idx=None):
        """Mean force (3) and torque about the origin (3) that the MPM material exerted on
        this collider over the last step, [6] or [n_envs, 6]."""
        self._check_built()
        t = self._rt.collider_force[self._sel(envs_idx)] / max(1, self._rt.last_step_substeps)
        return t[0] if self._scene.n_envs == 0 else t
