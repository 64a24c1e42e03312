"""Tool entities as kinematic colliders of the MPM grid op.

The reference's ToolEntity (genesis/engine/entities/tool_entity/tool_entity.py:19-460) is a
mesh moved by its own solver; its Mesh (tool_entity/mesh.py:10-176) normalises the mesh to
unit extent, samples its signed distance on a sdf_res^3 grid over [-0.6, 0.6]^3
(utils/mesh.py:179-201) and couples MPM grid nodes to it (legacy_coupler.py:346-350).  Here
the grid is computed on the device (mpm_sdf_voxelize), the tool is one mpm_collider row per
environment of kind MPM_COLLIDER_TOOL, and its pose advances in the grid op's collider pass:
pos += vel dt (kept above the floor height), quat = exp(ang dt) quat, as its advect
(tool_entity.py:178-191) does.  set_position / set_quaternion / set_velocity write the row
directly, which the reference does at the start of the next step (process_input).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _native as nat
from .. import morphs as _morphs
from ..exceptions import GenesisException
from .rigid import R_to_quat, quat_to_R

_POS, _ROT, _LIN, _ANG = slice(0, 3), slice(3, 12), slice(15, 18), slice(18, 21)
SDF_RADIUS = 0.6  # utils/mesh.py:183


class ToolEntityState:
    """pos [B, 3], quat [B, 4] (w-x-y-z), vel [B, 3], ang [B, 3] (states/entities.py: ToolEntityState)."""

    def __init__(self, entity, s_global, pos, quat, vel, ang):
        self._entity, self._s_global = entity, s_global
        self.pos, self.quat, self.vel, self.ang = pos, quat, vel, ang

    @property
    def entity(self):
        return self._entity

    @property
    def s_global(self):
        return self._s_global

    def serializable(self):
        self._entity = None
        self.pos, self.quat, self.vel, self.ang = (t.detach() for t in (self.pos, self.quat, self.vel, self.ang))


def normalized_mesh(morph):
    """tool_entity/mesh.py:39-51: the file's vertices centred on their bounding box and divided
    by its largest extent, and the faces."""
    sc = np.broadcast_to(np.asarray(morph.scale, dtype=np.float64), (3,))
    raw = np.asarray(morph.vertices, dtype=np.float64) / sc
    lo, hi = raw.min(0), raw.max(0)
    ext = float(np.max(hi - lo))
    if not ext > 0:
        raise GenesisException("Tool mesh is degenerate.")
    return (raw - (lo + hi) / 2) / ext, np.asarray(morph.faces, dtype=np.int32)


def sdf_voxels(vertices, faces, res, device, radius=SDF_RADIUS):
    """The signed-distance grid [res, res, res] of a mesh (mpm_sdf_voxelize), on the device."""
    lib = nat.load()
    v = torch.as_tensor(np.ascontiguousarray(vertices, dtype=np.float32), device=device)
    f = torch.as_tensor(np.ascontiguousarray(faces, dtype=np.int32), device=device)
    if f.numel() == 0 or f.min() < 0 or f.max() >= v.shape[0]:
        raise GenesisException("Tool mesh has faces that index no vertex.")
    out = torch.empty((res, res, res), dtype=torch.float32, device=device)
    from .runtime import _cuda_stream_handle

    nat.check("mpm_sdf_voxelize", lib.mpm_sdf_voxelize(
        C.c_void_p(v.data_ptr()), int(v.shape[0]), C.c_void_p(f.data_ptr()), int(f.shape[0]), int(res),
        C.c_float(radius), C.c_void_p(out.data_ptr()), _cuda_stream_handle()))
    return out


class ToolEntity:
    """A gs.materials.Tool entity with a Mesh morph (tool_entity.py:19-45)."""

    def __init__(self, scene, idx, material, morph, surface=None):
        if not isinstance(morph, _morphs.Mesh):
            raise GenesisException("Tool entities take a Mesh morph (tool_entity/mesh.py:23-37).")
        self._scene = scene
        self._idx = idx
        self._material = material
        self._morph = morph
        self._surface = surface
        self._init_pos = np.asarray(morph.pos, dtype=np.float64)
        self._init_quat = np.asarray(morph.quat, dtype=np.float64)
        self._norm_verts, self._faces = normalized_mesh(morph)
        sc = np.broadcast_to(np.asarray(morph.scale, dtype=np.float64), (3,))
        # T_mesh_to_sdf of mesh.py:32-34, 58-59: voxel = (res - 1) / (2 r) * p / scale + (res - 1) / 2
        self._sdf_scale = (material.sdf_res - 1) / (2 * SDF_RADIUS) / sc
        self._rows = None
        self._rt = None

    # ------------------------------------------------------------- build
    def _collider(self, env, sdf_offset, floor):
        c = nat.Collider()
        c.kind = nat.COLLIDER_TOOL
        c.instance = int(env)
        R = quat_to_R(self._init_quat)
        for d in range(3):
            c.pos[d] = float(self._init_pos[d])
            c.sdf_scale[d] = float(self._sdf_scale[d])
        for k in range(9):
            c.rot[k] = float(R.reshape(9)[k])
        c.friction, c.softness, c.restitution = self._material.friction, self._material.coup_softness, 0.0
        c.sdf_res = self._material.sdf_res if self._material.collision else 0  # 0: no coupling
        c.sdf_offset = int(sdf_offset)
        c.floor = float(floor)
        return c

    def _sdf(self, device):
        return sdf_voxels(self._norm_verts, self._faces, self._material.sdf_res, device)

    def _bind(self, runtime, rows):
        self._rt = runtime
        self._rows = torch.as_tensor(rows, dtype=torch.int64, device=runtime.device)

    def _check_built(self):
        if self._rt is None:
            raise GenesisException("Scene is not built yet.")

    def _sel(self, envs_idx=None):
        envs = self._scene._sanitize_envs_idx(envs_idx)
        return self._rows[envs.to(self._rows.device)]

    def _set_cols(self, cols, vals, envs_idx=None):
        self._check_built()
        rows = self._sel(envs_idx)
        v = torch.as_tensor(vals, dtype=torch.float32).detach().to(self._rt.device)
        v = v.reshape(-1, cols.stop - cols.start).expand(len(rows), -1)
        self._rt.collider_table()[rows, cols] = v

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

    @property
    def surface(self):
        return self._surface

    @property
    def init_pos(self):
        return self._init_pos

    @property
    def init_quat(self):
        return self._init_quat

    @property
    def vertices(self):
        """The normalised mesh scaled by the morph's scale (mesh.py:24-35), in the tool frame."""
        return self._norm_verts * np.broadcast_to(np.asarray(self._morph.scale, dtype=np.float64), (3,))

    @property
    def faces(self):
        return self._faces

    def _tape(self):
        solver = getattr(self._scene._sim, "mpm_solver", None)
        return getattr(solver, "tape", None)

    def set_position(self, pos):
        if self._tape() is not None:  # a differentiable scene: an input of the next step
            self._tape().record_input(self, "tool_pos", pos, None)
            return
        self._set_cols(_POS, pos)

    def _apply_input(self, kind, value):
        self._set_cols({"tool_pos": _POS, "tool_vel": _LIN, "tool_ang": _ANG}[kind], value)

    def _input_grad(self, shape, g):
        """dL/d(value) of a set_position / set_velocity input from dL/d(the rows it wrote) g
        [n_envs, 3] (a value given once for every environment gets their sum)."""
        with torch.enable_grad():
            a = torch.zeros(shape, dtype=torch.float32, device=g.device, requires_grad=True)
            out = a.reshape(-1, 3).expand(g.shape[0], 3)
            (ga,) = torch.autograd.grad(out, a, grad_outputs=g)
        return ga

    def set_quaternion(self, quat):
        q = np.asarray(torch.as_tensor(quat).detach().cpu(), dtype=np.float64).reshape(-1, 4)
        self._set_cols(_ROT, np.stack([quat_to_R(qq).reshape(9) for qq in q]))

    def set_velocity(self, vel=None, ang=None):
        tape = self._tape()
        if vel is not None:
            if tape is not None:
                tape.record_input(self, "tool_vel", vel, None)
            else:
                self._set_cols(_LIN, vel)
        if ang is not None:
            if tape is not None:
                tape.record_input(self, "tool_ang", ang, None)
            else:
                self._set_cols(_ANG, ang)

    def set_state(self, f, state):
        """Pose and velocities of every environment from a ToolEntityState (tool_entity.py:291-293)."""
        self._set_cols(_POS, state.pos.reshape(-1, 3))
        self.set_quaternion(state.quat)
        self._set_cols(_LIN, state.vel.reshape(-1, 3))
        self._set_cols(_ANG, state.ang.reshape(-1, 3))

    def get_state(self, f=None):
        self._check_built()
        t = self._rt.collider_table()[self._sel(None)]
        R = t[:, _ROT].detach().cpu().numpy().reshape(-1, 3, 3)
        quat = torch.as_tensor(np.stack([R_to_quat(r) for r in R]), dtype=torch.float32, device=t.device)
        return ToolEntityState(self, self._scene._sim.cur_step_global, t[:, _POS].clone(), quat, t[:, _LIN].clone(),
                               t[:, _ANG].clone())
