"""MPMEntity: particle sampling and per-entity state I/O
(genesis/engine/entities/mpm_entity.py, particle_entity.py)."""

from __future__ import annotations

import uuid

import numpy as np
import torch

from .. import morphs as _morphs
from ..exceptions import GenesisException
from .states import MPMEntityState


def _as_tensor(x, dtype, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype)
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=device)


def skinning_supports(particles, vverts, K):
    """particle_entity.py:192-226: the K nearest particles of each visual vertex, and
    weights b with sum 1 that reproduce the vertex from them, b[:-1] = pinv(P) (v - p_K)
    where the columns of P are p_j - p_K.  Returns (local indices int32 [V, K], weights
    float32 [V, K])."""
    from scipy.spatial import cKDTree

    particles = np.asarray(particles, dtype=np.float64)
    _, idx = cKDTree(particles).query(vverts, k=K)
    idx = np.clip(np.asarray(idx).reshape(len(vverts), K), 0, len(particles) - 1)
    ps = particles[idx]
    P = np.swapaxes(ps[:, :-1], -2, -1) - ps[:, -1][..., None]
    b = np.einsum("vij,vj->vi", np.linalg.pinv(P), vverts - ps[:, -1])
    w = np.concatenate([b, 1.0 - b.sum(axis=1, keepdims=True)], axis=1)
    return idx.astype(np.int32), w.astype(np.float32)


class MPMEntity:
    def __init__(self, scene, solver, material, morph, surface, particle_size, idx, particle_start, rng=None):
        self._scene = scene
        self._solver = solver
        self._sim = solver.sim
        self._material = material
        self._morph = morph
        self._surface = surface
        self._particle_size = particle_size
        self._idx = idx
        self._uid = uuid.uuid4().hex[:7]
        self._particle_start = particle_start
        sampler = material.sampler
        self.sampler = sampler
        self._particles = np.asarray(morph.sample(particle_size, sampler, rng), dtype=np.float64)
        if self._particles.size == 0:
            raise GenesisException("Entity has zero particles.")
        self.active = not isinstance(morph, _morphs.Nowhere)
        if self.active and not solver.boundary.is_inside(self._particles):
            # particle_entity.py:330-336
            raise GenesisException(
                "Entity has particles outside solver boundary. Note that for MPMSolver, boundary is slightly "
                "tighter than the specified domain due to safety padding.\n\n"
                f"Current boundary:\n{solver.boundary}\n\nEntity to be added:\nmin: {self._particles.min(0)}\n"
                f"max: {self._particles.max(0)}\n"
            )
        self._n_particles = len(self._particles)
        self._init_skinning(scene)
        origin = np.asarray(morph.pos, dtype=np.float64)
        self._init_particles_offset = self._particles - origin
        self._tgt = {"pos": None, "vel": None, "act": None, "actu": None}

    # ------------------------------------------------------------ skinning
    def _init_skinning(self, scene):
        """Visual vertices of the morph's mesh, each a fixed affine combination of nearby
        particles (mpm_entity.py:55-57, particle_entity.py:192-226): Liquid, Sand and Snow
        are not skinned, nor are Nowhere entities (no mesh)."""
        from .. import mesh as _mesh
        from ..materials import MPM

        self._vverts = np.zeros((0, 3))
        self._vfaces = np.zeros((0, 3), dtype=np.int64)
        self._support_idx = np.zeros((0, 0), dtype=np.int32)
        self._support_w = np.zeros((0, 0), dtype=np.float32)
        skinned = not isinstance(self._material, (MPM.Liquid, MPM.Sand, MPM.Snow))
        if not skinned or isinstance(self._morph, _morphs.Nowhere):
            return
        if isinstance(self._morph, _morphs.Box):
            v, f = _mesh.box_mesh(self._morph.size)
        elif isinstance(self._morph, _morphs.Sphere):
            v, f = _mesh.icosphere(3, self._morph.radius)
        elif isinstance(self._morph, _morphs.Cylinder):
            v, f = _mesh.cylinder_mesh(self._morph.radius, self._morph.height)
        elif isinstance(self._morph, _morphs.MeshSet):
            v, f = self._morph.visual_mesh()  # already placed
            self._vverts, self._vfaces = v, f
            K = int(getattr(getattr(scene, "vis_options", None), "n_support_neighbors", 12))
            self._support_idx, self._support_w = skinning_supports(self._particles, self._vverts, K)
            return
        elif isinstance(self._morph, _morphs.Mesh):
            v, f = self._morph.vertices, self._morph.faces
        else:
            return
        R = _morphs._quat_to_R(self._morph.quat)
        self._vverts = v @ R.T + np.asarray(self._morph.pos, dtype=np.float64)
        self._vfaces = f
        K = int(getattr(getattr(scene, "vis_options", None), "n_support_neighbors", 12))
        self._support_idx, self._support_w = skinning_supports(self._particles, self._vverts, K)

    @property
    def mesh_set_group_ids(self):
        """For a MeshSet entity, the index of the mesh each particle came from."""
        return getattr(self._morph, "group_ids", None)

    @property
    def vverts(self):
        """Visual vertices at build time, [n_vverts, 3]."""
        return self._vverts

    @property
    def vfaces(self):
        return self._vfaces

    @property
    def n_vfaces(self):
        return len(self._vfaces)

    def _v_offsets(self):
        """(first visual vertex, first visual face) of this entity in the solver's
        concatenation of the entities' visual meshes, in the order they were added."""
        vv = vf = 0
        for e in self._solver.entities:
            if e is self:
                return vv, vf
            vv += e.n_vverts
            vf += e.n_vfaces
        return vv, vf

    @property
    def vvert_start(self):
        return self._v_offsets()[0]

    @property
    def vvert_end(self):
        return self.vvert_start + self.n_vverts

    @property
    def vface_start(self):
        return self._v_offsets()[1]

    @property
    def vface_end(self):
        return self.vface_start + self.n_vfaces

    @property
    def n_vverts(self):
        return len(self._vverts)

    # ------------------------------------------------------------ properties
    @property
    def scene(self):
        return self._scene

    @property
    def sim(self):
        return self._sim

    @property
    def solver(self):
        return self._solver

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
    def idx(self):
        return self._idx

    @property
    def uid(self):
        return self._uid

    @property
    def n_particles(self):
        return self._n_particles

    @property
    def particle_start(self):
        return self._particle_start

    @property
    def particle_end(self):
        return self._particle_start + self._n_particles

    @property
    def particle_size(self):
        return self._particle_size

    @property
    def init_particles(self):
        return self._particles

    @property
    def is_built(self):
        return self._scene.is_built

    # ---------------------------------------------------------------- helpers
    def _envs(self, envs_idx):
        return self._scene._sanitize_envs_idx(envs_idx)

    def _flat_idx(self, particles_idx_local, envs_idx):
        """Runtime (flattened over environments) indices, shape (M, K)."""
        envs = self._envs(envs_idx)
        N = self._solver.n_particles
        dev = self._solver.device
        if particles_idx_local is None:
            local = torch.arange(self._n_particles, device=dev).expand(len(envs), -1)
        else:
            local = _as_tensor(particles_idx_local, torch.int64, dev)
            if local.ndim == 1:
                local = local.expand(len(envs), -1)
            if (local < 0).any() or (local >= self._n_particles).any():
                raise GenesisException("particle index out of range for this entity.")
        return envs[:, None] * N + self._particle_start + local

    def _values(self, vals, shape_tail, n_envs, n_p, dtype):
        t = _as_tensor(vals, dtype, self._solver.device)
        t = t.reshape((-1,) + tuple(shape_tail)) if t.ndim == len(shape_tail) else t
        return t.expand((n_envs, n_p) + tuple(shape_tail)).reshape((-1,) + tuple(shape_tail)).contiguous()

    def _check_built(self):
        if not self._scene.is_built:
            raise GenesisException("Scene is not built yet.")

    # --------------------------------------------------------------- setters
    def set_particles_pos(self, poss, particles_idx_local=None, envs_idx=None):
        """Set positions; also resets v=0, F=I, C=0, Jp=default_Jp (mpm_solver.py:804-822)."""
        self._check_built()
        idx = self._flat_idx(particles_idx_local, envs_idx)
        vals = self._values(poss, (3,), idx.shape[0], idx.shape[1], torch.float32)
        self._solver.runtime.set_particles_pos(idx.reshape(-1), vals)

    def set_particles_vel(self, vels, particles_idx_local=None, envs_idx=None):
        self._check_built()
        idx = self._flat_idx(particles_idx_local, envs_idx)
        vals = self._values(vels, (3,), idx.shape[0], idx.shape[1], torch.float32)
        self._solver.runtime.set_particles_vel(idx.reshape(-1), vals)

    def set_particles_active(self, actives, particles_idx_local=None, envs_idx=None):
        self._check_built()
        idx = self._flat_idx(particles_idx_local, envs_idx)
        vals = self._values(actives, (), idx.shape[0], idx.shape[1], torch.uint8)
        self._solver.runtime.set_particles_active(idx.reshape(-1), vals)

    def set_free(self, free, particles_idx_local=None):
        """Non-free particles act as boundary conditions (mpm_solver.py:388-389)."""
        self._check_built()
        idx = self._flat_idx(particles_idx_local, None)
        vals = self._values(free, (), idx.shape[0], idx.shape[1], torch.uint8)
        self._solver.runtime.set_particles_free(idx.reshape(-1), vals)

    def get_free(self):
        """Free (True) or fixed (False) flag of each particle, shape (n_particles,)
        (mpm_entity.py:571-583)."""
        self._check_built()
        return self._solver.runtime.get_particles_free(self._flat_idx(None, None)[0])

    # buffered targets applied at the next step (particle_entity.py:418-458, 503-578); in a
    # differentiable scene they go to the scene's tape, which applies them at the next step and
    # hands back their gradients (particle_entity.py:460-481)
    def _tape(self):
        return getattr(self._solver, "tape", None) if self._scene.requires_grad else None

    def _actu_groups(self, a, n_envs, n):
        """Per-group actuation values of shape ([M,] [n_particles,] [n_groups,]) broadcast to
        [n_envs, n, n_groups] (mpm_entity.py:412-451): a 2-D value is per environment when
        the scene is batched and its first dimension matches the environments, else per
        particle."""
        G = self._material.n_groups
        if a.ndim == 0:
            a = a.reshape(1).expand(G)
        a = a.reshape(a.shape[:-1] + (G,))
        if a.ndim == 2 and self._scene.n_envs > 0 and a.shape[0] == n_envs and a.shape[0] != n:
            a = a[:, None, :]
        return a.expand(n_envs, n, G)

    def _input_map(self, kind, value, envs_idx):
        """What a set_position / set_velocity / set_actuation value writes, per environment and
        particle (differentiable in value): positions / velocities [n_envs, n, 3], actuation
        [n_envs, n]."""
        n_envs, n = len(self._envs(envs_idx)), self._n_particles
        if kind == "pos":
            v = value
            if v.ndim == 1 or (v.ndim == 2 and v.shape[0] != n):
                off = torch.as_tensor(self._init_particles_offset, dtype=torch.float32, device=v.device)
                v = off + v[..., None, :]
            return v.expand(n_envs, n, 3)
        if kind == "vel":
            return value.expand(n_envs, n, 3)
        a = self._actu_groups(value, n_envs, n)
        idx = self._flat_idx(None, envs_idx)
        grp = self._solver.runtime.muscle_group[idx.reshape(-1)].reshape(n_envs, n, 1)
        return torch.gather(a, 2, grp).squeeze(2)

    def _input_grad(self, kind, shape, g, envs_idx):
        """dL/d(value) of a set_* input from dL/d(what it wrote) g."""
        with torch.enable_grad():
            a = torch.zeros(shape, dtype=torch.float32, device=g.device, requires_grad=True)
            out = self._input_map(kind, a, envs_idx)
            (ga,) = torch.autograd.grad(out, a, grad_outputs=g.reshape(out.shape), allow_unused=True)
        return torch.zeros(shape, device=g.device) if ga is None else ga

    def _apply_position(self, value, envs_idx):
        self.set_particles_pos(self._input_map("pos", value, envs_idx), envs_idx=envs_idx)

    def _apply_velocity(self, value, envs_idx):
        self.set_particles_vel(self._input_map("vel", value, envs_idx), envs_idx=envs_idx)

    def _apply_actuation(self, value, envs_idx):
        idx = self._flat_idx(None, envs_idx)
        self._solver.runtime.actu[idx.reshape(-1)] = self._input_map("actu", value, envs_idx).reshape(-1)

    def set_position(self, value, envs_idx=None):
        if self._tape() is not None:
            self._tape().record_input(self, "pos", value, envs_idx)
            return
        poss = _as_tensor(value, torch.float32, self._solver.device)
        if poss.ndim == 1 or (poss.ndim == 2 and poss.shape[0] != self._n_particles):
            off = torch.as_tensor(self._init_particles_offset, dtype=torch.float32, device=poss.device)
            poss = off + poss[..., None, :]
        self._tgt["pos"] = (poss, envs_idx)

    def set_velocity(self, vels, envs_idx=None):
        if self._tape() is not None:
            self._tape().record_input(self, "vel", vels, envs_idx)
            return
        self._tgt["vel"] = (_as_tensor(vels, torch.float32, self._solver.device), envs_idx)

    def set_active(self, active, envs_idx=None):
        a = _as_tensor(active, torch.uint8, self._solver.device)
        self._tgt["act"] = (a, envs_idx)
        self.active = bool((a != 0).any())

    def activate(self):
        """Every particle of the entity takes part in the next step (particle_entity.py:639-644)."""
        self.set_active(1)

    def deactivate(self):
        """Every particle of the entity is frozen from the next step on (particle_entity.py:646-651)."""
        self.set_active(0)

    # ---------------------------------------------------------------- muscle
    def _assert_muscle(self):
        from ..materials.MPM import Muscle

        if not isinstance(self._material, Muscle):
            raise GenesisException("This method is only supported by entities with a 'MPM.Muscle' material.")

    def set_actuation(self, actus, envs_idx=None):
        """Buffered per-group actuation applied at the next step (mpm_entity.py:412-427):
        actus of shape ([M,] [n_particles,] [n_groups,]); a scalar applies to every group."""
        self._assert_muscle()
        if self._tape() is not None:
            self._tape().record_input(self, "actu", actus, envs_idx)
            return
        a = _as_tensor(actus, torch.float32, self._solver.device)
        if a.ndim == 0:
            a = a.reshape((1,)).expand((self._material.n_groups,))
        self._tgt["actu"] = (a, envs_idx)

    def set_particles_actu(self, actus, particles_idx_local=None, envs_idx=None):
        """Each particle takes the value of its muscle group (mpm_entity.py:429-451,
        mpm_solver.py:922-934); actus of shape ([M,] [n_particles,] [n_groups,])."""
        self._assert_muscle()
        self._check_built()
        idx = self._flat_idx(particles_idx_local, envs_idx)
        G = self._material.n_groups
        a = _as_tensor(actus, torch.float32, self._solver.device)
        a = self._actu_groups(a, idx.shape[0], idx.shape[1]).reshape(-1, G)
        self._solver.runtime.set_actu_by_group(idx.reshape(-1), a)

    def get_particles_actu(self, envs_idx=None):
        self._assert_muscle()
        self._check_built()
        idx = self._flat_idx(None, envs_idx)
        return self._squeeze(self._solver.runtime.get_actu(idx.reshape(-1)).reshape(idx.shape))

    def _all_env_idx(self):
        return self._flat_idx(None, None)  # (B, n_particles)

    def set_muscle_group(self, muscle_group):
        """Muscle group of each particle, shape (n_particles,) (mpm_entity.py:475-493)."""
        self._assert_muscle()
        self._check_built()
        idx = self._all_env_idx()
        g = _as_tensor(muscle_group, torch.int64, self._solver.device).reshape(-1).expand(idx.shape)
        self._solver.runtime.set_muscle_group(idx.reshape(-1), g.reshape(-1))

    def get_muscle_group(self):
        self._assert_muscle()
        self._check_built()
        return self._solver.runtime.get_muscle_group(self._all_env_idx()[0]).to(torch.int32)

    def set_muscle_direction(self, muscle_direction):
        """Fibre direction of each particle, shape ([n_particles,] 3) (mpm_entity.py:495-517)."""
        self._assert_muscle()
        self._check_built()
        idx = self._all_env_idx()
        d = _as_tensor(muscle_direction, torch.float32, self._solver.device).reshape(-1, 3)
        d = d.expand(idx.shape[1], 3) if d.shape[0] == 1 else d
        self._solver.runtime.set_muscle_direction(idx.reshape(-1), d.expand(idx.shape + (3,)).reshape(-1, 3))

    def set_muscle(self, muscle_group=None, muscle_direction=None):
        if muscle_group is not None:
            self.set_muscle_group(muscle_group)
        if muscle_direction is not None:
            self.set_muscle_direction(muscle_direction)

    def process_input(self, in_backward=False):
        # positions first: setting positions resets velocities (particle_entity.py:439-440)
        if self._tgt["pos"] is not None:
            v, e = self._tgt["pos"]
            if v.ndim == 1 or (v.ndim == 2 and v.shape[-1] == 3 and v.shape[0] != self._n_particles):
                v = v.expand(self._n_particles, 3)
            self.set_particles_pos(v, envs_idx=e)
        if self._tgt["vel"] is not None:
            v, e = self._tgt["vel"]
            if v.ndim == 1:
                v = v.expand(self._n_particles, 3)
            self.set_particles_vel(v, envs_idx=e)
        if self._tgt["act"] is not None:
            v, e = self._tgt["act"]
            if v.ndim == 0:
                v = v.expand(self._n_particles)
            self.set_particles_active(v, envs_idx=e)
        if self._tgt.get("actu") is not None:
            v, e = self._tgt["actu"]
            self.set_particles_actu(v, envs_idx=e)
        for k in self._tgt:
            self._tgt[k] = None

    # --------------------------------------------------------------- getters
    def _get(self, keys, envs_idx):
        self._check_built()
        envs = self._envs(envs_idx)
        if self._tape() is not None:  # differentiable: slices of a query node of the tape
            full = self._solver.get_state()
            return {k: getattr(full, k)[envs, self._particle_start : self.particle_end] for k in keys}
        st = self._solver.runtime.get_state(keys)
        B, N = self._solver.B, self._solver.n_particles
        out = {}
        for k, v in st.items():
            v = v.reshape((B, N) + tuple(v.shape[1:]))[envs, self._particle_start : self.particle_end]
            if k in ("C", "F"):
                v = v.reshape(v.shape[:2] + (3, 3))
            out[k] = v
        return out

    def _squeeze(self, t):
        return t[0] if self._scene.n_envs == 0 else t

    def get_particles_pos(self, envs_idx=None):
        return self._squeeze(self._get(("pos",), envs_idx)["pos"])

    def get_particles_vel(self, envs_idx=None):
        return self._squeeze(self._get(("vel",), envs_idx)["vel"])

    def get_particles_active(self, envs_idx=None):
        return self._squeeze(self._get(("active",), envs_idx)["active"])

    def find_closest_particle(self, pos, envs_idx=None):
        """Local index of the particle closest to pos ([M,] 3) per environment
        (particle_entity.py:709-738); a scalar tensor without environments."""
        self._check_built()
        p = _as_tensor(pos, torch.float32, self._solver.device)
        envs = self._envs(envs_idx)
        if p.ndim == 1:
            p = p.reshape(1, 3).expand(len(envs), 3)
        if p.shape != (len(envs), 3):
            raise GenesisException(f"Invalid tensor shape {tuple(p.shape)} (expected ({len(envs)}, 3)).")
        cur = self._get(("pos",), envs_idx)["pos"]
        idx = torch.argmin(torch.linalg.norm(cur - p[:, None], dim=-1), dim=-1).to(torch.int32)
        return idx[0] if self._scene.n_envs == 0 else idx

    def get_frame(self, f, pos, vel, C, F, Jp, active):
        """Copy the entity's state into the given tensors (mpm_entity.py:293-340): pos/vel
        [B, n, 3], C/F [B, n, 3, 3], Jp/active [B, n].  Only the current frame is kept here, so
        f must be the current local substep (sim.cur_substep_local)."""
        if int(f) != self._sim.cur_substep_local:
            raise GenesisException(f"Only the current frame ({self._sim.cur_substep_local}) is kept, not {f}.")
        st = self._get(("pos", "vel", "C", "F", "Jp", "active"), None)
        for dst, key in ((pos, "pos"), (vel, "vel"), (C, "C"), (F, "F"), (Jp, "Jp"), (active, "active")):
            dst.copy_(st[key].to(dst.device, dst.dtype).reshape(dst.shape))

    def get_state(self):
        st = self._get(("pos", "vel", "C", "F", "Jp", "active"), None)
        return MPMEntityState(self, self._sim.cur_step_global, st["pos"], st["vel"], st["C"], st["F"], st["Jp"],
                              st["active"])

    def get_mass(self):
        """Total mass in kg, the 1e3 volume scale divided back out (mpm_solver.py:1000-1009)."""
        return float(self._n_particles * self._solver.particle_volume * self._material.rho
                     / self._solver.particle_volume_scale)
