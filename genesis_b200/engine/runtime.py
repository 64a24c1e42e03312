"""Device-resident MPM problem: PyTorch owns every buffer, the C ABI does the work.

One ``MPMRuntime`` advances one or more *instances* (independent scenes, or the
``n_envs`` copies of one scene) together.  The layout is the one documented in
include/genesis_b200_mpm.h: particles in planar SoA channels sorted by grid block,
the grid block-major inside one workspace blob.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from .. import _native as nat

F32_EPS = float(np.finfo(np.float32).eps)


@dataclass
class InstanceSpec:
    """Constants of one scene (MPMSolver.__init__, mpm_solver.py:31-78)."""

    grid_density: float
    lower_bound: tuple
    upper_bound: tuple
    particle_size: float
    dt: float  # substep dt
    gravity: tuple
    materials: list  # objects with ._native(p_vol) -> nat.Material
    n_particles: int
    eps: float = F32_EPS
    # derived
    dx: float = field(init=False)
    inv_dx: float = field(init=False)
    lower_cell: np.ndarray = field(init=False)
    upper_cell: np.ndarray = field(init=False)
    grid_res: np.ndarray = field(init=False)
    p_vol: float = field(init=False)
    bnd_lo: np.ndarray = field(init=False)
    bnd_hi: np.ndarray = field(init=False)

    def __post_init__(self):
        self.dx = float(1.0 / self.grid_density)
        self.inv_dx = float(self.grid_density)
        lo = np.asarray(self.lower_bound, dtype=np.float64)
        hi = np.asarray(self.upper_bound, dtype=np.float64)
        self.lower_cell = np.round(self.grid_density * lo).astype(np.int64)
        self.upper_cell = np.round(self.grid_density * hi).astype(np.int64)
        self.grid_res = self.upper_cell - self.lower_cell + 1
        self.p_vol = float(self.particle_size**3) * 1e3
        pad = 3 * self.dx
        self.bnd_lo = lo + pad
        self.bnd_hi = hi - pad
        if np.any(self.grid_res > 4 * 1023):
            raise ValueError("grid_res above 4092 nodes per axis is not supported (10-bit block coordinates)")

    @property
    def nblk(self) -> np.ndarray:
        return (self.grid_res + nat.MPM_BLOCK - 1) // nat.MPM_BLOCK

    @property
    def n_blocks(self) -> int:
        return int(np.prod(self.nblk))


def _h2d(a: np.ndarray, dev) -> torch.Tensor:
    """Host array -> device tensor through pinned memory, stream-ordered without blocking the
    host (a copy from pageable memory would wait for the GPU to reach it: a runtime built while
    another one's substeps run, as the server's repacks are, would stall the host until they end)."""
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().to(dev, non_blocking=True)


def _cuda_stream_handle():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream or None)


class MPMRuntime:
    """Buffers + C-ABI calls for a set of instances.

    Parameters
    ----------
    specs : list[InstanceSpec]
    chunk_particles : particles per p2g/g2p work item (128, 256 or 512)
    sort_interval : re-bin particles every this many substeps
    per_particle_lame : allocate per-particle (mu, lam) overrides
    """

    def __init__(
        self,
        specs: list[InstanceSpec],
        device=None,
        chunk_particles: int = 128,
        sort_interval: int = 50,
        per_particle_lame: bool = False,
        grid_ctas: int = 0,
        use_graphs: bool = True,
        colliders: list | None = None,
        sdf_voxels: torch.Tensor | None = None,
        cpic: bool = False,
        force_fields: list | None = None,
        ff_perm: np.ndarray | None = None,
    ):
        if not torch.cuda.is_available():
            raise RuntimeError("genesis_b200 needs a CUDA device (sm_100a); there is no CPU path")
        self.lib = nat.load()
        self.device = torch.device(device or "cuda")
        self.specs = list(specs)
        self.sort_interval = int(sort_interval)
        self.use_graphs = bool(use_graphs)
        self._graphs: dict = {}
        self._count = 0  # substeps executed
        self._nonfree = False
        self._dirty = False  # positions written since the last sort

        insts, mats = [], []
        p_begin = 0
        blk_base = 0
        for sp in self.specs:
            I = nat.Instance()
            I.p_begin = p_begin
            I.p_count = int(sp.n_particles)
            for d in range(3):
                I.res[d] = int(sp.grid_res[d])
                I.nblk[d] = int(sp.nblk[d])
                I.lower_cell[d] = int(sp.lower_cell[d])
                I.gravity[d] = float(sp.gravity[d])
                I.bnd_lo[d] = float(sp.bnd_lo[d])
                I.bnd_hi[d] = float(sp.bnd_hi[d])
            I.mat_base = len(mats)
            I.blk_base = blk_base
            I.dx = sp.dx
            I.inv_dx = sp.inv_dx
            I.dt = float(sp.dt)
            I.eps = float(sp.eps)
            # (-dt * particle_volume * 4 * inv_dx * inv_dx) folded in float64 (mpm_solver.py:344)
            I.stress_scale = -sp.dt * sp.p_vol * 4 * sp.inv_dx * sp.inv_dx
            I.c_scale = 4 * sp.inv_dx
            insts.append(I)
            for m in sp.materials:
                mats.append(m._native(sp.p_vol))
            p_begin += int(sp.n_particles)
            blk_base += sp.n_blocks
        self.n = p_begin
        self.n_blocks = blk_base
        self.stride = max(64, (self.n + 63) // 64 * 64)
        self._insts = insts
        self._mats = mats

        P = int(chunk_particles)
        mc = C.c_int32()
        nat.check("mpm_max_chunks", self.lib.mpm_max_chunks(self.n, self.n_blocks, P, C.byref(mc)))
        self.prob = nat.Problem(
            n_instances=len(insts),
            n_particles=self.n,
            n_blocks=self.n_blocks,
            n_materials=len(mats),
            chunk_particles=P,
            max_chunks=mc.value,
            grid_ctas=int(grid_ctas),
            flags=0,
        )
        dev = self.device
        self.inst_table = _h2d(nat.instances_to_bytes(insts), dev)
        self.mat_table = _h2d(nat.materials_to_bytes(mats), dev)
        # kinematic rigid colliders of the grid op (mpm_collider rows) and their reaction
        # force / torque accumulators
        colliders = list(colliders or [])
        self.n_colliders = len(colliders)
        self.last_step_substeps = 0
        if colliders:
            arr = (nat.Collider * len(colliders))(*colliders)
            self.coll_table = _h2d(np.frombuffer(bytes(arr), dtype=np.uint8).copy(), dev)
            self.coll_init = self.coll_table.clone()
            self.collider_force = torch.zeros((len(colliders), 6), dtype=torch.float32, device=dev)
        else:
            self.coll_table = None
            self.collider_force = None
        # the tools' signed-distance voxel grids (mpm_collider.sdf_offset indexes into it)
        self.sdf_voxels = None
        if sdf_voxels is not None and sdf_voxels.numel() > 0:
            self.sdf_voxels = sdf_voxels.to(dev, torch.float32).contiguous()
        if any(c.kind == nat.COLLIDER_TOOL for c in colliders):
            n_vox = 0 if self.sdf_voxels is None else self.sdf_voxels.numel()
            for c in colliders:
                if c.kind == nat.COLLIDER_TOOL and c.sdf_res != 0 and (
                        c.sdf_res < 2 or c.sdf_offset < 0 or c.sdf_offset + c.sdf_res ** 3 > n_vox):
                    raise ValueError("a tool collider's voxel grid lies outside sdf_voxels")
        # external force fields of the grid op (mpm_force_field rows) and the turbulence fields'
        # permutation tables (mpm_force_field.perm_offset indexes into them)
        force_fields = list(force_fields or [])
        self.n_force_fields = len(force_fields)
        self.ff_table = self.ff_perm = None
        if force_fields:
            perm_n = 0 if ff_perm is None else int(np.asarray(ff_perm).size)
            for f in force_fields:
                if f.kind == nat.FF_TURBULENCE and (f.perm_offset < 0 or f.perm_offset + 3 * 512 > perm_n):
                    raise ValueError("a turbulence field's permutation tables lie outside ff_perm")
            arr = (nat.ForceField * len(force_fields))(*force_fields)
            self.ff_table = _h2d(np.frombuffer(bytes(arr), dtype=np.uint8).copy(), dev)
            if perm_n:
                self.ff_perm = torch.as_tensor(np.asarray(ff_perm, dtype=np.int32).reshape(-1), device=dev)
        self.tables = nat.Tables(
            self.inst_table.data_ptr(), self.mat_table.data_ptr(),
            self.coll_table.data_ptr() if colliders else None, len(colliders), 0,
            self.collider_force.data_ptr() if colliders else None,
            self.sdf_voxels.data_ptr() if self.sdf_voxels is not None else None,
            self.ff_table.data_ptr() if force_fields else None, len(force_fields), 0,
            self.ff_perm.data_ptr() if self.ff_perm is not None else None,
        )

        self.state = torch.zeros((nat.MPM_STATE_CH, self.stride), dtype=torch.float32, device=dev)
        self.mat = torch.zeros(max(self.n, 1), dtype=torch.uint8, device=dev)
        self.pflags = torch.full((max(self.n, 1),), nat.PFLAG_ACTIVE | nat.PFLAG_FREE, dtype=torch.uint8, device=dev)
        self.gid = torch.arange(max(self.n, 1), dtype=torch.int32, device=dev)
        self.slot = torch.arange(max(self.n, 1), dtype=torch.int32, device=dev)
        self.mu_p = self.lam_p = None
        if per_particle_lame:
            self.mu_p = torch.zeros(max(self.n, 1), dtype=torch.float32, device=dev)
            self.lam_p = torch.zeros(max(self.n, 1), dtype=torch.float32, device=dev)
        # muscle inputs in API order (mpm_solver.py:787-788, 801: group 0, direction +z,
        # actuation 0), allocated only when a Muscle material is present
        self.actu = self.muscle_dir = self.muscle_group = None
        if any(m.flags & nat.MATF_MUSCLE for m in mats):
            nn = max(self.n, 1)
            self.actu = torch.zeros(nn, dtype=torch.float32, device=dev)
            self.muscle_dir = torch.zeros((nn, 3), dtype=torch.float32, device=dev)
            self.muscle_dir[:, 2] = 1.0
            self.muscle_group = torch.zeros(nn, dtype=torch.int64, device=dev)
        # CPIC (with colliders only): the collider-side normal each particle remembers, per
        # collider in API order, and the separated stencil nodes of the last p2g, per slot
        self.cpic_normal = self.cpic_sep = None
        if cpic and colliders:
            self.cpic_normal = torch.zeros((3 * len(colliders), self.stride), dtype=torch.float32, device=dev)
            self.cpic_sep = torch.zeros((7, self.stride), dtype=torch.int32, device=dev)
            self.prob.flags |= nat.PROBF_CPIC
        self.par = nat.Particles(
            state=self.state.data_ptr(),
            state_stride=self.stride,
            mat=self.mat.data_ptr(),
            pflags=self.pflags.data_ptr(),
            gid=self.gid.data_ptr(),
            slot=self.slot.data_ptr(),
            mu_p=self.mu_p.data_ptr() if self.mu_p is not None else None,
            lam_p=self.lam_p.data_ptr() if self.lam_p is not None else None,
            actu=self.actu.data_ptr() if self.actu is not None else None,
            muscle_dir=self.muscle_dir.data_ptr() if self.muscle_dir is not None else None,
            cpic_normal=self.cpic_normal.data_ptr() if self.cpic_normal is not None else None,
            cpic_sep=self.cpic_sep.data_ptr() if self.cpic_sep is not None else None,
        )
        nbytes = C.c_uint64()
        nat.check("mpm_workspace_bytes", self.lib.mpm_workspace_bytes(C.byref(self.prob), C.byref(nbytes)))
        self.workspace_bytes = int(nbytes.value)
        self.workspace = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=dev)
        self._ws = C.c_void_p(self.workspace.data_ptr())
        self._call("mpm_workspace_init", C.byref(self.prob), self._ws, _cuda_stream_handle())

    # ------------------------------------------------------------------ utils
    def _call(self, name, *args):
        rc = getattr(self.lib, name)(*args)
        nat.check(name, rc)

    @property
    def instance_offsets(self) -> list[int]:
        return [int(I.p_begin) for I in self._insts]

    def memory_bytes(self) -> int:
        t = self.state.numel() * 4 + self.mat.numel() * 10 + self.workspace_bytes
        if self.mu_p is not None:
            t += self.mu_p.numel() * 8
        if self.actu is not None:
            t += self.actu.numel() * 24
        return int(t)

    # -------------------------------------------------------------- state I/O
    def init_particles(self, pos, mat_idx, active=None, vel=None, default_jp=None):
        """Initialise all particles in API order (the _kernel_add_particles semantics,
        mpm_solver.py:768-801): v=0 (or vel), F=I, C=0, Jp=default_Jp, free=True."""
        n = self.n
        pos = np.asarray(pos, dtype=np.float32).reshape(n, 3)
        host = np.zeros((nat.MPM_STATE_CH, n), dtype=np.float32)
        host[nat.CH_X : nat.CH_X + 3] = pos.T
        if vel is not None:
            host[nat.CH_V : nat.CH_V + 3] = np.asarray(vel, dtype=np.float32).reshape(n, 3).T
        for k in (0, 4, 8):
            host[nat.CH_F + k] = 1.0
        mat_idx = np.asarray(mat_idx, dtype=np.uint8).reshape(n)
        if default_jp is None:
            default_jp = np.zeros(n, dtype=np.float32)
            for sp_i, I in enumerate(self._insts):
                sl = slice(I.p_begin, I.p_begin + I.p_count)
                djp = np.array([self._mats[I.mat_base + k].default_Jp for k in range(len(self.specs[sp_i].materials))],
                               dtype=np.float32)
                default_jp[sl] = djp[mat_idx[sl]]
        host[nat.CH_JP] = np.asarray(default_jp, dtype=np.float32)
        flags = np.full(n, nat.PFLAG_ACTIVE | nat.PFLAG_FREE, dtype=np.uint8)
        if active is not None:
            flags = np.where(np.asarray(active, dtype=bool).reshape(n), flags, nat.PFLAG_FREE).astype(np.uint8)
        with torch.no_grad():
            self.state[:, :n].copy_(torch.from_numpy(host))
            self.mat[:n].copy_(torch.from_numpy(mat_idx))
            self.pflags[:n].copy_(torch.from_numpy(flags))
            self.gid[:n].copy_(torch.arange(n, dtype=torch.int32))
            self.slot[:n].copy_(torch.arange(n, dtype=torch.int32))
        self._count = 0
        self._dirty = True

    def set_lame(self, mu, lam):
        """Per-particle Lame parameters in API order (requires per_particle_lame=True)."""
        if self.mu_p is None:
            raise RuntimeError("runtime was built without per-particle Lame parameters")
        mu = torch.as_tensor(mu, dtype=torch.float32, device=self.device).reshape(self.n)
        lam = torch.as_tensor(lam, dtype=torch.float32, device=self.device).reshape(self.n)
        sl = self.slot[: self.n].long()
        self.mu_p[sl] = mu
        self.lam_p[sl] = lam

    def reset_colliders(self):
        """Back to the poses and velocities the colliders were built with; the particles
        forget their CPIC sides (legacy_coupler.py:120-123)."""
        if self.coll_table is not None:
            self.coll_table.copy_(self.coll_init)
        if self.cpic_normal is not None:
            self.cpic_normal.zero_()
            self.cpic_sep.zero_()

    def get_cpic_normals(self) -> torch.Tensor:
        """The remembered collider-side normals, [n_colliders, n, 3] in API order."""
        if self.cpic_normal is None:
            raise RuntimeError("runtime has no CPIC state")
        return self.cpic_normal[:, : self.n].reshape(-1, 3, self.n).permute(0, 2, 1)

    def set_force_field_active(self, k: int, active: bool):
        """ForceField.activate / deactivate (force_fields.py:21-32) of row k, stream-ordered."""
        if self.ff_table is None or not 0 <= k < self.n_force_fields:
            raise IndexError("no such force field")
        off = k * C.sizeof(nat.ForceField) + nat.ForceField.active.offset
        self.ff_table.view(torch.int32)[off // 4] = 1 if active else 0

    def collider_table(self) -> torch.Tensor:
        """The collider rows as float32 [n_colliders, 32] (pos 0:3, rot 3:12, data 12:15,
        lin_vel 15:18, ang_vel 18:21, friction, softness, restitution 21:24, then the tool
        fields: sdf_res and its pad 24:26 and sdf_offset 26:28 as integer bits, sdf_scale
        28:31, floor 31), a view of the device table after each row's two int32 fields;
        writes go straight to the table."""
        if self.coll_table is None:
            raise RuntimeError("runtime has no colliders")
        stride = C.sizeof(nat.Collider) // 4
        return self.coll_table.view(torch.float32).view(self.n_colliders, stride)[:, 2:]

    # ---------------------------------------------------------------- muscle
    def _need_muscle(self):
        if self.actu is None:
            raise RuntimeError("runtime has no Muscle material")

    def set_actu_by_group(self, idx, actus):
        """_kernel_set_particles_actu (mpm_solver.py:922-934): particle idx[i] takes
        actus[i, muscle_group[idx[i]]]; idx are API-order indices, actus [len(idx), n_groups]."""
        self._need_muscle()
        idx = torch.as_tensor(idx, dtype=torch.int64, device=self.device).reshape(-1)
        actus = torch.as_tensor(actus, dtype=torch.float32, device=self.device).reshape(idx.numel(), -1)
        g = self.muscle_group[idx].clamp(0, actus.shape[1] - 1)
        self.actu[idx] = torch.gather(actus, 1, g[:, None])[:, 0]

    def get_actu(self, idx):
        self._need_muscle()
        return self.actu[torch.as_tensor(idx, dtype=torch.int64, device=self.device).reshape(-1)]

    def set_muscle_group(self, idx, group):
        self._need_muscle()
        idx = torch.as_tensor(idx, dtype=torch.int64, device=self.device).reshape(-1)
        self.muscle_group[idx] = torch.as_tensor(group, dtype=torch.int64, device=self.device).reshape(-1)

    def get_muscle_group(self, idx):
        self._need_muscle()
        return self.muscle_group[torch.as_tensor(idx, dtype=torch.int64, device=self.device).reshape(-1)]

    def set_muscle_direction(self, idx, direction):
        self._need_muscle()
        idx = torch.as_tensor(idx, dtype=torch.int64, device=self.device).reshape(-1)
        self.muscle_dir[idx] = torch.as_tensor(direction, dtype=torch.float32, device=self.device).reshape(-1, 3)

    def get_state(self, which=("pos", "vel", "C", "F", "Jp", "active")):
        """State in API order as device tensors: pos/vel [n,3], C/F [n,3,3], Jp [n], active [n] bool."""
        n = self.n
        dev = self.device
        out = {}
        shapes = {"pos": (n, 3), "vel": (n, 3), "C": (n, 3, 3), "F": (n, 3, 3), "Jp": (n,)}
        ptr = {}
        for k in ("pos", "vel", "C", "F", "Jp"):
            if k in which:
                out[k] = torch.empty(shapes[k], dtype=torch.float32, device=dev)
                ptr[k] = out[k].data_ptr()
            else:
                ptr[k] = None
        if "active" in which:
            out["active"] = torch.empty(n, dtype=torch.uint8, device=dev)
            ptr["active"] = out["active"].data_ptr()
        else:
            ptr["active"] = None
        self._call(
            "mpm_get_state", C.byref(self.prob), C.byref(self.par),
            ptr["pos"], ptr["vel"], ptr["C"], ptr["F"], ptr["Jp"], ptr["active"], _cuda_stream_handle(),
        )
        if "active" in out:
            out["active"] = out["active"].bool()
        return out

    # state channels in API order: (name, dtype, values per particle)
    _STATE_IO = (("pos", torch.float32, 3), ("vel", torch.float32, 3), ("C", torch.float32, 9),
                 ("F", torch.float32, 9), ("Jp", torch.float32, 1), ("active", torch.uint8, 1))

    def set_state(self, pos=None, vel=None, C_=None, F=None, Jp=None, active=None):
        """Overwrite any subset of the state, arrays in API order (device or host).

        When every given array is a contiguous pinned host tensor of the channel's dtype
        (float32; bool or uint8 for ``active``) the upload is asynchronous: the arrays are
        copied on a side stream into a device staging buffer, and the scatter into the
        sorted state waits for that copy on the current stream.  The host does not block,
        so the copy overlaps whatever the device is still running."""
        vals = dict(pos=pos, vel=vel, C=C_, F=F, Jp=Jp, active=active)
        n = self.n
        if pos is not None:
            self._dirty = True
        given = {k: v for k, v in vals.items() if v is not None}
        if given and all(self._stageable(k, v) for k, v in given.items()):
            return self._set_state_staged(given)
        dev = self.device
        keep = []

        def dptr(k, dtype, width):
            x = vals[k]
            if x is None:
                return None
            t = torch.as_tensor(x).to(device=dev, dtype=dtype).reshape((n, width) if width > 1 else (n,)).contiguous()
            keep.append(t)
            return t.data_ptr()

        self._call("mpm_set_state", C.byref(self.prob), C.byref(self.par),
                   *[dptr(k, dt, w) for k, dt, w in self._STATE_IO], _cuda_stream_handle())
        return keep

    def _stageable(self, k, v) -> bool:
        if not isinstance(v, torch.Tensor) or v.device.type != "cpu" or not v.is_contiguous():
            return False
        if k == "active":
            ok = v.dtype in (torch.bool, torch.uint8)
        else:
            ok = v.dtype == torch.float32
        width = dict((a, w) for a, _, w in self._STATE_IO)[k]
        return ok and v.numel() == self.n * width and v.is_pinned()

    def _set_state_staged(self, given):
        n = self.n
        if getattr(self, "_staging", None) is None:
            self._staging = torch.empty(n * 25 * 4 + n, dtype=torch.uint8, device=self.device)
            self._copy_stream = torch.cuda.Stream(device=self.device)
            self._staging_free = None
        main = torch.cuda.current_stream(self.device)
        cs = self._copy_stream
        if self._staging_free is not None:
            cs.wait_event(self._staging_free)  # the previous scatter has read the staging buffer
        ptrs, off = [], 0
        with torch.cuda.stream(cs):
            for k, dt, w in self._STATE_IO:
                nbytes = n * w * (4 if dt == torch.float32 else 1)
                if k in given:
                    dst = self._staging[off:off + nbytes]
                    dst.copy_(given[k].reshape(-1).view(torch.uint8), non_blocking=True)
                    ptrs.append(dst.data_ptr())
                else:
                    ptrs.append(None)
                off += nbytes
        done = torch.cuda.Event()
        done.record(cs)
        main.wait_event(done)
        self._call("mpm_set_state", C.byref(self.prob), C.byref(self.par), *ptrs, _cuda_stream_handle())
        self._staging_free = torch.cuda.Event()
        self._staging_free.record(main)
        return []

    def status_enqueue(self):
        """Start an asynchronous read of the status word on the current stream; returns a
        (pinned host tensor, event) pair, valid once the event has completed."""
        out = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self._call("mpm_status_enqueue", C.byref(self.prob), self._ws, C.c_void_p(out.data_ptr()),
                   _cuda_stream_handle())
        ev = torch.cuda.Event()
        ev.record()
        return out, ev

    def _idx_call(self, name, idx, values, vdtype, vshape, with_tables=False):
        dev = self.device
        idx = torch.as_tensor(idx).to(device=dev, dtype=torch.int32).reshape(-1).contiguous()
        n = idx.numel()
        vals = torch.as_tensor(values).to(device=dev, dtype=vdtype).reshape((n,) + vshape).contiguous()
        args = [C.byref(self.prob)]
        if with_tables:
            args.append(C.byref(self.tables))
        args += [C.byref(self.par), n, idx.data_ptr(), vals.data_ptr(), _cuda_stream_handle()]
        self._call(name, *args)
        return idx, vals

    def set_particles_pos(self, idx, pos):
        self._dirty = True
        return self._idx_call("mpm_set_particles_pos", idx, pos, torch.float32, (3,), with_tables=True)

    def set_particles_vel(self, idx, vel):
        return self._idx_call("mpm_set_particles_vel", idx, vel, torch.float32, (3,))

    def set_particles_active(self, idx, active):
        return self._idx_call("mpm_set_particles_active", idx, active, torch.uint8, ())

    def get_particles_free(self, idx):
        """Free flags (bool) of API-order particles idx."""
        idx = torch.as_tensor(idx, dtype=torch.int64, device=self.device).reshape(-1)
        return (self.pflags[self.slot[idx].long()] & nat.PFLAG_FREE) != 0

    def set_particles_free(self, idx, free):
        keep = self._idx_call("mpm_set_particles_free", idx, free, torch.uint8, ())
        if not bool(torch.as_tensor(free).bool().all()):
            self._nonfree = True
            self.prob.flags |= nat.PROBF_NONFREE
            self._drop_graphs()
        return keep

    def retune(self, chunk_particles=None, sort_interval=None, grid_ctas=None):
        """Change the launch configuration between substeps (the particle state is kept;
        the workspace is re-laid-out and the particles re-binned)."""
        if chunk_particles is not None and int(chunk_particles) != self.prob.chunk_particles:
            P = int(chunk_particles)
            mc = C.c_int32()
            nat.check("mpm_max_chunks", self.lib.mpm_max_chunks(self.n, self.n_blocks, P, C.byref(mc)))
            self.prob.chunk_particles = P
            self.prob.max_chunks = mc.value
            nbytes = C.c_uint64()
            nat.check("mpm_workspace_bytes", self.lib.mpm_workspace_bytes(C.byref(self.prob), C.byref(nbytes)))
            if int(nbytes.value) > self.workspace.numel():
                self.workspace = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
                self._ws = C.c_void_p(self.workspace.data_ptr())
            self.workspace_bytes = int(nbytes.value)
            self._call("mpm_workspace_init", C.byref(self.prob), self._ws, _cuda_stream_handle())
            self._sorted_once = False
        if sort_interval is not None:
            self.sort_interval = int(sort_interval)
        if grid_ctas is not None:
            self.prob.grid_ctas = int(grid_ctas)
        self._drop_graphs()

    @property
    def config(self) -> dict:
        return {"chunk_particles": int(self.prob.chunk_particles), "sort_interval": int(self.sort_interval),
                "grid_ctas": int(self.prob.grid_ctas)}

    # ---------------------------------------------------------------- stepping
    def sort(self):
        self._call("mpm_sort_particles", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                   _cuda_stream_handle())

    def p2g(self):
        self._call("mpm_p2g", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                   _cuda_stream_handle())

    def grid_op(self):
        self._call("mpm_grid_op", C.byref(self.prob), C.byref(self.tables), self._ws, _cuda_stream_handle())

    def g2p(self):
        self._call("mpm_g2p", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                   _cuda_stream_handle())

    def g2p2g(self):
        self._call("mpm_g2p2g", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                   _cuda_stream_handle())

    def ensure_sorted(self):
        """Re-bin before a p2g that starts a sort interval, the first one, or one after
        positions were overwritten (particles far from their bins would all take the
        slow out-of-tile path)."""
        if self._count % max(self.sort_interval, 1) == 0 or not getattr(self, "_sorted_once", False) or self._dirty:
            self.sort()
            self._sorted_once = True
            self._dirty = False

    def substeps(self, n: int):
        """Advance n substeps (p2g, grid op, g2p), re-sorting every sort_interval
        (sort_interval <= 0: sort once, before the first substep, and never again)."""
        n = int(n)
        stream = _cuda_stream_handle()
        if self.sort_interval <= 0:
            if not getattr(self, "_sorted_once", False) or self._dirty:
                self.sort()
                self._sorted_once = True
                self._dirty = False
            if n > 0:
                if self.use_graphs:
                    # one captured graph per run length (a rollout's checkpoint segments repeat it)
                    self._call("mpm_graph_launch", self._graph_unsorted(n), stream)
                else:
                    self._call("mpm_substeps", C.byref(self.prob), C.byref(self.tables), C.byref(self.par),
                               self._ws, n, 0, self._count, stream)
                self._count += n
            return
        K = max(self.sort_interval, 1)
        while n > 0:
            phase = self._count % K
            if not getattr(self, "_sorted_once", False) or (self._dirty and phase != 0):
                self.sort()
                self._sorted_once = True
            self._dirty = False
            if self.use_graphs and phase == 0 and n >= K:
                g = self._graph(K)
                self._call("mpm_graph_launch", g, stream)
                n -= K
                self._count += K
                continue
            m = min(n, K - phase) if phase else min(n, K)
            self._call("mpm_substeps", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                       m, K, self._count, stream)
            n -= m
            self._count += m

    def _graph_unsorted(self, n: int):
        """A graph of n substeps without a sort (the runtime never re-sorts)."""
        key = ("unsorted", n, self.prob.flags)
        g = self._graphs.get(key)
        if g is None:
            side = torch.cuda.Stream(device=self.device)
            side.wait_stream(torch.cuda.current_stream())
            h = C.c_void_p()
            with torch.cuda.stream(side):
                self._call("mpm_graph_create", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                           n, 0, 0, C.c_void_p(side.cuda_stream), C.byref(h))
            torch.cuda.current_stream().wait_stream(side)
            g = h
            self._graphs[key] = g
        return g

    def _graph(self, K: int):
        key = (K, self.prob.flags)
        g = self._graphs.get(key)
        if g is None:
            side = torch.cuda.Stream(device=self.device)
            side.wait_stream(torch.cuda.current_stream())
            h = C.c_void_p()
            with torch.cuda.stream(side):
                self._call("mpm_graph_create", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                           K, K, 0, C.c_void_p(side.cuda_stream), C.byref(h))
            torch.cuda.current_stream().wait_stream(side)
            g = h
            self._graphs[key] = g
        return g

    def _drop_graphs(self):
        for g in self._graphs.values():
            self.lib.mpm_graph_destroy(g)
        self._graphs.clear()

    def status(self, clear: bool = False) -> int:
        v = C.c_uint32()
        self._call("mpm_status", C.byref(self.prob), self._ws, int(clear), C.byref(v), _cuda_stream_handle())
        return int(v.value)

    def instance_status(self, clear: bool = False) -> np.ndarray:
        out = np.zeros(len(self._insts), dtype=np.uint32)
        self._call("mpm_instance_status", C.byref(self.prob), self._ws, int(clear),
                   out.ctypes.data_as(C.c_void_p), _cuda_stream_handle())
        return out

    def instance_status_enqueue(self, clear: bool = False):
        """Enqueue the read of the per-instance status words: returns (pinned uint32 host
        tensor, event), valid once the event has completed."""
        out = torch.zeros(max(len(self._insts), 1), dtype=torch.int32, pin_memory=True)
        self._call("mpm_instance_status_enqueue", C.byref(self.prob), self._ws, int(clear),
                   C.c_void_p(out.data_ptr()), _cuda_stream_handle())
        ev = torch.cuda.Event()
        ev.record()
        return out, ev

    def load_state(self, pos, vel, C_, F, Jp, active, mat):
        """Overwrite the whole particle state from device tensors in API order
        (pos/vel [n,3], C/F [n,9] or [n,3,3], Jp [n], active [n] bool, mat [n] uint8) and
        reset the slot permutation to the identity; the next substep re-bins."""
        n = self.n
        with torch.no_grad():
            self.gid[:n].copy_(torch.arange(n, dtype=torch.int32, device=self.device))
            self.slot[:n].copy_(self.gid[:n])
            self.state[0:3, :n].copy_(pos.reshape(n, 3).t())
            self.state[3:6, :n].copy_(vel.reshape(n, 3).t())
            self.state[6:15, :n].copy_(C_.reshape(n, 9).t())
            self.state[15:24, :n].copy_(F.reshape(n, 9).t())
            self.state[24, :n].copy_(Jp.reshape(n))
            self.mat[:n].copy_(mat.reshape(n).to(torch.uint8))
            act = active.reshape(n).to(torch.bool)
            self.pflags[:n].copy_(torch.where(act, nat.PFLAG_ACTIVE | nat.PFLAG_FREE, nat.PFLAG_FREE).to(torch.uint8))
        self._dirty = True
        self._sorted_once = False

    def export_instances(self):
        """Per-instance state in API order as device tensors (for repacking): a list of dicts
        with pos, vel, C, F, Jp, active, mat."""
        st = self.get_state()
        n = self.n
        mat = torch.empty(n, dtype=torch.uint8, device=self.device)
        mat[self.gid[:n].long()] = self.mat[:n]
        out = []
        for I in self._insts:
            sl = slice(int(I.p_begin), int(I.p_begin) + int(I.p_count))
            d = {k: v[sl] for k, v in st.items()}
            d["mat"] = mat[sl]
            out.append(d)
        return out

    def profile_substeps(self, n: int) -> dict:
        """Advance n substeps as substeps() does, without CUDA graphs, timing every launch
        group with CUDA events (mpm_substeps_profile).  Returns {kind: (ms, launches)} summed
        over the run; the kinds' times add up to the run's device time."""
        n = int(n)
        stream = _cuda_stream_handle()
        K = max(self.sort_interval, 0)
        nk = len(nat.KIND_NAMES)
        ms, cnt = (C.c_float * nk)(), (C.c_int32 * nk)()
        tot = {k: [0.0, 0] for k in nat.KIND_NAMES}
        while n > 0:
            phase = self._count % K if K else 1
            if not getattr(self, "_sorted_once", False) or (self._dirty and phase != 0):
                self.sort()
                self._sorted_once = True
            self._dirty = False
            m = min(n, K - self._count % K) if K else n
            self._call("mpm_substeps_profile", C.byref(self.prob), C.byref(self.tables), C.byref(self.par), self._ws,
                       m, K, self._count, ms, cnt, stream)
            for i, k in enumerate(nat.KIND_NAMES):
                tot[k][0] += float(ms[i])
                tot[k][1] += int(cnt[i])
            n -= m
            self._count += m
        return {k: (v[0], v[1]) for k, v in tot.items()}

    def fallback_count(self, clear: bool = False) -> int:
        v = C.c_uint64()
        self._call("mpm_fallback_count", C.byref(self.prob), self._ws, int(clear), C.byref(v), _cuda_stream_handle())
        return int(v.value)

    @property
    def substep_count(self) -> int:
        return self._count

    def __del__(self):
        try:
            self._drop_graphs()
        except Exception:
            pass


def _grid_views(rt: MPMRuntime):
    mm_off, gv_off = C.c_uint64(), C.c_uint64()
    nat.check("mpm_grid_offsets", rt.lib.mpm_grid_offsets(C.byref(rt.prob), C.byref(mm_off), C.byref(gv_off)))
    nodes = rt.n_blocks * nat.MPM_BLOCK**3
    mm = rt.workspace[mm_off.value : mm_off.value + nodes * 16].view(torch.float32).view(nodes, 4)
    gv = rt.workspace[gv_off.value : gv_off.value + nodes * 16].view(torch.float32).view(nodes, 4)
    return mm, gv


MPMRuntime.grid_views = _grid_views


def block_major_to_dense(arr: np.ndarray, spec: InstanceSpec, blk_base: int) -> np.ndarray:
    """[nodes, c] block-major grid slice of one instance -> dense [res_x, res_y, res_z, c]."""
    B = nat.MPM_BLOCK
    nb = spec.nblk
    n_inst = int(np.prod(nb)) * B**3
    a = arr[blk_base * B**3 : blk_base * B**3 + n_inst]
    c = a.shape[-1]
    a = a.reshape(nb[0], nb[1], nb[2], B, B, B, c).transpose(0, 3, 1, 4, 2, 5, 6)
    a = a.reshape(nb[0] * B, nb[1] * B, nb[2] * B, c)
    r = spec.grid_res
    return a[: r[0], : r[1], : r[2]]


def spec_from_desc(desc, materials) -> InstanceSpec:
    return InstanceSpec(
        grid_density=desc.grid_density,
        lower_bound=tuple(desc.lower_bound),
        upper_bound=tuple(desc.upper_bound),
        particle_size=desc.particle_size,
        dt=desc.dt,
        gravity=tuple(desc.gravity),
        materials=materials,
        n_particles=desc.n_particles,
    )


def runtime_from_descs(descs, **kw) -> MPMRuntime:
    """MPMRuntime advancing the given workloads.SceneDesc scenes together."""
    from .. import workloads
    from ..materials import MPM

    specs = [spec_from_desc(d, workloads.make_materials(d, MPM)) for d in descs]
    per_particle = any(d.E_particle is not None for d in descs)
    rt = MPMRuntime(specs, per_particle_lame=per_particle, **kw)
    pos = np.concatenate([d.pos for d in descs]) if descs else np.zeros((0, 3))
    vel = np.concatenate([d.vel for d in descs]) if descs else np.zeros((0, 3))
    mat = np.concatenate([d.mat_idx for d in descs]) if descs else np.zeros(0)
    rt.init_particles(pos, mat, vel=vel)
    if per_particle:
        mus, lams = [], []
        for d, sp in zip(descs, specs):
            nu = sp.materials[0].nu
            E = d.E_particle if d.E_particle is not None else np.full(d.n_particles, sp.materials[0].E)
            mus.append(E / (2.0 * (1.0 + nu)))
            lams.append(E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)))
        rt.set_lame(np.concatenate(mus), np.concatenate(lams))
    return rt
