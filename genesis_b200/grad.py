"""Differentiable MPM rollouts: a hand-written, checkpointed adjoint behind
torch.autograd.Function.

The forward pass advances the scene with the ordinary kernels and keeps the particle
state every ``checkpoint_every`` substeps.  The backward pass walks the segments in
reverse: it restores a segment's checkpoint, recomputes the segment once while recording each
substep's input state and grid (mpm_substeps_record), and runs the adjoint of each substep
from the last to the first on those records (mpm_substeps_adjoint_recorded), so no substep's
forward is evaluated twice in the reverse pass.  The recompute of the segment before runs on a
second stream beside that adjoint (neither reads what the other writes), which fills a GPU
that one small scene leaves mostly idle; both are replayed as CUDA graphs captured on first
use (per record buffer and run length).  Memory is one state per checkpoint plus two
segments of states and grids, instead of every substep.

Supported: scenes of any mix of MPM materials (Elastic corotated or neo-Hookean, Muscle,
ElastoPlastic von Mises or clamp, Liquid, Sand, Snow) with per-particle Young's modulus (each
particle's Poisson ratio is its material's); gradients with respect to the initial velocity
(a uniform v0 (3,), as entity.set_velocity sets it, or per particle (N, 3)), the initial
positions (an offset (3,) of the scene's positions, as entity.set_position moves an entity, or
absolute positions (N, 3)), per-particle E (N,) and, for Muscle, per-particle actuation (N,)
(mpm_solver.py:922-949: the reference's actuation gradients; particle_entity.py:415-481: its
state-input gradients).  The plastic materials' state (F and Jp) is carried through the
adjoint.  This replaces the reference's requires_grad path (simulator.py:294-303,
mpm_solver.py:485-517, with the gstaichi autodiff kernels and backward_svd at
mpm_solver.py:1112-1129).
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _native as nat
from .engine.runtime import MPMRuntime, runtime_from_descs, _cuda_stream_handle
from .exceptions import GenesisException


class DifferentiableRollout:
    def __init__(self, desc, checkpoint_every: int = 20, nu: float | None = None):
        kinds = {k for k, _ in desc.materials}
        if not kinds <= {"elastic", "muscle", "elastoplastic", "liquid", "sand", "snow"}:
            raise GenesisException(f"no adjoint for materials {sorted(kinds)}")
        self.muscle = "muscle" in kinds
        self.desc = desc
        self.k = int(checkpoint_every)
        self.T = int(desc.n_substeps)
        # one sort before the rollout, none after: the adjoint walks the same slot order
        self.rt: MPMRuntime = runtime_from_descs([desc], sort_interval=0)
        mats = self.rt.specs[0].materials
        mi = torch.as_tensor(desc.mat_idx, dtype=torch.long, device=self.rt.device)
        nus = torch.tensor([m.nu for m in mats], dtype=torch.float32, device=self.rt.device)
        # each particle's Poisson ratio (the nu argument overrides every material's) and default Jp
        self.nu_p = torch.full_like(mi, float(nu), dtype=torch.float32) if nu is not None else nus[mi]
        self.nu = float(nu if nu is not None else mats[0].nu)
        self.mat_idx = mi.to(torch.uint8)
        self.jp0 = torch.tensor([m.default_Jp for m in mats], dtype=torch.float32, device=self.rt.device)[mi]
        if self.rt.mu_p is None:
            raise GenesisException("the differentiable scene needs per-particle E")
        lib = self.rt.lib
        nbytes = C.c_uint64()
        nat.check("mpm_adjoint_workspace_bytes", lib.mpm_adjoint_workspace_bytes(C.byref(self.rt.prob), C.byref(nbytes)))
        self.adj_ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.rt.device)
        self.adj = torch.zeros_like(self.rt.state)
        # dL/dmu, dL/dlam and (Muscle) dL/dactu per slot
        self.lame_bar = torch.zeros((3, self.rt.stride), dtype=torch.float32, device=self.rt.device)
        if self.muscle:
            mdir = desc.meta.get("muscle_dir")
            if mdir is not None:
                self.rt.muscle_dir[: self.rt.n] = torch.as_tensor(mdir, dtype=torch.float32, device=self.rt.device)
        self.checkpoints: list[torch.Tensor] = []
        self.generation = 0  # forwards so far: a backward must follow its own forward

    def _lame(self, E):
        nu = self.nu_p
        return E / (2.0 * (1.0 + nu)), E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def forward(self, v0: torch.Tensor, E: torch.Tensor, actu: torch.Tensor | None = None,
                x0: torch.Tensor | None = None, record=None) -> torch.Tensor:
        """Final positions [N,3]; with record (substep counts in [0, T]) the positions after each
        of them, [len(record), N, 3] (a loss over a trajectory, as the reference's scripts build
        from get_state() every step)."""
        rt, d = self.rt, self.desc
        self.generation += 1
        self.record = None if record is None else [int(r) for r in record]
        if self.record is not None and any(r < 0 or r > self.T for r in self.record):
            raise GenesisException(f"record substeps must lie in [0, {self.T}]")
        n = rt.n
        dev = rt.device
        v0 = v0.detach().to(dev, torch.float32)
        v0 = v0.reshape(1, 3).expand(n, 3) if v0.numel() == 3 else v0.reshape(n, 3)
        pos = torch.as_tensor(d.pos, dtype=torch.float32, device=dev)
        if x0 is not None:
            x0 = x0.detach().to(dev, torch.float32)
            pos = pos + x0.reshape(1, 3) if x0.numel() == 3 else x0.reshape(n, 3)
        E = E.detach().to(dev, torch.float32).reshape(n)
        if self.muscle:
            a = torch.zeros(n, device=dev) if actu is None else actu.detach().to(dev, torch.float32).reshape(n)
            rt.actu[:n] = a
        rt.load_state(
            pos.contiguous(),
            v0.contiguous(),
            torch.zeros((n, 9), device=dev),
            torch.eye(3, device=dev).reshape(1, 9).repeat(n, 1),
            self.jp0,
            torch.ones(n, dtype=torch.bool, device=dev),
            self.mat_idx,
        )
        mu, lam = self._lame(E)
        rt.set_lame(mu, lam)
        rt._count = 0
        rt.ensure_sorted()  # fixes the slot order for the whole rollout and its adjoint
        self.checkpoints = []
        rec = {}
        if self.record is not None and 0 in self.record:
            rec[0] = rt.get_state(("pos",))["pos"]
        t = 0
        while t < self.T:
            m = min(self.k, self.T - t)
            self.checkpoints.append(rt.state.clone())
            # split at the recorded substeps (the same results: this runtime never re-sorts, and a
            # fused g2p + p2g equals a g2p followed by a p2g)
            stops = sorted({r for r in (self.record or []) if t < r < t + m} | {t + m})
            for r in stops:
                rt.substeps(r - t)
                t = r
                if self.record is not None and r in self.record:
                    rec[r] = rt.get_state(("pos",))["pos"]
        if self.record is None:
            return rt.get_state(("pos",))["pos"]
        return torch.stack([rec[r] for r in self.record])

    def _adjoint_substep(self, state: torch.Tensor):
        rt = self.rt
        par = nat.Particles(
            state=state.data_ptr(), state_stride=rt.stride, mat=rt.mat.data_ptr(), pflags=rt.pflags.data_ptr(),
            gid=rt.gid.data_ptr(), slot=rt.slot.data_ptr(), mu_p=rt.mu_p.data_ptr(), lam_p=rt.lam_p.data_ptr(),
            actu=rt.actu.data_ptr() if self.muscle else None,
            muscle_dir=rt.muscle_dir.data_ptr() if self.muscle else None)
        nat.check("mpm_substep_adjoint", rt.lib.mpm_substep_adjoint(
            C.byref(rt.prob), C.byref(rt.tables), C.byref(par), C.c_void_p(self.adj.data_ptr()),
            C.c_void_p(self.lame_bar.data_ptr()), rt._ws, C.c_void_p(self.adj_ws.data_ptr()), _cuda_stream_handle()))

    def _records(self):
        """Two buffers of per-substep records of one checkpoint segment (one being written
        while the adjoint reads the other): input states [k, 25, stride] and grid records
        (momentum + mass after p2g, velocity after the grid op, the active-block list;
        mpm_record_grid_bytes each), kept across backward calls."""
        rt = self.rt
        if getattr(self, "_rec", None) is None:
            gb = C.c_uint64()
            nat.check("mpm_record_grid_bytes", rt.lib.mpm_record_grid_bytes(C.byref(rt.prob), C.byref(gb)))
            self._rec = [(torch.empty((self.k,) + tuple(rt.state.shape), dtype=torch.float32, device=rt.device),
                          torch.empty(self.k * int(gb.value), dtype=torch.uint8, device=rt.device))
                         for _ in range(2)]
        return self._rec

    def _replay(self, key, launch):
        """Run `launch` (library calls on the current stream, fixed buffers) as a CUDA graph
        captured on first use and replayed on the current stream after."""
        if getattr(self, "_graphs", None) is None:
            self._graphs = {}
        g = self._graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                launch()
            self._graphs[key] = g
        g.replay()

    def _adjoint_recorded(self, first: int, count: int, buf: int):
        if count <= 0:
            return
        rt = self.rt
        rs, rg = self._rec[buf]

        def launch():
            nat.check("mpm_substeps_adjoint_recorded", rt.lib.mpm_substeps_adjoint_recorded(
                C.byref(rt.prob), C.byref(rt.tables), C.byref(rt.par), first, count,
                C.c_void_p(rs.data_ptr()), C.c_void_p(rg.data_ptr()), C.c_void_p(self.adj.data_ptr()),
                C.c_void_p(self.lame_bar.data_ptr()), C.c_void_p(self.adj_ws.data_ptr()), _cuda_stream_handle()))

        self._replay(("adjoint", buf, first, count), launch)

    def backward(self, pos_grad: torch.Tensor):
        """pos_grad: dL/dx_final [N,3] in API order (or, after a forward with record,
        [len(record), N, 3]) -> (dL/dv0 [3], dL/dE [N], dL/dactu [N] or None).  The per-particle
        gradients of the initial positions and velocities, [N,3] in API order, are left in
        x0_grad and v0_grad."""
        rt = self.rt
        n = rt.n
        slot = rt.slot[:n].long()
        self.adj.zero_()
        self.lame_bar.zero_()
        g = pos_grad.to(rt.device, torch.float32)
        # dL/dx at each recorded substep, added to the adjoint when the walk back reaches it
        inject = {}
        if self.record is None:
            inject[self.T] = g.reshape(n, 3)
        else:
            for i, r in enumerate(self.record):
                inject[r] = inject[r] + g[i].reshape(n, 3) if r in inject else g[i].reshape(n, 3)

        def add(r):
            if r in inject:
                self.adj[0:3, slot] += inject[r].t()

        add(self.T)
        final = rt.state.clone()
        recs = self._records()
        main = torch.cuda.current_stream(rt.device)
        if getattr(self, "_side", None) is None:
            self._side = torch.cuda.Stream(device=rt.device)
        side = self._side
        lib = rt.lib
        nseg = len(self.checkpoints)
        rec_done: list = [None] * nseg
        adj_done: list = [None] * nseg

        def record(c):
            # recompute segment c once on the side stream, recording each substep's input state
            # and grid into buffer c % 2, after the adjoint that last read that buffer (c + 2)
            t0, t1 = c * self.k, min((c + 1) * self.k, self.T)
            rs, rg = recs[c % 2]

            def launch():
                nat.check("mpm_substeps_record", lib.mpm_substeps_record(
                    C.byref(rt.prob), C.byref(rt.tables), C.byref(rt.par), rt._ws, t1 - t0,
                    C.c_void_p(rs.data_ptr()), C.c_void_p(rg.data_ptr()), _cuda_stream_handle()))

            with torch.cuda.stream(side):
                if c + 2 < nseg:
                    side.wait_event(adj_done[c + 2])
                rt.state.copy_(self.checkpoints[c])
                self._replay(("record", c % 2, t1 - t0), launch)
                rec_done[c] = torch.cuda.Event()
                rec_done[c].record(side)

        side.wait_stream(main)
        record(nseg - 1)
        for ci in range(nseg - 1, -1, -1):
            if ci > 0:
                record(ci - 1)  # runs beside this segment's adjoint: it reads only the records
            t0, t1 = ci * self.k, min((ci + 1) * self.k, self.T)
            m = t1 - t0
            main.wait_event(rec_done[ci])
            # the adjoint of substeps m-1 .. 0, split where dL/dx of an interior substep enters
            hi = m
            for j in range(m - 1, -1, -1):
                r = t0 + j + 1
                if r != self.T and r in inject:
                    self._adjoint_recorded(j + 1, hi - j - 1, ci % 2)
                    add(r)
                    hi = j + 1
            self._adjoint_recorded(0, hi, ci % 2)
            adj_done[ci] = torch.cuda.Event()
            adj_done[ci].record(main)
        main.wait_stream(side)
        add(0)
        rt.state.copy_(final)
        gid = rt.gid[:n].long()
        self.x0_grad = torch.empty((n, 3), dtype=torch.float32, device=rt.device)
        self.x0_grad[gid] = self.adj[0:3, :n].t()
        self.v0_grad = torch.empty((n, 3), dtype=torch.float32, device=rt.device)
        self.v0_grad[gid] = self.adj[3:6, :n].t()
        vbar = self.adj[3:6, :n].sum(dim=1)
        nu = self.nu_p[gid]  # the slot order's Poisson ratios
        Ebar_slot = self.lame_bar[0, :n] / (2.0 * (1.0 + nu)) + self.lame_bar[1, :n] * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        Ebar = torch.empty(n, dtype=torch.float32, device=rt.device)
        Ebar[gid] = Ebar_slot
        abar = None
        if self.muscle:
            abar = torch.empty(n, dtype=torch.float32, device=rt.device)
            abar[gid] = self.lame_bar[2, :n]
        return vbar, Ebar, abar


class _RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v0, E, actu, x0, sim, record):
        ctx.sim = sim
        ctx.generation = sim.generation + 1
        ctx.v0_per_particle = v0.numel() != 3
        ctx.x0_shape = None if x0 is None else tuple(x0.shape)
        return sim.forward(v0, E, actu, x0, record)

    @staticmethod
    def backward(ctx, grad_pos):
        sim = ctx.sim
        if sim.generation != ctx.generation:
            raise GenesisException("this rollout's checkpoints were replaced by a later forward of the same "
                                   "DifferentiableRollout; call backward before the next forward")
        v0b, Eb, ab = sim.backward(grad_pos)
        if ctx.v0_per_particle:
            v0b = sim.v0_grad
        x0b = None
        if ctx.x0_shape is not None:
            x0b = sim.x0_grad.sum(0).reshape(ctx.x0_shape) if len(ctx.x0_shape) < 2 else sim.x0_grad
        return v0b, Eb, ab, x0b, None, None


def rollout(v0: torch.Tensor, E: torch.Tensor, sim: DifferentiableRollout, actu: torch.Tensor | None = None,
            x0: torch.Tensor | None = None, record=None):
    """Final particle positions [N,3] of the rollout (or, with record, the positions after each
    listed substep count, [len(record), N, 3]), differentiable w.r.t. the initial velocity v0
    ((3,) uniform or (N,3)), the initial positions x0 (None: the scene's; (3,): an offset of
    them; (N,3): absolute), E and (for a Muscle scene) the per-particle actuation."""
    if sim.muscle and actu is None:
        actu = torch.zeros(sim.rt.n, device=sim.rt.device)
    return _RolloutFunction.apply(v0, E, actu, x0, sim, record)
