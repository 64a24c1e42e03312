"""Scene-level differentiation: `SimOptions(requires_grad=True)` scenes.

Replaces the reference's differentiable scene (simulator.py:294-344 `_step_grad` /
`sub_step_grad`, scene.py:1267-1281 `_backward`, grad/tensor.py:73-79 `gs.Tensor.backward`,
particle_entity.py:415-481 `process_input_grad`, mpm_entity.py:245-264) with torch autograd
nodes over the checkpointed CUDA adjoint (mpm_substep_adjoint):

* every `scene.step()` is one `_Step` node.  Its inputs are the previous step's handle (a
  one-element tensor that only orders the nodes) and the tensors given to the entities'
  `set_position` / `set_velocity` / `set_actuation` for that step; it saves the particle state
  after those inputs as its checkpoint and returns the next handle;
* every `scene.get_state()` (or entity `get_state()` / `get_particles_*`) is a `_Query` node on
  the current handle whose outputs are the state tensors.

`loss.backward()` then needs no scene call: autograd runs every query of a state and the step
that consumes it before the step that produced it, so when `_Step.backward` of step s runs, the
adjoint buffer holds dL/d(state after step s) minus the queries of that state, which it adds;
it recomputes the step's substeps from its checkpoint (once, recording each substep's input state
and grid, mpm_substeps_record, when no collider moves), runs their adjoints in reverse, reads
the gradients of the step's inputs (undoing them in reverse order: the state components an
input overwrote get a zero adjoint) and leaves dL/d(state before step s) for the step before.
Actuation persists until it is set again, so its gradient accumulates across steps and is
consumed by the step that set it.

Tools (tool_entity.py) are differentiated too: their `set_position` / `set_velocity` inputs are
step inputs like the particles', the step's checkpoint holds the collider table, and the backward
recomputes each substep's collider poses, runs mpm_substep_adjoint_colliders with each substep's
table (dL/d(tool position, linear velocity) through that substep's grid op) and chains
pos' = pos + lin_vel dt (kept above the floor) back through the substeps.  Rigid geoms act as
colliders whose pose carries no gradient; the particle-level coupling (CPIC) is refused.

Scope (the adjoint's): every MPM material (Elastic, Muscle, ElastoPlastic, Liquid, Sand,
Snow), tool and rigid colliders, no emitters; particle positions may be set only before the first
step (setting them later re-bins the particles, which would change the slot order the adjoint
walks in); tools' rotations and angular velocities carry no gradient.
"""

from __future__ import annotations

import ctypes as C

import torch

from .. import _native as nat
from ..exceptions import GenesisException
from .runtime import _cuda_stream_handle

# the order entity.process_input applies them in (tools: position, then velocities)
_KIND_ORDER = {"pos": 0, "vel": 1, "actu": 2, "tool_pos": 0, "tool_vel": 1, "tool_ang": 1}
_TOOL_KINDS = ("tool_pos", "tool_vel", "tool_ang")


class SceneTape:
    def __init__(self, solver):
        self.solver = solver
        rt = solver.runtime
        self.rt = rt
        if rt.mu_p is None:
            raise GenesisException("the differentiable runtime needs per-particle Lame parameters")
        nbytes = C.c_uint64()
        nat.check("mpm_adjoint_workspace_bytes", rt.lib.mpm_adjoint_workspace_bytes(C.byref(rt.prob), C.byref(nbytes)))
        self.adj_ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=rt.device)
        self.adj = torch.zeros_like(rt.state)  # dL/d(state), slot order
        self.lame_bar = torch.zeros((3, rt.stride), dtype=torch.float32, device=rt.device)
        self.muscle = rt.actu is not None
        nc = rt.n_colliders if rt.coll_table is not None else 0
        self.n_colliders = nc
        # dL/d(collider position, linear velocity) at the cursor, and one substep's share
        self.tool_bar = torch.zeros((max(nc, 1), 6), dtype=torch.float32, device=rt.device)
        self.cbar = torch.zeros_like(self.tool_bar)
        if nc:
            if rt.prob.flags & nat.PROBF_CPIC:
                raise GenesisException("A differentiable scene does not take the particle-level rigid coupling "
                                       "(enable_CPIC).")
            head = rt.coll_table.view(torch.int32).view(nc, C.sizeof(nat.Collider) // 4)[:, :2].cpu()
            self._col_is_tool = (head[:, 0] == nat.COLLIDER_TOOL).to(rt.device)
            self._col_dt = torch.as_tensor([rt.specs[int(i)].dt for i in head[:, 1]], dtype=torch.float32,
                                           device=rt.device)
        self.reset()

    def reset(self):
        self.handle = torch.zeros(1, device=self.rt.device, requires_grad=True)
        self.n_steps = 0
        self.pending = []  # (entity, kind, value, envs_idx) for the next step
        self.inject = {}  # state index -> dL/d(state) of its queries, slot order
        self.cursor = None  # the state index the adjoint buffer currently stands for
        self.step_inputs = []  # the input tensors of every step
        self.bw_latest = None  # the latest step of the running backward pass

    # ------------------------------------------------------------------ forward
    def record_input(self, entity, kind, value, envs_idx):
        if kind in _TOOL_KINDS:
            if not isinstance(value, torch.Tensor):
                value = torch.as_tensor(value, dtype=torch.float32)
            self.pending.append((entity, kind, value.to(self.rt.device, torch.float32), envs_idx))
            return
        if kind == "pos" and self.n_steps > 0:
            raise GenesisException("In a differentiable scene, positions can be set only before the first step.")
        if not isinstance(value, torch.Tensor):
            value = torch.as_tensor(value, dtype=torch.float32)
        self.pending.append((entity, kind, value.to(self.rt.device, torch.float32), envs_idx))

    def step(self):
        inputs = sorted(self.pending, key=lambda t: (_KIND_ORDER[t[1]], t[0].idx))
        self.pending = []
        meta = [(e, k, envs) for e, k, _, envs in inputs]
        self.step_inputs.append([v for _, _, v, _ in inputs])
        self.handle = _Step.apply(self, self.n_steps, meta, self.handle, *[v for _, _, v, _ in inputs])
        self.n_steps += 1

    def _zero_later_inputs(self):
        """Inputs of the steps after the loss's latest state get a zero gradient (a leaf that
        requires grad and has none), as the reference's scene backward gives every input of the
        recorded steps one (gs.Tensor.backward, grad/tensor.py:73-79)."""
        for vals in self.step_inputs[self.bw_latest + 1:]:
            for v in vals:
                if v.is_leaf and v.requires_grad and v.grad is None:
                    v.grad = torch.zeros_like(v)

    def query(self):
        return _Query.apply(self, self.n_steps, self.handle)

    # ------------------------------------------------------------------ helpers
    def _apply(self, entity, kind, value, envs):
        if kind in _TOOL_KINDS:
            entity._apply_input(kind, value)
        elif kind == "pos":
            entity._apply_position(value, envs)
        elif kind == "vel":
            entity._apply_velocity(value, envs)
        else:
            entity._apply_actuation(value, envs)

    def _adjoint_substep(self, state):
        rt = self.rt
        par = nat.Particles(
            state=state.data_ptr(), state_stride=rt.stride, mat=rt.mat.data_ptr(), pflags=rt.pflags.data_ptr(),
            gid=rt.gid.data_ptr(), slot=rt.slot.data_ptr(), mu_p=rt.mu_p.data_ptr(), lam_p=rt.lam_p.data_ptr(),
            actu=rt.actu.data_ptr() if self.muscle else None,
            muscle_dir=rt.muscle_dir.data_ptr() if self.muscle else None)
        cb = None
        if self.n_colliders:
            self.cbar.zero_()
            cb = C.c_void_p(self.cbar.data_ptr())
        nat.check("mpm_substep_adjoint_colliders", rt.lib.mpm_substep_adjoint_colliders(
            C.byref(rt.prob), C.byref(rt.tables), C.byref(par), C.c_void_p(self.adj.data_ptr()),
            C.c_void_p(self.lame_bar.data_ptr()), cb, rt._ws, C.c_void_p(self.adj_ws.data_ptr()),
            _cuda_stream_handle()))
        if self.n_colliders:
            self.tool_bar += self.cbar

    def _adjoint_step_recorded(self, m: int):
        rt = self.rt
        if getattr(self, "_rec", None) is None or self._rec[0].shape[0] != m:
            gb = C.c_uint64()
            nat.check("mpm_record_grid_bytes", rt.lib.mpm_record_grid_bytes(C.byref(rt.prob), C.byref(gb)))
            self._rec = (torch.empty((m,) + tuple(rt.state.shape), dtype=torch.float32, device=rt.device),
                         torch.empty(m * int(gb.value), dtype=torch.uint8, device=rt.device))
        rs, rg = self._rec
        stream = _cuda_stream_handle()
        nat.check("mpm_substeps_record", rt.lib.mpm_substeps_record(
            C.byref(rt.prob), C.byref(rt.tables), C.byref(rt.par), rt._ws, m, C.c_void_p(rs.data_ptr()),
            C.c_void_p(rg.data_ptr()), stream))
        par = nat.Particles.from_buffer_copy(rt.par)
        if not self.muscle:
            par.actu = None
            par.muscle_dir = None
        nat.check("mpm_substeps_adjoint_recorded", rt.lib.mpm_substeps_adjoint_recorded(
            C.byref(rt.prob), C.byref(rt.tables), C.byref(par), 0, m, C.c_void_p(rs.data_ptr()),
            C.c_void_p(rg.data_ptr()), C.c_void_p(self.adj.data_ptr()), C.c_void_p(self.lame_bar.data_ptr()),
            C.c_void_p(self.adj_ws.data_ptr()), stream))

    def _chain_colliders(self, cols):
        """Carry dL/d(pose after a substep) back over its motion pos' = pos + lin_vel dt (a
        tool's z held at its floor where pos_z + v_z dt falls below it), cols the collider
        rows at the substep's start (collider_table layout)."""
        dt = self._col_dt
        pb = self.tool_bar[: self.n_colliders, 0:3].clone()
        z_next = cols[:, 2] + cols[:, 17] * dt
        held = self._col_is_tool & (z_next < cols[:, 31])
        pb[:, 2] = torch.where(held, torch.zeros_like(pb[:, 2]), pb[:, 2])
        self.tool_bar[: self.n_colliders, 0:3] = pb
        self.tool_bar[: self.n_colliders, 3:6] += pb * dt[:, None]


class _Step(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tape, s, meta, handle, *values):
        rt, solver = tape.rt, tape.solver
        for (entity, kind, envs), v in zip(meta, values):
            tape._apply(entity, kind, v.detach(), envs)
        solver.process_input()  # the non-differentiable targets (activeness) as usual
        if not getattr(rt, "_sorted_once", False) or rt._dirty:  # the slot order is fixed from here on
            rt.sort()
            rt._sorted_once = True
            rt._dirty = False
        ctx.tape, ctx.s, ctx.meta = tape, s, meta
        ctx.shapes = [tuple(v.shape) for v in values]
        ctx.ckpt = rt.state.clone()
        ctx.actu = rt.actu.clone() if tape.muscle else None
        ctx.cols = rt.collider_table().clone() if tape.n_colliders else None
        solver.advance(solver._sim.substeps)
        return handle.new_zeros(1)

    @staticmethod
    def backward(ctx, g_handle):
        tape, rt, s = ctx.tape, ctx.tape.rt, ctx.s
        if tape.cursor != s + 1:  # the latest step of this backward pass
            tape.adj.zero_()
            tape.lame_bar.zero_()
            tape.tool_bar.zero_()
            tape.bw_latest = s
        inj = tape.inject.pop(s + 1, None)
        if inj is not None:
            tape.adj += inj
        live = rt.state.clone()
        live_actu = rt.actu.clone() if tape.muscle else None
        live_cols = rt.collider_table().clone() if tape.n_colliders else None
        live_force = rt.collider_force.clone() if rt.collider_force is not None else None
        rt.state.copy_(ctx.ckpt)
        if tape.muscle:
            rt.actu.copy_(ctx.actu)
        if tape.n_colliders:
            rt.collider_table().copy_(ctx.cols)
        if tape.n_colliders:
            states = []
            for _ in range(tape.solver._sim.substeps):  # recompute the step, one state per substep
                states.append((rt.state.clone(), rt.collider_table().clone()))
                rt.substeps(1)
            for st, cols in reversed(states):
                tape._chain_colliders(cols)
                rt.collider_table().copy_(cols)  # the substep's poses, for its grid op's adjoint
                tape._adjoint_substep(st)
        else:
            # no collider moves between substeps: recompute the step once, recording each
            # substep's input state and grid, and run the adjoints on the records
            tape._adjoint_step_recorded(tape.solver._sim.substeps)
        rt.state.copy_(live)
        if tape.muscle:
            rt.actu.copy_(live_actu)
        if tape.n_colliders:
            rt.collider_table().copy_(live_cols)
        if live_force is not None:  # the recompute added to the reported reaction forces
            rt.collider_force.copy_(live_force)
        grads = [None] * len(ctx.meta)
        for i in range(len(ctx.meta) - 1, -1, -1):  # undo the inputs, the last applied first
            entity, kind, envs = ctx.meta[i]
            if kind in _TOOL_KINDS:
                rows = entity._rows
                cols = slice(0, 3) if kind == "tool_pos" else slice(3, 6)
                if kind == "tool_ang":
                    grads[i] = torch.zeros(ctx.shapes[i], device=rt.device)
                    continue
                g = tape.tool_bar[rows, cols].clone()
                tape.tool_bar[rows, cols] = 0.0  # the input overwrote that state
                grads[i] = entity._input_grad(ctx.shapes[i], g)
                continue
            idx = entity._flat_idx(None, envs)  # [n_envs, n_particles] runtime ids
            slots = rt.slot[idx.reshape(-1)].long()
            if kind == "actu":
                g = tape.lame_bar[2, slots].reshape(idx.shape)  # dL/dactu per particle
                tape.lame_bar[2, slots] = 0.0
            else:
                rows = slice(0, 3) if kind == "pos" else slice(3, 6)
                g = tape.adj[rows, slots].t().reshape(idx.shape + (3,))
                if kind == "pos":
                    tape.adj[:, slots] = 0.0  # set_particles_pos resets v, C, F and Jp as well
                else:
                    tape.adj[3:6, slots] = 0.0
            grads[i] = entity._input_grad(kind, ctx.shapes[i], g, envs)
        tape.cursor = s
        if s == 0:
            tape._zero_later_inputs()
        return (None, None, None, torch.zeros_like(g_handle), *grads)


class _Query(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tape, s, handle):
        rt, solver = tape.rt, tape.solver
        st = rt.get_state(("pos", "vel", "C", "F", "Jp"))
        B, N = solver._B, solver.n_particles
        ctx.tape, ctx.s = tape, s
        return (st["pos"].reshape(B, N, 3), st["vel"].reshape(B, N, 3), st["C"].reshape(B, N, 3, 3),
                st["F"].reshape(B, N, 3, 3), st["Jp"].reshape(B, N))

    @staticmethod
    def backward(ctx, g_pos, g_vel, g_C, g_F, g_Jp):
        tape = ctx.tape
        rt = tape.rt
        n = rt.n
        slot = rt.slot[:n].long()
        inj = torch.zeros_like(rt.state)
        for g, rows, w in ((g_pos, slice(0, 3), 3), (g_vel, slice(3, 6), 3), (g_C, slice(6, 15), 9),
                           (g_F, slice(15, 24), 9), (g_Jp, slice(24, 25), 1)):
            if g is not None:
                inj[rows, slot] = g.reshape(n, w).t().to(torch.float32)
        prev = tape.inject.get(ctx.s)
        tape.inject[ctx.s] = inj if prev is None else prev + inj
        return None, None, torch.zeros(1, device=rt.device)
