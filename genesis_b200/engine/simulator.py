"""Simulator: substep orchestration (genesis/engine/simulator.py:268-344)."""

from __future__ import annotations

import numpy as np

from .. import _globals
from .. import _native as nat
from ..exceptions import GenesisException
from .mpm_solver import NAN_MESSAGE, LegacyCoupler, MPMSolver
from .states import MPM_INDEX, SOLVER_NAMES, SimState, ToolSolverState


class Simulator:
    def __init__(self, scene, options, mpm_options, b200_options):
        self._scene = scene
        self.options = options
        self._dt = options.dt
        self._substep_dt = options.dt / options.substeps
        self._substeps = options.substeps
        self._substeps_local = options.substeps_local
        self._requires_grad = options.requires_grad
        self._steps_local = options._steps_local
        self._cur_substep_global = 0
        self._gravity = np.array(options.gravity, dtype=np.float64)
        self._B = 1
        # solver options inherit dt/gravity from SimOptions (scene.py:168-175)
        if mpm_options.dt is None:
            mpm_options.dt = options.dt
        self.mpm_solver = MPMSolver(scene, self, mpm_options, b200_options)
        self._coupler = LegacyCoupler(self)
        self._b200 = b200_options
        self._queried_states = []
        self._pending_status = []  # (pinned status word, event) of steps not yet checked

    def build(self):
        self._B = self._scene._B
        self.mpm_solver.build()

    # -------------------------------------------------------------- stepping
    def step(self, in_backward=False):
        """process_input, then `substeps` substeps (simulator.py:268-292)."""
        self.poll_status()
        if self.mpm_solver.is_active and self.mpm_solver.tape is not None:
            self.mpm_solver.tape.step()  # inputs, substeps and their checkpoint as one autograd node
        else:
            self.process_input(in_backward=in_backward)
            if self.mpm_solver.is_active:
                self.mpm_solver.advance(self._substeps)
        self._cur_substep_global += self._substeps
        if self.mpm_solver.is_active and self._b200.check_nan == "step":
            self.mpm_solver.check_state()
        elif self.mpm_solver.is_active and self._b200.check_nan == "async":
            self._pending_status.append(self.mpm_solver.runtime.status_enqueue())

    def poll_status(self, wait=False):
        """Raise for a NaN found by an earlier step's asynchronous status read (check_nan
        'async'); with wait=True, wait for every pending read first."""
        while self._pending_status:
            word, ev = self._pending_status[0]
            if wait:
                ev.synchronize()
            elif not ev.query():
                return
            self._pending_status.pop(0)
            if int(word[0]) & nat.MPM_STATUS_NAN:
                self._pending_status.clear()
                raise GenesisException(NAN_MESSAGE)

    def process_input(self, in_backward=False):
        if self.mpm_solver.is_active:
            self.mpm_solver.process_input(in_backward=in_backward)

    def substep(self, f):
        """One substep through the solver/coupler plugin interface (simulator.py:317-321)."""
        self._coupler.preprocess(f)
        self.substep_pre_coupling(f)
        self._coupler.couple(f)
        self.substep_post_coupling(f)
        self._cur_substep_global += 1

    def substep_pre_coupling(self, f):
        if self.mpm_solver.is_active:
            self.mpm_solver.substep_pre_coupling(f)

    def substep_post_coupling(self, f):
        if self.mpm_solver.is_active:
            self.mpm_solver.substep_post_coupling(f)

    def get_state(self):
        self.poll_status()
        slots = [None] * len(SOLVER_NAMES)
        slots[MPM_INDEX] = self.mpm_solver.get_state(self.cur_substep_local)
        tools = getattr(self._scene, "_tool_entities", [])
        if tools and self.mpm_solver.is_active:
            ts = ToolSolverState(self._scene)
            ts.entities = [t.get_state() for t in tools]
            slots[SOLVER_NAMES.index("tool")] = ts
        state = SimState(self._scene, self.cur_step_global, slots)
        self._queried_states.append(state)
        return state

    def set_gravity(self, gravity, envs_idx=None):
        raise GenesisException("set_gravity after build is not supported on this path; pass gravity in SimOptions.")

    # ----------------------------------------------------------- properties
    @property
    def scene(self):
        return self._scene

    @property
    def device(self):
        return _globals.device

    @property
    def dt(self):
        return self._dt

    @property
    def substep_dt(self):
        return self._substep_dt

    @property
    def substeps(self):
        return self._substeps

    @property
    def substeps_local(self):
        return self._substeps_local

    @property
    def requires_grad(self):
        return self._requires_grad

    @property
    def gravity(self):
        return self._gravity

    @property
    def coupler(self):
        return self._coupler

    @property
    def cur_substep_global(self):
        return self._cur_substep_global

    @property
    def cur_substep_local(self):
        return self._cur_substep_global % self._substeps_local

    @property
    def cur_step_global(self):
        return self._cur_substep_global // self._substeps

    @property
    def cur_t(self):
        return self._cur_substep_global * self._substep_dt

    @property
    def solvers(self):
        return [self.mpm_solver]

    @property
    def active_solvers(self):
        return [s for s in self.solvers if s.is_active]
