"""Scene: the user-facing build/step/state API (genesis/engine/scene.py:91-936)."""

from __future__ import annotations

import logging

import torch

from .. import _globals
from .. import materials as _materials
from ..exceptions import GenesisException
from ..options import B200Options, LegacyCouplerOptions, MPMOptions, SimOptions
from .simulator import Simulator
from .states import MPM_INDEX, SimState

log = logging.getLogger("genesis_b200")


class Scene:
    def __init__(
        self,
        sim_options: SimOptions | None = None,
        coupler_options=None,
        mpm_options: MPMOptions | None = None,
        vis_options=None,
        viewer_options=None,
        profiling_options=None,
        renderer=None,
        show_viewer: bool | None = None,
        show_FPS: bool | None = None,
        b200_options: B200Options | None = None,
        **other_solver_options,
    ):
        if not _globals.initialized:
            raise GenesisException("Genesis hasn't been initialized. Did you call `gs.init()`?")
        if show_viewer:
            log.warning("show_viewer ignored: this build has no viewer (graphics are out of scope).")
        self.sim_options = sim_options or SimOptions()
        self.coupler_options = coupler_options or LegacyCouplerOptions()
        self.mpm_options = mpm_options or MPMOptions()
        self.b200_options = b200_options or B200Options()
        from ..options import VisOptions

        self.vis_options = vis_options or VisOptions()
        self._other = other_solver_options
        self._sim = Simulator(self, self.sim_options, self.mpm_options, self.b200_options)
        self._entities = []
        self._rigid_entities = []  # kinematic colliders of the MPM grid op
        self._tool_entities = []  # tools, coupled before the rigid geoms
        self._emitters = []
        self._force_fields = []
        self._is_built = False
        self._B = 1
        self._n_envs = 0
        self._envs_idx = torch.zeros(1, dtype=torch.int64)
        self._init_state = None

    # ---------------------------------------------------------------- build
    def add_entity(self, morph, material=None, surface=None, visualize_contact=False, vis_mode=None):
        if self._is_built:
            raise GenesisException("Scene is already built.")
        if material is None:  # scene.py:355-356: a Rigid entity by default
            material = _materials.Rigid()
        if isinstance(material, _materials.Rigid):
            from .rigid import KinematicRigidEntity

            ent = KinematicRigidEntity(self, len(self._entities), material, morph,
                                       exact_box_sdf=self.b200_options.exact_box_sdf)
            self._entities.append(ent)
            if material.needs_coup:
                self._rigid_entities.append(ent)
            return ent
        if isinstance(material, _materials.Tool):
            from .tool import ToolEntity

            ent = ToolEntity(self, len(self._entities), material, morph, surface)
            self._entities.append(ent)
            self._tool_entities.append(ent)
            return ent
        if material is None or not isinstance(material, _materials.MPM.Base):
            raise GenesisException("Only gs.materials.MPM.*, gs.materials.Rigid and gs.materials.Tool entities are "
                                   "supported by this build.")
        ent = self._sim.mpm_solver.add_entity(len(self._entities), material, morph, surface, rng=_globals.rng)
        self._entities.append(ent)
        return ent

    def add_emitter(self, material, max_particles=20000, surface=None):
        """A particle emitter backed by a Nowhere entity of max_particles inactive particles
        (scene.py:664-718); particles are recycled once the limit is reached."""
        from ..morphs import Nowhere
        from .emitter import Emitter

        if self.sim_options.requires_grad:
            raise GenesisException("Emitter is not supported in differentiable mode.")
        if not isinstance(material, _materials.MPM.Base):
            raise GenesisException("Non-supported material for emitter. Supported materials are: `gs.materials.MPM.Base`.")
        emitter = Emitter(max_particles)
        entity = self.add_entity(morph=Nowhere(n_particles=max_particles), material=material, surface=surface)
        emitter.set_entity(entity)
        self._emitters.append(emitter)
        return emitter

    @property
    def emitters(self):
        return self._emitters

    def add_force_field(self, force_field):
        """Register an external acceleration field of the MPM grid op (scene.py:720-736); it acts
        once activated."""
        from .. import force_fields as _ff

        if self._is_built:
            raise GenesisException("Scene is already built.")
        if not isinstance(force_field, _ff.ForceField):
            raise GenesisException("`force_field` must be a gs.force_fields.ForceField.")
        if isinstance(force_field, _ff.Custom):
            raise GenesisException("Custom force fields (a gstaichi function) are not supported.")
        if self.sim_options.requires_grad and isinstance(force_field, _ff.Noise):
            raise GenesisException("The Noise force field is not supported in differentiable mode (its draws are "
                                   "not replayed by the backward pass).")
        force_field.scene = self
        self._force_fields.append(force_field)
        return force_field

    @property
    def force_fields(self):
        return self._force_fields

    def build(self, n_envs=0, env_spacing=(0.0, 0.0), n_envs_per_row=None, center_envs_at_origin=True,
              compile_kernels=None):
        if self._is_built:
            raise GenesisException("Scene is already built.")
        self._n_envs = int(n_envs)
        self._B = max(1, self._n_envs)
        self._envs_idx = torch.arange(self._B, dtype=torch.int64, device=_globals.device)
        self._sim.build()
        self._is_built = True
        self._init_state = self.get_state() if self._sim.mpm_solver.is_active else None
        if self._init_state is not None:
            self._init_state.serializable()
        self._sim._queried_states.clear()

    def _sanitize_envs_idx(self, envs_idx=None):
        if envs_idx is None:
            return self._envs_idx
        t = torch.as_tensor(envs_idx, dtype=torch.int64, device=self._envs_idx.device).reshape(-1)
        if (t < 0).any() or (t >= self._B).any():
            raise GenesisException("`envs_idx` exceeds valid range.")
        return t

    # ---------------------------------------------------------------- step
    def step(self, update_visualizer=True, refresh_visualizer=True):
        if not self._is_built:
            raise GenesisException("Scene is not built yet.")
        self._sim.step()

    def check_state(self):
        """Explicit NaN check (one host sync); also settles the pending asynchronous checks."""
        self._sim.poll_status(wait=True)
        return self._sim.mpm_solver.check_state()

    def get_state(self):
        return self._sim.get_state()

    def reset(self, state: SimState | None = None, envs_idx=None):
        if not self._is_built:
            raise GenesisException("Scene is not built yet.")
        self._sim.poll_status()
        if state is None:
            state = self._init_state
        if state is not None:
            mpm_state = state.solvers_state[MPM_INDEX] if isinstance(state, SimState) else state
            self._sim.mpm_solver.set_state(0, mpm_state, envs_idx=envs_idx)
        self._sim._queried_states.clear()  # simulator.py:227, 238
        for emitter in self._emitters:  # scene.py:893-895
            emitter.reset()
        if envs_idx is None:
            self._sim._cur_substep_global = 0
            if self._sim.mpm_solver.is_active:
                self._sim.mpm_solver.runtime.reset_colliders()
                if self._sim.mpm_solver.tape is not None:
                    self._sim.mpm_solver.tape.reset()  # a new differentiable rollout
                tool_state = state.solvers_state[0] if isinstance(state, SimState) else None
                if tool_state is not None:  # the tool solver's set_state (tool_solver.py:70-74)
                    for t, ts in zip(self._tool_entities, tool_state.entities):
                        t.set_state(0, ts)

    def save_checkpoint(self, path):
        st = self.get_state()[MPM_INDEX]
        torch.save({k: getattr(st, k).cpu() for k in ("pos", "vel", "C", "F", "Jp", "active")} |
                   {"cur_substep_global": self._sim.cur_substep_global}, path)

    def load_checkpoint(self, path):
        d = torch.load(path)
        from .states import MPMSolverState

        st = MPMSolverState(self, d["pos"], d["vel"], d["C"], d["F"], d["Jp"], d["active"])
        self._sim.mpm_solver.set_state(0, st)
        self._sim._cur_substep_global = int(d["cur_substep_global"])

    # ----------------------------------------------------------- properties
    @property
    def sim(self):
        return self._sim

    @property
    def mpm_solver(self):
        return self._sim.mpm_solver

    @property
    def entities(self):
        return self._entities

    @property
    def is_built(self):
        return self._is_built

    @property
    def n_envs(self):
        return self._n_envs

    @property
    def dt(self):
        return self._sim.dt

    @property
    def substeps(self):
        return self._sim.substeps

    @property
    def t(self):
        return self._sim.cur_step_global

    @property
    def cur_t(self):
        return self._sim.cur_t

    @property
    def requires_grad(self):
        return self._sim.requires_grad

    @property
    def solvers(self):
        return self._sim.solvers

    @property
    def active_solvers(self):
        return self._sim.active_solvers
