"""State containers (genesis/engine/states/solvers.py:5-198, states/entities.py)."""

from __future__ import annotations


class MPMSolverState:
    """Dynamic state of the MPM solver: pos/vel [B,N,3], C/F [B,N,3,3], Jp [B,N], active [B,N] bool."""

    def __init__(self, scene, pos, vel, C, F, Jp, active):
        self._scene = scene
        self._pos, self._vel, self._C, self._F, self._Jp, self._active = pos, vel, C, F, Jp, active

    def serializable(self):
        self._scene = None
        for k in ("_pos", "_vel", "_C", "_F", "_Jp", "_active"):
            setattr(self, k, getattr(self, k).detach())

    @property
    def scene(self):
        return self._scene

    @property
    def pos(self):
        return self._pos

    @property
    def vel(self):
        return self._vel

    @property
    def C(self):
        return self._C

    @property
    def F(self):
        return self._F

    @property
    def Jp(self):
        return self._Jp

    @property
    def active(self):
        return self._active


class MPMEntityState(MPMSolverState):
    """Per-entity slice of the solver state (states/entities.py: MPMEntityState)."""

    def __init__(self, entity, s_global, pos, vel, C, F, Jp, active):
        super().__init__(entity.scene, pos, vel, C, F, Jp, active)
        self._entity = entity
        self._s_global = s_global

    @property
    def entity(self):
        return self._entity

    @property
    def s_global(self):
        return self._s_global


class ToolSolverState:
    """The tools' states, one ToolEntityState per tool entity (states/solvers.py:114-133)."""

    def __init__(self, scene):
        self.scene = scene
        self.entities = []

    def serializable(self):
        self.scene = None
        for st in self.entities:
            st.serializable()

    def __len__(self):
        return len(self.entities)

    def __getitem__(self, index):
        return self.entities[index]


# the reference's solver order (simulator.py:129-140): a scene's state has one entry per solver,
# None for the solvers that are not active; only the MPM solver exists here
SOLVER_NAMES = ("tool", "rigid", "avatar", "mpm", "sph", "pbd", "fem", "sf")
MPM_INDEX = SOLVER_NAMES.index("mpm")


class SimState:
    """Scene-level state: one entry per solver, in the reference's order, so the MPM state is
    solvers_state[3] as scripts written for the reference index it (states/solvers.py:5-45)."""

    def __init__(self, scene, s_global, solvers_state):
        self._scene = scene
        self._s_global = s_global
        self._solvers_state = list(solvers_state)

    def serializable(self):
        self._scene = None
        for st in self._solvers_state:
            if st is not None:
                st.serializable()

    @property
    def scene(self):
        return self._scene

    @property
    def s_global(self):
        return self._s_global

    @property
    def solvers_state(self):
        return self._solvers_state

    def __iter__(self):
        return iter(self._solvers_state)

    def __getitem__(self, i):
        return self._solvers_state[i]
