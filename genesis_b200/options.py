"""gs.options for the MPM path: SimOptions, MPMOptions (genesis/options/solvers.py)
plus B200Options, the tuning knobs of this implementation."""

from __future__ import annotations

from typing import Optional

import numpy as np

from .exceptions import GenesisException


class Options:
    """Keyword-only option record with defaults taken from class attributes."""

    def __init__(self, **data):
        fields = self._fields()
        for k in data:
            if k not in fields:
                raise GenesisException(f"Unrecognized attribute: {k} for {type(self).__name__}")
        for k, default in fields.items():
            setattr(self, k, data.get(k, default))

    @classmethod
    def _fields(cls):
        out = {}
        for klass in reversed(cls.__mro__):
            for k, v in vars(klass).items():
                if not k.startswith("__") and not callable(v) and not isinstance(v, (property, classmethod, staticmethod)):
                    out[k] = v
        return out

    def copy_attributes_from(self, other, override=False):
        for k in self._fields():
            if hasattr(other, k) and (override or getattr(self, k) is None):
                setattr(self, k, getattr(other, k))

    def __repr__(self):
        body = ", ".join(f"{k}={getattr(self, k)!r}" for k in self._fields() if not k.startswith("_"))
        return f"{type(self).__name__}({body})"


class SimOptions(Options):
    """Top-level simulator options (options/solvers.py:15-68)."""

    dt: float = 1e-2
    substeps: int = 1
    substeps_local: Optional[int] = None
    gravity: tuple = (0.0, 0.0, -9.81)
    floor_height: float = 0.0
    requires_grad: bool = False
    _steps_local: Optional[int] = None

    def __init__(self, **data):
        super().__init__(**data)
        if self.substeps_local is None:
            self.substeps_local = self.substeps if self.requires_grad else 1
        if self.requires_grad:
            if self.substeps_local % self.substeps != 0:
                raise GenesisException("`substeps_local` must be divisible by `substeps` when `requires_grad` is True.")
            self._steps_local = int(self.substeps_local / self.substeps)
        else:
            self._steps_local = None


class ToolOptions(Options):
    """Tool solver options (options/solvers.py:265-290): floor_height None takes the
    SimOptions one; dt is the simulator's."""

    dt: Optional[float] = None
    floor_height: Optional[float] = None


class LegacyCouplerOptions(Options):
    """Accepted for API compatibility; only the MPM grid update of the legacy coupler is on this path."""

    dt: Optional[float] = None
    enable_collision: bool = False


class MPMOptions(Options):
    """MPMSolver options (options/solvers.py:443-493)."""

    dt: Optional[float] = None
    gravity: Optional[tuple] = None
    particle_size: Optional[float] = None
    grid_density: float = 64
    enable_CPIC: bool = False
    lower_bound: tuple = (-1.0, -1.0, 0.0)
    upper_bound: tuple = (1.0, 1.0, 1.0)
    use_sparse_grid: bool = False
    leaf_block_size: int = 8

    def __init__(self, **data):
        super().__init__(**data)
        if not np.all(np.asarray(self.upper_bound) > np.asarray(self.lower_bound)):
            raise GenesisException("Invalid pair of upper_bound and lower_bound.")
        if self.particle_size is None:
            self.particle_size = 0.01 * 64.0 / self.grid_density


class B200Options(Options):
    """Tuning of the CUDA path (no reference counterpart).

    sort_interval    re-bin particles by grid block every this many substeps
    chunk_particles  particles per p2g/g2p work item: 128, 256 or 512
    use_cuda_graph   replay sort_interval substeps as one captured CUDA graph
    check_nan        'step' (raise at the end of a step, one host sync per step),
                     'async' (the step enqueues a non-blocking read of the status word;
                     the first scene call after it has arrived raises; scene.check_state()
                     waits for it),
                     'never' (call scene.check_state() yourself)
    exact_box_sdf    couple Box rigid entities through the exact box distance instead of the
                     sampled signed-distance grid the reference uses for every non-analytic geom
    """

    sort_interval: int = 50
    chunk_particles: int = 128
    use_cuda_graph: bool = True
    check_nan: str = "step"
    grid_ctas: int = 0
    exact_box_sdf: bool = False

    def __init__(self, **data):
        super().__init__(**data)
        if self.check_nan not in ("step", "async", "never"):
            raise GenesisException(f"check_nan must be 'step', 'async' or 'never', got {self.check_nan!r}")


class VisOptions(Options):
    """Accepted and ignored: there is no visualiser on this path."""

    visualize_mpm_boundary: bool = False
    n_support_neighbors: int = 12


class ViewerOptions(Options):
    """Accepted and ignored: there is no viewer on this path."""

    camera_pos: tuple = (3.5, 0.5, 2.5)
    camera_lookat: tuple = (0.0, 0.0, 0.5)
    camera_fov: float = 40
    res: Optional[tuple] = None
    max_FPS: Optional[int] = 60


__all__ = ["SimOptions", "MPMOptions", "ToolOptions", "LegacyCouplerOptions", "B200Options", "VisOptions", "ViewerOptions"]
