"""Particle emitter (genesis/engine/entities/emitter.py:11-244).

An emitter owns a Nowhere entity of `max_particles` inactive particles (scene.add_emitter);
each emit() samples a droplet on the host, places it at the nozzle and writes positions,
velocities and the active flag of the next run of particle slots through the entity
setters (device kernels k_set_pos / k_set_vel / k_set_flag).  Slots are recycled from the
start once the next droplet would not fit.  Writing positions marks the particle binning
dirty, so the next substep re-sorts and the new particles join the work items of their
grid blocks.
"""

from __future__ import annotations

import logging

import numpy as np
import torch

from .. import _globals
from .. import geom as gu
from .. import particle as pu
from ..exceptions import GenesisException

log = logging.getLogger("genesis_b200")


class Emitter:
    def __init__(self, max_particles):
        self._entity = None
        self._max_particles = int(max_particles)
        self._acc_droplet_len = 0.0  # accumulated droplet length not yet emitted
        self._next_particle = 0
        self._rng = None

    def set_entity(self, entity):
        self._entity = entity
        self._sim = entity.sim
        self._solver = entity.solver
        self._next_particle = 0
        self._rng = _globals.rng if getattr(_globals, "rng", None) is not None else np.random.default_rng()

    def reset(self):
        self._next_particle = 0

    @property
    def entity(self):
        return self._entity

    @property
    def max_particles(self):
        return self._max_particles

    @property
    def next_particle(self):
        return self._next_particle

    def _activate(self, positions, vels):
        if not self._solver.boundary.is_inside(positions):
            raise GenesisException("Emitted particles are outside the boundary.")
        n = len(positions)
        if n > self._entity.n_particles:
            raise GenesisException(
                f"Number of particles to emit ({n}) at the current step is larger than the maximum "
                f"number of particles ({self._entity.n_particles})."
            )
        idx = torch.arange(self._next_particle, self._next_particle + n, dtype=torch.int64)
        self._entity.set_particles_pos(positions, idx)
        self._entity.set_particles_vel(vels, idx)
        self._entity.set_particles_active(1, idx)
        self._next_particle += n
        if self._next_particle + n > self._entity.n_particles:  # recycle
            self._next_particle = 0
        log.debug(f"Emitted {n} particles. Next particle index: {self._next_particle}.")
        return n

    def emit(self, droplet_shape, droplet_size, droplet_length=None, pos=(0.5, 0.5, 1.0), direction=(0, 0, -1),
             theta=0.0, speed=1.0, p_size=None):
        """Emit one droplet ("circle", "sphere", "square" or "rectangle") from a nozzle at
        `pos` along `direction` (emitter.py:58-197).  Returns the number emitted."""
        if self._entity is None:
            raise GenesisException("Emitter has no entity.")
        if droplet_shape in ("circle", "sphere", "square"):
            if not isinstance(droplet_size, (int, float)):
                raise GenesisException("droplet_size must be a number for this shape.")
        elif droplet_shape == "rectangle":
            if not (isinstance(droplet_size, (tuple, list)) and len(droplet_size) == 2):
                raise GenesisException("droplet_size must be (width, height) for a rectangle.")
        else:
            raise GenesisException(f"Unsupported nozzle shape: {droplet_shape}.")
        direction = np.asarray(direction, dtype=np.float64)
        if np.linalg.norm(direction) < _globals.EPS:
            raise GenesisException("Zero-length direction.")
        direction = gu.normalize(direction)
        p_size = self._entity.particle_size if p_size is None else p_size

        if droplet_length is None:
            # the droplet covers the distance travelled in one step at `speed`
            droplet_length = speed * self._solver.substep_dt * self._sim.substeps + self._acc_droplet_len
            if droplet_length < p_size:  # too short: accumulate and emit later
                self._acc_droplet_len = droplet_length
                droplet_length = 0.0
            else:
                self._acc_droplet_len = 0.0
        if droplet_length <= 0.0:
            log.debug("Droplet length is too short for current step. Skipping to next step.")
            return 0

        sampler = self._entity.sampler
        if droplet_shape == "circle":
            positions = pu.cylinder_to_particles(p_size, radius=droplet_size / 2, height=droplet_length,
                                                 sampler=sampler, rng=self._rng)
        elif droplet_shape == "sphere":  # ignores droplet_length
            positions = pu.sphere_to_particles(p_size, radius=droplet_size / 2, sampler=sampler, rng=self._rng)
        elif droplet_shape == "square":
            positions = pu.box_to_particles(p_size, size=(droplet_size, droplet_size, droplet_length),
                                            sampler=sampler, rng=self._rng)
        else:
            positions = pu.box_to_particles(p_size, size=(droplet_size[0], droplet_size[1], droplet_length),
                                            sampler=sampler, rng=self._rng)
        R = gu.z_up_to_R(direction) @ gu.axis_angle_to_R(np.array([0.0, 0.0, 1.0]), theta)
        positions = gu.transform_by_trans_R(positions, np.asarray(pos, dtype=np.float64), R)
        vels = np.tile(speed * direction, (len(positions), 1))
        return self._activate(positions, vels)

    def emit_omni(self, source_radius=0.1, pos=(0.5, 0.5, 1.0), speed=1.0, particle_size=None):
        """Emit a shell of particles (radii 0.4 r .. r) moving radially outwards
        (emitter.py:199-244).  Returns the number emitted."""
        if self._entity is None:
            raise GenesisException("Emitter has no entity.")
        pos = np.asarray(pos, dtype=np.float64)
        if particle_size is None:
            particle_size = self._entity.particle_size
        local = pu.shell_to_particles(particle_size, outer_radius=source_radius, inner_radius=source_radius * 0.4,
                                      sampler=self._entity.sampler, rng=self._rng)
        positions = pos + local
        if not self._solver.boundary.is_inside(positions):
            raise GenesisException("Emitted particles are outside the boundary.")
        dists = np.linalg.norm(local, axis=1)
        positions[dists < _globals.EPS] = _globals.EPS
        vels = (speed / (dists[:, None] + _globals.EPS)) * local
        return self._activate(positions, vels)
