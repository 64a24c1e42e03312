"""Batched scenes: many independent MPM scenes with uneven particle counts and grid
sizes advanced by the same kernel launches.

Each scene is one *instance* in the runtime's instance table (its particle range, grid
block base, dx, dt, gravity, boundary and material entries), so a substep of all scenes
is one p2g/g2p2g launch over the union of their work items plus one grid-op launch over
the union of their active blocks; a sort interval of substeps is replayed as one CUDA
graph.  There is no counterpart in the reference, whose batching (n_envs) copies one
scene B times.
"""

from __future__ import annotations

import torch

from . import autotune
from .engine.runtime import MPMRuntime, runtime_from_descs


class BatchedScenes:
    def __init__(self, descs, tune: bool = True, tune_cache: bool = True, **runtime_kw):
        self.descs = list(descs)
        self.rt: MPMRuntime = runtime_from_descs(self.descs, **runtime_kw)
        self.offsets = self.rt.instance_offsets
        self.tuning = None
        if tune:
            self.tuning = autotune.tune(self.rt, use_cache=tune_cache)

    @property
    def n_particles(self) -> int:
        return self.rt.n

    def substeps(self, n: int):
        self.rt.substeps(n)

    def scene_state(self, i: int, keys=("pos", "vel")) -> dict:
        st = self.rt.get_state(keys)
        sl = slice(self.offsets[i], self.offsets[i] + self.descs[i].n_particles)
        return {k: v[sl] for k, v in st.items()}

    def states(self, keys=("pos", "vel")) -> list[dict]:
        st = self.rt.get_state(keys)
        return [{k: v[o : o + d.n_particles] for k, v in st.items()} for o, d in zip(self.offsets, self.descs)]


def run_sequential(descs, n_substeps: int, per_scene: bool = False, **runtime_kw):
    """The plain one-scene-at-a-time path: each scene gets its own runtime and runs alone.
    Returns device seconds (CUDA events around each scene's substeps, summed), or with
    per_scene=True the list of each scene's seconds."""
    total = 0.0
    times = []
    for d in descs:
        rt = runtime_from_descs([d], **runtime_kw)
        rt.substeps(min(n_substeps, rt.sort_interval))  # warm: first sort + graph capture
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        rt.substeps(n_substeps)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) * 1e-3)
        total += times[-1]
        del rt
    return times if per_scene else total
