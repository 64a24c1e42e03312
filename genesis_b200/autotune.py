"""Launch-configuration autotuner for an MPMRuntime.

Picks, by timing short runs on the problem itself, the particles per work item
(chunk_particles: 128/256, i.e. threads per CTA of p2g/g2p/g2p2g), the re-sort
interval and the persistent CTA count (grid_ctas; the candidates are given per SM:
0 is the library default of one CTA per resident slot, i.e. SMs x occupancy, 4 per SM
leaves slots free for a concurrent stream, 14 per SM is two waves of the 128-particle
kernels, which evens out the tail when the work items are few and uneven).  The grid block edge is fixed at 4 nodes (it sets
the block-major grid layout and the 8^3 shared tile).  Results are cached per problem
signature (particle and grid-block counts rounded to powers of two) in a JSON file so a
served or batched workload tunes once.
"""

from __future__ import annotations

import json
import math
import os
import threading

import torch

DEFAULT_CANDIDATES = {
    "chunk_particles": (128, 256),
    "sort_interval": (25, 50, 100),
    "grid_ctas_per_sm": (0, 4, 14),
}

_lock = threading.Lock()


def signature(rt) -> str:
    b = lambda x: 1 << max(0, int(math.ceil(math.log2(max(1, x)))))
    return f"n{b(rt.n)}_blk{b(rt.n_blocks)}_inst{b(len(rt.specs))}"


def _cache_path():
    return os.environ.get("GENESIS_B200_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache",
                                                                   "genesis_b200_tune.json"))


def _load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def time_substeps(rt, n: int) -> float:
    """Device milliseconds per substep over n substeps (after the state is already binned)."""
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    rt.substeps(n)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / max(n, 1)


def tune(rt, candidates=None, trial_substeps: int = 100, use_cache: bool = True, restore_state: bool = True):
    """Time every candidate configuration on rt and leave rt configured with the fastest.

    The particle state advanced by the trials is restored afterwards (restore_state) so
    tuning does not change the simulation.  Returns (best_config, {config: ms/substep})."""
    cand = dict(DEFAULT_CANDIDATES)
    cand.update(candidates or {})
    if "grid_ctas" not in cand:
        sms = torch.cuda.get_device_properties(rt.device).multi_processor_count
        cand["grid_ctas"] = tuple(int(k) * sms for k in cand["grid_ctas_per_sm"])
    sig = signature(rt)
    if use_cache:
        with _lock:
            cache = _load_cache()
        if sig in cache:
            best = cache[sig]["best"]
            rt.retune(**best)
            return best, cache[sig].get("times", {})
    # every candidate starts from the same particle state: timed on a simulation that moves
    # on between candidates, the ones tried first would see an earlier (and, as a scene
    # settles into contact and plastic flow, cheaper) stretch of it
    saved = (rt.state.clone(), rt.mat.clone(), rt.pflags.clone(), rt.gid.clone(), rt.slot.clone(),
             None if rt.mu_p is None else rt.mu_p.clone(), None if rt.lam_p is None else rt.lam_p.clone(),
             rt._count)
    # the colliders move with the substeps and accumulate reaction forces
    cols = rt.collider_table().clone() if getattr(rt, "coll_table", None) is not None else None
    cforce = rt.collider_force.clone() if getattr(rt, "collider_force", None) is not None else None

    def restore():
        if cols is not None:
            rt.collider_table().copy_(cols)
        if cforce is not None:
            rt.collider_force.copy_(cforce)
        st, mat, pf, gid, slot, mu, lam, count = saved
        rt.state.copy_(st)
        rt.mat.copy_(mat)
        rt.pflags.copy_(pf)
        rt.gid.copy_(gid)
        rt.slot.copy_(slot)
        if mu is not None:
            rt.mu_p.copy_(mu)
            rt.lam_p.copy_(lam)
        rt._count = count
        rt._sorted_once = False  # the binning in the workspace belongs to the advanced state

    times = {}
    best, best_t = None, float("inf")
    for P in cand["chunk_particles"]:
        for K in cand["sort_interval"]:
            for G in cand["grid_ctas"]:
                restore()
                rt.retune(chunk_particles=P, sort_interval=K, grid_ctas=G)
                rt._count = 0
                n = max(trial_substeps, K)
                rt.substeps(K)  # warm-up (graph capture, first sort)
                t = time_substeps(rt, (n // K) * K)
                key = f"P{P}_K{K}_G{G}"
                times[key] = t
                if t < best_t:
                    best, best_t = {"chunk_particles": P, "sort_interval": K, "grid_ctas": G}, t
    if restore_state:
        restore()
    rt.retune(**best)
    rt._sorted_once = False
    if use_cache:
        with _lock:
            cache = _load_cache()
            cache[sig] = {"best": best, "times": times}
            _store_cache(cache)
    return best, times
