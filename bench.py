#!/usr/bin/env python
"""MPM particle-substeps/s of the B200-native MLS-MPM substep.

Workload (N=1): the 500,000-particle mixed-material scene -- four seeded 50^3 jittered
lattices (Liquid E=1e5 nu=0.2, Sand friction 45 deg, Snow yield 2.5e-2/7.5e-3,
ElastoPlastic von Mises 1e4), v ~ N(0, 0.5 m/s), grid_density 128 (129^3 nodes),
dt = 5e-5.  One bench step = one scene.step() of 100 substeps (the 2000-substep rollout
is 20 steps).

  value  particle-substeps/s with the state resident in HBM (CUDA events on the launch
         stream, L2 flushed between timed steps)
  e2e    the same through the public API (gs.Scene): every step uploads the full particle
         state from pinned host memory, runs scene.step() and reads positions and
         velocities back (uploads and read-backs on copy streams, overlapping compute)
  roofline  the dominant kernel's algorithmic bytes / its measured duration, against the
         measured HBM copy bandwidth
  cpu_baseline  the C/OpenMP restatement of the reference algorithm on the host cores

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Under torchrun with N>1 every rank advances its own replica of the scene (the plain
single-scene path has no exchange step): value = N x per-rank work / max rank time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MPM particle-substeps/s"
UNIT = "particle-substeps/s"
WORKLOAD = (
    "mixed_500k: 4 x 125,000 particles (Liquid, Sand, Snow, ElastoPlastic), grid_density 128 (129^3 nodes), "
    "dt 5e-5, 100 substeps per step"
)
# algorithmic bytes per particle / per active grid node, per kernel kind
BYTES = {
    "p2g": (148, 16),  # read x,v,C,F,Jp (100) + material idx & mass (8); write F,Jp (40); grid m+mom (16)
    "grid_op": (0, 28),  # read m+mom (16), write v (12)
    "g2p": (60, 12),  # write x,v,C (60); read grid v (12)  (x read counted in p2g)
    # fused g2p of substep n + p2g of n+1: one substep's particle bytes (208) + grid v read
    # (12) and m+mom write (16).  v and C never leave registers, so the DRAM bytes it must
    # move are lower (x, F, Jp read + written: ~106 B/particle); 'traffic' reports ncu's count.
    "g2p2g": (208, 28),
    "sort": (220, 0),  # read + write the 25 state channels, material, flags, ids (~2 x 110)
}
SUBSTEP_BYTES = (208, 56)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--substeps-per-step", type=int, default=100)
    ap.add_argument("--sort-interval", type=int, default=50)
    ap.add_argument("--chunk", type=int, default=128)
    ap.add_argument("--n-side", type=int, default=50, help="particles per box edge (50 -> 500k)")
    ap.add_argument("--grid-density", type=int, default=128,
                    help="grid nodes per metre (128 -> 129^3; with --n-side 100 / 200, 256 / 512 keep the "
                         "particles per cell of the default scene)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-sequential comparison")
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--batch-substeps", type=int, default=500, help="substeps per scene (500 = the batching config)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving run")
    ap.add_argument("--no-grad", action="store_true", help="skip the differentiation run")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests in the Poisson stream (2000 = the full serving config)")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_name(args, d):
    """The default scene's name, or the same mix at another size."""
    if args.n_side == 50 and args.grid_density == 128:
        return WORKLOAD
    return (f"mixed_{d.n_particles}: 4 x {d.n_particles // 4:,} particles (Liquid, Sand, Snow, ElastoPlastic), "
            f"grid_density {args.grid_density} ({d.grid_res}^3 nodes), dt 5e-5, {args.substeps_per_step} "
            "substeps per step")


def ncu_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            line = line.strip()
            if line and not line.startswith("#") and "=" in line:
                k, v = line.split("=", 1)
                try:
                    out[k.strip()] = float(v.split()[0])
                except ValueError:
                    pass
    return out


class Clocks:
    """SM clock and clock-event reasons sampled every 10 ms during the timed region, through
    NVML in a background thread (read-only queries); nvidia-smi at 200 ms if NVML is
    unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self.proc = None
        self.path = None

    def start(self):
        try:
            import threading

            import pynvml

            pynvml.nvmlInit()
            h = None
            try:  # the CUDA device's own GPU, whatever CUDA_VISIBLE_DEVICES renumbered
                import torch

                h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(torch.cuda.get_device_properties(self.gpu).uuid))
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            masks = [(name, getattr(pynvml, attr, 0)) for name, attr in self.REASONS]
            self._stop = threading.Event()

            def run():
                while not self._stop.is_set():
                    try:
                        mhz = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                        r = int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                        self.samples.append((mhz, [n for n, m in masks if m and (r & m)]))
                    except Exception:
                        pass
                    self._stop.wait(0.01)

            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
            return
        except Exception:
            self._thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)
            if not self.samples:
                return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"], "source": "nvml"}
            sm = [m for m, _ in self.samples]
            loaded = [x for x in sm if x > 0.5 * (self.max_mhz or max(sm))] or sm
            reasons = sorted({r for _, rs in self.samples for r in rs})
            return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(self.samples), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms"}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def reduce_max(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ CPU (reference arm)
CPU_SUB = 2  # substeps per timed CPU step: a bounded sample of the 100-substep step


def cpu_sample(desc, threads, steps, sub=CPU_SUB):
    """The CPU sample both CPU legs time: the C/OpenMP restatement in float32 from the
    workload's initial state, one untimed warm-up substep, then `steps` timed steps of `sub`
    substeps each.  Returns (per-step seconds, final state)."""
    import numpy as np

    from oracle import bridge, cref

    p, mats, st = bridge.from_desc(desc, np.float32)
    st, _ = cref.substeps(p, mats, st, 1, n_threads=threads)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        st, _ = cref.substeps(p, mats, st, sub, n_threads=threads)
        times.append(time.perf_counter() - t0)
    return times, st


def cpu_port_rate(desc, steps, single_thread_steps=5):
    """cpu_baseline leg: the same sample as the reference arm on all host threads, and a
    shorter prefix of it on one thread."""
    threads = os.cpu_count() or 1
    times, _ = cpu_sample(desc, threads, steps)
    rate = desc.n_particles * CPU_SUB * steps / sum(times)
    t1, _ = cpu_sample(desc, 1, single_thread_steps)
    rate1 = desc.n_particles * CPU_SUB * single_thread_steps / sum(t1)
    sample = (f"{desc.n_particles:,} particles, float32: 1 warm-up substep, then {steps} steps x {CPU_SUB} substeps "
              "(the reference arm's sample)")
    single = {"value": rate1, "unit": UNIT, "cores": 1,
              "sample": f"{desc.n_particles:,} particles, float32: 1 warm-up substep, then "
                        f"{single_thread_steps} steps x {CPU_SUB} substeps"}
    return rate, threads, sample, single


def run_reference(args, world, rank):
    if rank != 0:
        return None
    from genesis_b200 import workloads as W

    d = W.mixed_500k(n_side=args.n_side, grid_density=args.grid_density)
    threads = os.cpu_count() or 1
    sub = CPU_SUB
    times, _ = cpu_sample(d, threads, args.steps)
    el = sum(times)
    value = d.n_particles * sub * args.steps / el
    sample = (f"{d.n_particles:,} particles, float32, {threads} threads: 1 warm-up substep, then {args.steps} steps x "
              f"{sub} substeps")
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload_name(args, d), "particles": d.n_particles, "grid": f"{d.grid_res}^3",
                   "substeps_per_step": sub, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference = C/OpenMP restatement of Genesis's MPM substep (gstaichi, the reference's "
                "runtime, is not installed on this image)",
    }


# ------------------------------------------------------------------ GPU (our arm)
def kernel_breakdown(rt, n_substeps):
    """Per-kernel-kind device time over n_substeps of the mpm_substeps schedule, from CUDA
    events recorded between consecutive launch groups (mpm_substeps_profile): returns
    {kind: (ms per launch group, launch groups, kernel launches)} and the total ms.  The GPU
    is kept busy while the launches are enqueued, so the events bracket kernels back to back."""
    import torch

    torch.cuda.synchronize()
    torch.cuda._sleep(int(2e8))
    prof = rt.profile_substeps(n_substeps)
    total = sum(ms for ms, _ in prof.values())
    out = {}
    for k, (ms, launches) in prof.items():
        groups = launches // (SORT_KERNELS if k == "sort" else 1)
        if groups:
            out[k] = (ms / groups, groups, launches)
    return out, total


SORT_KERNELS = 7  # keys, 3 scan passes, chunk table, scatter, lane deal


def launches_per_step(S, K):
    """Kernel launches of one timed step (S substeps from a sort boundary): the runtime replays
    one CUDA graph per sort interval of K substeps, each the mpm_substeps schedule: the sort,
    p2g and grid op, K - 1 times the fused g2p/p2g and the grid op, and the last g2p."""
    graphs, rest = divmod(S, K)
    per = lambda k: SORT_KERNELS + 2 + 2 * (k - 1) + 1
    return graphs * per(K) + (per(rest) if rest else 0)


def active_nodes(rt):
    import torch

    from genesis_b200.engine.runtime import F32_EPS

    rt.ensure_sorted()
    rt.p2g()
    mm, _ = rt.grid_views()
    n = int((mm[:, 3] > F32_EPS).sum().item())
    rt.grid_op()
    rt.g2p()
    rt._count += 1
    torch.cuda.synchronize()
    return n


def build_scene(d, S, check_nan="step"):
    import genesis_b200 as gs

    gs.init(backend=gs.gpu, precision="32", seed=0, logging_level="warning")
    scene = gs.Scene(
        sim_options=gs.options.SimOptions(dt=d.dt * S, substeps=S, gravity=d.gravity),
        mpm_options=gs.options.MPMOptions(lower_bound=d.lower_bound, upper_bound=d.upper_bound,
                                          grid_density=d.grid_density, particle_size=d.particle_size),
        b200_options=gs.options.B200Options(sort_interval=50, check_nan=check_nan),
    )
    from genesis_b200 import workloads as W

    mats = W.make_materials(d, gs.materials.MPM)
    ents = []
    for mi, m in enumerate(mats):
        sel = d.mat_idx == mi
        lo, hi = d.pos[sel].min(0) - 1e-4, d.pos[sel].max(0) + 1e-4
        ents.append((scene.add_entity(gs.morphs.Box(lower=tuple(lo), upper=tuple(hi)), material=m), sel))
    scene.build()
    for ent, sel in ents:
        n = ent.n_particles
        if n != int(sel.sum()):
            raise RuntimeError("entity sampling does not match the workload particle count")
        ent.set_particles_pos(d.pos[sel])
        ent.set_particles_vel(d.vel[sel])
    return scene


def run_e2e(d, S, K, W_):
    """Through gs.Scene with host buffers.  Every step uploads the full particle state from
    pinned host memory (scene.reset), runs scene.step() (S substeps) and reads pos/vel back
    into pinned host memory.  The upload takes the scene's asynchronous staged path and the
    read-back runs on a copy stream, so step k's read-back and step k+1's upload overlap the
    compute; the NaN check is the asynchronous one (check_nan='async'), settled by
    scene.check_state() after the timed loop.  Timed with CUDA events around all K steps."""
    import torch

    scene = build_scene(d, S, check_nan="async")
    st = scene.get_state()[3]
    host = {k: getattr(st, k).cpu().pin_memory() for k in ("pos", "vel", "C", "F", "Jp", "active")}
    from genesis_b200.engine.states import MPMSolverState

    out_pos = torch.empty_like(host["pos"]).pin_memory()
    out_vel = torch.empty_like(host["vel"]).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    d2h = out_pos.numel() * 4 + out_vel.numel() * 4
    main = torch.cuda.current_stream()
    d2h_stream = torch.cuda.Stream()

    def one():
        s = MPMSolverState(scene, host["pos"], host["vel"], host["C"], host["F"], host["Jp"], host["active"])
        scene.reset(s)
        scene.step()
        cur = scene.get_state()[3]
        d2h_stream.wait_stream(main)
        with torch.cuda.stream(d2h_stream):
            out_pos.copy_(cur.pos, non_blocking=True)
            out_vel.copy_(cur.vel, non_blocking=True)
        cur.pos.record_stream(d2h_stream)
        cur.vel.record_stream(d2h_stream)

    for _ in range(W_):
        one()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(K):
        one()
    main.wait_stream(d2h_stream)
    b.record()
    torch.cuda.synchronize()
    scene.check_state()
    ms = a.elapsed_time(b) / K
    return d.n_particles * S / (ms * 1e-3), ms, h2d, d2h


def run_ours(args, world, rank, local):
    import torch

    from genesis_b200 import workloads as W
    from genesis_b200.engine.runtime import runtime_from_descs

    S = args.substeps_per_step
    d = W.mixed_500k(n_side=args.n_side, grid_density=args.grid_density)
    rt = runtime_from_descs([d], sort_interval=args.sort_interval, chunk_particles=args.chunk)
    for _ in range(args.warmup):
        rt.substeps(S)
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    step_ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)  # evict L2 between timed steps (not timed)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        rt.substeps(S)
        b.record()
        step_ms.append((a, b))
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    dev_ms = sum(a.elapsed_time(b) for a, b in step_ms)
    dev_s = reduce_max(world, dev_ms * 1e-3)
    status = rt.status()
    units = d.n_particles * S * args.steps * world
    value = units / dev_s

    # per-kernel breakdown + roofline of the dominant kernel
    n_act = active_nodes(rt)
    nsub = 2 * S
    kb, prof_ms = kernel_breakdown(rt, nsub)
    hbm, src = peaks()
    dom = max(kb, key=lambda k: kb[k][0] * kb[k][1])
    bp, bc = BYTES[dom]
    alg = bp * d.n_particles + bc * n_act
    step_sub_ms = dev_ms / (args.steps * S)
    t_dom = kb[dom][0] * 1e-3
    achieved = alg / t_dom / 1e9
    tr = ncu_traffic()
    # the committed ncu figure is the default scene's; other sizes report none
    traffic = tr.get(f"{dom}_dram_bytes_per_launch") if workload_name(args, d) == WORKLOAD else None
    sub_alg = SUBSTEP_BYTES[0] * d.n_particles + SUBSTEP_BYTES[1] * n_act
    gpu_launches = args.steps * launches_per_step(S, args.sort_interval)

    res = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_s * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": workload_name(args, d),
            "particles": d.n_particles,
            "grid": f"{d.grid_res}^3",
            "substeps_per_step": S,
            "sort_interval": args.sort_interval,
            "chunk_particles": args.chunk,
            "l2": "flushed between timed steps (256 MB write, untimed)",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "wall_s": wall,
        },
        "roofline": {
            "bound": "hbm",
            "kernel": dom,
            "achieved": achieved,
            "peak": hbm,
            "unit": "GB/s",
            "frac": achieved / hbm,
            "peak_source": src,
            "traffic": traffic,
            "alg_bytes_per_launch": alg,
            "active_nodes": n_act,
            "kernel_ms": {k: round(v[0], 5) for k, v in kb.items()},
            "kernel_share": {k: round(v[0] * v[1] / prof_ms, 4) for k, v in kb.items()},
            "launches_per_substep": {k: round(v[2] / nsub, 4) for k, v in kb.items()},
            "timing": f"CUDA events between consecutive launch groups over {nsub} substeps of the same "
                      "schedule (mpm_substeps_profile, no graph); kernel_ms is per launch group (a sort is 7 "
                      "kernels)",
            "profile_ms_per_substep": prof_ms / nsub,
            "substep_ms": step_sub_ms,
            "profile_vs_step": (prof_ms / nsub) / step_sub_ms,
            # the profiled shares applied to the graph-replayed step (the events' own gaps,
            # ~13% of the profiled run, spread in proportion): these sum to substep_ms
            "kernel_ms_in_step": {k: round(v[0] * step_sub_ms * nsub / prof_ms, 5) for k, v in kb.items()},
            "substep_alg_GBs": sub_alg / (step_sub_ms * 1e-3) / 1e9,
            "substep_frac": sub_alg / (step_sub_ms * 1e-3) / 1e9 / hbm,
        },
        "gpu_launches": gpu_launches,
        "clocks": clk,
        "status_word": status,
    }
    return res, d, rt


def run_batched(args, world, rank):
    """Batching config: 256 independent scenes (N log-uniform in [2e3, 2e5], grid density
    32/64/96, material uniform over the five, E log-uniform [1e4, 1e6]) advanced together by
    one launch sequence, against the same scenes run one at a time.  Under torchrun the
    scenes are sharded over ranks by work (genesis_b200.shard; no data-path collective)."""
    import torch

    from genesis_b200 import workloads as W
    from genesis_b200.batch import BatchedScenes, run_sequential

    from genesis_b200 import shard

    all_descs = W.batch_scenes(n_scenes=args.batch_scenes, n_substeps=args.batch_substeps)
    descs = shard.my_shard(all_descs, rank, world)
    n_total = sum(d.n_particles for d in all_descs)
    S = args.batch_substeps
    bs = BatchedScenes(descs, tune=True, tune_cache=False)
    tuning = bs.tuning[0] if bs.tuning else None
    K = bs.rt.sort_interval
    bs.substeps(K)
    torch.cuda.synchronize()
    barrier(world)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    bs.substeps(S)
    b.record()
    torch.cuda.synchronize()
    t_b = reduce_max(world, a.elapsed_time(b) * 1e-3)
    status = bs.rt.status()
    split, _ = kernel_breakdown(bs.rt, 2 * K)
    del bs
    torch.cuda.empty_cache()
    per_scene = run_sequential(descs, S, per_scene=True)
    t_s = reduce_max(world, sum(per_scene))
    return {
        "workload": f"{args.batch_scenes} scenes, N log-uniform [2e3, 2e5], grid 33^3/65^3/97^3, 5 materials, "
                    f"E log-uniform [1e4, 1e6], {S} substeps each",
        "scenes": args.batch_scenes,
        "particles": n_total,
        "substeps": S,
        "value": n_total * S / t_b,
        "unit": UNIT,
        "sequential_value": n_total * S / t_s,
        "speedup_vs_sequential": t_s / t_b,
        "tuning": tuning,
        "kernel_ms": {k: round(v[0], 5) for k, v in split.items()},
        "status_word": status,
        "amdahl": amdahl_ceiling(descs, per_scene, S, t_b),
    }


def amdahl_ceiling(descs, seq_times, S, t_batched, large=50_000):
    """How far batching alone can go on this scene set.  Batching removes per-scene costs
    (launches, grid-op passes, sort and graph boundaries, a persistent grid's tail) that
    weigh on small scenes; a large scene already runs at the fused kernel's per-particle rate.
    The ceiling assumes every scene ran at the per-particle-substep rate that the plain path
    reaches on the large scenes (>= `large` particles) -- removing all per-scene overhead and
    nothing else -- and divides the sequential time by that."""
    big = [i for i, d in enumerate(descs) if d.n_particles >= large]
    work = [d.n_particles * S for d in descs]
    t_seq = sum(seq_times)
    t_big = sum(seq_times[i] for i in big)
    w_big = sum(work[i] for i in big)
    rate_big = w_big / t_big if t_big > 0 else None
    t_ideal = sum(work) / rate_big if rate_big else None
    return {
        "large_scene_particles": large,
        "large_scenes": len(big),
        "sequential_time_fraction_in_large": t_big / t_seq if t_seq else None,
        "work_fraction_in_large": w_big / sum(work) if work else None,
        "large_scene_rate": rate_big,
        "max_speedup_if_all_at_large_rate": t_seq / t_ideal if t_ideal else None,
        "batched_vs_large_rate": (sum(work) / t_batched) / rate_big if rate_big else None,
        "three_x_reachable_by_batching_alone": (t_seq / t_ideal >= 3.0) if t_ideal else None,
    }


def run_served(args, world, rank, capacity):
    """Serving config: Poisson arrivals of rollout requests (N log-uniform [1e3, 5e5], grid
    density 32-128, substeps U[100, 2000], the mixed_500k material mix), mean rate 80% of the
    measured batched capacity; continuous batching under a 150 GB HBM budget.  Reports
    p50/p99 end-to-end latency (arrival -> result on the host) and throughput, beside the plain
    one-request-at-a-time path under the same arrivals.  Under torchrun each rank serves the
    requests of its work-balanced shard (genesis_b200.shard)."""
    import torch

    from genesis_b200 import serve
    from genesis_b200 import workloads as W
    from genesis_b200.engine.runtime import runtime_from_descs

    base = W.serving_stream(n_requests=args.serve_requests, rate=1.0)
    work = [r.scene.n_particles * r.scene.n_substeps for r in base]
    mean_work = sum(work) / len(work)
    rate = 0.8 * capacity / mean_work  # requests per second over all ranks
    from genesis_b200 import shard

    reqs = shard.my_shard([W.Request(r.rid, r.arrival / rate, r.scene) for r in base], rank, world)
    my_work = sum(r.scene.n_particles * r.scene.n_substeps for r in reqs)
    srv = serve.MPMServer(budget_bytes=150e9, tick_substeps=50, keep_results=False)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    res = srv.serve(reqs, realtime=True)
    wall = reduce_max(world, time.perf_counter() - t0)
    lat = [r.latency for r in res if r.error is None]
    errors = sum(1 for r in res if r.error is not None)
    # the plain path: each request alone (own runtime, graphs), in arrival order
    durs = []
    for r in reqs:
        rt = runtime_from_descs([r.scene])
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        rt.substeps(r.scene.n_substeps)
        b.record()
        torch.cuda.synchronize()
        durs.append(a.elapsed_time(b) * 1e-3)
        del rt
    seq_lat = serve.sequential_timeline(reqs, durs)
    total_work = sum(work)
    # capacity at saturation: the same requests all queued at t = 0 (offered load >= capacity)
    srv_sat = serve.MPMServer(budget_bytes=150e9, tick_substeps=50, keep_results=False)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    res_sat = srv_sat.serve(reqs, realtime=False)
    wall_sat = reduce_max(world, time.perf_counter() - t0)
    sat_stats = {"ticks": srv_sat.ticks, "repacks": srv_sat.repacks, "repack_host_s": srv_sat.repack_s,
                 "substeps_per_tick": srv_sat.substeps_run / max(1, srv_sat.ticks)}
    del srv_sat
    seq_rate = my_work / sum(durs)
    return {
        "workload": f"{args.serve_requests} Poisson requests (rate {rate:.2f}/s = 80% of measured batched capacity), "
                    "N log-uniform [1e3, 5e5], grid density 32-128, substeps U[100, 2000], 150 GB budget",
        "requests": args.serve_requests,
        "value": total_work / wall,
        "unit": UNIT,
        "p50_latency_s": serve.percentile(lat, 50),
        "p99_latency_s": serve.percentile(lat, 99),
        "errors": errors,
        "ticks": srv.ticks,
        "repacks": srv.repacks,
        "repack_host_s": srv.repack_s,
        "sequential_value": seq_rate,
        "sequential_p50_latency_s": serve.percentile(seq_lat, 50),
        "sequential_p99_latency_s": serve.percentile(seq_lat, 99),
        "wall_s": wall,
        "note": "at 80% offered load the served throughput is the offered load by construction; "
                "saturation.value is the server's capacity",
        "saturation": {
            "value": total_work / wall_sat,
            "unit": UNIT,
            "wall_s": wall_sat,
            "errors": sum(1 for r in res_sat if r.error is not None),
            "speedup_vs_sequential": (total_work / wall_sat) / (seq_rate * world),
            "offered": "all requests queued at t = 0",
            **sat_stats,
        },
    }


def run_grad(args):
    """Differentiation config: Elastic block of 20,000 particles with per-particle E, 200
    substeps at dt 1e-4, loss |mean(x_T) - target|^2, gradients w.r.t. v0 and E through the
    checkpointed adjoint (checkpoints every 20 substeps); device time of forward+backward."""
    import torch

    from genesis_b200 import workloads as W
    from genesis_b200.grad import DifferentiableRollout, rollout

    d = W.diff_elastic()
    sim = DifferentiableRollout(d, checkpoint_every=20)
    v0 = torch.tensor(d.meta["v0"], dtype=torch.float32, device="cuda", requires_grad=True)
    E = torch.tensor(d.E_particle, dtype=torch.float32, device="cuda", requires_grad=True)
    tgt = torch.tensor(d.meta["target"], dtype=torch.float32, device="cuda")
    times = []
    for it in range(3):
        v0.grad = None
        E.grad = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x = rollout(v0, E, sim)
        loss = ((x.mean(0) - tgt) ** 2).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        times.append((t1 - t0, t2 - t1))
    fwd, bwd = times[-1]
    return {
        "workload": "Elastic block, 20,000 particles, per-particle E, 200 substeps, checkpoints every 20",
        "forward_s": fwd,
        "backward_s": bwd,
        "loss": float(loss.detach()),
        "grad_v0": [float(g) for g in v0.grad.cpu()],
        "grad_E_norm": float(E.grad.norm().cpu()),
        "check": "tests/test_gpu_grad.py compares these gradients with float64 central finite differences",
    }


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
        if out is not None:
            print(json.dumps(out))
        return
    import torch

    from genesis_b200 import build as B

    B.build()
    res, d, rt = run_ours(args, world, rank, local)
    del rt
    torch.cuda.empty_cache()
    S = args.substeps_per_step
    if not args.no_e2e:
        rate, ms, h2d, d2h = run_e2e(d, S, args.steps, args.warmup)
        rate = reduce_max(world, -rate) * -1 if world > 1 else rate
        res["e2e"] = {"value": rate * (world if world > 1 else 1), "unit": UNIT, "h2d_bytes_per_step": h2d,
                      "d2h_bytes_per_step": d2h, "ms_per_step": ms, "api": "gs.Scene.reset(state)+step()+get_state()",
                      "copies": "H2D staged on a side stream, D2H on a copy stream; check_nan='async'"}
    if not args.no_batch:
        res["batched"] = run_batched(args, world, rank)
        torch.cuda.empty_cache()
    if not args.no_grad and rank == 0:
        res["differentiation"] = run_grad(args)
        torch.cuda.empty_cache()
    if not args.no_serve:
        cap = res["batched"]["value"] if "batched" in res else res["value"]
        res["served"] = run_served(args, world, rank, cap)
        torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, threads, sample, single = cpu_port_rate(d, args.steps)
        res["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                               "single_thread": single}
    if rank == 0:
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
