"""CUDA path vs the CPU oracle on the same seeded inputs (parity tests proper).

Tolerances (float32 kernels, float32/float64 oracle):
  * grid mass and momentum sums after p2g: 1e-6 relative;
  * per-node grid values: 1e-5 of the largest node value;
  * particle positions after 100 substeps: 1e-5 of the domain size (1 m); velocities
    1e-5 m/s (the elastic cube);
  * single-substep state per material: the CUDA error against the float64 oracle must be
    within 20x the float32 oracle's own error (+ a small absolute floor), because
    atomics sum in a different order than the oracle.
Atomic accumulation order on the GPU is nondeterministic; tests compare against the
oracle, never against a previous GPU run bit for bit.
"""

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _rt(descs, **kw):
    from genesis_b200.engine.runtime import runtime_from_descs

    return runtime_from_descs(descs, **kw)


def _oracle(desc, dtype):
    from oracle import bridge

    return bridge.from_desc(desc, dtype)


def _state_np(rt):
    st = rt.get_state()
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in st.items()}


def _dense_grid(rt, inst=0):
    from genesis_b200.engine.runtime import block_major_to_dense

    mm, gv = rt.grid_views()
    torch.cuda.synchronize()
    sp = rt.specs[inst]
    base = int(rt._insts[inst].blk_base)
    return (block_major_to_dense(mm.cpu().numpy(), sp, base), block_major_to_dense(gv.cpu().numpy(), sp, base))


@pytest.mark.parametrize("n_side", [16, 32])
def test_p2g_grid_matches_oracle(n_side):
    """Grid mass/momentum after the first p2g; n_side 32 is the full 32,768-particle cube."""
    from oracle import mpm_ref as R

    d = W.elastic_cube(n_side=n_side)
    d.vel = np.random.default_rng(5).normal(0, 0.5, size=d.vel.shape)
    rt = _rt([d])
    rt.sort()
    rt.p2g()
    mm, _ = _dense_grid(rt)
    p, mats, st = _oracle(d, np.float64)
    gm, gp, _, _ = R.p2g(p, mats, st)
    assert np.isclose(mm[..., 3].sum(), gm.sum(), rtol=1e-6)
    mom_scale = np.abs(gp).sum()
    assert np.allclose(mm[..., :3].sum(axis=(0, 1, 2)), gp.sum(axis=(0, 1, 2)), rtol=0, atol=1e-6 * mom_scale)
    assert np.abs(mm[..., 3] - gm).max() <= 1e-5 * gm.max()
    assert np.abs(mm[..., :3] - gp).max() <= 1e-5 * np.abs(gp).max()


def _deformed(desc, rng, fscale, cscale):
    n = desc.n_particles
    F = np.eye(3)[None] + fscale * rng.normal(size=(n, 3, 3))
    C = cscale * rng.normal(size=(n, 3, 3))
    return F, C


@pytest.mark.parametrize("kind,kw", [
    ("elastic", dict(E=1e5, nu=0.3)),
    ("elastic", dict(E=1e5, nu=0.3, model="neohooken")),
    ("elastoplastic", dict(von_mises_yield_stress=1e4)),
    ("elastoplastic", dict(use_von_mises=False)),
    ("liquid", dict(E=1e5)),
    ("liquid", dict(E=1e5, viscous=True)),
    ("sand", dict(friction_angle=45)),
    ("snow", dict(yield_lower=2.5e-2, yield_higher=7.5e-3)),
])
def test_one_substep_per_material(kind, kw):
    from oracle import mpm_ref as R

    rng = np.random.default_rng(6)
    d = W.elastic_cube(n_side=12)
    d.materials = [(kind, dict(kw))]
    d.vel = rng.normal(0, 0.5, size=d.vel.shape)
    F, Cm = _deformed(d, rng, 0.04, 2.0)
    rt = _rt([d])
    n = d.n_particles
    Jp0 = np.full(n, 0.0 if kind == "sand" else 1.0)
    if kind == "snow":
        Jp0 = rng.uniform(0.95, 1.05, size=n)
    rt.set_state(C_=Cm.reshape(n, 9), F=F.reshape(n, 9), Jp=Jp0)
    rt.substeps(1)
    g = _state_np(rt)
    outs = {}
    for dt in (np.float64, np.float32):
        p, mats, st = _oracle(d, dt)
        st["F"] = F.astype(dt)
        st["C"] = Cm.astype(dt)
        st["Jp"] = Jp0.astype(dt)
        outs[dt] = R.substep(p, mats, st)
    o64, o32 = outs[np.float64], outs[np.float32]
    gm = {"x": g["pos"], "v": g["vel"], "C": g["C"].reshape(n, 3, 3), "F": g["F"].reshape(n, 3, 3), "Jp": g["Jp"]}
    for k in ("x", "v", "C", "F", "Jp"):
        ref_err = np.abs(o32[k] - o64[k]).max()
        err = np.abs(gm[k] - o64[k]).max()
        floor = 1e-6 * max(1.0, np.abs(o64[k]).max())
        assert err <= 20 * ref_err + floor, f"{k}: gpu err {err:.3e} vs f32-oracle err {ref_err:.3e}"


def test_100_substeps_elastic_cube_full_size():
    """Elastic cube of 32,768 particles, 65^3 grid, dt 1e-4: 100 substeps vs the f64 oracle."""
    from oracle import cref

    d = W.elastic_cube()
    rt = _rt([d])
    rt.substeps(100)
    g = _state_np(rt)
    o, rc = cref.substeps(*_oracle(d, np.float64), 100)
    assert rc == 0
    ex = np.abs(g["pos"] - o["x"]).max()
    ev = np.abs(g["vel"] - o["v"]).max()
    assert ex <= 1e-5, ex
    assert ev <= 1e-5, ev  # m/s (measured ~2e-7)
    assert rt.status() == 0


def test_100_substeps_mixed_materials_reduced():
    """Four boxes (Liquid, Sand, Snow, ElastoPlastic) at 12^3 particles each on the 129^3 grid.

    Per material, positions after 100 substeps within 1e-5 m of the reference's precision-32
    model computed in float64 (float64 arithmetic with the float32 gs.EPS, which the plastic
    return mappings use in Matrix.norm(EPS): sand.py:61, elasto_plastic.py:74)."""
    from oracle import bridge, cref

    d = W.mixed_500k(n_side=12)
    rt = _rt([d])
    rt.substeps(100)
    g = _state_np(rt)
    o, rc = cref.substeps(*bridge.from_desc(d, np.float64, model_dtype=np.float32), 100)
    assert rc == 0
    for m in range(4):
        sel = d.mat_idx == m
        ex = np.abs(g["pos"][sel] - o["x"][sel]).max()
        assert ex <= 1e-5, (m, ex)


def test_state_roundtrip_and_sort_permutation():
    d = W.mixed_500k(n_side=10)
    rt = _rt([d], sort_interval=1)
    before = _state_np(rt)
    rt.sort()
    after = _state_np(rt)
    for k in before:
        assert np.array_equal(before[k], after[k]), k
    # gid/slot stay inverse permutations
    gid = rt.gid[: rt.n].cpu().numpy()
    slot = rt.slot[: rt.n].cpu().numpy()
    assert np.array_equal(slot[gid], np.arange(rt.n))


def test_sort_interval_does_not_change_results():
    d = W.mixed_500k(n_side=10)
    a = _rt([d], sort_interval=1, use_graphs=False)
    b = _rt([d], sort_interval=1000, use_graphs=False)
    a.substeps(40)
    b.substeps(40)
    sa, sb = _state_np(a), _state_np(b)
    # a different binning changes only the float32 summation order; the scene holds Sand,
    # whose float32 rounding sensitivity is ~3e-5 per 100 substeps, so the parity bar
    # (1e-5 of the domain) applies rather than bitwise agreement
    assert np.abs(sa["pos"] - sb["pos"]).max() < 1e-5
    assert a.fallback_count() == 0  # re-binned before every p2g: no particle leaves its tile


def test_graph_replay_matches_eager():
    d = W.elastic_cube(n_side=16)
    a = _rt([d], sort_interval=8, use_graphs=True)
    b = _rt([d], sort_interval=8, use_graphs=False)
    a.substeps(32)
    b.substeps(32)
    sa, sb = _state_np(a), _state_np(b)
    assert np.abs(sa["pos"] - sb["pos"]).max() < 1e-6


def test_set_particles_pos_resets_state():
    d = W.elastic_cube(n_side=8)
    rt = _rt([d])
    rt.substeps(5)
    idx = torch.tensor([0, 7, 100], dtype=torch.int32)
    new = torch.tensor([[0.5, 0.5, 0.5], [0.45, 0.5, 0.5], [0.5, 0.55, 0.5]])
    rt.set_particles_pos(idx, new)
    s = _state_np(rt)
    assert np.allclose(s["pos"][[0, 7, 100]], new.numpy())
    assert np.all(s["vel"][[0, 7, 100]] == 0)
    assert np.allclose(s["F"][[0, 7, 100]], np.eye(3))
    assert np.all(s["C"][[0, 7, 100]] == 0)
    assert np.all(s["Jp"][[0, 7, 100]] == 1.0)


def test_inactive_particles_are_frozen():
    d = W.elastic_cube(n_side=8)
    rt = _rt([d])
    idx = torch.arange(0, 50, dtype=torch.int32)
    rt.set_particles_active(idx, torch.zeros(50, dtype=torch.uint8))
    s0 = _state_np(rt)
    rt.substeps(10)
    s1 = _state_np(rt)
    assert np.array_equal(s0["pos"][:50], s1["pos"][:50])
    assert not s1["active"][:50].any() and s1["active"][50:].all()
    assert not np.array_equal(s0["pos"][50:], s1["pos"][50:])


def test_nan_is_reported_not_propagated_to_memory():
    d = W.elastic_cube(n_side=8)
    rt = _rt([d])
    pos = d.pos.copy()
    pos[3] = np.nan
    rt.set_state(pos=pos)
    rt.substeps(2)
    from genesis_b200 import _native as nat

    assert rt.status() & nat.MPM_STATUS_NAN


def test_batched_instances_match_individual_runs():
    """Several scenes of different sizes and grids in one launch == each run alone."""
    descs = W.batch_scenes(n_scenes=5, n_range=(500, 3000), densities=(32, 64))
    together = _rt(descs)
    together.substeps(20)
    st = _state_np(together)
    offs = together.instance_offsets
    for i, d in enumerate(descs):
        alone = _rt([d])
        alone.substeps(20)
        sa = _state_np(alone)
        sl = slice(offs[i], offs[i] + d.n_particles)
        assert np.abs(st["pos"][sl] - sa["pos"]).max() < 1e-6, i


def test_full_size_mixed_500k_conservation():
    """Config with 500,000 particles on the 129^3 grid: p2g conserves mass exactly (to f32
    summation) and momentum; 20 substeps keep every particle finite and inside the boundary."""
    d = W.mixed_500k()
    rt = _rt([d])
    rt.sort()
    rt.p2g()
    mm, _ = _dense_grid(rt)
    mats = rt._mats
    masses = np.array([mats[int(k)].mass for k in d.mat_idx])
    assert np.isclose(mm[..., 3].sum(dtype=np.float64), masses.sum(), rtol=1e-6)
    mom = (masses[:, None] * d.vel).sum(0)
    scale = (masses[:, None] * np.abs(d.vel)).sum()
    assert np.allclose(mm[..., :3].sum(axis=(0, 1, 2), dtype=np.float64), mom, atol=1e-6 * scale)
    rt.grid_op()
    rt.g2p()
    rt._count += 1
    rt.substeps(19)
    s = _state_np(rt)
    sp = rt.specs[0]
    assert np.all(np.isfinite(s["pos"]))
    assert np.all(s["pos"] >= sp.bnd_lo.astype(np.float32)) and np.all(s["pos"] <= sp.bnd_hi.astype(np.float32))
    assert rt.status() == 0


def test_retune_and_autotune_preserve_the_simulation():
    from genesis_b200 import autotune

    d = W.mixed_500k(n_side=10)
    a = _rt([d], use_graphs=False)
    b = _rt([d], use_graphs=False)
    best, times = autotune.tune(b, candidates={"chunk_particles": (128, 256), "sort_interval": (10, 20),
                                               "grid_ctas_per_sm": (0, 14)}, trial_substeps=20, use_cache=False)
    assert set(best) == {"chunk_particles", "sort_interval", "grid_ctas"} and len(times) == 8
    assert np.array_equal(_state_np(a)["pos"], _state_np(b)["pos"])  # trials were rolled back
    a.substeps(30)
    b.substeps(30)
    assert np.abs(_state_np(a)["pos"] - _state_np(b)["pos"]).max() < 1e-6


def test_batched_many_small_scenes_faster_than_sequential():
    from genesis_b200.batch import BatchedScenes, run_sequential

    descs = W.batch_scenes(n_scenes=24, n_range=(2e3, 5e3), densities=(32,))
    bs = BatchedScenes(descs, tune=False)
    bs.substeps(bs.rt.sort_interval)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    bs.substeps(100)
    b.record()
    torch.cuda.synchronize()
    t_batched = a.elapsed_time(b) * 1e-3
    t_seq = run_sequential(descs, 100)
    assert t_seq > 2.0 * t_batched, (t_seq, t_batched)
