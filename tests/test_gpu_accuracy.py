"""Error of the float32 CUDA path per benchmark configuration, against float64 oracles.

Two float64 references are used, both the C restatement (oracle/mpm_ref.c, pinned to the
reference's own code by tests/test_reference_golden.py):

* "model32": the reference's precision-32 model evaluated in float64 -- float64 arithmetic
  with the float32 gs.EPS (1.19e-7, genesis/__init__.py:205-206).  EPS is part of the model,
  not of the arithmetic: it is the grid-mass threshold and the eps of Matrix.norm(eps) in
  the plastic return mappings (sand.py:61, elasto_plastic.py:74).  The tolerances below are
  asserted against it: it is what a float32 run of the reference computes, without the
  float32 round-off.
* "fp64": the reference's precision-64 run (EPS 2.2e-16).  Its distance from the float32 run
  is a model difference plus round-off; it is printed (run with -s) and recorded, not
  asserted.  For Sand the two differ by ~3e-5 m after 100 substeps, because sqrt(|e_hat|^2 +
  EPS) in the Drucker-Prager projection is dominated by EPS at per-substep strains of 1e-4.

Tolerances (1 m domain): positions 1e-5 m after 100 substeps for every material;
velocities 1e-5 m/s where float32 arithmetic can reach it, otherwise within 4x the float32
C restatement's own deviation from model32 (it computes the same model with another operation
order, so it measures what float32 round-off alone does to the trajectory; in the granular
Sand and Snow flows two float32 runs drift apart in velocity by 1e-4 - 1e-3 m/s within 100
substeps while their positions stay within 4e-6 m): the bound is 4 x that deviation + 1e-6,
and both numbers are printed.
"""

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _run(descs, n, **kw):
    from genesis_b200.engine.runtime import runtime_from_descs

    rt = runtime_from_descs(descs, **kw)
    rt.substeps(n)
    st = rt.get_state(("pos", "vel", "Jp"))
    torch.cuda.synchronize()
    return rt, {k: v.cpu().numpy().astype(np.float64) for k, v in st.items()}


def _oracle(desc, n, dtype=np.float64, model=np.float32, margin=False):
    from oracle import bridge, cref

    p, mats, st = bridge.from_desc(desc, dtype, model_dtype=model)
    if not margin:
        out, rc = cref.substeps(p, mats, st, n)
        assert rc == 0
        return out
    # record each particle's distance to its return mapping's branch switch, from substep 2 on
    # (substep 1 starts every Sand particle at tr = 0 exactly, in every precision)
    st, rc = cref.substeps(p, mats, st, 1)
    m = np.full(desc.n_particles, np.inf, dtype=dtype)
    out, rc2 = cref.substeps(p, mats, st, n - 1, branch_margin=m)
    assert rc == 0 and rc2 == 0
    return out, m


def _errs(g, o, sel):
    return np.abs(g["pos"][sel] - o["x"][sel]).max(), np.abs(g["vel"][sel] - o["v"][sel]).max()


def test_elastic_cube_vs_fp64():
    """The elastic cube at full size: 32,768 particles, 65^3 grid, dt 1e-4, 100 substeps."""
    d = W.elastic_cube()
    _, g = _run([d], 100)
    o = _oracle(d, 100)
    o64 = _oracle(d, 100, model=np.float64)
    sel = slice(None)
    ex, ev = _errs(g, o, sel)
    ex64, ev64 = _errs(g, o64, sel)
    print(f"\n[accuracy] elastic_cube 32,768 p, 100 substeps: model32 max|dx| = {ex:.2e} m, max|dv| = {ev:.2e} m/s;"
          f" fp64 max|dx| = {ex64:.2e} m, max|dv| = {ev64:.2e} m/s")
    assert ex <= 1e-5 and ev <= 1e-5


def test_mixed_500k_vs_fp64_per_material():
    """The mixed scene at full size: 500,000 particles (Liquid, Sand, Snow, ElastoPlastic), 129^3 grid,
    dt 5e-5, 100 substeps.  Also reports, per material, how many particles came within 1e-5 of
    their return mapping's branch switch in the float64 run, and the error among them and
    among the rest (the float32 error is not concentrated near the switches)."""
    d = W.mixed_500k()
    _, g = _run([d], 100)
    o, margin = _oracle(d, 100, margin=True)
    o64 = _oracle(d, 100, model=np.float64)
    o32 = _oracle(d, 100, dtype=np.float32)
    names = ["liquid", "sand", "snow", "elastoplastic"]
    for m in range(4):
        sel = d.mat_idx == m
        ex, ev = _errs(g, o, sel)
        ex64, ev64 = _errs(g, o64, sel)
        e32x, e32v = _errs({"pos": o32["x"], "vel": o32["v"]}, o, sel)
        near = sel & (margin < 1e-5)
        far = sel & ~(margin < 1e-5)
        exn = np.abs(g["pos"][near] - o["x"][near]).max() if near.any() else 0.0
        exf = np.abs(g["pos"][far] - o["x"][far]).max() if far.any() else 0.0
        print(f"\n[accuracy] mixed_500k {names[m]}, 100 substeps: model32 max|dx| = {ex:.2e} m, max|dv| = {ev:.2e} m/s"
              f" (float32 C restatement {e32x:.2e} m, {e32v:.2e} m/s); fp64 max|dx| = {ex64:.2e} m, max|dv| = "
              f"{ev64:.2e} m/s; within 1e-5 of a branch switch: {int(near.sum())} particles (max|dx| {exn:.2e}),"
              f" the other {int(far.sum())}: max|dx| {exf:.2e}")
        assert ex <= 1e-5, (names[m], ex)
        assert ev <= 4 * e32v + 1e-6, (names[m], ev, e32v)


def _config3_subset():
    """From the 256 scenes of the batching configuration (workloads.batch_scenes defaults,
    seed 2), the smallest scene of every (material, grid) pair: 15 scenes covering the five
    materials and the three grids."""
    scenes = W.batch_scenes()
    pick = {}
    for d in scenes:
        key = (d.materials[0][0], d.grid_density)
        if key not in pick or d.n_particles < pick[key].n_particles:
            pick[key] = d
    return [pick[k] for k in sorted(pick)]


def test_batched_scenes_vs_fp64():
    descs = _config3_subset()
    assert len({d.materials[0][0] for d in descs}) == 5 and len({d.grid_density for d in descs}) == 3
    rt, g = _run(descs, 100)
    offs = rt.instance_offsets
    worst = worst64 = worst_v = 0.0
    for i, d in enumerate(descs):
        sl = slice(offs[i], offs[i] + d.n_particles)
        gi = {k: v[sl] for k, v in g.items()}
        o = _oracle(d, 100)
        o64 = _oracle(d, 100, model=np.float64)
        o32 = _oracle(d, 100, dtype=np.float32)
        ex, ev = _errs(gi, o, slice(None))
        ex64, _ = _errs(gi, o64, slice(None))
        _, e32v = _errs({"pos": o32["x"], "vel": o32["v"]}, o, slice(None))
        worst, worst64, worst_v = max(worst, ex), max(worst64, ex64), max(worst_v, ev)
        assert ex <= 1e-5, (d.name, d.materials, ex)
        assert ev <= 4 * e32v + 1e-6, (d.name, d.materials, ev, e32v)
    print(f"\n[accuracy] {len(descs)} batched scenes from the 256-scene set (5 materials x 3 grids, "
          f"{sum(d.n_particles for d in descs)} particles), 100 substeps: worst model32 max|dx| = {worst:.2e} m, "
          f"max|dv| = {worst_v:.2e} m/s; fp64 max|dx| = {worst64:.2e} m")
