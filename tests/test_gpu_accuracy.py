"""Error of the float32 CUDA path against the float64 oracle, per benchmark configuration.

Each test prints its measured errors (run with -s to see them) and asserts the stated
tolerance.  Position errors are in metres (domain size 1 m), after the stated number of
substeps, as max over particles.
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
    return rt, {k: v.cpu().numpy() for k, v in st.items()}


def _f64(desc, n, dtype=np.float64):
    from oracle import bridge, cref

    out, rc = cref.substeps(*bridge.from_desc(desc, dtype), n)
    assert rc == 0
    return out


def test_elastic_cube_vs_fp64():
    d = W.elastic_cube()
    _, g = _run([d], 100)
    o = _f64(d, 100)
    ex = np.abs(g["pos"] - o["x"]).max()
    ev = np.abs(g["vel"] - o["v"]).max()
    print(f"\n[accuracy] elastic_cube 32,768 p, 100 substeps: max|dx| = {ex:.2e} m, max|dv| = {ev:.2e} m/s")
    assert ex <= 1e-5


def test_mixed_500k_vs_fp64_per_material():
    d = W.mixed_500k()
    _, g = _run([d], 100)
    o = _f64(d, 100)
    o32 = _f64(d, 100, np.float32)
    names = ["liquid", "sand", "snow", "elastoplastic"]
    for m in range(4):
        sel = d.mat_idx == m
        ex = np.abs(g["pos"][sel] - o["x"][sel]).max()
        e32 = np.abs(o32["x"][sel] - o["x"][sel]).max()
        print(f"\n[accuracy] mixed_500k {names[m]}, 100 substeps: max|dx| = {ex:.2e} m "
              f"(float32 CPU restatement: {e32:.2e} m)")
        assert ex <= max(1e-5, 2 * e32)


def test_batched_scenes_vs_fp64():
    descs = W.batch_scenes(n_scenes=8, n_range=(2e3, 2e4))
    rt, g = _run(descs, 100)
    offs = rt.instance_offsets
    worst = 0.0
    for i, d in enumerate(descs):
        o = _f64(d, 100)
        sl = slice(offs[i], offs[i] + d.n_particles)
        o32 = _f64(d, 100, np.float32)
        ex = np.abs(g["pos"][sl] - o["x"]).max()
        e32 = np.abs(o32["x"] - o["x"]).max()
        worst = max(worst, ex)
        assert ex <= max(1e-5, 2 * e32), (i, d.materials, ex, e32)
    print(f"\n[accuracy] 8 batched scenes (5 materials, 3 grids), 100 substeps: worst max|dx| = {worst:.2e} m")
