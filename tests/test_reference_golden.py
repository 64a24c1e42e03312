"""Both oracles against fixtures made by the REFERENCE's own code (tests/golden/ref_*.npz,
written by make_reference_golden.py, which imports Genesis's mpm_solver.py,
legacy_coupler.py, boundaries.py and materials/MPM/*.py unchanged and runs their kernels on
a numpy stand-in for gstaichi).  This pins the oracle to the reference: every material's
return mapping and stress, the boundary, the SVD adjoint, and whole substeps (p2g, grid op,
g2p) over 9 material variants and a cube thrown at the floor.  All float64.  No GPU."""

import json
import os

import numpy as np
import pytest

from oracle import cref
from oracle import mpm_adjoint as A
from oracle import mpm_ref as R

HERE = os.path.join(os.path.dirname(__file__), "golden")


def _fx(suffix=""):
    z = np.load(os.path.join(HERE, f"ref_functions{suffix}.npz"))
    return z, json.loads(str(z["meta"]))


def _rel(a, b):
    return float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))


@pytest.mark.parametrize("suffix", ["", "_m32"])
@pytest.mark.parametrize("vi", range(9))
def test_material_functions_match_reference(vi, suffix):
    """update_F_S_Jp and update_stress of oracle/mpm_ref.py against the reference's own methods
    (elastic.py, elasto_plastic.py, liquid.py, sand.py, snow.py, muscle.py) on F_tmp with
    singular values 0.3-1.6, some nearly repeated; at float64 gs.EPS and at the precision-32
    model's float32 gs.EPS (_m32)."""
    z, meta = _fx(suffix)
    kind, kw = meta["variants"][vi]
    m = R.make_material(kind, **dict(kw))
    F = z[f"m{vi}_F_tmp"]
    U, S, V = R.svd3(F)
    J = S[:, 0] * (S[:, 1] * S[:, 2])
    Jp = z[f"m{vi}_Jp"]
    Fn, Sn, Jn = R.update_F_S_Jp(m, meta["eps"], J, F, U, S, V, Jp)
    assert _rel(Fn, z[f"m{vi}_F_new"]) < 1e-12
    assert _rel(Sn, np.diagonal(z[f"m{vi}_S_new"], axis1=1, axis2=2)) < 1e-12
    assert np.abs(Jn - z[f"m{vi}_Jp_new"]).max() < 1e-12
    st = R.update_stress(m, U, Sn, V, F, Fn, J, Jp, z[f"m{vi}_actu"], z[f"m{vi}_mdir"])
    assert _rel(st, z[f"m{vi}_stress"]) < 1e-11


def test_sand_fixture_covers_both_branches():
    z, meta = _fx()
    vi = [k for k, _ in meta["variants"]].index("sand")
    _, S, _ = R.svd3(z[f"m{vi}_F_tmp"])
    tr = np.log(np.maximum(np.abs(S), 1e-4)).sum(1) + z[f"m{vi}_Jp"]
    assert (tr >= 0).sum() >= 10 and (tr < 0).sum() >= 10


def test_boundary_matches_reference():
    """CubeBoundary.impose_pos_vel (boundaries.py:23-33) at, inside and beyond the walls."""
    z, _ = _fx()
    p = R.Params(grid_density=64)
    assert np.allclose(p.bnd_lo, z["bnd_lo"]) and np.allclose(p.bnd_hi, z["bnd_hi"])
    pos, vel = R.boundary(p, z["bnd_pos"].copy(), z["bnd_vel"].copy())
    assert np.array_equal(pos, z["bnd_pos_out"])
    assert np.array_equal(vel, z["bnd_vel_out"])


def test_backward_svd_matches_reference():
    """The oracle's restatement of backward_svd (mpm_solver.py:1106-1129, signmax guard
    included) against the reference's function on random adjoints."""
    z, _ = _fx()
    out = A.backward_svd(z["bsvd_gU"], z["bsvd_gS"], z["bsvd_gV"], z["bsvd_U"], z["bsvd_S"], z["bsvd_V"])
    assert _rel(out, z["bsvd_out"]) < 1e-10


def _scene(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    p = R.Params(grid_density=meta["grid_density"], lower_bound=tuple(meta["lower_bound"]),
                 upper_bound=tuple(meta["upper_bound"]), particle_size=meta["particle_size"], dt=meta["dt"],
                 gravity=tuple(meta["gravity"]), dtype=np.float64)
    p.eps = meta.get("eps", p.eps)  # the *_m32 fixtures: the precision-32 model (float32 gs.EPS)
    mats = [R.make_material(k, **dict(kw)) for k, kw in meta["materials"]]
    st = R.make_state(z["pos"], mats, z["mat_idx"], np.float64, v=z["vel"], active=z["active"])
    st.update(C=z["C"].copy(), F=z["F"].copy(), Jp=z["Jp"].astype(np.float64).copy())
    if "muscle_idx" in z.files:
        n = len(z["pos"])
        actu = np.zeros(n)
        mdir = np.tile([0.0, 0.0, 1.0], (n, 1))
        actu[z["muscle_idx"]] = z["muscle_actu"][z["muscle_group"]]
        mdir[z["muscle_idx"]] = z["muscle_dir"]
        st.update(actu=actu, mdir=mdir)
    return z, meta, p, mats, st


SCENES = ["ref_mixed", "ref_cube", "ref_mixed_m32", "ref_cube_m32"]


@pytest.mark.parametrize("name", SCENES)
def test_numpy_oracle_reproduces_reference_substeps(name):
    z, meta, p, mats, st = _scene(name)
    gm, gp, _, _ = R.p2g(p, mats, st)
    assert np.abs(gm - z["grid_mass"]).max() <= 1e-15 * max(1.0, z["grid_mass"].max())
    assert np.abs(gp - z["grid_mom"]).max() <= 1e-12 * max(1.0, np.abs(z["grid_mom"]).max())
    done = 0
    for n in meta["snapshots"]:
        st = R.run(p, mats, st, n - done)
        done = n
        assert np.abs(st["x"] - z[f"x_{n}"]).max() < 1e-12, n
        assert np.abs(st["v"] - z[f"v_{n}"]).max() < 1e-9, n
        assert _rel(st["C"], z[f"C_{n}"]) < 1e-9, n
        assert np.abs(st["F"] - z[f"F_{n}"]).max() < 1e-10, n
        assert np.abs(st["Jp"] - z[f"Jp_{n}"]).max() < 1e-10, n


@pytest.mark.parametrize("name", SCENES)
def test_c_oracle_reproduces_reference_substeps(name):
    z, meta, p, mats, st = _scene(name)
    done = 0
    for n in meta["snapshots"]:
        st, rc = cref.substeps(p, mats, st, n - done)
        assert rc == 0
        done = n
        assert np.abs(st["x"] - z[f"x_{n}"]).max() < 1e-12, n
        assert np.abs(st["v"] - z[f"v_{n}"]).max() < 1e-9, n
        assert _rel(st["C"], z[f"C_{n}"]) < 1e-9, n
        assert np.abs(st["F"] - z[f"F_{n}"]).max() < 1e-10, n
        assert np.abs(st["Jp"] - z[f"Jp_{n}"]).max() < 1e-10, n
