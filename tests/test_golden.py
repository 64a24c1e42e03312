"""The oracle against the committed golden fixtures (tests/golden/, made by
make_golden.py from the float64 numpy restatement): both restatements must reproduce
them.  No GPU."""

import glob
import json
import os

import numpy as np
import pytest

from oracle import cref
from oracle import mpm_ref as R

# fixtures of the float64 oracle (make_golden.py); the ref_*.npz made by running the reference's
# own code are checked by test_reference_golden.py
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith("ref_"))


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    p = R.Params(grid_density=meta["grid_density"], lower_bound=tuple(meta["lower_bound"]),
                 upper_bound=tuple(meta["upper_bound"]), particle_size=meta["particle_size"], dt=meta["dt"],
                 gravity=tuple(meta["gravity"]), dtype=np.float64)
    mats = [R.make_material(k, **dict(kw)) for k, kw in meta["materials"]]
    st = R.make_state(z["pos"], mats, z["mat_idx"], np.float64, v=z["vel"], active=z["active"])
    return z, meta, p, mats, st


def test_fixtures_present():
    names = {os.path.basename(g)[:-4] for g in GOLDEN}
    assert {"elastic_cube", "elastic_neohookean", "mixed", "mixed_partly_active", "batch_0"} <= names


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_c_oracle_reproduces_golden(path):
    z, meta, p, mats, st = load(path)
    done = 0
    for n in meta["snapshots"]:
        st, rc = cref.substeps(p, mats, st, n - done)
        assert rc == 0
        done = n
        assert np.abs(st["x"] - z[f"x_{n}"]).max() < 1e-11, n
        assert np.abs(st["v"] - z[f"v_{n}"]).max() < 1e-8, n
        assert np.abs(st["F"] - z[f"F_{n}"]).max() < 1e-9, n
        assert np.abs(st["Jp"] - z[f"Jp_{n}"]).max() < 1e-9, n


@pytest.mark.parametrize("path", GOLDEN[:3], ids=lambda p: os.path.basename(p)[:-4])
def test_numpy_oracle_reproduces_golden_and_grid_sums(path):
    z, meta, p, mats, st = load(path)
    gm, gp, _, _ = R.p2g(p, mats, st)
    assert np.isclose(gm.sum(), float(z["grid_mass"]), rtol=1e-13)
    assert np.allclose(gp.reshape(-1, 3).sum(0), z["grid_momentum"], rtol=1e-12, atol=1e-15)
    out = R.run(p, mats, st, 10)
    assert np.abs(out["x"] - z["x_10"]).max() < 1e-13
