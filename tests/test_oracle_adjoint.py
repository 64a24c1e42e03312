"""The oracle's hand-derived substep adjoint against float64 central finite differences
(CPU only).  The differentiation scene starts just above the floor with a downward
velocity so both the velocity and the per-particle-E gradients are non-trivial."""

import numpy as np

from genesis_b200 import workloads as W
from oracle import bridge
from oracle import mpm_adjoint as AD
from oracle import mpm_ref as R


def test_adjoint_matches_central_differences():
    d = W.diff_elastic(n=64, n_substeps=30)
    p, mats, st = bridge.from_desc(d, np.float64)
    n = st["x"].shape[0]
    mass = np.full(n, R.particle_mass(p, mats[0]))
    v0 = d.meta["v0"]
    st["v"] = np.tile(v0, (n, 1))
    target = d.meta["target"]
    E = d.E_particle
    loss, gv0, gE, _ = AD.rollout_loss_and_grad(p, st, E, 0.3, mass, d.n_substeps, target)

    def L(v, Ev):
        s = dict(st)
        s["v"] = np.tile(v, (n, 1))
        return AD.rollout_loss(p, s, Ev, 0.3, mass, d.n_substeps, target)

    h = 1e-4
    for c in range(3):
        e = np.zeros(3)
        e[c] = h
        fd = (L(v0 + e, E) - L(v0 - e, E)) / (2 * h)
        assert abs(gv0[c] - fd) <= 1e-6 * max(abs(fd), 1e-8), (c, gv0[c], fd)
    k = int(np.argmax(np.abs(gE)))
    hE = 1e-4 * E[k]  # relative step for E
    Ep, Em = E.copy(), E.copy()
    Ep[k] += hE
    Em[k] -= hE
    fd = (L(v0, Ep) - L(v0, Em)) / (2 * hE)
    assert abs(fd) > 0 and abs(gE[k] - fd) <= 1e-4 * abs(fd), (gE[k], fd)
