"""The adjoint of every MPM material, on the CPU (float64).

* The restatement of the reference's own backward (oracle/mpm_adjoint.py: the materials'
  update_F_S_Jp / update_stress differentiated with U, S, V, F_tmp and Jp as inputs, then
  backward_svd, mpm_solver.py:1112-1129) against central finite differences of whole
  rollouts, per material: the initial velocity, one particle's mu and lam, and (Snow) its Jp.
* The kernel's formulation (the spectral form of mpm_adjoint.cuh, restated in numpy) against
  that restatement at random non-degenerate F_tmp: equal to round-off.
* At the rest state F_tmp = I the reference's backward_svd loses the rotation's derivative
  (its signmax guard makes the 1 / (s_j^2 - s_i^2) factors symmetric, so the U and V terms
  cancel), which should cancel the skew part of the stress's direct derivative: the reference's
  gradient keeps a spurious 2 mu skew(P_bar), while the spectral form matches finite
  differences there.
"""

import numpy as np
import pytest

from oracle import mpm_adjoint as A
from oracle import mpm_ref as R

MATERIALS = [
    ("elastic", dict(E=1e5, nu=0.3)),
    ("elastic", dict(E=1e5, nu=0.3, model="neohooken")),
    ("muscle", dict(E=1e5, nu=0.3)),
    ("elastoplastic", dict(E=1e5, nu=0.3, von_mises_yield_stress=1e3)),
    ("elastoplastic", dict(E=1e5, nu=0.3, use_von_mises=False)),
    ("liquid", dict(E=1e5, nu=0.2, viscous=True)),
    ("liquid", dict(E=1e5, nu=0.2)),
    ("sand", dict(E=1e5, friction_angle=40)),
    ("snow", dict(E=1e5, yield_lower=2.5e-2, yield_higher=7.5e-3)),
]


def _scene(kind, kw, seed, n=48):
    rng = np.random.default_rng(seed)
    mats = [R.make_material(kind, **kw)]
    p = R.Params(grid_density=32, upper_bound=(0.5, 0.5, 0.5), particle_size=0.01, dt=2e-4, gravity=(0, 0, -9.8))
    pos = 0.2 + rng.uniform(0, 0.1, size=(n, 3))
    st = R.make_state(pos, mats, np.zeros(n, int), np.float64, v=rng.normal(0, 0.3, (n, 3)))
    st["F"] = (0.97 if kind == "sand" else 1.0) * np.eye(3) + rng.normal(0, 0.03, (n, 3, 3))
    st["C"] = rng.normal(0, 2.0, (n, 3, 3))
    if kind == "sand":
        st["Jp"] = rng.uniform(-0.02, 0.02, n)
    if kind == "snow":
        st["Jp"] = rng.uniform(0.95, 1.05, n)
    if kind == "muscle":
        d = rng.normal(size=(n, 3))
        st["actu"] = rng.uniform(-0.3, 0.3, n)
        st["mdir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    m = mats[0]
    mu = np.full(n, m.mu) * rng.uniform(0.8, 1.2, n)
    lam = np.full(n, m.lam) * rng.uniform(0.8, 1.2, n)
    W = rng.normal(size=(n, 3))
    return p, mats, st, mu, lam, W


@pytest.mark.parametrize("kind,kw", MATERIALS, ids=lambda x: str(x)[:30])
def test_rollout_gradient_matches_central_differences(kind, kw):
    p, mats, st, mu, lam, W = _scene(kind, kw, seed=3)
    T = 4
    loss, gv0, gmu, glam, adj = A.rollout_materials(p, mats, st, mu, lam, T, None, weights=W)

    def L(st2=st, mu2=mu, lam2=lam):
        return A.rollout_materials(p, mats, st2, mu2, lam2, T, None, grad=False, weights=W)

    def with_(key, i, delta):
        s2 = dict(st)
        s2[key] = st[key].copy()
        s2[key][i] += delta
        return s2

    h = 1e-6
    for c in range(3):
        fd = (L(with_("v", (slice(None), c), h)) - L(with_("v", (slice(None), c), -h))) / (2 * h)
        assert abs(gv0[c] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gv0).max()), (c, gv0[c], fd)
    for i in (5, 17):
        if mats[0].mu:
            hm = 1e-4 * mu[i]
            mp, mm = mu.copy(), mu.copy()
            mp[i] += hm
            mm[i] -= hm
            fd = (L(mu2=mp) - L(mu2=mm)) / (2 * hm)
            assert abs(gmu[i] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(gmu).max()), (i, gmu[i], fd)
        hl = 1e-4 * lam[i]
        lp, lm = lam.copy(), lam.copy()
        lp[i] += hl
        lm[i] -= hl
        fd = (L(lam2=lp) - L(lam2=lm)) / (2 * hl)
        assert abs(glam[i] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(glam).max()), (i, glam[i], fd)
        if kind in ("snow", "sand"):
            fd = (L(with_("Jp", i, 1e-5)) - L(with_("Jp", i, -1e-5))) / 2e-5
            assert abs(adj["Jp"][i] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(adj["Jp"]).max()), (i, adj["Jp"][i], fd)


@pytest.mark.parametrize("kind,kw", [m for m in MATERIALS if m[0] != "muscle"], ids=lambda x: str(x)[:30])
def test_spectral_form_equals_reference_backward(kind, kw):
    rng = np.random.default_rng(11)
    m = R.make_material(kind, **kw)
    n = 300
    s = rng.uniform(0.93, 1.02, (n, 3)) if kind == "sand" else rng.uniform(0.85, 1.15, (n, 3))
    q1 = np.linalg.qr(rng.normal(size=(n, 3, 3)))[0]
    q2 = np.linalg.qr(rng.normal(size=(n, 3, 3)))[0]
    Ft = q1 @ (s[:, :, None] * np.swapaxes(q2, 1, 2))
    U, S, V = R.svd3(Ft)
    Jp = rng.uniform(0.95, 1.05, n) if kind == "snow" else (rng.uniform(-0.05, 0.05, n) if kind == "sand" else np.ones(n))
    mu = (m.mu if m.mu else 0.0) * rng.uniform(0.8, 1.2, n)
    lam = m.lam * rng.uniform(0.8, 1.2, n)
    Gb, Pb = rng.normal(size=(2, n, 3, 3))
    Jb = rng.normal(size=n)
    Sd = np.zeros((n, 3, 3))
    Sd[:, [0, 1, 2], [0, 1, 2]] = S
    ftb, ub, sb, vb, jb, mb, lb, _ = A.material_vjp(m, 2.2e-16, U, S, V, Ft, Jp, mu, lam, None, None, Gb, Jb, Pb)
    Sb = np.zeros_like(Sd)
    Sb[:, [0, 1, 2], [0, 1, 2]] = sb
    ref = ftb + A.backward_svd(ub, Sb, vb, U, Sd, V)
    got, gj, gm, gl = A.material_vjp_spectral(m, 2.2e-16, U, S, V, Ft, Jp, mu, lam, Gb, Jb, Pb)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.abs(gj - jb).max() <= 1e-10 * max(1.0, np.abs(jb).max())
    assert np.abs(gm - mb).max() <= 1e-10 * max(1e-30, np.abs(mb).max())
    assert np.abs(gl - lb).max() <= 1e-10 * max(1e-30, np.abs(lb).max())


def test_rest_state_rotation_gradient():
    """F_tmp = I (every particle at rest): dP = 2 mu (dF - dR) + lam tr(dF) I with dR =
    skew(dF), so the true F_tmp_bar = 2 mu sym(P_bar) + lam tr(P_bar) I is symmetric.  The
    reference's backward_svd drops the dR term (its guarded factors are +1e6 on both sides of
    the diagonal and the U and V terms cancel) and keeps 2 mu skew(P_bar); the spectral form
    matches finite differences."""
    m = R.make_material("elastic", E=1e5, nu=0.3)
    n = 1
    rng = np.random.default_rng(2)
    Ft = np.eye(3)[None].copy()
    U, S, V = R.svd3(Ft)
    mu, lam = np.array([m.mu]), np.array([m.lam])
    Pb = rng.normal(size=(1, 3, 3))
    zero = np.zeros((1, 3, 3))

    def stress(F):
        u, s_, v = np.linalg.svd(F[0])
        Rm = u @ v
        J = np.linalg.det(F[0])
        return 2 * mu[0] * (F[0] - Rm) @ F[0].T + lam[0] * J * (J - 1) * np.eye(3)

    fd = np.zeros((3, 3))
    h = 1e-6
    for a in range(3):
        for b in range(3):
            dF = np.zeros((1, 3, 3))
            dF[0, a, b] = h
            fd[a, b] = ((stress(Ft + dF) - stress(Ft - dF)) * Pb[0]).sum() / (2 * h)
    spectral, _, _, _ = A.material_vjp_spectral(m, 2.2e-16, U, S, V, Ft, np.ones(n), mu, lam, zero, np.zeros(n), Pb)
    assert np.abs(spectral[0] - fd).max() <= 1e-6 * np.abs(fd).max()
    Sd = np.eye(3)[None]
    ftb, ub, sb, vb, _, _, _, _ = A.material_vjp(m, 2.2e-16, U, S, V, Ft, np.ones(n), mu, lam, None, None, zero,
                                                np.zeros(n), Pb)
    Sb = np.zeros((1, 3, 3))
    Sb[:, [0, 1, 2], [0, 1, 2]] = sb
    reference = ftb + A.backward_svd(ub, Sb, vb, U, Sd, V)
    assert np.abs(fd - fd.T).max() <= 1e-6 * np.abs(fd).max()  # the true gradient is symmetric
    spurious = mu[0] * (Pb[0] - Pb[0].T)  # 2 mu skew(P_bar)
    assert np.abs(reference[0] - fd - spurious).max() <= 1e-6 * np.abs(fd).max()
