"""Reverse-mode adjoint of one MPM substep (Elastic, corotated) -- TEST INFRASTRUCTURE ONLY.

numpy restatement of the hand-derived adjoint that the CUDA kernels implement, used to
check them.  It differentiates exactly the forward of ``mpm_ref.substep`` for Elastic
materials with per-particle Lame parameters:

  F_tmp = (I + dt C) F                                  mpm_solver.py:264-266
  F_tmp = U S V^T, R = U V^T, J = det F_tmp             mpm_solver.py:273, 305
  P = 2 mu (F_tmp - R) F_tmp^T + lam J (J - 1) I        elastic.py:70-75
  A = s P + m C,  s = -dt vol 4 inv_dx^2                mpm_solver.py:344-345
  grid: m_i = sum w m,  p_i = sum w (m v + A d_i)       mpm_solver.py:347-386
  v_i = bc(p_i / m_i + dt g)                            legacy_coupler.py:369-372, 495-496
  v' = sum w v_i,  C' = c sum w v_i u_i^T,  x' = x + dt v', then the boundary
                                                        mpm_solver.py:396-437
with d_i = (off - fx) dx = x_i - x_p, u_i = off - fx (cell units), c = 4 inv_dx.

The polar-rotation part of the SVD backward uses the closed form
  Fbar += U [(M_ij - M_ji) / (s_i + s_j)] V^T,   M = U^T Rbar V,
which is what the reference's backward_svd (mpm_solver.py:1112-1129, the PyTorch SVD
adjoint) reduces to for R = U V^T, written without the 1 / (s_j^2 - s_i^2) factors that
its signmax(., 1e-6) guard clamps when singular values nearly coincide.
"""

from __future__ import annotations

import numpy as np

from . import mpm_ref as R


def _mT(A):
    return np.swapaxes(A, -1, -2)


def backward_svd(gU, gS, gV, U, S, V):
    """Restatement of the reference's backward_svd (mpm_solver.py:1106-1129, the PyTorch
    SVD adjoint), batched over the leading axis: given the adjoints of U, S (a 3x3 matrix,
    diagonal in the forward) and V of F = U S V^T, the adjoint of F is
      U [(F o (U^T gU - gU^T U)) S] V^T + U [S ((F o (V^T gV - gV^T V)) V^T)] + U gS V^T,
    with F_ij = 1 / signmax(s_j^2 - s_i^2, 1e-6) off the diagonal and 0 on it, s_i = S_ii,
    signmax(a, e) = sign(a) max(|a|, e) (sign(0) = +1)."""
    vt, ut = _mT(V), _mT(U)
    s2 = np.diagonal(S, axis1=-2, axis2=-1) ** 2
    diff = s2[..., None, :] - s2[..., :, None]  # [i, j] = s_j^2 - s_i^2
    sm = np.where(diff >= 0, 1.0, -1.0) * np.maximum(np.abs(diff), 1e-6)
    Fm = 1.0 / sm
    idx = np.arange(3)
    Fm[..., idx, idx] = 0.0
    s_term = U @ gS @ vt
    u_term = U @ ((Fm * (ut @ gU - _mT(gU) @ U)) @ S) @ vt
    v_term = U @ (S @ ((Fm * (vt @ gV - _mT(gV) @ V)) @ vt))
    return u_term + v_term + s_term


def _weights_and_grads(fx):
    w = [0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2]
    dw = [-(1.5 - fx), -2.0 * (fx - 1.0), fx - 0.5]
    return w, dw


def _stencil(p, x):
    xi = x * p.inv_dx
    base = np.floor(xi - 0.5).astype(np.int64)
    fx = xi - base
    w, dw = _weights_and_grads(fx)
    node0 = base - p.lower_cell[None, :]
    return base, fx, w, dw, node0


def _offsets():
    for i in range(3):
        for j in range(3):
            for k in range(3):
                yield i, j, k


def forward(p, st, mu, lam, mass):
    """One substep for all (active, Elastic) particles with per-particle mu/lam; returns the
    new state and the intermediates the adjoint needs."""
    x, v, C, F = st["x"], st["v"], st["C"], st["F"]
    n = x.shape[0]
    eye = np.eye(3)
    Ft = (eye + p.dt * C) @ F
    U, S, V = R.svd3(Ft)
    Rm = U @ _mT(V)
    J = np.linalg.det(Ft)
    P = 2 * mu[:, None, None] * (Ft - Rm) @ _mT(Ft) + (lam * J * (J - 1))[:, None, None] * eye
    s = -p.dt * p.p_vol * 4 * p.inv_dx * p.inv_dx
    A = s * P + mass[:, None, None] * C
    base, fx, w, dw, node0 = _stencil(p, x)
    res = tuple(int(r) for r in p.grid_res)
    G = int(np.prod(res))
    gm = np.zeros(G)
    gp = np.zeros((G, 3))
    lin_all = []
    for i, j, k in _offsets():
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        d = (off[None, :] - fx) * p.dx
        lin = np.ravel_multi_index((node0 + off).T, res)
        lin_all.append(lin)
        gm += np.bincount(lin, weights=wt * mass, minlength=G)
        contrib = wt[:, None] * (mass[:, None] * v + np.einsum("nij,nj->ni", A, d))
        for c in range(3):
            gp[:, c] += np.bincount(lin, weights=contrib[:, c], minlength=G)
    # grid op
    act = gm > p.eps
    vg = np.zeros((G, 3))
    vg[act] = gp[act] / gm[act][:, None] + p.dt * np.asarray(p.gravity)[None, :]
    idx = np.array(np.unravel_index(np.arange(G), res)).T
    gpos = (idx + p.lower_cell[None, :]) * p.dx
    gmask = np.ones((G, 3))
    for c in range(3):
        up = (gpos[:, c] >= p.bnd_hi[c]) & (vg[:, c] >= 0)
        dn = (~up) & (gpos[:, c] <= p.bnd_lo[c]) & (vg[:, c] <= 0)
        gmask[:, c] = np.where(up | dn, 0.0, 1.0)
    gmask[~act] = 0.0
    vh = vg * gmask
    # g2p
    c4 = 4 * p.inv_dx
    nv = np.zeros((n, 3))
    nC = np.zeros((n, 3, 3))
    for (i, j, k), lin in zip(_offsets(), lin_all):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        u = off[None, :] - fx
        nv += wt[:, None] * vh[lin]
        nC += (c4 * wt)[:, None, None] * vh[lin][:, :, None] * u[:, None, :]
    xs = x + p.dt * nv
    pmask = np.ones((n, 3))
    vmask = np.ones((n, 3))
    for c in range(3):
        up = (xs[:, c] >= p.bnd_hi[c]) & (nv[:, c] >= 0)
        dn = (~up) & (xs[:, c] <= p.bnd_lo[c]) & (nv[:, c] <= 0)
        vmask[:, c] = np.where(up | dn, 0.0, 1.0)
        pmask[:, c] = np.where((xs[:, c] > p.bnd_hi[c]) | (xs[:, c] < p.bnd_lo[c]), 0.0, 1.0)
    xn = np.clip(xs, p.bnd_lo, p.bnd_hi)
    out = dict(st)
    out.update(x=xn, v=nv * vmask, C=nC, F=Ft)
    inter = dict(Ft=Ft, U=U, S=S, V=V, Rm=Rm, J=J, P=P, A=A, fx=fx, w=w, dw=dw, lin=lin_all, gm=gm, gp=gp,
                 vh=vh, gmask=gmask, act=act, nv=nv, pmask=pmask, vmask=vmask, s=s)
    return out, inter


def backward(p, st, mu, lam, mass, inter, adj):
    """adj: dict with x, v, C, F adjoints of the substep's output.  Returns the adjoints of
    its input state and of mu, lam."""
    x, v, C, F = st["x"], st["v"], st["C"], st["F"]
    n = x.shape[0]
    G = inter["gm"].shape[0]
    fx, w, dw = inter["fx"], inter["w"], inter["dw"]
    c4 = 4 * p.inv_dx
    # ---- g2p adjoint
    gx = adj["x"] * inter["pmask"]
    vbar = adj["v"] * inter["vmask"] + p.dt * gx
    Cbar = adj["C"]
    xbar = gx.copy()
    vh_bar = np.zeros((G, 3))
    for (i, j, k), lin in zip(_offsets(), inter["lin"]):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        gw = np.stack([dw[i][:, 0] * w[j][:, 1] * w[k][:, 2], w[i][:, 0] * dw[j][:, 1] * w[k][:, 2],
                       w[i][:, 0] * w[j][:, 1] * dw[k][:, 2]], 1) * p.inv_dx
        u = off[None, :] - fx
        vh = inter["vh"][lin]
        Cu = np.einsum("nij,nj->ni", Cbar, u)
        contrib = wt[:, None] * vbar + (c4 * wt)[:, None] * Cu
        for c in range(3):
            vh_bar[:, c] += np.bincount(lin, weights=contrib[:, c], minlength=G)
        wbar = (vbar * vh).sum(1) + c4 * (vh * Cu).sum(1)
        ubar = (c4 * wt)[:, None] * np.einsum("nji,nj->ni", Cbar, vh)
        xbar += wbar[:, None] * gw - p.inv_dx * ubar
    # ---- grid op adjoint
    vg_bar = vh_bar * inter["gmask"]
    act = inter["act"]
    pbar = np.zeros((G, 3))
    mbar = np.zeros(G)
    pbar[act] = vg_bar[act] / inter["gm"][act][:, None]
    mbar[act] = -(vg_bar[act] * inter["gp"][act]).sum(1) / inter["gm"][act] ** 2
    # ---- p2g adjoint
    A = inter["A"]
    Abar = np.zeros((n, 3, 3))
    vbar_n = np.zeros((n, 3))
    for (i, j, k), lin in zip(_offsets(), inter["lin"]):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        gw = np.stack([dw[i][:, 0] * w[j][:, 1] * w[k][:, 2], w[i][:, 0] * dw[j][:, 1] * w[k][:, 2],
                       w[i][:, 0] * w[j][:, 1] * dw[k][:, 2]], 1) * p.inv_dx
        d = (off[None, :] - fx) * p.dx
        pb = pbar[lin]
        mb = mbar[lin]
        q = mass[:, None] * v + np.einsum("nij,nj->ni", A, d)
        wbar = mb * mass + (pb * q).sum(1)
        vbar_n += (wt * mass)[:, None] * pb
        Abar += wt[:, None, None] * pb[:, :, None] * d[:, None, :]
        xbar += wbar[:, None] * gw - wt[:, None] * np.einsum("nji,nj->ni", A, pb)
    Pbar = inter["s"] * Abar
    Cbar_n = mass[:, None, None] * Abar
    Ft, U, S, V, Rm, J = inter["Ft"], inter["U"], inter["S"], inter["V"], inter["Rm"], inter["J"]
    D = Ft - Rm
    mu_bar = 2 * np.einsum("nij,nij->n", Pbar, D @ _mT(Ft))
    trP = np.trace(Pbar, axis1=1, axis2=2)
    lam_bar = trP * J * (J - 1)
    Ft_bar = 2 * mu[:, None, None] * (Pbar @ Ft + _mT(Pbar) @ D)
    Rbar = -2 * mu[:, None, None] * Pbar @ Ft
    Jbar = lam * (2 * J - 1) * trP
    Ft_bar += Jbar[:, None, None] * J[:, None, None] * np.linalg.inv(_mT(Ft))
    M = _mT(U) @ Rbar @ V
    den = S[:, :, None] + S[:, None, :]
    X = (M - _mT(M)) / np.where(np.abs(den) > 1e-12, den, 1e-12)
    Ft_bar += U @ X @ _mT(V)
    Ft_bar += adj["F"]  # F_new = F_tmp for Elastic
    eye = np.eye(3)
    F_bar_n = _mT(eye + p.dt * C) @ Ft_bar
    Cbar_n += p.dt * Ft_bar @ _mT(F)
    return dict(x=xbar, v=vbar_n, C=Cbar_n, F=F_bar_n), mu_bar, lam_bar


def lame_of_E(E, nu):
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


def rollout_loss_and_grad(p, st0, E, nu, mass, n_substeps, target):
    """loss = |mean(x_T) - target|^2 and its gradient w.r.t. the initial velocity (summed
    over particles, i.e. w.r.t. a uniform v0) and per-particle E, storing every state."""
    mu, lam = lame_of_E(E, nu)
    states, inters = [st0], []
    st = st0
    for _ in range(n_substeps):
        st, it = forward(p, st, mu, lam, mass)
        states.append(st)
        inters.append(it)
    n = st0["x"].shape[0]
    xm = states[-1]["x"].mean(0)
    loss = float(((xm - target) ** 2).sum())
    adj = dict(x=np.tile(2 * (xm - target) / n, (n, 1)), v=np.zeros((n, 3)), C=np.zeros((n, 3, 3)),
               F=np.zeros((n, 3, 3)))
    mu_bar = np.zeros(n)
    lam_bar = np.zeros(n)
    for t in range(n_substeps - 1, -1, -1):
        adj, mb, lb = backward(p, states[t], mu, lam, mass, inters[t], adj)
        mu_bar += mb
        lam_bar += lb
    E_bar = mu_bar / (2.0 * (1.0 + nu)) + lam_bar * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return loss, adj["v"].sum(0), E_bar, adj


def rollout_loss(p, st0, E, nu, mass, n_substeps, target):
    mu, lam = lame_of_E(E, nu)
    st = st0
    for _ in range(n_substeps):
        st, _ = forward(p, st, mu, lam, mass)
    return float(((st["x"].mean(0) - target) ** 2).sum())
